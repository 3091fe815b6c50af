// Copy tasks of the one-launch ghost fill (host code, no CUDA dependence
// beyond the int2/int4 vector types, so that a host-only test can compile it).
//
// The copies of a fill (destination, source node index) read only nodes the
// fill does not change, so their order is free.  Runs of copies whose
// destinations and sources both advance by one node (rows of a periodic or
// outflow ghost plane) become tasks, one GPU block each, a run longer than
// kGhostLong cut into pieces of at most that many (up to eight copies per
// thread, four in flight).  A task is (first destination, source offset,
// length, 0).  The copies of runs shorter than kGhostMinRun are returned one
// by one (`single`, a thread each).  Rows of a ghost plane are not merged
// into one task: on a 129^3 grid that made the fill slower.
#pragma once

#include <algorithm>
#include <vector>

constexpr int kGhostLong = 2048;
constexpr int kGhostMinRun = 32;

template <class Int2, class Int4>
void ghost_copy_tasks_of(const std::vector<Int2> &pairs, std::vector<Int4> &tasks, std::vector<Int2> &single)
{
    auto task = [&](size_t q, size_t len) {
        Int4 t;
        t.x = pairs[q].x;
        t.y = pairs[q].y - pairs[q].x;
        t.z = (int)len;
        t.w = 0;
        tasks.push_back(t);
    };
    for (size_t i = 0; i < pairs.size();) {
        size_t j = i + 1;
        while (j < pairs.size() && pairs[j].x == pairs[j - 1].x + 1 && pairs[j].y == pairs[j - 1].y + 1) {
            ++j;
        }
        if (j - i < (size_t)kGhostMinRun) {
            single.insert(single.end(), pairs.begin() + i, pairs.begin() + j);
        } else {
            for (size_t q = i; q < j; q += kGhostLong) task(q, std::min<size_t>(kGhostLong, j - q));
        }
        i = j;
    }
}

// The copies of a fill on the grid whose axes 0 and 1 are exchanged: node
// (i, j, k) of a grid with n1 nodes along axis 1 and row pitch `pitch` is
// node (j, i, k) of the transposed grid (n0 rows of pitch `xpitch`); the
// copies come back in destination order.  For a fill of copies (periodic and
// outflow faces) this is the same fill of the transposed grid.
template <class Int2>
std::vector<Int2> transposed_copies_of(const std::vector<Int2> &pairs, int pitch, int n0, int n1, int xpitch)
{
    auto tr = [&](int q) {
        const long long i = q % pitch, j = (q / pitch) % n1, k = q / ((long long)pitch * n1);
        return (int)((k * n0 + i) * xpitch + j);
    };
    std::vector<Int2> xc(pairs.size());
    for (size_t q = 0; q < xc.size(); ++q) {
        xc[q].x = tr(pairs[q].x);
        xc[q].y = tr(pairs[q].y);
    }
    std::sort(xc.begin(), xc.end(), [](const Int2 &a, const Int2 &b) { return a.x < b.x; });
    return xc;
}

#ifdef __CUDACC__
inline void ghost_copy_tasks(const std::vector<int2> &pairs, std::vector<int4> &tasks, std::vector<int2> &single)
{
    ghost_copy_tasks_of<int2, int4>(pairs, tasks, single);
}
#endif
