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

#ifdef __CUDACC__
inline void ghost_copy_tasks(const std::vector<int2> &pairs, std::vector<int4> &tasks, std::vector<int2> &single)
{
    ghost_copy_tasks_of<int2, int4>(pairs, tasks, single);
}
#endif
