// Geometry of the shared-memory bricks of the stage kernels (fast FP64 and
// FP32 forms), shared by the kernels and by the host code that encodes the
// TMA tensor maps.
//
// A block owns a tile of interfaces: T[s] interfaces along the sweep axis s
// (the first one is the left interface of the tile's first node, so the block
// updates T[s]-1 nodes per line) and T[t] lines along the transverse axes.
// Its brick is the tile's stencil region -- 3 nodes either side along s and,
// for viscous cases, one node either side along the transverse axes -- all
// five conservative variables of one time level, loaded by one 5-D TMA copy.
// The x origin of a brick is rounded down to an even node so that the copy
// starts on a 16-byte boundary; the x extent is padded accordingly.
#pragma once

namespace acfd {

template <int S, bool VISC>
struct Brick;

// X sweep: 32 interfaces along x, 4 lines in y, 2 in z (256 threads)
template <bool V>
struct Brick<0, V> {
    static constexpr int TX = 32, TY = 4, TZ = 2;
    static constexpr int BX = 38, BY = V ? 6 : 4, BZ = V ? 4 : 2;
    static constexpr int HX = 3, HY = V ? 1 : 0, HZ = V ? 1 : 0;  // halo before the tile origin
    static constexpr int SX = TX - 1, SY = TY, SZ = TZ;            // tile step in nodes
};

// Y sweep: 16 x-lines, 16 interfaces along y
template <bool V>
struct Brick<1, V> {
    static constexpr int TX = 16, TY = 16, TZ = 1;
    static constexpr int BX = V ? 20 : 18, BY = 21, BZ = V ? 3 : 1;
    static constexpr int HX = V ? 1 : 0, HY = 3, HZ = V ? 1 : 0;
    static constexpr int SX = TX, SY = TY - 1, SZ = TZ;
};

// Z sweep: 16 x-lines, 16 interfaces along z
template <bool V>
struct Brick<2, V> {
    static constexpr int TX = 16, TY = 1, TZ = 16;
    static constexpr int BX = V ? 20 : 18, BY = V ? 3 : 1, BZ = 21;
    static constexpr int HX = V ? 1 : 0, HY = V ? 1 : 0, HZ = 3;
    static constexpr int SX = TX, SY = TY, SZ = TZ - 1;
};

// box extents (x, y, z) of the tensor map of sweep s
inline void brick_box(int s, bool visc, int box[3])
{
#define ACFD_BOX(S_, V_)        \
    box[0] = Brick<S_, V_>::BX; \
    box[1] = Brick<S_, V_>::BY; \
    box[2] = Brick<S_, V_>::BZ;
    if (s == 0) {
        if (visc) { ACFD_BOX(0, true) } else { ACFD_BOX(0, false) }
    } else if (s == 1) {
        if (visc) { ACFD_BOX(1, true) } else { ACFD_BOX(1, false) }
    } else {
        if (visc) { ACFD_BOX(2, true) } else { ACFD_BOX(2, false) }
    }
#undef ACFD_BOX
}

}  // namespace acfd
