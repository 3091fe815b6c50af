// Geometry of the shared-memory bricks of the stage kernels (fast FP64, FP32
// and hybrid forms), shared by the kernels and by the host code that encodes
// the TMA tensor maps.
//
// A block owns a tile of interfaces: T[s] interfaces along the sweep axis s
// (the first one is the left interface of the tile's first node, so the block
// updates T[s]-1 nodes per line) and T[t] lines along the transverse axes.
// Its brick is the tile's stencil region -- 3 nodes either side along s and,
// for viscous cases, one node either side along the transverse axes -- all
// five conservative variables of one time level, loaded by one 5-D TMA copy.
// The x origin of a brick is rounded down to an even node so that the copy
// starts on a 16-byte boundary; the x extent is padded accordingly.
//
// Each axis has kTileVariants tile shapes (VAR); acfd_autotune times them on
// the case and keeps the fastest.
#pragma once

namespace acfd {

constexpr int kTileVariants = 2;

template <int S, bool VISC, int VAR = 0>
struct Brick;

// X sweep: VAR 0: 32 interfaces along x x 4 (y) x 2 (z); VAR 1: 64 x 2 x 2
template <bool V, int VAR>
struct Brick<0, V, VAR> {
    static constexpr int TX = VAR ? 64 : 32, TY = VAR ? 2 : 4, TZ = 2;
    static constexpr int BX = TX + 6, BY = TY + (V ? 2 : 0), BZ = TZ + (V ? 2 : 0);
    static constexpr int HX = 3, HY = V ? 1 : 0, HZ = V ? 1 : 0;  // halo before the tile origin
    static constexpr int SX = TX - 1, SY = TY, SZ = TZ;            // tile step in nodes
};

// Y sweep: VAR 0: 16 x-lines x 16 interfaces along y; VAR 1: 32 x 8
template <bool V, int VAR>
struct Brick<1, V, VAR> {
    static constexpr int TX = VAR ? 32 : 16, TY = VAR ? 8 : 16, TZ = 1;
    static constexpr int BX = TX + (V ? 4 : 2), BY = TY + 5, BZ = V ? 3 : 1;
    static constexpr int HX = V ? 1 : 0, HY = 3, HZ = V ? 1 : 0;
    static constexpr int SX = TX, SY = TY - 1, SZ = TZ;
};

// Z sweep: VAR 0: 16 x-lines x 16 interfaces along z; VAR 1: 32 x 8
template <bool V, int VAR>
struct Brick<2, V, VAR> {
    static constexpr int TX = VAR ? 32 : 16, TY = 1, TZ = VAR ? 8 : 16;
    static constexpr int BX = TX + (V ? 4 : 2), BY = V ? 3 : 1, BZ = TZ + 5;
    static constexpr int HX = V ? 1 : 0, HY = V ? 1 : 0, HZ = 3;
    static constexpr int SX = TX, SY = TY, SZ = TZ - 1;
};

// Node-update box of a tile (persistent FP32 stage kernel): the nodes the
// tile updates, with x from the even node at or below the first one, read by
// one TMA copy of U[to] (or U[tm]); the x extent is even (16-byte rule).
template <int S, int VAR>
struct OBox;
template <int VAR>
struct OBox<0, VAR> {
    static constexpr int OX = Brick<0, false, VAR>::TX, OY = Brick<0, false, VAR>::TY, OZ = Brick<0, false, VAR>::TZ;
};
template <int VAR>
struct OBox<1, VAR> {
    static constexpr int OX = Brick<1, false, VAR>::TX + 2, OY = Brick<1, false, VAR>::TY - 1,
                         OZ = Brick<1, false, VAR>::TZ;
};
template <int VAR>
struct OBox<2, VAR> {
    static constexpr int OX = Brick<2, false, VAR>::TX + 2, OY = Brick<2, false, VAR>::TY,
                         OZ = Brick<2, false, VAR>::TZ - 1;
};

inline void update_box(int s, int var, int box[3])
{
#define ACFD_OBOX(S_, R_)           \
    box[0] = OBox<S_, R_>::OX;      \
    box[1] = OBox<S_, R_>::OY;      \
    box[2] = OBox<S_, R_>::OZ;
    if (s == 0) {
        if (var) { ACFD_OBOX(0, 1) } else { ACFD_OBOX(0, 0) }
    } else if (s == 1) {
        if (var) { ACFD_OBOX(1, 1) } else { ACFD_OBOX(1, 0) }
    } else {
        if (var) { ACFD_OBOX(2, 1) } else { ACFD_OBOX(2, 0) }
    }
#undef ACFD_OBOX
}

// tile steps (nodes updated per tile along x, y, z) of sweep s, variant var
inline void brick_step(int s, bool visc, int var, int st[3])
{
#define ACFD_STEP(S_, V_, R_)             \
    st[0] = Brick<S_, V_, R_>::SX;        \
    st[1] = Brick<S_, V_, R_>::SY;        \
    st[2] = Brick<S_, V_, R_>::SZ;
#define ACFD_STEP_V(S_, R_)                                   \
    if (visc) { ACFD_STEP(S_, true, R_) } else { ACFD_STEP(S_, false, R_) }
    if (s == 0) {
        if (var) { ACFD_STEP_V(0, 1) } else { ACFD_STEP_V(0, 0) }
    } else if (s == 1) {
        if (var) { ACFD_STEP_V(1, 1) } else { ACFD_STEP_V(1, 0) }
    } else {
        if (var) { ACFD_STEP_V(2, 1) } else { ACFD_STEP_V(2, 0) }
    }
#undef ACFD_STEP_V
#undef ACFD_STEP
}

// box extents (x, y, z) of the tensor map of sweep s, tile variant var
inline void brick_box(int s, bool visc, int var, int box[3])
{
#define ACFD_BOX(S_, V_, R_)            \
    box[0] = Brick<S_, V_, R_>::BX;     \
    box[1] = Brick<S_, V_, R_>::BY;     \
    box[2] = Brick<S_, V_, R_>::BZ;
#define ACFD_BOX_V(S_, R_)                                   \
    if (visc) { ACFD_BOX(S_, true, R_) } else { ACFD_BOX(S_, false, R_) }
    if (s == 0) {
        if (var) { ACFD_BOX_V(0, 1) } else { ACFD_BOX_V(0, 0) }
    } else if (s == 1) {
        if (var) { ACFD_BOX_V(1, 1) } else { ACFD_BOX_V(1, 0) }
    } else {
        if (var) { ACFD_BOX_V(2, 1) } else { ACFD_BOX_V(2, 0) }
    }
#undef ACFD_BOX_V
#undef ACFD_BOX
}

}  // namespace acfd
