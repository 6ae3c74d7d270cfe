// grid19.cuh -- the coarse offsets of the level-1 operator of a parity-split
// 7-point grid, in the order a coarse row stores them.
//
// Level 0's C cells are the even cells (i+j+k even); the Galerkin row of an
// even cell couples it to the even cells at offsets 0, +-2e_a and
// +-e_a+-e_b.  Rows keep their columns in ascending coarse id = ascending
// fine index; for nx >= 4 and ny >= 4 that order of the 19 offsets is the
// same for every cell, and q19 numbers them in it.
#pragma once

namespace hm {

constexpr int kQ19 = 19;

__host__ __device__ constexpr int q19x(int q)
{
    return (q == 2 || q == 6 || q == 11 || q == 15) ? -1
         : (q == 3 || q == 7 || q == 12 || q == 16) ? 1
         : q == 8 ? -2 : q == 10 ? 2 : 0;
}
__host__ __device__ constexpr int q19y(int q)
{
    return (q == 1 || q == 6 || q == 7 || q == 14) ? -1
         : (q == 4 || q == 11 || q == 12 || q == 17) ? 1
         : q == 5 ? -2 : q == 13 ? 2 : 0;
}
__host__ __device__ constexpr int q19z(int q)
{
    return q == 0 ? -2 : q == 18 ? 2 : (q >= 1 && q <= 4) ? -1 : (q >= 14 && q <= 17) ? 1 : 0;
}

// the q of offset (dx, dy, dz), or -1
__host__ __device__ constexpr int q19_of(int dx, int dy, int dz)
{
    int r = -1;
    for (int q = 0; q < kQ19; q++)
        if (q19x(q) == dx && q19y(q) == dy && q19z(q) == dz) r = q;
    return r;
}

// fine-index offset of q on an nx * ny grid
__host__ __device__ constexpr long q19_lin(int q, long nx, long nxy)
{
    return q19x(q) + q19y(q) * nx + q19z(q) * nxy;
}

constexpr bool q19_ascending(long nx, long ny)
{
    for (int q = 1; q < kQ19; q++)
        if (!(q19_lin(q - 1, nx, nx * ny) < q19_lin(q, nx, nx * ny))) return false;
    return true;
}
static_assert(q19_ascending(4, 4) && q19_ascending(256, 256) && q19_ascending(4, 1000) &&
                  q19_ascending(1000, 4),
              "q19 order");
static_assert(q19_of(0, 0, 0) == 9, "q19 centre");

}  // namespace hm
