// rap_stencil.cu -- the first coarsening step of a matrix assembled on the
// device (hmfem_assemble), computed from its known 7-point structure.
//
// For the TPFA stencil in natural order the reference's greedy C/F split
// (amg.h:1-32, 219-223) is the parity colouring: a cell is C iff i+j+k is
// even (every odd cell has a lower even neighbour, every even cell's lower
// neighbours are odd).  P then takes each F cell's neighbours (all C) with
// weight 1/degree, and the Galerkin row of a coarse cell c involves only c
// and its six F neighbours: the 19 coarse cells at offsets 0, +-2e_a and
// +-e_a+-e_b.  Each coarse row is formed here by one thread, adding every
// contribution in the same order sparse_multiply_transpose would
// (amg.h:520-546: A P in A-row order d,l,c,r,u,t,b, then P^T (A P) over
// fine rows in ascending order), without FMA contraction -- so the result
// is bit-identical to the generic Galerkin kernels (and to the reference),
// at a fraction of their cost.
#include "grid19.cuh"
#include "hm.cuh"

namespace hm {

namespace {

// storage order of a level-0 row (solve_linearsystem_AMG.c:103-139)
enum { DD = 0, DL, DC, DR, DU, DT, DB };

struct SG {
    int nx, ny, nz;
    long nxy;
};

__device__ __forceinline__ unsigned present(const SG &g, int i, int j, int k)
{
    return (unsigned)(j > 0) << DD | (unsigned)(i > 0) << DL | 1u << DC |
           (unsigned)(i < g.nx - 1) << DR | (unsigned)(j < g.ny - 1) << DU |
           (unsigned)(k < g.nz - 1) << DT | (unsigned)(k > 0) << DB;
}

// a_{s, s+dir} of row s (dir present)
__device__ __forceinline__ double aval(const int *__restrict__ rowptr,
                                       const double *__restrict__ val, long s,
                                       unsigned pm, int dir)
{
    return val[rowptr[s] + __popc(pm & ((1u << dir) - 1))];
}

// The same entries from the level-0 stencil form (Grid7, stencil_cycle.cu):
// a_cc and the +x, +y, +z couplings of each cell slice-interleaved; the -x
// coupling of s is the +x coupling of s - 1 and so on.  Setup extracts that
// form from the CSR values and checks the matrix bitwise symmetric, so every
// entry is the CSR value bit for bit -- without the row-pointer look-up in
// front of each load.
struct CsrA {
    const int *__restrict__ rowptr;
    const double *__restrict__ val;
    __device__ __forceinline__ double operator()(const SG &, long s, unsigned pm, int dir) const
    {
        return aval(rowptr, val, s, pm, dir);
    }
};
struct G7A {
    const double *__restrict__ cf;
    __device__ __forceinline__ double operator()(const SG &g, long s, unsigned, int dir) const
    {
        switch (dir) {
        case DC: return cf[slice_at(s, 0, 4)];
        case DR: return cf[slice_at(s, 1, 4)];
        case DL: return cf[slice_at(s - 1, 1, 4)];
        case DU: return cf[slice_at(s, 2, 4)];
        case DD: return cf[slice_at(s - g.nx, 2, 4)];
        case DT: return cf[slice_at(s, 3, 4)];
        default: return cf[slice_at(s - g.nxy, 3, 4)];
        }
    }
};

// The 19 coarse offsets of a level-1 row, by slot: 0, +-2e_x, +-2e_y,
// +-2e_z, then the 12 offsets +-e_a +- e_b.
__host__ __device__ constexpr int OX(int t)
{
    return t == 1 ? 2 : t == 2 ? -2 : (t == 7 || t == 8 || t == 11 || t == 12) ? 1
         : (t == 9 || t == 10 || t == 13 || t == 14) ? -1 : 0;
}
__host__ __device__ constexpr int OY(int t)
{
    return t == 3 ? 2 : t == 4 ? -2 : (t == 7 || t == 9 || t == 15 || t == 16) ? 1
         : (t == 8 || t == 10 || t == 17 || t == 18) ? -1 : 0;
}
__host__ __device__ constexpr int OZ(int t)
{
    return t == 5 ? 2 : t == 6 ? -2 : (t == 11 || t == 13 || t == 15 || t == 17) ? 1
         : (t == 12 || t == 14 || t == 16 || t == 18) ? -1 : 0;
}

// Per-grid slot table: the fine-index offset of each slot and, for each
// slot, the mask of slots with a smaller offset.  Two in-grid coarse
// neighbours never share an offset, so the rank of a present slot among the
// present ones, popc(present & less[slot]), is its position in the coarse
// row (columns ascend with fine index).
struct SGT {
    long lin[19];
    unsigned less[19];
};

SGT slot_table(const SG &g)
{
    SGT t;
    for (int a = 0; a < 19; a++)
        t.lin[a] = OX(a) + (long)OY(a) * g.nx + (long)OZ(a) * g.nxy;
    for (int a = 0; a < 19; a++) {
        t.less[a] = 0;
        for (int b = 0; b < 19; b++)
            if (t.lin[b] < t.lin[a] || (t.lin[b] == t.lin[a] && b < a)) t.less[a] |= 1u << b;
    }
    return t;
}

// mask of the slots whose coarse neighbour of even cell (i,j,k) is in grid
__device__ __forceinline__ unsigned in_grid(const SG &g, int i, int j, int k)
{
    unsigned m = 0;
#pragma unroll
    for (int t = 0; t < 19; t++) {
        const int a = i + OX(t), b = j + OY(t), c = k + OZ(t);
        m |= (unsigned)(a >= 0 && a < g.nx && b >= 0 && b < g.ny && c >= 0 && c < g.nz) << t;
    }
    return m;
}

// Threads walk the even cells only: (nx+1)/2 per x-row.
__device__ __forceinline__ bool even_cell(const SG &g, long t, int &i, int &j, int &k)
{
    const int hx = (g.nx + 1) >> 1;
    const long r = t / hx;
    j = (int)(r % g.ny);
    k = (int)(r / g.ny);
    i = 2 * (int)(t - r * hx) + ((j + k) & 1);
    return i < g.nx;
}

__global__ void k_parity(SG g, signed char *sel)
{
    const long n = g.nxy * g.nz;
    for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < n;
         s += (long)gridDim.x * blockDim.x) {
        const int i = (int)(s % g.nx), j = (int)((s / g.nx) % g.ny), k = (int)(s / g.nxy);
        sel[s] = ((i + j + k) & 1) == 0 ? 1 : 2;
    }
}

__global__ void k_sg_count(SG g, const int *__restrict__ cid, int *cnt)
{
    const long n = (long)((g.nx + 1) >> 1) * g.ny * g.nz;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
         t += (long)gridDim.x * blockDim.x) {
        int i, j, k;
        if (!even_cell(g, t, i, j, k)) continue;
        cnt[cid[i + (long)j * g.nx + (long)k * g.nxy]] = __popc(in_grid(g, i, j, k));
    }
}

__host__ __device__ constexpr int slot_of(int dx, int dy, int dz)
{
    return (dx == 0 && dy == 0 && dz == 0) ? 0
         : (dx == 2 && dy == 0 && dz == 0) ? 1 : (dx == -2 && dy == 0 && dz == 0) ? 2
         : (dx == 0 && dy == 2 && dz == 0) ? 3 : (dx == 0 && dy == -2 && dz == 0) ? 4
         : (dx == 0 && dy == 0 && dz == 2) ? 5 : (dx == 0 && dy == 0 && dz == -2) ? 6
         : (dx == 1 && dy == 1 && dz == 0) ? 7 : (dx == 1 && dy == -1 && dz == 0) ? 8
         : (dx == -1 && dy == 1 && dz == 0) ? 9 : (dx == -1 && dy == -1 && dz == 0) ? 10
         : (dx == 1 && dy == 0 && dz == 1) ? 11 : (dx == 1 && dy == 0 && dz == -1) ? 12
         : (dx == -1 && dy == 0 && dz == 1) ? 13 : (dx == -1 && dy == 0 && dz == -1) ? 14
         : (dx == 0 && dy == 1 && dz == 1) ? 15 : (dx == 0 && dy == 1 && dz == -1) ? 16
         : (dx == 0 && dy == -1 && dz == 1) ? 17 : (dx == 0 && dy == -1 && dz == -1) ? 18
         : -1;
}

__host__ __device__ constexpr int DX(int d) { return d == DL ? -1 : d == DR ? 1 : 0; }
__host__ __device__ constexpr int DY(int d) { return d == DD ? -1 : d == DU ? 1 : 0; }
__host__ __device__ constexpr int DZ(int d) { return d == DB ? -1 : d == DT ? 1 : 0; }

// acc[slot] += t in order; the first contribution initialises the slot
#define SG_ADD(slot, t)                                                        \
    do {                                                                       \
        const double t_ = (t);                                                 \
        if (hv & (1u << (slot))) acc[slot] = dadd(acc[slot], t_);              \
        else { acc[slot] = t_; hv |= 1u << (slot); }                           \
    } while (0)

// One coarse row c: Ac[c][q] = sum over the fine rows f of R(c) in ascending
// index order {c-nxy, c-nx, c-1, c, c+1, c+nx, c+nxy} of AP[f][q] * w_f,
// where
//   AP[c][q] = sum over c's row in stored order (d,l,c,r,u,t,b) of
//              a_cj * w_j for each F neighbour j adjacent to q, and a_cc for
//              q = c;
//   AP[f][q] = a_fq + a_ff * w_f for an F neighbour f and each of its C
//              neighbours q (a sum of two terms, so its order is free).
// Slots are numbered as in OX/OY/OZ; every index below is a compile-time
// constant once the direction loops are unrolled, so acc stays in
// registers.
template <class AV>
__global__ void __launch_bounds__(128)
k_sg_fill(SG g, const SGT tb, AV aval, const double *__restrict__ pw,
          const int *__restrict__ cid, const int *__restrict__ crow, int *ccol,
          double *cval, double *g19v, long nc)
{
    const long n = (long)((g.nx + 1) >> 1) * g.ny * g.nz;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
         t += (long)gridDim.x * blockDim.x) {
        int i, j, k;
        if (!even_cell(g, t, i, j, k)) continue;
        const long s = i + (long)j * g.nx + (long)k * g.nxy;
        const unsigned pmc = present(g, i, j, k);
        // ---- AP[c][.], in c's row order
        double ap[19];
        unsigned hv = 0;
        double *acc = ap;
        const int adir[7] = {DD, DL, DC, DR, DU, DT, DB};
#pragma unroll
        for (int aa = 0; aa < 7; aa++) {
            const int e = adir[aa];
            if (!(pmc & (1u << e))) continue;
            const double a_ce = aval(g, s, pmc, e);
            if (e == DC) {
                SG_ADD(0, a_ce);
                continue;
            }
            const long f = s + DX(e) + (long)DY(e) * g.nx + (long)DZ(e) * g.nxy;
            const double t = dmul(a_ce, pw[f]);
            // the C neighbours of f = c + e: c, c + 2e, c + e +- (perpendicular)
#pragma unroll
            for (int b2 = 0; b2 < 7; b2++) {
                if (b2 == DC) continue;
                const int qx = DX(e) + DX(b2), qy = DY(e) + DY(b2), qz = DZ(e) + DZ(b2);
                const int sl = slot_of(qx, qy, qz);
                if (sl < 0) continue;
                if (!(present(g, i + DX(e), j + DY(e), k + DZ(e)) & (1u << b2))) continue;
                SG_ADD(sl, t);
            }
        }
        const unsigned hap = hv;
        // ---- P^T (A P): fine rows of R(c) in ascending order
        double out[19];
        hv = 0;
        acc = out;
        const int rdir[7] = {DB, DD, DL, DC, DR, DU, DT};
#pragma unroll
        for (int rr = 0; rr < 7; rr++) {
            const int d = rdir[rr];
            if (!(pmc & (1u << d))) continue;
            if (d == DC) {
#pragma unroll
                for (int sl = 0; sl < 19; sl++)
                    if (hap & (1u << sl)) SG_ADD(sl, ap[sl]);  // * w_c = 1
                continue;
            }
            const long f = s + DX(d) + (long)DY(d) * g.nx + (long)DZ(d) * g.nxy;
            const unsigned pmf = present(g, i + DX(d), j + DY(d), k + DZ(d));
            const double wf = pw[f];
            const double dg = dmul(aval(g, f, pmf, DC), wf);
#pragma unroll
            for (int b2 = 0; b2 < 7; b2++) {
                if (b2 == DC || !(pmf & (1u << b2))) continue;
                const int sl = slot_of(DX(d) + DX(b2), DY(d) + DY(b2), DZ(d) + DZ(b2));
                if (sl < 0) continue;
                SG_ADD(sl, dmul(dadd(aval(g, f, pmf, b2), dg), wf));
            }
        }
        // ---- emit in coarse-id order (ascending fine index)
        const unsigned in = in_grid(g, i, j, k);
        const int c = cid[s];
        const long o = crow[c];
#pragma unroll
        for (int sl = 0; sl < 19; sl++) {
            const bool on = in & (1u << sl);
            if (g19v) g19v[slice_at(c, q19_of(OX(sl), OY(sl), OZ(sl)), kQ19)] = on ? out[sl] : 0.0;
            if (!on) continue;
            const long e = o + __popc(in & tb.less[sl]);
            ccol[e] = cid[s + tb.lin[sl]];
            cval[e] = out[sl];
        }
    }
}

// Level 1 of the exact red-black reduction (hmfem_options.schur0): the
// Schur complement S = A_CC - A_CF A_FF^-1 A_FC of the parity split, which
// is P^T A P for the interpolation P_F = -A_FF^-1 A_FC, P_C = I (the F
// equations solved exactly for given C values).  Same rows, columns and
// slot layout as k_sg_fill.  Values, evaluated in this order without FMA
// contraction: diagonal a_cc, minus (a_cf a_cf) / a_ff for each neighbour
// f of c in row order d,l,r,u,t,b; slot q: minus the sum, in that order of
// f and then of f's row order, of (a_cf a_fq) / a_ff over the F cells f
// adjacent to both c and q.  AV reads level 0's entries (CsrA, or G7A
// from the stencil form: the same values).
template <class AV>
__global__ void __launch_bounds__(128)
k_schur_fill(SG g, const SGT tb, AV aval, const int *__restrict__ cid,
             const int *__restrict__ crow, int *ccol, double *cval, double *g19v)
{
    const long n = (long)((g.nx + 1) >> 1) * g.ny * g.nz;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
         t += (long)gridDim.x * blockDim.x) {
        int i, j, k;
        if (!even_cell(g, t, i, j, k)) continue;
        const long s = i + (long)j * g.nx + (long)k * g.nxy;
        const unsigned pmc = present(g, i, j, k);
        double out[19];
        unsigned hv = 0;
        double *acc = out;
        double dsum = aval(g, s, pmc, DC);
        const int adir[6] = {DD, DL, DR, DU, DT, DB};
#pragma unroll
        for (int aa = 0; aa < 6; aa++) {
            const int e = adir[aa];
            if (!(pmc & (1u << e))) continue;
            const double a_ce = aval(g, s, pmc, e);
            const long f = s + DX(e) + (long)DY(e) * g.nx + (long)DZ(e) * g.nxy;
            const unsigned pmf = present(g, i + DX(e), j + DY(e), k + DZ(e));
            const double a_ff = aval(g, f, pmf, DC);
            dsum = dsub(dsum, dmul(a_ce, a_ce) / a_ff);
#pragma unroll
            for (int b2 = 0; b2 < 7; b2++) {
                if (b2 == DC || !(pmf & (1u << b2))) continue;
                const int sl = slot_of(DX(e) + DX(b2), DY(e) + DY(b2), DZ(e) + DZ(b2));
                if (sl <= 0) continue;  // back to c (its diagonal is above)
                SG_ADD(sl, dmul(a_ce, aval(g, f, pmf, b2)) / a_ff);
            }
        }
        out[0] = dsum;
        hv |= 1u;
#pragma unroll
        for (int sl = 1; sl < 19; sl++) out[sl] = -out[sl];
        const unsigned in = in_grid(g, i, j, k);
        const int c = cid[s];
        const long o = crow[c];
#pragma unroll
        for (int sl = 0; sl < 19; sl++) {
            const bool on = in & (1u << sl);
            if (g19v) g19v[slice_at(c, q19_of(OX(sl), OY(sl), OZ(sl)), kQ19)] = on ? out[sl] : 0.0;
            if (!on) continue;
            const long e = o + __popc(in & tb.less[sl]);
            ccol[e] = cid[s + tb.lin[sl]];
            cval[e] = out[sl];
        }
    }
}

// R = P^T of the parity split in closed form: coarse row c (C cell s) holds
// s and its in-grid neighbours (all F, all interpolating from s), fine rows
// ascending -- what the stable sort of P's coarse ids gives.
__global__ void k_parity_rcount(SG g, const int *__restrict__ cid, int *cnt)
{
    const long n = (long)((g.nx + 1) >> 1) * g.ny * g.nz;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
         t += (long)gridDim.x * blockDim.x) {
        int i, j, k;
        if (!even_cell(g, t, i, j, k)) continue;
        cnt[cid[i + (long)j * g.nx + (long)k * g.nxy]] = __popc(present(g, i, j, k));
    }
}

__global__ void k_parity_rfill(SG g, const int *__restrict__ cid,
                               const int *__restrict__ rrow, int *rcol)
{
    const long n = (long)((g.nx + 1) >> 1) * g.ny * g.nz;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
         t += (long)gridDim.x * blockDim.x) {
        int i, j, k;
        if (!even_cell(g, t, i, j, k)) continue;
        const long s = i + (long)j * g.nx + (long)k * g.nxy;
        const unsigned pm = present(g, i, j, k);
        long o = rrow[cid[s]];
        // ascending fine index: b, d, l, c, r, u, t
        const int order[7] = {DB, DD, DL, DC, DR, DU, DT};
#pragma unroll
        for (int q = 0; q < 7; q++) {
            const int d = order[q];
            if (pm & (1u << d)) rcol[o++] = (int)(s + DX(d) + (long)DY(d) * g.nx + (long)DZ(d) * g.nxy);
        }
    }
}

constexpr bool slots_consistent()
{
    for (int t = 0; t < 19; t++)
        if (slot_of(OX(t), OY(t), OZ(t)) != t) return false;
    return true;
}
static_assert(slots_consistent(), "slot numbering");

int nbk(long n)
{
    long b = ceil_div(n, 256);
    if (b < 1) b = 1;
    return (int)(b < 148L * 16 ? b : 148L * 16);
}

// ---- the C/F split of level 1 from its 19-offset structure ---------------
//
// The reference's greedy split (amg.h:1-32, node_selection in natural
// order, strength all-true at eps = 0) makes a node C iff none of its
// lower-numbered neighbours is C.  On level 1 (even cells, coarse id
// s >> 1 for nx even) the lower neighbours of the even cell (i,j,k) are the
// offsets q19 = 0..8: (0,0,-2), (0,-1,-1), (-1,0,-1), (1,0,-1), (0,1,-1),
// (0,-2,0), (-1,-1,0), (1,-1,0) -- in the x-rows (j,k-2), (j-1,k-1),
// (j,k-1), (j+1,k-1), (j-2,k), (j-1,k) -- and (-2,0,0), the previous cell of
// the same x-row.  So an x-row depends only on rows with a smaller
// t = j + 2k.  Inside a row, with "blocked" = some lower neighbour in
// another row is C, the row recurrence C_b = !blocked_b && !C_{b-1} makes
// every run of unblocked cells alternate C, F, C, ... from its first cell
// (or from the carried state of the previous 32-cell chunk).
//
// One launch for the whole wavefront: warps take x-rows from a ticket in
// (t, k) order and resolve them 32 cells (one chunk) at a time.  A row
// publishes each chunk as one 64-bit word, its C bits in the low half and a
// valid bit above them (an aligned 64-bit store is seen whole or not at
// all), so a reader needs no flag, fence or second load: lanes 0-17 poll
// the words c-1, c, c+1 of the six rows below (bounded waits) and every
// lane picks its neighbours' bits from them.  Those rows have smaller t,
// so earlier tickets, held by warps that are already running: every wait
// ends.  Chunk c of a row waits only for chunk c+1 of the rows before it,
// so consecutive rows of the wavefront overlap chunk by chunk.

constexpr int kWaveThreads = 128;
// 256 warps cover the wavefront's width at 256^3 (alone: 1.3 ms for its 766
// diagonals) and leave most SMs to the level-0 kernels it runs beside; one
// CTA on every SM slowed those 1.4x (setup 24.4 against 23.5 ms at 256^3)
constexpr int kWaveBlocks = 64;

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// x-rows (j, k) of an ny x nz plane with j + 2k < t
__host__ __device__ __forceinline__ long long rows_before(long long t, int ny, int nz)
{
    if (t <= 0) return 0;
    long long kf = t >= ny ? (t - ny) / 2 + 1 : 0;  // rows with t - 2k >= ny: all ny
    long long kp = (t + 1) / 2;                     // rows with t - 2k > 0
    if (kf > nz) kf = nz;
    if (kp > nz) kp = nz;
    return (long long)ny * kf + (kp - kf) * t - (kp - kf) * (kf + kp - 1);
}

// words: [ny * nz rows][W chunks] (W = chunks of nx / 2 cells), zero on entry
__global__ void __launch_bounds__(kWaveThreads)
k_mis19_wave(SG g, signed char *sel, unsigned long long *words, int W, unsigned *ticket,
             int *err, long long max_polls)
{
    const unsigned full = 0xffffffffu;
    const unsigned long long valid = 1ull << 32;
    const int lane = threadIdx.x & 31;
    const unsigned rows = (unsigned)g.ny * (unsigned)g.nz;
    const long long tmax = (g.ny - 1) + 2LL * (g.nz - 1);
    const int m = g.nx >> 1;  // cells of every x-row of level 1 (nx even)
    volatile int *verr = err;
    // lane L < 18 watches word c + (L % 3) - 1 of row L / 3: (j,k-2),
    // (j-1,k-1), (j,k-1), (j+1,k-1), (j-2,k), (j-1,k)
    const int ri = lane / 3, wo = lane % 3 - 1;
    const int dj = ri == 1 || ri == 5 ? -1 : ri == 3 ? 1 : ri == 4 ? -2 : 0;
    const int dk = ri == 0 ? -2 : ri <= 3 ? -1 : 0;
    for (;;) {
        unsigned tk = 0;
        if (lane == 0) tk = atomicAdd(ticket, 1u);
        tk = __shfl_sync(full, tk, 0);
        if (tk >= rows) return;
        long long lo = 0, hi = tmax;  // the largest t with rows_before(t) <= tk
        while (lo < hi) {
            const long long mid = (lo + hi + 1) >> 1;
            if (rows_before(mid, g.ny, g.nz) <= (long long)tk) lo = mid;
            else hi = mid - 1;
        }
        const int t = (int)lo;
        const int kmin = t > g.ny - 1 ? (t - g.ny + 2) / 2 : 0;
        const int k = kmin + (int)((long long)tk - rows_before(t, g.ny, g.nz));
        const int j = t - 2 * k;
        const int p = (j + k) & 1;
        // the x-neighbours -1 / +1 of cell b sit at bit b + dm / b + dp of
        // the rows of the other parity
        const int dm = p == 0 ? -1 : 0, dp = p == 0 ? 0 : 1;
        const int jj = j + dj, kk = k + dk;
        const bool row_in = lane < 18 && jj >= 0 && jj < g.ny && kk >= 0 && kk < g.nz;
        const unsigned long long *nrow = words + (row_in ? ((long)jj + (long)g.ny * kk) * W : 0);
        unsigned long long *own = words + ((long)j + (long)g.ny * k) * W;
        const long rowbase = (long)j * g.nx + (long)k * g.nxy;
        bool prev_c = false;
        for (int c = 0; c < W; c++) {
            const int w = c + wo;
            const bool need = row_in && w >= 0 && w < W;
            unsigned long long v = 0;
            long long polls = 0;
            for (;;) {
                if (need && !(v & valid)) v = ld_relaxed_u64(nrow + w);
                if (__all_sync(full, !need || (v & valid))) break;
                if (__any_sync(full, ++polls > max_polls || *verr != 0)) {
                    if (lane == 0) atomicExch(err, 1);
                    return;  // the whole warp: the rest of its row stays unpublished
                }
                __nanosleep(polls > 8 ? 128 : 16);
            }
            unsigned x[18];
#pragma unroll
            for (int q = 0; q < 18; q++) x[q] = __shfl_sync(full, (unsigned)v, q);
            auto bit = [&](int r, int d) -> bool {
                const int pos = lane + d;
                return pos < 0 ? (x[3 * r] >> 31) & 1u
                     : pos > 31 ? x[3 * r + 2] & 1u : (x[3 * r + 1] >> pos) & 1u;
            };
            const int b = 32 * c + lane;
            const bool blocked = b >= m || bit(0, 0) || bit(1, 0) || bit(2, dm) || bit(2, dp) ||
                                 bit(3, 0) || bit(4, 0) || bit(5, dm) || bit(5, dp);
            const unsigned B = __ballot_sync(full, blocked);
            const unsigned lower = B & ((1u << lane) - 1u);
            bool is_c;
            if (lower) is_c = !blocked && (((lane - (31 - __clz(lower)) - 1) & 1) == 0);
            else is_c = !blocked && ((lane & 1) == (prev_c ? 1 : 0));
            const unsigned cm = __ballot_sync(full, is_c);
            if (lane == 0) st_relaxed_u64(own + c, valid | cm);
            if (b < m) sel[(rowbase + p + 2 * b) >> 1] = is_c ? 1 : 2;
            prev_c = (cm >> 31) & 1u;
        }
    }
}

}  // namespace

// work: the rows' chunk words (two ints each), then the ticket and the
// error word
static long wave_chunks(int nx) { return ((long)(nx >> 1) + 31) >> 5; }

long stencil19_split_work_ints(int nx, int ny, int nz)
{
    return 2 * (long)ny * nz * wave_chunks(nx) + 2;
}

int stencil19_split(int nx, int ny, int nz, signed char *sel, int *work, cudaStream_t st)
{
    SG g{nx, ny, nz, (long)nx * ny};
    const long rows = (long)ny * nz;
    if (rows <= 0 || nx < 2) return HMFEM_OK;
    if (rows > 0x7fffffffL || (nx & 1)) {
        set_last_error("level-1 split: needs an even nx and fewer than 2^31 x-rows",
                       __FILE__, __LINE__);
        return HMFEM_E_CAPACITY;
    }
    const long wi = stencil19_split_work_ints(nx, ny, nz);
    HM_CUDA(cudaMemsetAsync(work, 0, sizeof(int) * wi, st));
    const long warps = kWaveThreads / 32;
    long blocks = (rows + warps - 1) / warps;
    if (blocks > kWaveBlocks) blocks = kWaveBlocks;
    k_mis19_wave<<<(int)blocks, kWaveThreads, 0, st>>>(
        g, sel, (unsigned long long *)work, (int)wave_chunks(nx), (unsigned *)(work + wi - 2),
        work + wi - 1, split_poll_limit());
    HM_LAUNCHED();
    return HMFEM_OK;
}

int stencil_parity_split(int nx, int ny, int nz, signed char *sel, cudaStream_t st)
{
    SG g{nx, ny, nz, (long)nx * ny};
    k_parity<<<nbk(g.nxy * nz), 256, 0, st>>>(g, sel);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int stencil_galerkin(int nx, int ny, int nz, const Level &L, Csr &out,
                     double *g19v, cudaStream_t st, bool schur)
{
    SG g{nx, ny, nz, (long)nx * ny};
    const long n = g.nxy * nz;
    out.n = L.nc;
    out.rowptr = (int *)dalloc(sizeof(int) * (L.nc + 1));
    if (!out.rowptr) return HMFEM_E_CUDA;
    k_sg_count<<<nbk(n / 2), 256, 0, st>>>(g, L.cid, out.rowptr);
    HM_LAUNCHED();
    HM_CHECK(rowptr_from_counts(out.rowptr, L.nc, st, &out.nnz));
    out.col = (int *)dalloc(sizeof(int) * (out.nnz > 0 ? out.nnz : 1));
    out.val = (double *)dalloc(sizeof(double) * (out.nnz > 0 ? out.nnz : 1));
    if (!out.col || !out.val) return HMFEM_E_CUDA;
    if (schur && L.g7.cf)
        k_schur_fill<<<nbk(n / 2), 128, 0, st>>>(g, slot_table(g), G7A{L.g7.cf}, L.cid,
                                                 out.rowptr, out.col, out.val, g19v);
    else if (schur)
        k_schur_fill<<<nbk(n / 2), 128, 0, st>>>(g, slot_table(g), CsrA{L.A.rowptr, L.A.val},
                                                 L.cid, out.rowptr, out.col, out.val, g19v);
    else
    {
        if (L.g7.cf)
            k_sg_fill<<<nbk(n / 2), 128, 0, st>>>(g, slot_table(g), G7A{L.g7.cf}, L.pw, L.cid,
                                                  out.rowptr, out.col, out.val, g19v,
                                                  (long)L.nc);
        else
            k_sg_fill<<<nbk(n / 2), 128, 0, st>>>(g, slot_table(g), CsrA{L.A.rowptr, L.A.val},
                                                  L.pw, L.cid, out.rowptr, out.col, out.val,
                                                  g19v, (long)L.nc);
    }
    HM_LAUNCHED();
    return HMFEM_OK;
}

int stencil_parity_R(int nx, int ny, int nz, const int *cid, int nc, Csr &R, cudaStream_t st)
{
    SG g{nx, ny, nz, (long)nx * ny};
    const long n = g.nxy * nz;
    R.n = nc;
    HM_CUDA(cudaMemsetAsync(R.rowptr, 0, sizeof(int) * ((long)nc + 1), st));
    k_parity_rcount<<<nbk(n / 2), 256, 0, st>>>(g, cid, R.rowptr);
    HM_LAUNCHED();
    long nnz = 0;
    HM_CHECK(rowptr_from_counts(R.rowptr, nc, st, &nnz));
    if (nnz != R.nnz) {
        set_last_error("parity split: R size differs from P", __FILE__, __LINE__);
        return HMFEM_E_CAPACITY;
    }
    k_parity_rfill<<<nbk(n / 2), 256, 0, st>>>(g, cid, R.rowptr, R.col);
    HM_LAUNCHED();
    return HMFEM_OK;
}

}  // namespace hm
