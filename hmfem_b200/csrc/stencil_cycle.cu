// stencil_cycle.cu -- solve-phase kernels for the two finest levels of a
// matrix assembled on the device, stored by their grid structure instead of
// SELL-32, so no column index is read.
//
// Level 0 is the 7-point TPFA stencil: per cell a_cc and the couplings to
// the +x, +y, +z neighbours; the coupling to -x is the -x neighbour's +x
// one, and so on.  That needs the assembled matrix to be bitwise symmetric
// (hm(a,b) = 2ab/(a+b) is, and every pair is checked before this form is
// used).  A row costs 4 coefficients instead of 7 values + 7 column
// indices.  Level 1 -- the Galerkin operator of the parity split -- couples
// each even cell to the even cells at the 19 offsets of grid19.cuh; with nx
// even the even cell s has coarse id s >> 1, so the 19 coefficients of a
// row sit in 19 unit-stride arrays.
//
// Every row is summed in the CSR's column order (level 0: d,l,c,r,u,t,b as
// solve_linearsystem_AMG.c:103-139 packs it; level 1: ascending), with the
// operations of the SELL kernels, so FP64 results are bit-identical to
// them; the level-0 transfers follow the parity split's P and R rows
// (C rows: the cell itself; F rows: the six neighbours, in row order).
#include "cycle.cuh"
#include "grid19.cuh"

namespace hm {

namespace {

// (i, j, k) of cell s
__device__ __forceinline__ void cell_ijk(unsigned s, unsigned nx, unsigned ny, int &i,
                                         int &j, int &k)
{
    const unsigned r = s / nx;
    i = (int)(s - r * nx);
    k = (int)(r / ny);
    j = (int)(r - (unsigned)k * ny);
}

template <class V> struct G7v {
    const V *cf;  // slice-interleaved: a_cc, +x, +y, +z
    int nx, ny, nz;
};

// t -/+ sum over row s of a_sj x(j), in the order d,l,c,r,u,t,b
template <class T, bool SUB, class V, class X>
__device__ __forceinline__ T g7_row(T t, const G7v<V> &g, long s, int i, int j, int k,
                                    X x)
{
    using A = Ar<T>;
    const long nx = g.nx, nxy = (long)g.nx * g.ny;
    const bool hd = j > 0, hl = i > 0, hr = i < g.nx - 1, hu = j < g.ny - 1,
               ht = k < g.nz - 1, hb = k > 0;
    // all loads first, so they overlap
    const T ad = hd ? (T)ld(g.cf, slice_at(s - nx, 2, 4)) : (T)0, xd = hd ? x(s - nx) : (T)0;
    const T al = hl ? (T)ld(g.cf, slice_at(s - 1, 1, 4)) : (T)0, xl = hl ? x(s - 1) : (T)0;
    const T ac = (T)ld(g.cf, slice_at(s, 0, 4)), xc = x(s);
    const T ar = hr ? (T)ld(g.cf, slice_at(s, 1, 4)) : (T)0, xr = hr ? x(s + 1) : (T)0;
    const T au = hu ? (T)ld(g.cf, slice_at(s, 2, 4)) : (T)0, xu = hu ? x(s + nx) : (T)0;
    const T at = ht ? (T)ld(g.cf, slice_at(s, 3, 4)) : (T)0, xt = ht ? x(s + nxy) : (T)0;
    const T ab = hb ? (T)ld(g.cf, slice_at(s - nxy, 3, 4)) : (T)0, xb = hb ? x(s - nxy) : (T)0;
    auto acc = [&](T a, T xv) {
        const T p = A::mul(a, xv);
        t = SUB ? A::sub(t, p) : A::add(t, p);
    };
    if (hd) acc(ad, xd);
    if (hl) acc(al, xl);
    acc(ac, xc);
    if (hr) acc(ar, xr);
    if (hu) acc(au, xu);
    if (ht) acc(at, xt);
    if (hb) acc(ab, xb);
    return t;
}

// number of neighbours of cell (i,j,k) = the P-row length of an F cell
__device__ __forceinline__ int g7_degree(int i, int j, int k, int nx, int ny, int nz)
{
    return (j > 0) + (i > 0) + (i < nx - 1) + (j < ny - 1) + (k < nz - 1) + (k > 0);
}

template <class V> struct G19v {
    const V *v;   // slice-interleaved, 19 per row
    int n;        // coarse rows
    int nx, ny, nz;
    // coarse row c = (x-pair, j, k) by multiplication: c / (nx/2) and
    // row / ny as __umul64hi(., m) with m = floor(2^64 / d) + 1 (exact for
    // 32-bit operands and 2 <= d < 2^32)
    unsigned long long mhx, mny;
    // coarse id of neighbour q: c + dq[parity][q] (the fine cell of c is
    // s = 2c + parity, parity = (j + k) & 1, and (s + off_q) >> 1 =
    // c + ((parity + off_q) >> 1))
    int dq[2][kQ19];
};

// t -/+ sum over level-1 row c of a_cq x(q), ascending q.  No bounds test:
// the coefficient of a neighbour outside the grid is stored as +0, and its
// x index is clamped into the vector, so it adds t -/+ 0 * x = t (x finite;
// the SELL kernels' zero padding behaves the same).  Entries are loaded in
// chunks (five in FP64, ten in FP32: two rounds of gathers) so the gathers
// overlap without holding all 19 in registers; the summation order is
// unchanged.
// BF16 coefficients of level 1 are stored four per 8-byte word: in slice t
// (rows 32t..32t+31), word j of row 32t + l holds coefficients 4j..4j+3 at
// ((5t + j) * 32 + l) (coefficient 19 is a zero pad), so a row's 19
// coefficients are five 8-byte loads, all issued before the gathers.
constexpr int kG19Words = 5;
__host__ __device__ __forceinline__ long long g19q_len(long long n)
{
    return ((n + 31) >> 5) * (long long)kG19Words * 32 * 4;
}

template <class T, bool SUB, class V, class X>
__device__ __forceinline__ T g19_row(T t, const G19v<V> &g, int c, X x)
{
    using A = Ar<T>;
    constexpr int CH = sizeof(T) == 8 ? 5 : 10;
    constexpr bool Q4 = std::is_same<V, __nv_bfloat16>::value;
    const unsigned cu = (unsigned)c;
    const unsigned row = (unsigned)__umul64hi(cu, g.mhx);
    const unsigned k = (unsigned)__umul64hi(row, g.mny), j = row - k * (unsigned)g.ny;
    const bool odd = ((j + k) & 1) != 0;
    const int last = g.n - 1;
    uint2 wq[kG19Words];
    if constexpr (Q4) {
        const uint2 *w = reinterpret_cast<const uint2 *>(g.v) +
                         (long long)(cu >> 5) * (kG19Words * 32) + (cu & 31);
#pragma unroll
        for (int jw = 0; jw < kG19Words; jw++) wq[jw] = __ldg(w + jw * 32);
    }
#pragma unroll
    for (int q0 = 0; q0 < kQ19; q0 += CH) {
        T a[CH], xv[CH];
#pragma unroll
        for (int d = 0; d < CH; d++) {
            const int q = q0 + d;
            if (q < kQ19) {
                if constexpr (Q4) {
                    // BF16 -> FP32 exactly (the bits of the upper half)
                    const unsigned wv = (q & 2) ? wq[q >> 2].y : wq[q >> 2].x;
                    a[d] = (T)__uint_as_float((q & 1) ? (wv & 0xffff0000u) : (wv << 16));
                } else {
                    a[d] = (T)ld(g.v, slice_at(c, q, kQ19));
                }
                int e = c + (odd ? g.dq[1][q] : g.dq[0][q]);
                e = e < 0 ? 0 : (e > last ? last : e);
                xv[d] = x(e);
            }
        }
#pragma unroll
        for (int d = 0; d < CH; d++) {
            if (q0 + d < kQ19) {
                const T p = A::mul(a[d], xv[d]);
                t = SUB ? A::sub(t, p) : A::add(t, p);
            }
        }
    }
    return t;
}

// ---- level 0 ------------------------------------------------------------

// r = f - A u (u the seeded first Jacobi iterate);  rs = r / |P row|
// (k_pre on the stencil)
template <class T, class V>
__global__ void __launch_bounds__(256)
k_g7_pre(G7v<V> g, int n, const T *__restrict__ f, const T *__restrict__ u,
         T *__restrict__ rs, const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    using A = Ar<T>;
    GRID_STRIDE(s, n) {
        int i, j, k;
        cell_ijk((unsigned)s, g.nx, g.ny, i, j, k);
        const T t = g7_row<T, true>(f[s], g, s, i, j, k, [&](long c) { return u[c]; });
        const int pc = ((i + j + k) & 1) ? g7_degree(i, j, k, g.nx, g.ny, g.nz) : 1;
        rs[s] = pc == 1 ? t : A::div(t, (T)pc);
    }
}

// f_c = sum over R(c) of rs, fine rows ascending: b, d, l, c, r, u, t
template <class T>
__global__ void __launch_bounds__(256)
k_g7_restrict(int nx, int ny, int nz, const int *__restrict__ cid,
              const T *__restrict__ rs, T *__restrict__ fc, Seed<T> sd, const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    using A = Ar<T>;
    const unsigned hx = (unsigned)(nx + 1) >> 1;
    const long nxy = (long)nx * ny, m = (long)hx * ny * nz;
    GRID_STRIDE(t, m) {
        const unsigned tu = (unsigned)t, r = tu / hx, kk0 = r / (unsigned)ny;
        const int j = (int)(r - kk0 * (unsigned)ny), k = (int)kk0;
        const int i = 2 * (int)(tu - r * hx) + ((j + k) & 1);
        if (i >= nx) continue;
        const long s = i + (long)r * nx;
        const T vb = k > 0 ? rs[s - nxy] : (T)0, vd = j > 0 ? rs[s - nx] : (T)0;
        const T vl = i > 0 ? rs[s - 1] : (T)0, vc = rs[s];
        const T vr = i < nx - 1 ? rs[s + 1] : (T)0, vu = j < ny - 1 ? rs[s + nx] : (T)0;
        const T vt = k < nz - 1 ? rs[s + nxy] : (T)0;
        T acc = (T)0;
        if (k > 0) acc = A::add(acc, vb);
        if (j > 0) acc = A::add(acc, vd);
        if (i > 0) acc = A::add(acc, vl);
        acc = A::add(acc, vc);
        if (i < nx - 1) acc = A::add(acc, vr);
        if (j < ny - 1) acc = A::add(acc, vu);
        if (k < nz - 1) acc = A::add(acc, vt);
        const int e = cid ? cid[s] : (int)(s >> 1);
        fc[e] = acc;
        sd.put(e, acc);
    }
}

// u += P u_c: C cells take their own coarse value, F cells the average of
// their neighbours' in row order d, l, r, u, t, b (k_prolong_add's sums)
template <class T>
__global__ void __launch_bounds__(256)
k_g7_prolong(int nx, int ny, int nz, const int *__restrict__ cid,
             const T *__restrict__ uc, T *__restrict__ u, const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    using A = Ar<T>;
    const long nxy = (long)nx * ny, n = nxy * nz;
    GRID_STRIDE(s, n) {
        int i, j, k;
        cell_ijk((unsigned)s, nx, ny, i, j, k);
        T add;
        if (((i + j + k) & 1) == 0) {
            add = uc[cid[s]];
        } else {
            const bool h[6] = {j > 0, i > 0, i < nx - 1, j < ny - 1, k < nz - 1, k > 0};
            const long o[6] = {-nx, -1, 1, nx, nxy, -nxy};
            T v[6];
#pragma unroll
            for (int d = 0; d < 6; d++) v[d] = h[d] ? uc[cid[s + o[d]]] : (T)0;
            T t = (T)0;
            int c = 0;
#pragma unroll
            for (int d = 0; d < 6; d++) {
                if (!h[d]) continue;
                t = c == 0 ? v[d] : A::add(t, v[d]);
                c++;
            }
            add = c == 1 ? t : A::div(t, (T)c);
        }
        u[s] = A::add(u[s], add);
    }
}

// The same for nx even, a thread per x-neighbour pair (2t, 2t+1): one of
// the two is a C cell, the other an F cell, so no warp diverges on the
// cell type; coarse ids are s >> 1 (no index array) and every load of a
// thread is independent.
template <class T>
__global__ void __launch_bounds__(256)
k_g7_prolong2(int nx, int ny, int nz, const T *__restrict__ uc, T *__restrict__ u,
              const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    using A = Ar<T>;
    const long nxy = (long)nx * ny, npair = nxy * nz / 2;
    GRID_STRIDE(t, npair) {
        const long s0 = 2 * t;
        int i0, j, k;
        cell_ijk((unsigned)s0, nx, ny, i0, j, k);
        const bool c_first = ((j + k) & 1) == 0;  // i0 is even
        const long sc = c_first ? s0 : s0 + 1, sf = c_first ? s0 + 1 : s0;
        const int fi = c_first ? i0 + 1 : i0;
        const T vc = uc[sc >> 1];
        const bool h[6] = {j > 0, fi > 0, fi < nx - 1, j < ny - 1, k < nz - 1, k > 0};
        const long o[6] = {-nx, -1, 1, nx, nxy, -nxy};
        T v[6];
#pragma unroll
        for (int d = 0; d < 6; d++) v[d] = h[d] ? uc[(sf + o[d]) >> 1] : (T)0;
        T acc = (T)0;
        int c = 0;
#pragma unroll
        for (int d = 0; d < 6; d++) {
            if (!h[d]) continue;
            acc = c == 0 ? v[d] : A::add(acc, v[d]);
            c++;
        }
        const T vf = c == 1 ? acc : A::div(acc, (T)c);
        u[sc] = A::add(u[sc], vc);
        u[sf] = A::add(u[sf], vf);
    }
}

// ---- level 0, exact red-black reduction (hmfem_options.schur0) -----------
//
// With the interpolation P_F = -A_FF^-1 A_FC (level 1 = the Schur
// complement, k_schur_fill) level 0 needs no smoothing: the F equations are
// solved exactly.  Restriction: u0 = A_FF^-1 f on F cells, 0 on C cells,
// leaves a residual that is zero on F cells, so the coarse right-hand side
// is f_c - sum over c's neighbours f of a_cf f_f / a_ff.  Prolongation: C
// cells take the coarse value, F cells solve their equation with it,
// (f_f - sum over f's neighbours c of a_fc u_c) / a_ff.  Neighbours in row
// order d, l, r, u, t, b; the coupling a_{s,s+e} comes from the stencil form
// (the +x/+y/+z entry of the lower cell).
template <class T, class V>
__device__ __forceinline__ T g7_coupling(const G7v<V> &g, long s, long nx, long nxy, int e)
{
    // e: 0 d, 1 l, 2 r, 3 u, 4 t, 5 b
    switch (e) {
    case 0: return (T)ld(g.cf, slice_at(s - nx, 2, 4));
    case 1: return (T)ld(g.cf, slice_at(s - 1, 1, 4));
    case 2: return (T)ld(g.cf, slice_at(s, 1, 4));
    case 3: return (T)ld(g.cf, slice_at(s, 2, 4));
    case 4: return (T)ld(g.cf, slice_at(s, 3, 4));
    default: return (T)ld(g.cf, slice_at(s - nxy, 3, 4));
    }
}

// fc[c] = f_s - sum_f a_sf (f_f dinv_f) over the C cells s (coarse id cid[s],
// or s >> 1 for nx even)
template <class T, class V>
__global__ void __launch_bounds__(256)
k_g7_sred(G7v<V> g, const T *__restrict__ f, const T *__restrict__ dinv,
          const int *__restrict__ cid, T *__restrict__ fc, Seed<T> sd, const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    using A = Ar<T>;
    const unsigned hx = (unsigned)(g.nx + 1) >> 1;
    const long nx = g.nx, nxy = (long)g.nx * g.ny, m = (long)hx * g.ny * g.nz;
    GRID_STRIDE(t, m) {
        const unsigned tu = (unsigned)t, r = tu / hx, kk0 = r / (unsigned)g.ny;
        const int j = (int)(r - kk0 * (unsigned)g.ny), k = (int)kk0;
        const int i = 2 * (int)(tu - r * hx) + ((j + k) & 1);
        if (i >= g.nx) continue;
        const long s = i + (long)r * nx;
        const bool h[6] = {j > 0, i > 0, i < g.nx - 1, j < g.ny - 1, k < g.nz - 1, k > 0};
        const long o[6] = {-nx, -1, 1, nx, nxy, -nxy};
        T a[6], v[6];
#pragma unroll
        for (int e = 0; e < 6; e++) {
            a[e] = h[e] ? g7_coupling<T>(g, s, nx, nxy, e) : (T)0;
            v[e] = h[e] ? A::mul(f[s + o[e]], dinv[s + o[e]]) : (T)0;
        }
        T acc = f[s];
#pragma unroll
        for (int e = 0; e < 6; e++)
            if (h[e]) acc = A::sub(acc, A::mul(a[e], v[e]));
        const int c = cid ? cid[s] : (int)(s >> 1);
        fc[c] = acc;
        sd.put(c, acc);
    }
}

// z on one F cell: (f_s - sum_c a_sc uc[c]) dinv_s
template <class T, class V, class CI>
__device__ __forceinline__ T g7_fsolve(const G7v<V> &g, long s, int i, int j, int k,
                                       const T *__restrict__ f, const T *__restrict__ dinv,
                                       const T *__restrict__ uc, CI coarse_id)
{
    using A = Ar<T>;
    const long nx = g.nx, nxy = (long)g.nx * g.ny;
    const bool h[6] = {j > 0, i > 0, i < g.nx - 1, j < g.ny - 1, k < g.nz - 1, k > 0};
    const long o[6] = {-nx, -1, 1, nx, nxy, -nxy};
    T a[6], v[6];
#pragma unroll
    for (int e = 0; e < 6; e++) {
        a[e] = h[e] ? g7_coupling<T>(g, s, nx, nxy, e) : (T)0;
        v[e] = h[e] ? uc[coarse_id(s + o[e])] : (T)0;
    }
    T acc = f[s];
#pragma unroll
    for (int e = 0; e < 6; e++)
        if (h[e]) acc = A::sub(acc, A::mul(a[e], v[e]));
    return A::mul(acc, dinv[s]);
}

// nx even: a thread per x-neighbour pair (one C cell, one F cell), coarse
// ids s >> 1
template <class T, class V>
__global__ void __launch_bounds__(256)
k_g7_sprol2(G7v<V> g, const T *__restrict__ f, const T *__restrict__ dinv,
            const T *__restrict__ uc, T *__restrict__ z, const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    const long npair = (long)g.nx * g.ny * g.nz / 2;
    GRID_STRIDE(t, npair) {
        const long s0 = 2 * t;
        int i0, j, k;
        cell_ijk((unsigned)s0, g.nx, g.ny, i0, j, k);
        const bool c_first = ((j + k) & 1) == 0;
        const long sc = c_first ? s0 : s0 + 1, sf = c_first ? s0 + 1 : s0;
        const int fi = c_first ? i0 + 1 : i0;
        z[sc] = uc[sc >> 1];
        z[sf] = g7_fsolve<T>(g, sf, fi, j, k, f, dinv, uc, [](long q) { return q >> 1; });
    }
}

// k_g7_sprol2 that also forms the CG's dots of the z it writes: sigma =
// (z, r) and, after the first application, (z, v) with v = A s_old; the
// last block derives beta (zdots_finish, flexible CG) -- the work of
// k_finish_z, without reading z again.
template <class T, class V>
__global__ void __launch_bounds__(256)
k_g7_sprol2_zd(G7v<V> g, const T *__restrict__ f, const T *__restrict__ dinv,
               const T *__restrict__ uc, T *__restrict__ z, const double *__restrict__ r,
               const double *__restrict__ v, Ctl *ctl, double *part, int first)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    const long npair = (long)g.nx * g.ny * g.nz / 2;
    double d1 = 0.0, d2 = 0.0;
    GRID_STRIDE(t, npair) {
        const long s0 = 2 * t;
        int i0, j, k;
        cell_ijk((unsigned)s0, g.nx, g.ny, i0, j, k);
        const bool c_first = ((j + k) & 1) == 0;
        const long sc = c_first ? s0 : s0 + 1, sf = c_first ? s0 + 1 : s0;
        const int fi = c_first ? i0 + 1 : i0;
        const T zc = uc[sc >> 1];
        const T zf = g7_fsolve<T>(g, sf, fi, j, k, f, dinv, uc, [](long q) { return q >> 1; });
        z[sc] = zc;
        z[sf] = zf;
        const double z0 = (double)(c_first ? zc : zf), z1 = (double)(c_first ? zf : zc);
        d1 += z0 * r[s0];
        d1 += z1 * r[s0 + 1];
        if (!first) {
            d2 += z0 * v[s0];
            d2 += z1 * v[s0 + 1];
        }
    }
    double *p2 = part + kRedBlocks;
    if (!first)
        grid_reduce_sum(d2, p2, &ctl->tickets[RED_A], [&](double t) { ctl->rz_old = t; });
    grid_reduce_sum(d1, part, &ctl->tickets[RED_SIGMA],
                    [&](double s) { zdots_finish(ctl, s, first, 1); });
}

// any nx: a thread per cell, coarse ids from cid
template <class T, class V>
__global__ void __launch_bounds__(256)
k_g7_sprol(G7v<V> g, const T *__restrict__ f, const T *__restrict__ dinv,
           const int *__restrict__ cid, const T *__restrict__ uc, T *__restrict__ z,
           const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    const long n = (long)g.nx * g.ny * g.nz;
    GRID_STRIDE(s, n) {
        int i, j, k;
        cell_ijk((unsigned)s, g.nx, g.ny, i, j, k);
        if (((i + j + k) & 1) == 0) z[s] = uc[cid[s]];
        else z[s] = g7_fsolve<T>(g, s, i, j, k, f, dinv, uc, [&](long q) { return cid[q]; });
    }
}

// v = f - A u;  u_out = u + w v D^-1;  optionally sigma = (u_out, f)
template <class T, class V, bool DOT>
__global__ void __launch_bounds__(256)
k_g7_post(G7v<V> g, int n, const T *__restrict__ f, const T *__restrict__ dinv, T w,
          const T *__restrict__ u, T *__restrict__ uo, Ctl *ctl, double *part, int first)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    using A = Ar<T>;
    double dot = 0.0;
    GRID_STRIDE(s, n) {
        int i, j, k;
        cell_ijk((unsigned)s, g.nx, g.ny, i, j, k);
        const T fr = f[s];
        const T t = g7_row<T, true>(fr, g, s, i, j, k, [&](long c) { return u[c]; });
        const T un = A::add(u[s], A::mul(A::mul(w, t), dinv[s]));
        uo[s] = un;
        if (DOT) dot += (double)un * (double)fr;
    }
    if (DOT)
        grid_reduce_sum(dot, part, &ctl->tickets[RED_SIGMA],
                        [&](double s) { sigma_finish(ctl, s, first); });
}

// v = A s; tau = (s, v); alpha = sigma / tau   (k_spmv_dot on the stencil)
__global__ void __launch_bounds__(256)
k_g7_spmv_dot(G7v<double> g, int n, const double *__restrict__ x, double *__restrict__ y,
              Ctl *ctl, double *part)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    double d = 0.0;
    GRID_STRIDE(s, n) {
        int i, j, k;
        cell_ijk((unsigned)s, g.nx, g.ny, i, j, k);
        const double a = g7_row<double, false>(0.0, g, s, i, j, k, [&](long c) { return x[c]; });
        y[s] = a;
        d += x[s] * a;
    }
    grid_reduce_sum(d, part, &ctl->tickets[RED_TAU], [&](double t) { tau_finish(ctl, t); });
}

// The same SpMV for nx even, two x-adjacent cells (s, s + 1; s even) per
// thread with 16-byte loads: the pair's x values, those one row and one
// plane away and the pair's coefficients arrive in 10 loads of 16 bytes and
// 3 of 8 instead of 28 of 8 (more bytes in flight per thread).  Each cell's
// sum keeps the terms, operations and order of g7_row (d,l,c,r,u,t,b from
// 0.0), so y is bit-identical; tau's partial sums group differently.
// DOT = false: y = A x alone (the inspection SpMV).
__device__ __forceinline__ double2 ld2(const double *p)
{
    return *reinterpret_cast<const double2 *>(p);
}

template <bool DOT>
__global__ void __launch_bounds__(256)
k_g7_spmv_dot2(G7v<double> g, int n, const double *__restrict__ x, double *__restrict__ y,
               Ctl *ctl, double *part)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    using A = Ar<double>;
    const long nx = g.nx, nxy = (long)g.nx * g.ny;
    const double2 z2 = make_double2(0.0, 0.0);
    double d = 0.0;
    GRID_STRIDE(h, (long)n >> 1) {
        const long s = 2 * h;
        int i, j, k;
        cell_ijk((unsigned)s, g.nx, g.ny, i, j, k);  // i even, s + 1 = (i + 1, j, k)
        const bool hd = j > 0, hu = j < g.ny - 1, ht = k < g.nz - 1, hb = k > 0;
        const bool hl = i > 0, hr = i + 2 < g.nx;    // -x of s, +x of s + 1
        const double2 xd = hd ? ld2(x + s - nx) : z2;
        const double xl = hl ? x[s - 1] : 0.0;
        const double2 xc = ld2(x + s);
        const double xr = hr ? x[s + 2] : 0.0;
        const double2 xu = hu ? ld2(x + s + nx) : z2;
        const double2 xt = ht ? ld2(x + s + nxy) : z2;
        const double2 xb = hb ? ld2(x + s - nxy) : z2;
        const double2 ad = hd ? ld2(g.cf + slice_at(s - nx, 2, 4)) : z2;
        const double al = hl ? g.cf[slice_at(s - 1, 1, 4)] : 0.0;
        const double2 ac = ld2(g.cf + slice_at(s, 0, 4));
        const double2 ar = ld2(g.cf + slice_at(s, 1, 4));  // s -> s + 1, s + 1 -> s + 2
        const double2 au = hu ? ld2(g.cf + slice_at(s, 2, 4)) : z2;
        const double2 at = ht ? ld2(g.cf + slice_at(s, 3, 4)) : z2;
        const double2 ab = hb ? ld2(g.cf + slice_at(s - nxy, 3, 4)) : z2;
        double t0 = 0.0, t1 = 0.0;
        auto acc = [&](double &t, double a, double xv) { t = A::add(t, A::mul(a, xv)); };
        if (hd) acc(t0, ad.x, xd.x);
        if (hl) acc(t0, al, xl);
        acc(t0, ac.x, xc.x);
        acc(t0, ar.x, xc.y);
        if (hu) acc(t0, au.x, xu.x);
        if (ht) acc(t0, at.x, xt.x);
        if (hb) acc(t0, ab.x, xb.x);
        if (hd) acc(t1, ad.y, xd.y);
        acc(t1, ar.x, xc.x);  // -x of s + 1: the +x coupling of s
        acc(t1, ac.y, xc.y);
        if (hr) acc(t1, ar.y, xr);
        if (hu) acc(t1, au.y, xu.y);
        if (ht) acc(t1, at.y, xt.y);
        if (hb) acc(t1, ab.y, xb.y);
        *reinterpret_cast<double2 *>(y + s) = make_double2(t0, t1);
        if (DOT) {
            d += xc.x * t0;
            d += xc.y * t1;
        }
    }
    if (DOT)
        grid_reduce_sum(d, part, &ctl->tickets[RED_TAU], [&](double t) { tau_finish(ctl, t); });
}

// the pair form applies: nx even, every array 16-byte aligned
bool g7_pairs(const G7v<double> &g, const double *x, const double *y)
{
    return g.nx % 2 == 0 && (((uintptr_t)x | (uintptr_t)y | (uintptr_t)g.cf) & 15) == 0;
}

// plain y = A x (inspection)
__global__ void __launch_bounds__(256)
k_g7_spmv(G7v<double> g, int n, const double *__restrict__ x, double *__restrict__ y)
{
    PDL_ENTRY();
    GRID_STRIDE(s, n) {
        int i, j, k;
        cell_ijk((unsigned)s, g.nx, g.ny, i, j, k);
        y[s] = g7_row<double, false>(0.0, g, s, i, j, k, [&](long c) { return x[c]; });
    }
}

// r = b - A x; (r, r); (b, b)   (k_resid on the stencil)
__global__ void __launch_bounds__(256)
k_g7_resid(G7v<double> g, int n, const double *__restrict__ b, const double *__restrict__ x,
           double *__restrict__ r, Ctl *ctl, double *part, int init, Seed<double> sd,
           Demote dm)
{
    PDL_ENTRY();
    if (init == 0 && (finished(ctl) || !ctl->check)) return;
    double rr = 0.0, bb = 0.0;
    GRID_STRIDE(s, n) {
        int i, j, k;
        cell_ijk((unsigned)s, g.nx, g.ny, i, j, k);
        const double a = g7_row<double, false>(0.0, g, s, i, j, k, [&](long c) { return x[c]; });
        const double bi = b[s];
        const double ri = dsub(bi, a);
        r[s] = ri;
        if (init != 2) {
            sd.put(s, ri);
            dm.put(s, ri);
        }
        rr += ri * ri;
        bb += bi * bi;
    }
    double *p2 = part + kRedBlocks;
    grid_reduce_sum(bb, p2, &ctl->tickets[RED_BB], [&](double s) { ctl->bb = s; });
    grid_reduce_sum(rr, part, &ctl->tickets[RED_TRR],
                    [&](double s) { trr_finish(ctl, s, init); });
}

// ---- level 1 ------------------------------------------------------------

template <class T, class V>
__global__ void __launch_bounds__(256)
k_g19_pre(G19v<V> g, const T *__restrict__ f, const T *__restrict__ u,
          const int *__restrict__ prow, T *__restrict__ rs, const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    using A = Ar<T>;
    GRID_STRIDE(c, g.n) {
        const T t = g19_row<T, true>(f[c], g, (int)c, [&](long q) { return u[q]; });
        const int pc = prow[c + 1] - prow[c];
        rs[c] = pc == 1 ? t : A::div(t, (T)pc);
    }
}

template <class T, class V>
__global__ void __launch_bounds__(256)
k_g19_post(G19v<V> g, const T *__restrict__ f, const T *__restrict__ dinv, T w,
           const T *__restrict__ u, T *__restrict__ uo, const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    using A = Ar<T>;
    GRID_STRIDE(c, g.n) {
        const T fr = f[c];
        const T t = g19_row<T, true>(fr, g, (int)c, [&](long q) { return u[q]; });
        uo[c] = A::add(u[c], A::mul(A::mul(w, t), dinv[c]));
    }
}

__global__ void __launch_bounds__(256)
k_g19_spmv(G19v<double> g, const double *__restrict__ x, double *__restrict__ y)
{
    PDL_ENTRY();
    GRID_STRIDE(c, g.n) y[c] = g19_row<double, false>(0.0, g, (int)c, [&](long q) { return x[q]; });
}

// ---- setup ----------------------------------------------------------------

// a_cc, a_{c,c+1}, a_{c,c+nx}, a_{c,c+nxy} from the assembled rows (order
// d,l,c,r,u,t,b over the in-grid neighbours), and a bitwise check of
// a_{c,c+e} == a_{c+e,c} for the three + directions
__global__ void k_g7_extract(int nx, int ny, int nz, const int *__restrict__ rowptr,
                             const int *__restrict__ col, const double *__restrict__ val,
                             double *cf, float *cf32, int *bad)
{
    const long nxy = (long)nx * ny, n = nxy * nz;
    GRID_STRIDE(s, n) {
        int i, j, k;
        cell_ijk((unsigned)s, nx, ny, i, j, k);
        const int o = rowptr[s];
        // position of each direction in the row
        const int pd = o, pl = pd + (j > 0), pc = pl + (i > 0), pr = pc + 1;
        const int pu = pr + (i < nx - 1), pt = pu + (j < ny - 1), pb = pt + (k < nz - 1);
        const int e = pb + (k > 0);
        bool ok = e == rowptr[s + 1] && col[pc] == (int)s;
        const double vc = val[pc];
        double vr = 0.0, vu = 0.0, vt = 0.0;
        if (i < nx - 1) {
            vr = val[pr];
            const long q = s + 1;
            const int oq = rowptr[q] + (j > 0);  // its l entry
            ok = ok && col[pr] == (int)q && col[oq] == (int)s &&
                 __double_as_longlong(val[oq]) == __double_as_longlong(vr);
        }
        if (j < ny - 1) {
            vu = val[pu];
            const long q = s + nx;
            const int oq = rowptr[q];  // its d entry (first)
            ok = ok && col[pu] == (int)q && col[oq] == (int)s &&
                 __double_as_longlong(val[oq]) == __double_as_longlong(vu);
        }
        if (k < nz - 1) {
            vt = val[pt];
            const long q = s + nxy;
            const int oq = rowptr[q + 1] - 1;  // its b entry (last)
            ok = ok && col[pt] == (int)q && col[oq] == (int)s &&
                 __double_as_longlong(val[oq]) == __double_as_longlong(vt);
        }
        const double v4[4] = {vc, vr, vu, vt};
#pragma unroll
        for (int a = 0; a < 4; a++) {
            cf[slice_at(s, a, 4)] = v4[a];
            if (cf32) cf32[slice_at(s, a, 4)] = (float)v4[a];
        }
        if (!ok) atomicOr(bad, 1);
    }
}

__device__ __forceinline__ void cvt(double v, float *o) { *o = (float)v; }

template <class D>
__global__ void k_g19_cast(const double *__restrict__ v, long m, D *out)
{
    GRID_STRIDE(t, m) cvt(v[t], out + t);
}

// the BF16 copy in the four-per-word layout (g19q_at); rows past n and the
// pad coefficient are zero
__global__ void k_g19_cast16(const double *__restrict__ v, long n, __nv_bfloat16 *out)
{
    const long m = g19q_len(n);
    GRID_STRIDE(t, m) {
        const long r = ((t >> 2) / (kG19Words * 32)) * 32 + ((t >> 2) & 31);
        const int q = (int)((((t >> 2) >> 5) % kG19Words) * 4 + (t & 3));
        out[t] = (r < n && q < kQ19) ? __float2bfloat16((float)v[slice_at(r, q, kQ19)])
                                     : __float2bfloat16(0.0f);
    }
}

int nb(long n)
{
    long b = ceil_div(n, 256);
    if (b < 1) b = 1;
    return (int)(b < kRedBlocks ? b : kRedBlocks);
}

template <class V> G7v<V> g7v(const Grid7 &g);
template <> G7v<double> g7v<double>(const Grid7 &g) { return {g.cf, g.nx, g.ny, g.nz}; }
template <> G7v<float> g7v<float>(const Grid7 &g) { return {g.cf32, g.nx, g.ny, g.nz}; }

// floor(2^64 / d) + 1 (d >= 2)
unsigned long long mul_inverse(unsigned d)
{
    return (unsigned long long)(~0ull / d) + ((~0ull % d) == d - 1 ? 2ull : 1ull);
}

template <class V> G19v<V> g19v_of(const V *v, const Grid19 &g, int n)
{
    G19v<V> o;
    o.v = v;
    o.n = n;
    o.nx = g.nx; o.ny = g.ny; o.nz = g.nz;
    o.mhx = mul_inverse((unsigned)g.nx >> 1);
    o.mny = mul_inverse((unsigned)g.ny);
    const long nx = g.nx, nxy = (long)g.nx * g.ny;
    for (int par = 0; par < 2; par++)
        for (int q = 0; q < kQ19; q++) {
            const long off = q19x(q) + q19y(q) * nx + q19z(q) * nxy;
            const long y = par + off;
            o.dq[par][q] = (int)(y >= 0 ? y / 2 : -((-y + 1) / 2));  // floor(y / 2)
        }
    return o;
}

template <class V> G19v<V> g19v(const Grid19 &g, int n);
template <> G19v<double> g19v<double>(const Grid19 &g, int n) { return g19v_of(g.v, g, n); }
template <> G19v<float> g19v<float>(const Grid19 &g, int n) { return g19v_of(g.v32, g, n); }
template <> G19v<__nv_bfloat16> g19v<__nv_bfloat16>(const Grid19 &g, int n)
{
    return g19v_of(g.v16, g, n);
}

}  // namespace

bool g19_applies(int nx, int ny, int nz)
{
    (void)nz;
    return nx % 2 == 0 && nx >= 4 && ny >= 4;
}

void g7_free(Grid7 &g)
{
    dfree(g.cf);
    dfree(g.cf32);
    g = Grid7();
}

void g19_free(Grid19 &g)
{
    dfree(g.v); dfree(g.v32); dfree(g.v16);
    g = Grid19();
}

int g7_build(Level &L, int nx, int ny, int nz, bool f32, cudaStream_t st, int *dwork)
{
    g7_free(L.g7);
    const long n = (long)nx * ny * nz;
    if (n != L.A.n || n <= 0) return HMFEM_OK;
    Grid7 g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    const long long m = slice_len(n, 4);
    g.cf = (double *)dalloc(sizeof(double) * m);
    if (f32) g.cf32 = (float *)dalloc(sizeof(float) * m);
    if (!g.cf || (f32 && !g.cf32)) { g7_free(g); return HMFEM_E_CUDA; }
    HM_CUDA(cudaMemsetAsync(g.cf, 0, sizeof(double) * m, st));  // tail of the last slice
    if (f32) HM_CUDA(cudaMemsetAsync(g.cf32, 0, sizeof(float) * m, st));
    HM_CUDA(cudaMemsetAsync(dwork, 0, sizeof(int), st));
    k_g7_extract<<<nb(n), 256, 0, st>>>(nx, ny, nz, L.A.rowptr, L.A.col, L.A.val, g.cf,
                                        g.cf32, dwork);
    HM_LAUNCHED();
    int bad = 0;
    HM_CUDA(cudaMemcpyAsync(&bad, dwork, sizeof(int), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    if (bad) { g7_free(g); return HMFEM_OK; }
    L.g7 = g;
    return HMFEM_OK;
}

int g19_lowp(Grid19 &g, int n, bool f32, bool bf16, cudaStream_t st)
{
    const long m = (long)slice_len(n, kQ19);
    if (f32 && !g.v32) {
        g.v32 = (float *)dalloc(sizeof(float) * m);
        if (!g.v32) return HMFEM_E_CUDA;
        k_g19_cast<float><<<nb(m), 256, 0, st>>>(g.v, m, g.v32);
        HM_LAUNCHED();
    }
    if (bf16 && !g.v16) {
        const long m16 = (long)g19q_len(n);
        g.v16 = (__nv_bfloat16 *)dalloc(sizeof(__nv_bfloat16) * m16);
        if (!g.v16) return HMFEM_E_CUDA;
        k_g19_cast16<<<nb(m16), 256, 0, st>>>(g.v, n, g.v16);
        HM_LAUNCHED();
    }
    return HMFEM_OK;
}

// ---- launchers used by the cycle and the CG --------------------------------

template <class T, class V>
int g7_pre(const Level &L, const T *f, const T *u, T *rs, const Ctl *ctl, cudaStream_t st)
{
    const int n = L.A.n;
    const int nblk = occ_blocks((const void *)k_g7_pre<T, V>, n, 256, kRedBlocks);
    launch_pdl(k_g7_pre<T, V>, nblk, 256, st, g7v<V>(L.g7), n, f, u, rs, ctl);
    HM_LAUNCHED();
    return HMFEM_OK;
}

template <class T>
int g7_restrict(const Level &L, const T *rs, T *fc, Seed<T> sd, const Ctl *ctl,
                cudaStream_t st)
{
    const Grid7 &g = L.g7;
    const long m = (long)((g.nx + 1) >> 1) * g.ny * g.nz;
    const int nblk = occ_blocks((const void *)k_g7_restrict<T>, m, 256, kRedBlocks);
    // nx even: the C cell s has coarse id s >> 1, no index array needed
    const int *cid = g.nx % 2 ? L.cid : nullptr;
    launch_pdl(k_g7_restrict<T>, nblk, 256, st, g.nx, g.ny, g.nz, cid, rs, fc, sd, ctl);
    HM_LAUNCHED();
    return HMFEM_OK;
}

template <class T>
int g7_sred(const Level &L, const T *f, const T *dinv, T *fc, Seed<T> sd, const Ctl *ctl,
            cudaStream_t st)
{
    const Grid7 &g = L.g7;
    const long m = (long)((g.nx + 1) >> 1) * g.ny * g.nz;
    const G7v<T> gv = g7v<T>(g);
    const int nblk = occ_blocks((const void *)k_g7_sred<T, T>, m, 256, kRedBlocks);
    const int *cid = g.nx % 2 ? L.cid : nullptr;
    launch_pdl(k_g7_sred<T, T>, nblk, 256, st, gv, f, dinv, cid, fc, sd, ctl);
    HM_LAUNCHED();
    return HMFEM_OK;
}

template <class T>
int g7_sprol(const Level &L, const T *f, const T *dinv, const T *uc, T *z, const Ctl *ctl,
             cudaStream_t st)
{
    const Grid7 &g = L.g7;
    const G7v<T> gv = g7v<T>(g);
    if (g.nx % 2 == 0) {
        const long npair = (long)L.A.n / 2;
        const int nblk = occ_blocks((const void *)k_g7_sprol2<T, T>, npair, 256, kRedBlocks);
        launch_pdl(k_g7_sprol2<T, T>, nblk, 256, st, gv, f, dinv, uc, z, ctl);
        HM_LAUNCHED();
        return HMFEM_OK;
    }
    const int nblk = occ_blocks((const void *)k_g7_sprol<T, T>, L.A.n, 256, kRedBlocks);
    launch_pdl(k_g7_sprol<T, T>, nblk, 256, st, gv, f, dinv, (const int *)L.cid, uc, z, ctl);
    HM_LAUNCHED();
    return HMFEM_OK;
}

template <class T>
int g7_prolong(const Level &L, const T *uc, T *u, const Ctl *ctl, cudaStream_t st)
{
    const Grid7 &g = L.g7;
    if (g.nx % 2 == 0) {
        const long npair = (long)L.A.n / 2;
        const int nblk = occ_blocks((const void *)k_g7_prolong2<T>, npair, 256, kRedBlocks);
        launch_pdl(k_g7_prolong2<T>, nblk, 256, st, g.nx, g.ny, g.nz, uc, u, ctl);
        HM_LAUNCHED();
        return HMFEM_OK;
    }
    const int nblk = occ_blocks((const void *)k_g7_prolong<T>, L.A.n, 256, kRedBlocks);
    launch_pdl(k_g7_prolong<T>, nblk, 256, st, g.nx, g.ny, g.nz, L.cid, uc, u, ctl);
    HM_LAUNCHED();
    return HMFEM_OK;
}

template <class T, class V, bool DOT>
int g7_post(const Level &L, const T *f, const T *dinv, T w, const T *u, T *uo, Ctl *ctl,
             double *part, int first, cudaStream_t st)
{
    const int n = L.A.n;
    const int nblk = occ_blocks((const void *)k_g7_post<T, V, DOT>, n, 256, kRedBlocks);
    launch_pdl(k_g7_post<T, V, DOT>, nblk, 256, st, g7v<V>(L.g7), n, f, dinv, w, u, uo, ctl,
                                                part, first);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int g7_spmv_dot(const Level &L, const double *x, double *y, Ctl *ctl, double *part,
                 cudaStream_t st)
{
    const int n = L.A.n;
    const auto gv = g7v<double>(L.g7);
    if (g7_pairs(gv, x, y)) {
        const int nblk =
            occ_blocks((const void *)k_g7_spmv_dot2<true>, (long)n / 2, 256, kRedBlocks);
        launch_pdl(k_g7_spmv_dot2<true>, nblk, 256, st, gv, n, x, y, ctl, part);
    } else {
        const int nblk = occ_blocks((const void *)k_g7_spmv_dot, n, 256, kRedBlocks);
        launch_pdl(k_g7_spmv_dot, nblk, 256, st, gv, n, x, y, ctl, part);
    }
    HM_LAUNCHED();
    return HMFEM_OK;
}

template <class T>
int g7_sprol_zd(const Level &L, const T *f, const T *dinv, const T *uc, T *z,
                const double *r, const double *v, Ctl *ctl, double *part, int first,
                bool *fused, cudaStream_t st)
{
    *fused = false;
    if (L.g7.nx % 2 != 0) return g7_sprol<T>(L, f, dinv, uc, z, ctl, st);
    const G7v<T> gv = g7v<T>(L.g7);
    const long npair = (long)L.A.n / 2;
    const int nblk = occ_blocks((const void *)k_g7_sprol2_zd<T, T>, npair, 256, kRedBlocks);
    launch_pdl(k_g7_sprol2_zd<T, T>, nblk, 256, st, gv, f, dinv, uc, z, r, v, ctl, part, first);
    HM_LAUNCHED();
    *fused = true;
    return HMFEM_OK;
}
template int g7_sprol_zd<float>(const Level &, const float *, const float *, const float *,
                                float *, const double *, const double *, Ctl *, double *, int,
                                bool *, cudaStream_t);

int g7_resid(const Level &L, const double *b, const double *x, double *r, Ctl *ctl,
             double *part, int init, Seed<double> sd, Demote dm, cudaStream_t st)
{
    const int n = L.A.n;
    const int nblk = occ_blocks((const void *)k_g7_resid, n, 256, kRedBlocks);
    launch_pdl(k_g7_resid, nblk, 256, st, g7v<double>(L.g7), n, b, x, r, ctl, part, init, sd,
               dm);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int g7_spmv(const Level &L, const double *x, double *y, cudaStream_t st)
{
    const int n = L.A.n;
    const auto gv = g7v<double>(L.g7);
    if (g7_pairs(gv, x, y)) {  // the CG's kernel without its dot
        const int nblk =
            occ_blocks((const void *)k_g7_spmv_dot2<false>, (long)n / 2, 256, kRedBlocks);
        launch_pdl(k_g7_spmv_dot2<false>, nblk, 256, st, gv, n, x, y, (Ctl *)nullptr,
                   (double *)nullptr);
    } else {
        const int nblk = occ_blocks((const void *)k_g7_spmv, n, 256, kRedBlocks);
        launch_pdl(k_g7_spmv, nblk, 256, st, gv, n, x, y);
    }
    HM_LAUNCHED();
    return HMFEM_OK;
}

template <class T, class V>
int g19_pre(const Level &L, const T *f, const T *u, T *rs, const Ctl *ctl, cudaStream_t st)
{
    const G19v<V> g = g19v<V>(L.g19, L.A.n);
    const int nblk = occ_blocks((const void *)k_g19_pre<T, V>, g.n, 256, kRedBlocks);
    launch_pdl(k_g19_pre<T, V>, nblk, 256, st, g, f, u, L.P.rowptr, rs, ctl);
    HM_LAUNCHED();
    return HMFEM_OK;
}

template <class T, class V>
int g19_post(const Level &L, const T *f, const T *dinv, T w, const T *u, T *uo,
              const Ctl *ctl, cudaStream_t st)
{
    const G19v<V> g = g19v<V>(L.g19, L.A.n);
    const int nblk = occ_blocks((const void *)k_g19_post<T, V>, g.n, 256, kRedBlocks);
    launch_pdl(k_g19_post<T, V>, nblk, 256, st, g, f, dinv, w, u, uo, ctl);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int g19_spmv(const Level &L, const double *x, double *y, cudaStream_t st)
{
    const G19v<double> g = g19v<double>(L.g19, L.A.n);
    const int nblk = occ_blocks((const void *)k_g19_spmv, g.n, 256, kRedBlocks);
    launch_pdl(k_g19_spmv, nblk, 256, st, g, x, y);
    HM_LAUNCHED();
    return HMFEM_OK;
}

template int g7_pre<double, double>(const Level &, const double *, const double *, double *,
                                    const Ctl *, cudaStream_t);
template int g7_pre<float, float>(const Level &, const float *, const float *, float *,
                                  const Ctl *, cudaStream_t);
template int g7_restrict<double>(const Level &, const double *, double *, Seed<double>,
                                 const Ctl *, cudaStream_t);
template int g7_restrict<float>(const Level &, const float *, float *, Seed<float>,
                                const Ctl *, cudaStream_t);
template int g7_prolong<double>(const Level &, const double *, double *, const Ctl *,
                                cudaStream_t);
template int g7_prolong<float>(const Level &, const float *, float *, const Ctl *,
                               cudaStream_t);
template int g7_sred<float>(const Level &, const float *, const float *, float *,
                            Seed<float>, const Ctl *, cudaStream_t);
template int g7_sprol<float>(const Level &, const float *, const float *, const float *,
                             float *, const Ctl *, cudaStream_t);
template int g7_sred<double>(const Level &, const double *, const double *, double *,
                             Seed<double>, const Ctl *, cudaStream_t);
template int g7_sprol<double>(const Level &, const double *, const double *,
                              const double *, double *, const Ctl *, cudaStream_t);
template int g7_post<double, double, true>(const Level &, const double *, const double *,
                                           double, const double *, double *, Ctl *,
                                           double *, int, cudaStream_t);
template int g7_post<double, double, false>(const Level &, const double *, const double *,
                                            double, const double *, double *, Ctl *,
                                            double *, int, cudaStream_t);
template int g7_post<float, float, false>(const Level &, const float *, const float *,
                                          float, const float *, float *, Ctl *, double *,
                                          int, cudaStream_t);
template int g19_pre<double, double>(const Level &, const double *, const double *, double *,
                                     const Ctl *, cudaStream_t);
template int g19_pre<float, float>(const Level &, const float *, const float *, float *,
                                   const Ctl *, cudaStream_t);
template int g19_pre<float, __nv_bfloat16>(const Level &, const float *, const float *,
                                           float *, const Ctl *, cudaStream_t);
template int g19_post<double, double>(const Level &, const double *, const double *,
                                      double, const double *, double *, const Ctl *,
                                      cudaStream_t);
template int g19_post<float, float>(const Level &, const float *, const float *, float,
                                    const float *, float *, const Ctl *, cudaStream_t);
template int g19_post<float, __nv_bfloat16>(const Level &, const float *, const float *,
                                            float, const float *, float *, const Ctl *,
                                            cudaStream_t);

}  // namespace hm
