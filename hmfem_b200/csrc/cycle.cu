// cycle.cu -- V-cycle kernels (damped Jacobi on SELL-32, the device design
// of device_amg.h:11-43, 370-432) and the CG vector kernels.
//
// FP64 instantiations use non-contracted arithmetic, so one V-cycle is
// bit-identical to the oracle's Jacobi V-cycle; the FP32 ones (the mixed
// precision preconditioner) use FMA.  Every kernel takes the CG control
// block and returns at once when the solve is already finished, so a
// captured iteration can be replayed past convergence at no cost.
#include <cstdlib>

#include "cycle.cuh"

namespace hm {

thread_local std::vector<KRec> *t_kprof = nullptr;
thread_local int t_nopdl = 0;
thread_local int t_klevel = -1;

int g_pdl = [] {
    const char *e = getenv("HMFEM_PDL");
    return e ? atoi(e) : 1;
}();

// t - sum_k a_k x(c_k) (SUB) or t + sum_k a_k x(c_k) over one SELL-32 row
// (entries at o, o+32, ...), in stored order.  Column indices, values and
// the gathered x are loaded CH entries at a time (four in FP64, eight in
// FP32) so the dependent gathers overlap; the summation order is unchanged.
template <class T, bool SUB, int CH = (sizeof(T) == 8 ? 4 : 8), class M, class X>
__device__ __forceinline__ T row_acc(T t, const int *__restrict__ scol,
                                     const M *__restrict__ sval, long long o,
                                     int wd, X x)
{
    using A = Ar<T>;
    for (int k0 = 0; k0 < wd; k0 += CH, o += 32 * CH) {
        int c[CH];
        T a[CH], xv[CH];
#pragma unroll
        for (int q = 0; q < CH; q++) {
            const bool ok = k0 + q < wd;
            c[q] = ok ? scol[o + 32 * q] : 0;
            a[q] = ok ? (T)ld(sval, o + 32 * q) : (T)0;
        }
#pragma unroll
        for (int q = 0; q < CH; q++) xv[q] = k0 + q < wd ? x(c[q]) : (T)0;
#pragma unroll
        for (int q = 0; q < CH; q++) {
            if (k0 + q < wd) {
                const T ax = A::mul(a[q], xv[q]);
                t = SUB ? A::sub(t, ax) : A::add(t, ax);
            }
        }
    }
    return t;
}

// Sell::pk entries: the column is the row plus the high half (int16), the
// value the BF16 bits of the low half (exactly __bfloat162float of them);
// same terms, same order as row_acc over col + val16.
struct Pk16 {
    unsigned w;
};

template <class T, bool SUB, int CH = (sizeof(T) == 8 ? 4 : 8), class X>
__device__ __forceinline__ T row_acc_pk(T t, const Pk16 *__restrict__ pk, long long o, int wd,
                                        int row, X x)
{
    using A = Ar<T>;
    for (int k0 = 0; k0 < wd; k0 += CH, o += 32 * CH) {
        unsigned e[CH];
        T xv[CH];
#pragma unroll
        for (int q = 0; q < CH; q++) e[q] = k0 + q < wd ? __ldg(&pk[o + 32 * q].w) : 0u;
#pragma unroll
        for (int q = 0; q < CH; q++) xv[q] = k0 + q < wd ? x(row + ((int)e[q] >> 16)) : (T)0;
#pragma unroll
        for (int q = 0; q < CH; q++) {
            if (k0 + q < wd) {
                const T ax = A::mul((T)__uint_as_float(e[q] << 16), xv[q]);
                t = SUB ? A::sub(t, ax) : A::add(t, ax);
            }
        }
    }
    return t;
}

// row_acc over either storage of a SELL level
template <class T, bool SUB, class M, class X>
__device__ __forceinline__ T row_acc_r(T t, const int *__restrict__ scol,
                                       const M *__restrict__ sval, long long o, int wd,
                                       int row, X x)
{
    if constexpr (std::is_same<M, Pk16>::value) return row_acc_pk<T, SUB>(t, sval, o, wd, row, x);
    else return row_acc<T, SUB>(t, scol, sval, o, wd, x);
}

// Vector loads of the row functions below (a load policy, so a caller can
// route them differently without touching the arithmetic).
struct PlainLd {
    template <class T> __device__ __forceinline__ T operator()(const T *p, long i) const
    {
        return p[i];
    }
};

// ---- smoother / transfer row functions ---------------------------------
// One row (one coarse row for the restriction) of each Chebyshev-level
// kernel (the kernels below run these over their grid-stride rows).

template <class T, class M, class LD>
__device__ __forceinline__ void pre_row(long r, const long long *__restrict__ sptr,
                                        const int *__restrict__ scol,
                                        const M *__restrict__ sval, const T *f, const T *u,
                                        const int *__restrict__ prow, T *rs, LD ld)
{
    using A = Ar<T>;
    long q = r >> 5;
    int lane = (int)(r & 31);
    long long base = sptr[q];
    int wd = (int)((sptr[q + 1] - base) >> 5);
    T t = ld(f, r);
    t = row_acc_r<T, true>(t, scol, sval, base + lane, wd, (int)r,
                           [&](int c) { return ld(u, c); });
    int pc = prow[r + 1] - prow[r];
    rs[r] = pc == 1 ? t : A::div(t, (T)pc);
}

template <class T, class M, class LD>
__device__ __forceinline__ void cheb0_row(long i, const long long *__restrict__ sptr,
                                          const int *__restrict__ scol,
                                          const M *__restrict__ sval, const T *f,
                                          const T *__restrict__ dinv, T ith, const T *u,
                                          T *r, T *d, LD ld)
{
    using A = Ar<T>;
    const long q = i >> 5;
    const long long base = sptr[q];
    const int wd = (int)((sptr[q + 1] - base) >> 5);
    const T t = row_acc_r<T, true>(ld(f, i), scol, sval, base + (i & 31), wd, (int)i,
                                   [&](int c) { return ld(u, c); });
    const T di = dinv[i];
    r[i] = A::mul(di, t);
    d[i] = A::mul(A::mul(ith, t), di);
}

template <class T, class M, int MODE, class LD>
__device__ __forceinline__ void cheb_step_row(long i, const long long *__restrict__ sptr,
                                              const int *__restrict__ scol,
                                              const M *__restrict__ sval, const T *f,
                                              const T *__restrict__ dinv, T c1, T c2,
                                              const T *din, T *dout, T *r, T *u, int last,
                                              LD ld)
{
    using A = Ar<T>;
    const long q = i >> 5;
    const long long base = sptr[q];
    const int wd = (int)((sptr[q + 1] - base) >> 5);
    const T ad = row_acc_r<T, false>((T)0, scol, sval, base + (i & 31), wd, (int)i,
                                     [&](int c) { return ld(din, c); });
    const T di = dinv[i], dold = ld(din, i);
    const T rp = MODE == 0 ? A::mul(di, ld(f, i)) : ld(r, i);
    const T rn = A::sub(rp, A::mul(di, ad));
    const T dn = A::add(A::mul(c1, dold), A::mul(c2, rn));
    u[i] = MODE == 0 ? A::add(dold, dn)
         : MODE == 1 ? A::add(A::add(ld(u, i), dold), dn) : A::add(ld(u, i), dn);
    if (!last) {
        r[i] = rn;
        dout[i] = dn;
    }
}

// ---- smoother / transfer kernels --------------------------------------

// Residual after the pre-smoother from zero (device_jacobi 3-arg,
// device_amg.h:35-42), whose iterate u = w D^-1 f the producer of f has
// already written (Seed):  r = f - A u;  rs = r / |P row| (the 1/c of
// simple_restriction, generic_operator.h:97-122, applied here).
template <class T, class M>
__global__ void __launch_bounds__(256, 6)
k_pre(const long long *__restrict__ sptr, const int *__restrict__ scol,
      const M *__restrict__ sval, int n, const T *__restrict__ f,
      const T *__restrict__ u, const int *__restrict__ prow, T *__restrict__ rs,
      const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    GRID_STRIDE(r, n) pre_row<T>(r, sptr, scol, sval, f, u, prow, rs, PlainLd{});
}

// u = (w f) D^-1 on level 0 where no producer seeded it (a V-cycle applied
// on its own, hmfem_vcycle)
template <class T>
__global__ void k_seed(int n, const T *__restrict__ f, Seed<T> sd)
{
    PDL_ENTRY();
    GRID_STRIDE(i, n) sd.put(i, f[i]);
}

// f_c[e] = sum_{i in R(e), ascending} rs_i  (simple_restriction's
// accumulation order, generic_operator.h:86-128).
// Four rows (a grid stride apart) advance together in the prolongation so
// that their chains of dependent loads (row pointer, column, gathered value)
// overlap; each row's sum keeps its own ascending order.  (The restriction's
// rows -- columns of P -- are long and uneven: interleaved, every row waits
// for the longest, 36 -> 64 us on level 1 at 256^3, so it keeps one row at
// a time.)
constexpr int kRowsPerThread = 4;

template <class T>
__global__ void __launch_bounds__(256)
k_restrict(const int *__restrict__ rrow, const int *__restrict__ rcol, int nc,
           const T *__restrict__ rs, T *__restrict__ fc, Seed<T> sd, const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    using A = Ar<T>;
    GRID_STRIDE(e, nc)
    {
        T acc = (T)0;
        for (int k = rrow[e]; k < rrow[e + 1]; k++) acc = A::add(acc, ld(rs, rcol[k]));
        fc[e] = acc;
        sd.put(e, acc);
    }
}

template <class T>
__global__ void __launch_bounds__(256)
k_prolong_add(const int *__restrict__ prow, const int *__restrict__ pcol, int n,
              const T *__restrict__ uc, T *__restrict__ u, const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    using A = Ar<T>;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i0 = blockIdx.x * (long)blockDim.x + threadIdx.x; i0 < n;
         i0 += kRowsPerThread * stride) {
        int a[kRowsPerThread], c[kRowsPerThread];
        T t[kRowsPerThread];
        int cm = 0;
#pragma unroll
        for (int j = 0; j < kRowsPerThread; j++) {
            const long i = i0 + j * stride;
            a[j] = i < n ? prow[i] : 0;
            c[j] = i < n ? prow[i + 1] - a[j] : 0;
            cm = c[j] > cm ? c[j] : cm;
        }
#pragma unroll
        for (int j = 0; j < kRowsPerThread; j++) t[j] = c[j] > 0 ? ld(uc, pcol[a[j]]) : (T)0;
        for (int k = 1; k < cm; k++)
#pragma unroll
            for (int j = 0; j < kRowsPerThread; j++)
                if (k < c[j]) t[j] = A::add(t[j], ld(uc, pcol[a[j] + k]));
        // one C neighbour taken as is, else the mean (simple_prolongation)
#pragma unroll
        for (int j = 0; j < kRowsPerThread; j++) {
            const long i = i0 + j * stride;
            if (i < n && c[j] > 0)
                u[i] = A::add(ld(u, i), c[j] == 1 ? t[j] : A::div(t[j], (T)c[j]));
        }
    }
}

// Post-smoother (device_jacobi 2-arg, device_amg.h:27-34):
// v = f - A u;  u_out = u + w v D^-1.  Optionally accumulates
// dot(u_out, f) -> ctl->sigma (the PCG's (C r, r), pcg.h:66).
template <class T, class M, bool DOT>
__global__ void __launch_bounds__(256, 6)
k_post(const long long *__restrict__ sptr, const int *__restrict__ scol,
       const M *__restrict__ sval, int n, const T *__restrict__ f,
       const T *__restrict__ dinv, T w, const T *__restrict__ u,
       T *__restrict__ uo, Ctl *ctl, double *part, int first)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    using A = Ar<T>;
    double dot = 0.0;
    GRID_STRIDE(r, n) {
        long q = r >> 5;
        int lane = (int)(r & 31);
        long long base = sptr[q];
        int wd = (int)((sptr[q + 1] - base) >> 5);
        T fr = f[r];
        T t = fr;
        t = row_acc_r<T, true>(t, scol, sval, base + lane, wd, (int)r,
                               [&](int c) { return u[c]; });
        T un = A::add(u[r], A::mul(A::mul(w, t), dinv[r]));
        uo[r] = un;
        if (DOT) dot += (double)un * (double)fr;
    }
    if (DOT) {
        grid_reduce_sum(dot, part, &ctl->tickets[RED_SIGMA],
                        [&](double s) { sigma_finish(ctl, s, first); });
    }
}

// ---- Chebyshev smoothing (coarse levels) ---------------------------------
//
// K steps of the Chebyshev iteration on D^-1 A (D the l1 diagonal) over
// [1/30, 1]; the oracle's cheb_steps restates the same operations.  The
// first direction d0 = (1/theta * t) D^-1 (t = f from zero, seeded by the
// producer of f; t = f - A u after the prolongation, k_cheb0); then per
// step, in one pass: q = A d (row order, from 0), r = r - D^-1 q,
// d' = c1 d + c2 r, u = u + d' (first step: d0 + d' from zero, (u + d0) + d'
// otherwise).  d ping-pongs between two vectors because every row gathers
// it; r and u are only read at their own row.

// post-smoother, step 0: t = f - A u;  r = D^-1 t;  d0 = (ith t) D^-1
template <class T, class M>
__global__ void __launch_bounds__(256, 6)
k_cheb0(const long long *__restrict__ sptr, const int *__restrict__ scol,
        const M *__restrict__ sval, int n, const T *__restrict__ f,
        const T *__restrict__ dinv, T ith, const T *__restrict__ u, T *__restrict__ r,
        T *__restrict__ d, const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    GRID_STRIDE(i, n) cheb0_row<T>(i, sptr, scol, sval, f, dinv, ith, u, r, d, PlainLd{});
}

// one Chebyshev step; MODE 0: first step from zero, 1: first step after the
// prolongation, 2: later steps.  last: r and d' are not needed afterwards.
template <class T, class M, int MODE>
__global__ void __launch_bounds__(256, 6)
k_cheb_step(const long long *__restrict__ sptr, const int *__restrict__ scol,
            const M *__restrict__ sval, int n, const T *__restrict__ f,
            const T *__restrict__ dinv, T c1, T c2, const T *__restrict__ din,
            T *__restrict__ dout, T *__restrict__ r, T *__restrict__ u, int last,
            const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    GRID_STRIDE(i, n) cheb_step_row<T, M, MODE>(i, sptr, scol, sval, f, dinv, c1, c2, din,
                                                  dout, r, u, last, PlainLd{});
}

// ---- multicolour Gauss-Seidel (coarse levels) ---------------------------

// Forward sweep from zero, first colour: u_i = f_i / a_ii on colour 0,
// 0 elsewhere (exactly what the colour-0 update gives from u = 0).
template <class T>
__global__ void __launch_bounds__(256)
k_gs_init(int n, const signed char *__restrict__ color, const T *__restrict__ f,
          const T *__restrict__ dinv, T *__restrict__ u, const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    using A = Ar<T>;
    GRID_STRIDE(i, n) u[i] = color[i] == 0 ? A::mul(f[i], dinv[i]) : (T)0;
}

// sum_j a_ij x_j of CSR row `row` by the eight threads of a warp quarter
// (g = thread within the group): thread g adds entries g, g+8, ... in
// order (four entries per round, so the gathers overlap), the eight
// partial sums are combined by xor offsets 4, 2, 1 and thread 0's value is
// returned to the group -- the order the oracle's row_dot8 reproduces.
// Every thread of the warp must call this (a group with no row passes
// a = e = 0).
// CG: load x through L2 only (ld.global.cg) -- for a kernel that also
// writes x from other blocks between grid barriers, where the read-only and
// L1 paths could return stale values.
template <class T, class M, bool CG = false>
__device__ __forceinline__ T row_dot8(int a, int e, const int *__restrict__ col,
                                      const M *__restrict__ val, const T *x, int g)
{
    using A = Ar<T>;
    T p = (T)0;
    for (int k0 = a + g; k0 < e; k0 += 32) {
        int c[4];
        T v[4], xv[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int k = k0 + 8 * q;
            c[q] = k < e ? col[k] : 0;
            v[q] = k < e ? (T)ld(val, k) : (T)0;
        }
#pragma unroll
        for (int q = 0; q < 4; q++)
            xv[q] = k0 + 8 * q < e ? (CG ? __ldcg(x + c[q]) : x[c[q]]) : (T)0;
#pragma unroll
        for (int q = 0; q < 4; q++)
            if (k0 + 8 * q < e) p = A::add(p, A::mul(v[q], xv[q]));
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) p = A::add(p, __shfl_xor_sync(0xffffffffu, p, o));
    return __shfl_sync(0xffffffffu, p, (threadIdx.x & 31) & ~7);
}

// One colour of a Gauss-Seidel sweep, four rows per warp: rows crows[r0..r1)
// (no two rows of a colour couple), u_i += (f_i - sum_j a_ij u_j) / a_ii.
template <class T, class M>
__global__ void __launch_bounds__(256)
k_gs_sweep(const int *__restrict__ rowptr, const int *__restrict__ col,
           const M *__restrict__ val, const int *__restrict__ crows, long r0,
           long r1, const T *__restrict__ f, const T *__restrict__ dinv,
           T *__restrict__ u, const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    using A = Ar<T>;
    const int g = threadIdx.x & 7;
    const long nw = ((long)gridDim.x * blockDim.x) >> 5;
    for (long w = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
         r0 + 4 * w < r1; w += nw) {
        const long t = r0 + 4 * w + ((threadIdx.x & 31) >> 3);
        const bool on = t < r1;
        const int row = on ? crows[t] : 0;
        const int a = on ? rowptr[row] : 0, e = on ? rowptr[row + 1] : 0;
        const T sum = row_dot8<T>(a, e, col, val, u, g);
        if (on && g == 0) u[row] = A::add(u[row], A::mul(A::sub(f[row], sum), dinv[row]));
    }
}

// Residual after the pre-sweep, scaled for restriction, four rows per warp:
// rs = (f - A u) / |P row|.
template <class T, class M>
__global__ void __launch_bounds__(256)
k_resid_rs(const int *__restrict__ rowptr, const int *__restrict__ col,
           const M *__restrict__ val, int n, const T *__restrict__ f,
           const T *__restrict__ u, const int *__restrict__ prow,
           T *__restrict__ rs, const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    using A = Ar<T>;
    const int g = threadIdx.x & 7;
    const long nw = ((long)gridDim.x * blockDim.x) >> 5;
    for (long w = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5; 4 * w < n;
         w += nw) {
        const long r = 4 * w + ((threadIdx.x & 31) >> 3);
        const bool on = r < n;
        const int a = on ? rowptr[r] : 0, e = on ? rowptr[r + 1] : 0;
        const T sum = row_dot8<T>(a, e, col, val, u, g);
        if (on && g == 0) {
            const T t = A::sub(f[r], sum);
            const int pc = prow[r + 1] - prow[r];
            rs[r] = pc == 1 ? t : A::div(t, (T)pc);
        }
    }
}

// ---- one launch per Gauss-Seidel sweep -----------------------------------
//
// The colours of a sweep run in one cooperative launch (every block
// resident), separated by a grid barrier, instead of one launch per colour.
// Row work and arithmetic are those of k_gs_init / k_gs_sweep / k_resid_rs,
// so results are bit-identical to them.

// Grid barrier over bar = {arrivals, generation, error}.  The wait is
// bounded: after kBarrierPolls polls the block flags bar[2] (and the CG
// control block, which then reports HMFEM_E_TIMEOUT); every block that sees
// the flag leaves, so a failed barrier never hangs the grid.
constexpr unsigned kBarrierPolls = 1u << 24;

__device__ __forceinline__ bool grid_barrier(unsigned *bar, Ctl *ctl)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *vb = bar;
        const unsigned gen = vb[1];
        __threadfence();
        if (atomicAdd(&bar[0], 1u) == gridDim.x - 1) {
            atomicExch(&bar[0], 0u);
            __threadfence();
            atomicAdd(&bar[1], 1u);
        } else {
            unsigned polls = 0;
            while (vb[1] == gen && vb[2] == 0u) {
                if (++polls > kBarrierPolls) {
                    atomicExch(&bar[2], 1u);
                    if (ctl) { ctl->status = HMFEM_E_TIMEOUT; ctl->done = 1; }
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ((volatile unsigned *)bar)[2] == 0u;
}

// rows [r0, r1) of crows, four per warp, eight threads per row
template <class T, class M>
__device__ __forceinline__ void gs_colour(const int *__restrict__ rowptr,
                                          const int *__restrict__ col,
                                          const M *__restrict__ val,
                                          const int *__restrict__ crows, int r0, int r1,
                                          const T *__restrict__ f,
                                          const T *__restrict__ dinv, T *u)
{
    using A = Ar<T>;
    const int g = threadIdx.x & 7;
    const long nw = ((long)gridDim.x * blockDim.x) >> 5;
    for (long w = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5; r0 + 4 * w < r1;
         w += nw) {
        const long t = r0 + 4 * w + ((threadIdx.x & 31) >> 3);
        const bool on = t < r1;
        const int row = on ? crows[t] : 0;
        const int a = on ? rowptr[row] : 0, e = on ? rowptr[row + 1] : 0;
        const T sum = row_dot8<T, M, true>(a, e, col, val, u, g);
        if (on && g == 0)
            u[row] = A::add(__ldcg(u + row), A::mul(A::sub(f[row], sum), dinv[row]));
    }
}

// Pre-smoothing of a Gauss-Seidel level: forward sweep from zero (colour 0
// = D^-1 f, then colours 1..nc-1), then rs = (f - A u) / |P row|.
template <class T, class M>
__global__ void __launch_bounds__(512)
k_gs_pre_fused(const int *__restrict__ rowptr, const int *__restrict__ col,
               const M *__restrict__ val, int n, const signed char *__restrict__ color,
               const int *__restrict__ crows, const int *__restrict__ cslot, int ncolors,
               const T *__restrict__ f, const T *__restrict__ dinv, T *u,
               const int *__restrict__ prow, T *__restrict__ rs, unsigned *bar, Ctl *ctl)
{
    if (finished(ctl) || ((volatile unsigned *)bar)[2]) return;
    using A = Ar<T>;
    GRID_STRIDE(i, n) u[i] = color[i] == 0 ? A::mul(f[i], dinv[i]) : (T)0;
    for (int c = 1; c < ncolors; c++) {
        if (!grid_barrier(bar, ctl)) return;
        gs_colour<T>(rowptr, col, val, crows, cslot[c], cslot[c + 1], f, dinv, u);
    }
    if (!grid_barrier(bar, ctl)) return;
    const int g = threadIdx.x & 7;
    const long nw = ((long)gridDim.x * blockDim.x) >> 5;
    for (long w = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5; 4 * w < n; w += nw) {
        const long r = 4 * w + ((threadIdx.x & 31) >> 3);
        const bool on = r < n;
        const int a = on ? rowptr[r] : 0, e = on ? rowptr[r + 1] : 0;
        const T sum = row_dot8<T, M, true>(a, e, col, val, u, g);
        if (on && g == 0) {
            const T t = A::sub(f[r], sum);
            const int pc = prow[r + 1] - prow[r];
            rs[r] = pc == 1 ? t : A::div(t, (T)pc);
        }
    }
}

// Post-smoothing of a Gauss-Seidel level: backward sweep, colours nc-1..0.
template <class T, class M>
__global__ void __launch_bounds__(512)
k_gs_post_fused(const int *__restrict__ rowptr, const int *__restrict__ col,
                const M *__restrict__ val, const int *__restrict__ crows,
                const int *__restrict__ cslot, int ncolors, const T *__restrict__ f,
                const T *__restrict__ dinv, T *u, unsigned *bar, Ctl *ctl)
{
    if (finished(ctl) || ((volatile unsigned *)bar)[2]) return;
    for (int c = ncolors - 1; c >= 0; c--) {
        gs_colour<T>(rowptr, col, val, crows, cslot[c], cslot[c + 1], f, dinv, u);
        if (c > 0 && !grid_barrier(bar, ctl)) return;
    }
}

// coarsest level: v = D^-1 f (diagonal_solver, amg.h:1074-1097)
template <class T>
__global__ void k_diag_solve(int n, const T *__restrict__ dinv,
                             const T *__restrict__ f, T *__restrict__ u,
                             const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    using A = Ar<T>;
    GRID_STRIDE(i, n) u[i] = A::mul(dinv[i], f[i]);
}

// Coarse solve by the explicit inverse: u = A^-1 f, a warp per row (FP64
// accumulation, the inverse stored row-major).
template <class T>
__global__ void __launch_bounds__(256)
k_dense_solve(int n, const double *__restrict__ Minv, const T *__restrict__ f,
              T *__restrict__ u, const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    const int lane = threadIdx.x & 31;
    for (long i = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5; i < n;
         i += ((long)gridDim.x * blockDim.x) >> 5) {
        const double *row = Minv + i * (long)n;
        double acc = 0.0;
        for (int j = lane; j < n; j += 32) acc += row[j] * (double)f[j];
        acc = warp_sum(acc);
        if (lane == 0) u[i] = (T)acc;
    }
}

// ---- CG kernels ---------------------------------------------------------

// r = b - A x; rr = (r,r); bb = (b,b)
__global__ void __launch_bounds__(256, 6)
k_resid(const long long *__restrict__ sptr, const int *__restrict__ scol,
        const double *__restrict__ sval, int n, const double *__restrict__ b,
        const double *__restrict__ x, double *__restrict__ r, Ctl *ctl,
        double *part, int init, Seed<double> sd, Demote dm)
{
    PDL_ENTRY();
    // init: 1 = start of the solve, 0 = convergence check (residual
    // replacement), 2 = report only
    if (init == 0 && (finished(ctl) || !ctl->check)) return;
    double rr = 0.0, bb = 0.0;
    GRID_STRIDE(i, n) {
        long q = i >> 5;
        int lane = (int)(i & 31);
        long long base = sptr[q];
        int wd = (int)((sptr[q + 1] - base) >> 5);
        double s = 0.0;
        s = row_acc<double, false>(s, scol, sval, base + lane, wd, [&](int c) { return x[c]; });
        double bi = b[i];
        double ri = dsub(bi, s);
        r[i] = ri;
        if (init != 2) {
            sd.put(i, ri);
            dm.put(i, ri);
        }
        rr += ri * ri;
        bb += bi * bi;
    }
    // two sums: reuse the single-value reduction twice through separate
    // partial rows
    double *p2 = part + kRedBlocks;
    grid_reduce_sum(bb, p2, &ctl->tickets[RED_BB], [&](double s) { ctl->bb = s; });
    grid_reduce_sum(rr, part, &ctl->tickets[RED_TRR],
                    [&](double s) { trr_finish(ctl, s, init); });
}

// v = A s; tau = (s, v); alpha = sigma / tau (pcg.h:59-63)
__global__ void __launch_bounds__(256, 6)
k_spmv_dot(const long long *__restrict__ sptr, const int *__restrict__ scol,
           const double *__restrict__ sval, int n, const double *__restrict__ s,
           double *__restrict__ v, Ctl *ctl, double *part)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    double d = 0.0;
    GRID_STRIDE(i, n) {
        long q = i >> 5;
        int lane = (int)(i & 31);
        long long base = sptr[q];
        int wd = (int)((sptr[q + 1] - base) >> 5);
        double a = 0.0;
        a = row_acc<double, false>(a, scol, sval, base + lane, wd, [&](int c) { return s[c]; });
        v[i] = a;
        d += s[i] * a;
    }
    grid_reduce_sum(d, part, &ctl->tickets[RED_TAU],
                    [&](double t) { tau_finish(ctl, t); });
}

// x += alpha s; r -= alpha v; rr = (r, r)  (pcg.h:64-65)
__global__ void __launch_bounds__(256)
k_update(int n, double *__restrict__ x, double *__restrict__ r,
         const double *__restrict__ s, const double *__restrict__ v, Ctl *ctl,
         double *part, Seed<double> sd, Demote dm)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    const double al = ctl->alpha;
    double rr = 0.0;
    // two cells per thread with 16-byte loads and stores (more bytes in
    // flight per load); the same operations per cell
    auto cell = [&](long i, double xi, double si, double ri, double vi, double &xo,
                    double &ro) {
        xo = dadd(xi, dmul(si, al));
        ro = dsub(ri, dmul(vi, al));
        sd.put(i, ro);
        dm.put(i, ro);
        rr += ro * ro;
    };
    GRID_STRIDE(h, (long)n >> 1) {
        const double2 xv = reinterpret_cast<const double2 *>(x)[h];
        const double2 sv = reinterpret_cast<const double2 *>(s)[h];
        const double2 rv = reinterpret_cast<const double2 *>(r)[h];
        const double2 vv = reinterpret_cast<const double2 *>(v)[h];
        double2 xo, ro;
        cell(2 * h, xv.x, sv.x, rv.x, vv.x, xo.x, ro.x);
        cell(2 * h + 1, xv.y, sv.y, rv.y, vv.y, xo.y, ro.y);
        reinterpret_cast<double2 *>(x)[h] = xo;
        reinterpret_cast<double2 *>(r)[h] = ro;
    }
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const long i = n - 1;
        cell(i, x[i], s[i], r[i], v[i], x[i], r[i]);
    }
    grid_reduce_sum(rr, part, &ctl->tickets[RED_RR], [&](double t) {
        ctl->rr = t;
        int it = ++ctl->iters;
        if (ctl->stop_rule == 0 && t <= ctl->tol2 * ctl->bb) ctl->check = 1;
        if (it >= ctl->max_iter) { ctl->status = HMFEM_E_NOTCONV; ctl->done = 1; }
    });
}

// s = s * beta + z  (scale_add, pcg.h:69); sigma_last = sigma (pcg.h:70).
// beta = 0 (the first direction) reads no s, whose buffer holds nothing yet.
template <class T>
__global__ void __launch_bounds__(256)
k_sdir(int n, double *__restrict__ s, const T *__restrict__ z, Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    const double be = ctl->beta;
    // two cells per thread, 16-byte accesses to s (same operations per cell)
    using Z2 = typename std::conditional<std::is_same<T, double>::value, double2, float2>::type;
    if (be == 0.0) {
        GRID_STRIDE(h, (long)n >> 1) {
            const Z2 zv = reinterpret_cast<const Z2 *>(z)[h];
            reinterpret_cast<double2 *>(s)[h] = make_double2((double)zv.x, (double)zv.y);
        }
    } else {
        GRID_STRIDE(h, (long)n >> 1) {
            const Z2 zv = reinterpret_cast<const Z2 *>(z)[h];
            const double2 sv = reinterpret_cast<const double2 *>(s)[h];
            reinterpret_cast<double2 *>(s)[h] = make_double2(
                dadd(dmul(sv.x, be), (double)zv.x), dadd(dmul(sv.y, be), (double)zv.y));
        }
    }
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const long i = n - 1;
        s[i] = be == 0.0 ? (double)z[i] : dadd(dmul(s[i], be), (double)z[i]);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl->sigma_last = ctl->sigma;
}

// z = (double) src; sigma = (z, r); for the flexible CG also (z, v) with
// v = A s_old, giving beta = -(z, A s_old) / (s_old, A s_old) (one-term
// flexible CG; equals the Polak-Ribiere formula).  Used after an FP32
// V-cycle, and after a V-cycle that ends in the coarsest solve.
template <class T>
__global__ void __launch_bounds__(256)
k_finish_z(int n, const T *__restrict__ src, const double *__restrict__ r,
           const double *__restrict__ v, double *__restrict__ z, Ctl *ctl,
           double *part, int first, int flexible)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    double d1 = 0.0, d2 = 0.0;
    GRID_STRIDE(i, n) {
        double zi = (double)src[i];
        if (z) z[i] = zi;
        d1 += zi * r[i];
        if (flexible && !first) d2 += zi * v[i];
    }
    double *p2 = part + kRedBlocks;
    if (flexible && !first)
        grid_reduce_sum(d2, p2, &ctl->tickets[RED_A], [&](double t) { ctl->rz_old = t; });
    grid_reduce_sum(d1, part, &ctl->tickets[RED_SIGMA],
                    [&](double s) { zdots_finish(ctl, s, first, flexible); });
}

__global__ void k_demote(int n, const double *__restrict__ r, float *__restrict__ f,
                         Seed<float> sd, const Ctl *ctl)
{
    PDL_ENTRY();
    if (finished(ctl)) return;
    GRID_STRIDE(i, n) {
        const float fi = (float)r[i];
        f[i] = fi;
        sd.put(i, fi);
    }
}

// ---- host side ------------------------------------------------------------

static int nb(long n, int threads = 256)
{
    long b = ceil_div(n, threads);
    if (b < 1) b = 1;
    return (int)(b < kRedBlocks ? b : kRedBlocks);
}

// Where a level leaves its correction: ub for Jacobi levels (ping-pong),
// ua for Gauss-Seidel levels (in place) and for the coarse solves.
template <class T>
static T *cycle_out(Solver &s, int l)
{
    const int last = s.nlevels - 1;
    if (l == last || l == s.direct_level || s.lv[l].gs || s.lv[l].cheb) return s.vec_ua<T>(l);
    return s.vec_ub<T>(l);
}

// Chebyshev coefficients on [1/30, 1] (the oracle's cheb_coeffs, same
// expressions, same doubles): 1/theta and, for steps k >= 1, c1_k, c2_k
struct ChebCoef {
    double ith, c1[10], c2[10];
};

static ChebCoef cheb_coef(int K)
{
    const double lo = 1.0 / 30.0, hi = 1.0;
    const double th = (hi + lo) / 2, de = (hi - lo) / 2;
    const double sg = th / de;
    ChebCoef c{};
    double rho = 1.0 / sg;
    c.ith = 1.0 / th;
    for (int k = 1; k < K && k < 10; k++) {
        const double rn = 1.0 / (2.0 * sg - rho);
        c.c1[k] = rn * rho;
        c.c2[k] = 2.0 * rn / de;
        rho = rn;
    }
    return c;
}

// Cooperative launch (all blocks co-resident, as the fused sweeps' grid
// barrier needs), capturable into the CG iteration's graph.
template <class... KArgs, class... Args>
static cudaError_t coop_launch(void (*kernel)(KArgs...), int grid, int block,
                               cudaStream_t st, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Blocks of a fused sweep: at most two 512-thread blocks per SM (fewer
// arrivals per barrier), at most one 32-row pass over n rows, never more
// than can be co-resident.
static int gs_blocks(const void *kernel, long n)
{
    int nsm = 0, dev = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 512, 0);
    if (per_sm > 2) per_sm = 2;
    long b = ceil_div(n, 64);
    const long full = (long)nsm * (per_sm > 0 ? per_sm : 1);
    if (b > full) b = full;
    return (int)(b < 1 ? 1 : b);
}

// The seed (first Jacobi iterate) a producer of level l's right-hand side
// writes: none unless level l is Jacobi-smoothed.
template <class T>
static Seed<T> seed_of(Solver &s, int l)
{
    const int last = s.nlevels - 1;
    if (l >= last || l == s.direct_level || s.lv[l].gs) return {nullptr, nullptr, (T)0};
    if (l == 0 && s.use_schur0()) return {nullptr, nullptr, (T)0};  // not smoothed
    // Chebyshev: the first direction d0 = (1/theta f) D^-1, kept in ub
    if (s.lv[l].cheb)
        return {s.vec_ub<T>(l), s.vec_dinv<T>(l), (T)cheb_coef(s.opt.cheb_degree).ith};
    return {s.vec_ua<T>(l), s.vec_dinv<T>(l), (T)s.opt.omega};
}

template <class T> static T *vec_dx(Solver &s, int l);
template <> double *vec_dx<double>(Solver &s, int l) { return s.lv[l].dx; }
template <> float *vec_dx<float>(Solver &s, int l) { return s.lv[l].dx32; }

// Launches fn(values) with the level's matrix values in the cycle's
// storage type: FP64, FP32, or BF16 on levels >= bf16_from (packed with the
// column offsets, Sell::pk, where they fit).
template <class T, class F>
static void with_vals(Solver &s, const Sell &S, int l, F fn)
{
    if constexpr (std::is_same<T, double>::value) fn(S.val);
    else if (s.use_bf16(l)) {
        if (S.pk) fn((const Pk16 *)S.pk);
        else fn(S.val16);
    } else fn(S.val32);
}

// One V-cycle from level l: f[l] holds the right-hand side, the result is
// left in cycle_out(l).
template <class T>
static int cycle_t(Solver &s, int l, cudaStream_t st, bool dot, bool seeded)
{
    t_klevel = l;
    Level &L = s.lv[l];
    const int last = s.nlevels - 1;
    const int n = L.A.n;
    Ctl *ctl = s.ctl_active ? s.ctl : nullptr;
    T *f = s.vec_f<T>(l), *ua = s.vec_ua<T>(l), *ub = s.vec_ub<T>(l);
    if (l == s.direct_level) {
        launch_pdl(k_dense_solve<T>, (int)ceil_div((long)n * 32, 256), 256, st, n, s.dense_L, f, ua,
                                                                         ctl);
        HM_LAUNCHED();
        return HMFEM_OK;
    }
    if (l == last) {
        launch_pdl(k_diag_solve<T>, nb(n), 256, st, n, s.vec_dtrue<T>(l), f, ua, ctl);
        HM_LAUNCHED();
        return HMFEM_OK;
    }
    if (l == 0 && s.use_schur0()) {
        // exact red-black reduction: coarse right-hand side, V-cycle on the
        // Schur complement, F cells solved with its result
        const T *d0 = s.vec_dtrue<T>(0);
        HM_CHECK((g7_sred<T>(L, f, d0, s.vec_f<T>(1), seed_of<T>(s, 1), ctl, st)));
        HM_CHECK(cycle_t<T>(s, 1, st, false, true));
        t_klevel = l;
        if constexpr (std::is_same<T, float>::value) {
            if (s.fuse_zdots) {
                bool fused = false;
                HM_CHECK((g7_sprol_zd<T>(L, f, d0, cycle_out<T>(s, 1), ub, s.r, s.v, s.ctl,
                                         s.part, s.first_sigma, &fused, st)));
                s.zdots_done = fused;
                return HMFEM_OK;
            }
        }
        HM_CHECK((g7_sprol<T>(L, f, d0, cycle_out<T>(s, 1), ub, ctl, st)));
        return HMFEM_OK;
    }
    const T w = (T)s.opt.omega;
    if (!seeded && seed_of<T>(s, l).u) {
        launch_pdl(k_seed<T>, nb(n), 256, st, n, f, seed_of<T>(s, l));
        HM_LAUNCHED();
    }
    const bool g7 = s.use_g7(l), g19 = s.use_g19(l);
    const bool bf16 = !std::is_same<T, double>::value && s.use_bf16(l);
    T *rs = s.vec_rs<T>(l);
    const T *dv = s.vec_dinv<T>(l);
    const T *dt = s.vec_dtrue<T>(l);
    auto csr_vals = [&](auto fn) {
        if constexpr (std::is_same<T, double>::value) fn(L.A.val);
        else if (s.use_bf16(l)) fn(L.aval16);
        else fn(L.aval32);
    };
    auto sweep = [&](int c) {
        const long r0 = L.color_slot[c], r1 = L.color_slot[c + 1];
        csr_vals([&](auto vals) {
            using M = typename std::remove_const<
                typename std::remove_pointer<decltype(vals)>::type>::type;
            launch_pdl(k_gs_sweep<T, M>, nb(ceil_div(r1 - r0, 4) * 32), 256, st,
                L.A.rowptr, L.A.col, vals, L.crows, r0, r1, f, dt, ua, ctl);
            HM_COUNT();
        });
    };
    // ---- pre-smoothing + residual (scaled for the restriction)
    if (L.gs && s.opt.gs_fused) {
        Ctl *cw = s.ctl_active ? s.ctl : nullptr;
        cudaError_t le = cudaSuccess;
        csr_vals([&](auto vals) {
            using M = typename std::remove_const<
                typename std::remove_pointer<decltype(vals)>::type>::type;
            auto kern = k_gs_pre_fused<T, M>;
            le = coop_launch(kern, gs_blocks((const void *)kern, n), 512, st, L.A.rowptr,
                             L.A.col, vals, n, (const signed char *)L.color,
                             (const int *)L.crows, (const int *)L.cslot, L.ncolors,
                             (const T *)f, dt, ua, (const int *)L.P.rowptr, rs, s.gsbar, cw);
            HM_COUNT();
        });
        HM_CUDA(le);
    } else if (L.gs) {
        launch_pdl(k_gs_init<T>, nb(n), 256, st, n, L.color, f, dt, ua, ctl);
        HM_COUNT();
        for (int c = 1; c < L.ncolors; c++) sweep(c);
        csr_vals([&](auto vals) {
            using M = typename std::remove_const<
                typename std::remove_pointer<decltype(vals)>::type>::type;
            launch_pdl(k_resid_rs<T, M>, nb(ceil_div(n, 4) * 32), 256, st,
                L.A.rowptr, L.A.col, vals, n, f, ua, L.P.rowptr, rs, ctl);
            HM_COUNT();
        });
    } else if (L.cheb) {
        // d0 was seeded into ub by the producer of f; K-1 steps, then the
        // residual for the restriction (r lives in rs until then)
        const int K = s.opt.cheb_degree;
        const ChebCoef cc = cheb_coef(K);
        T *dbuf[2] = {ub, vec_dx<T>(s, l)};
        with_vals<T>(s, L.S, l, [&](auto vals) {
            using M = typename std::remove_const<
                typename std::remove_pointer<decltype(vals)>::type>::type;
            for (int k = 1; k < K; k++) {
                auto kern = k == 1 ? k_cheb_step<T, M, 0> : k_cheb_step<T, M, 2>;
                launch_pdl(kern, nb(n), 256, st, L.S.sptr, L.S.col, vals, n, f, dv,
                           (T)cc.c1[k], (T)cc.c2[k], dbuf[(k - 1) & 1], dbuf[k & 1], rs, ua,
                           (int)(k == K - 1), ctl);
                HM_COUNT();
            }
            launch_pdl(k_pre<T, M>, nb(n), 256, st, L.S.sptr, L.S.col, vals, n, f, ua,
                       L.P.rowptr, rs, ctl);
            HM_COUNT();
        });
    } else if (g7) {
        HM_CHECK((g7_pre<T, T>(L, f, ua, rs, ctl, st)));
    } else if (g19) {
        if (bf16) HM_CHECK((g19_pre<T, __nv_bfloat16>(L, f, ua, rs, ctl, st)));
        else HM_CHECK((g19_pre<T, T>(L, f, ua, rs, ctl, st)));
    } else {
        with_vals<T>(s, L.S, l, [&](auto vals) {
            using M = typename std::remove_const<
                typename std::remove_pointer<decltype(vals)>::type>::type;
            launch_pdl(k_pre<T, M>, nb(n), 256, st, L.S.sptr, L.S.col, vals, n, f, ua,
                                           L.P.rowptr, rs, ctl);
            HM_COUNT();
        });
    }
    HM_LAUNCHED();
    if (g7) {
        HM_CHECK((g7_restrict<T>(L, rs, s.vec_f<T>(l + 1), seed_of<T>(s, l + 1), ctl, st)));
    } else {
        launch_pdl(k_restrict<T>, nb(L.nc), 256, st, L.R.rowptr, L.R.col, L.nc, rs,
                                                s.vec_f<T>(l + 1), seed_of<T>(s, l + 1),
                                                ctl);
        HM_LAUNCHED();
    }
    HM_CHECK(cycle_t<T>(s, l + 1, st, false, true));
    t_klevel = l;
    if (g7) {
        HM_CHECK((g7_prolong<T>(L, cycle_out<T>(s, l + 1), ua, ctl, st)));
    } else {
        launch_pdl(k_prolong_add<T>, nb(n), 256, st, L.P.rowptr, L.P.col, n,
                                                cycle_out<T>(s, l + 1), ua, ctl);
        HM_LAUNCHED();
    }
    // ---- post-smoothing
    if (L.gs && s.opt.gs_fused) {
        Ctl *cw = s.ctl_active ? s.ctl : nullptr;
        cudaError_t le = cudaSuccess;
        csr_vals([&](auto vals) {
            using M = typename std::remove_const<
                typename std::remove_pointer<decltype(vals)>::type>::type;
            auto kern = k_gs_post_fused<T, M>;
            le = coop_launch(kern, gs_blocks((const void *)kern, n), 512, st, L.A.rowptr,
                             L.A.col, vals, (const int *)L.crows, (const int *)L.cslot,
                             L.ncolors, (const T *)f, dt, ua, s.gsbar, cw);
            HM_COUNT();
        });
        HM_CUDA(le);
    } else if (L.gs) {
        for (int c = L.ncolors - 1; c >= 0; c--) sweep(c);
    } else if (L.cheb) {
        const int K = s.opt.cheb_degree;
        const ChebCoef cc = cheb_coef(K);
        T *dbuf[2] = {ub, vec_dx<T>(s, l)};
        with_vals<T>(s, L.S, l, [&](auto vals) {
            using M = typename std::remove_const<
                typename std::remove_pointer<decltype(vals)>::type>::type;
            launch_pdl(k_cheb0<T, M>, nb(n), 256, st, L.S.sptr, L.S.col, vals, n, f, dv,
                       (T)cc.ith, ua, rs, dbuf[0], ctl);
            HM_COUNT();
            for (int k = 1; k < K; k++) {
                auto kern = k == 1 ? k_cheb_step<T, M, 1> : k_cheb_step<T, M, 2>;
                launch_pdl(kern, nb(n), 256, st, L.S.sptr, L.S.col, vals, n, f, dv,
                           (T)cc.c1[k], (T)cc.c2[k], dbuf[(k - 1) & 1], dbuf[k & 1], rs, ua,
                           (int)(k == K - 1), ctl);
                HM_COUNT();
            }
        });
    } else if (g7) {
        if constexpr (std::is_same<T, double>::value) {
            if (dot) HM_CHECK((g7_post<T, T, true>(L, f, dv, w, ua, ub, s.ctl, s.part, s.first_sigma, st)));
            else HM_CHECK((g7_post<T, T, false>(L, f, dv, w, ua, ub, ctl, nullptr, 0, st)));
        } else {
            HM_CHECK((g7_post<T, T, false>(L, f, dv, w, ua, ub, ctl, nullptr, 0, st)));
        }
    } else if (g19 && !dot) {
        if (bf16) HM_CHECK((g19_post<T, __nv_bfloat16>(L, f, dv, w, ua, ub, ctl, st)));
        else HM_CHECK((g19_post<T, T>(L, f, dv, w, ua, ub, ctl, st)));
    } else if (dot) {
        launch_pdl(k_post<T, T, true>, nb(n), 256, st, L.S.sptr, L.S.col, s.sval<T>(l), n,
                                                   f, dv, w, ua, ub, s.ctl, s.part,
                                                   s.first_sigma);
        HM_COUNT();
    } else {
        with_vals<T>(s, L.S, l, [&](auto vals) {
            using M = typename std::remove_const<
                typename std::remove_pointer<decltype(vals)>::type>::type;
            launch_pdl(k_post<T, M, false>, nb(n), 256, st, L.S.sptr, L.S.col, vals, n, f,
                       dv, w, ua, ub, ctl, nullptr, 0);
            HM_COUNT();
        });
    }
    HM_LAUNCHED();
    return HMFEM_OK;
}

int cycle_fp64(Solver &s, int l, cudaStream_t st, bool dot, bool seeded)
{
    return cycle_t<double>(s, l, st, dot, seeded);
}

int cycle_fp32(Solver &s, int l, cudaStream_t st, bool dot, bool seeded)
{
    return cycle_t<float>(s, l, st, dot, seeded);
}

// ---- CG iteration bodies (enqueued once, captured into a graph) -----------

// The FP64 cycle's level-0 seed, written by the CG kernels that produce r
// (the FP32 cycle seeds in k_demote instead)
static Seed<double> cg_seed(Solver &s)
{
    if (s.opt.precision != 0) return {nullptr, nullptr, 0.0};
    return seed_of<double>(s, 0);
}

static Demote cg_demote(Solver &s)
{
    if (s.opt.precision != 1) return {nullptr, {nullptr, nullptr, 0.f}};
    return {s.lv[0].f32, seed_of<float>(s, 0)};
}

static const float *cg_z32(Solver &s)
{
    const bool top_is_coarse = s.nlevels == 1 || s.direct_level == 0;
    return top_is_coarse ? s.lv[0].ua32 : s.lv[0].ub32;
}

// z = C r, sigma = (z, r), beta (fused into the last V-cycle kernel where
// the V-cycle is FP64 and has a coarse level)
int cg_precondition(Solver &s, cudaStream_t st)
{
    Level &L0 = s.lv[0];
    const int n = L0.A.n;
    const bool top_is_coarse = s.nlevels == 1 || s.direct_level == 0;
    if (s.opt.precision == 0) {
        // the V-cycle reads f[0] = r in place; z lands in ub[0] = s.z
        HM_CHECK(cycle_fp64(s, 0, st, !top_is_coarse, true));
        t_klevel = -1;
        if (top_is_coarse) {
            launch_pdl(k_finish_z<double>, nb(n), 256, st, n, L0.ua, s.r, s.v, s.z,
                                                      s.ctl, s.part,
                                                      s.first_sigma, 0);
            HM_LAUNCHED();
        }
        return HMFEM_OK;
    }
    // f32 and its seed were written by the kernel that produced r; the
    // level-0 prolongation of the exact reduction forms the dots of z
    // itself where it can (fuse_zdots), else k_finish_z does
    s.fuse_zdots = true;
    s.zdots_done = false;
    const int rc = cycle_fp32(s, 0, st, false, true);
    s.fuse_zdots = false;
    HM_CHECK(rc);
    t_klevel = -1;
    if (!s.zdots_done) {
        launch_pdl(k_finish_z<float>, nb(n), 256, st, n, cg_z32(s), s.r, s.v,
                   (double *)nullptr, s.ctl, s.part, s.first_sigma, 1);
        HM_LAUNCHED();
    }
    return HMFEM_OK;
}

// s = s beta + z with z the preconditioned residual (FP32 cycle: read as
// FP32 straight from the cycle's output, never stored in FP64)
static int cg_sdir(Solver &s, cudaStream_t st)
{
    const int n = s.lv[0].A.n;
    if (s.opt.precision == 1) launch_pdl(k_sdir<float>, nb(n), 256, st, n, s.s, cg_z32(s), s.ctl);
    else launch_pdl(k_sdir<double>, nb(n), 256, st, n, s.s, (const double *)s.z, s.ctl);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int cg_init(Solver &s, cudaStream_t st)
{
    Level &L0 = s.lv[0];
    const int n = L0.A.n;
    if (s.use_g7(0)) {
        HM_CHECK(g7_resid(L0, s.b, s.x, s.r, s.ctl, s.part, 1, cg_seed(s), cg_demote(s), st));
    } else {
        launch_pdl(k_resid, nb(n), 256, st, L0.S.sptr, L0.S.col, L0.S.val, n, s.b, s.x,
                                       s.r, s.ctl, s.part, 1, cg_seed(s), cg_demote(s));
        HM_LAUNCHED();
    }
    s.first_sigma = 1;
    HM_CHECK(cg_precondition(s, st));
    s.first_sigma = 0;
    HM_CHECK(cg_sdir(s, st));
    return HMFEM_OK;
}

int cg_iteration(Solver &s, cudaStream_t st)
{
    t_klevel = -1;
    Level &L0 = s.lv[0];
    const int n = L0.A.n;
    const bool g7 = s.use_g7(0);
    if (g7) {
        HM_CHECK(g7_spmv_dot(L0, s.s, s.v, s.ctl, s.part, st));
    } else {
        launch_pdl(k_spmv_dot, nb(n), 256, st, L0.S.sptr, L0.S.col, L0.S.val, n, s.s,
                                          s.v, s.ctl, s.part);
        HM_LAUNCHED();
    }
    launch_pdl(k_update, nb(n), 256, st, n, s.x, s.r, s.s, s.v, s.ctl, s.part, cg_seed(s),
               cg_demote(s));
    HM_LAUNCHED();
    if (g7) {
        HM_CHECK(g7_resid(L0, s.b, s.x, s.r, s.ctl, s.part, 0, cg_seed(s), cg_demote(s), st));
    } else {
        launch_pdl(k_resid, nb(n), 256, st, L0.S.sptr, L0.S.col, L0.S.val, n, s.b, s.x,
                                       s.r, s.ctl, s.part, 0, cg_seed(s), cg_demote(s));
        HM_LAUNCHED();
    }
    HM_CHECK(cg_precondition(s, st));
    t_klevel = -1;
    HM_CHECK(cg_sdir(s, st));
    return HMFEM_OK;
}

// final true residual ||b - A x||^2 into ctl->trr (r is overwritten)
int cg_final_residual(Solver &s, cudaStream_t st)
{
    Level &L0 = s.lv[0];
    const int n = L0.A.n;
    if (s.use_g7(0)) {
        HM_CHECK(g7_resid(L0, s.b, s.x, s.r, s.ctl, s.part, 2, Seed<double>{}, Demote{}, st));
    } else {
        launch_pdl(k_resid, nb(n), 256, st, L0.S.sptr, L0.S.col, L0.S.val, n, s.b, s.x,
                                       s.r, s.ctl, s.part, 2, Seed<double>{}, Demote{});
        HM_LAUNCHED();
    }
    return HMFEM_OK;
}

// plain SpMV on level l (inspection / tests)
int level_spmv(Solver &s, int l, const double *x, double *y, cudaStream_t st)
{
    if (s.use_g7(l)) return g7_spmv(s.lv[l], x, y, st);
    if (s.use_g19(l)) return g19_spmv(s.lv[l], x, y, st);
    if (!s.lv[l].S.sptr) HM_CHECK(csr_to_sell(s.lv[l].A, s.lv[l].S, st));
    return launch_spmv(s.lv[l].S, x, y, st);
}

__global__ void k_fill_one(double *x, int n)
{
    GRID_STRIDE(i, n) x[i] = 1.0;
}

// Times `reps` back-to-back launches of one solve-phase kernel on level l
// with CUDA events on the solver stream; returns the mean duration and the
// kernel's algorithmic bytes per launch (no padding, every vector element
// moved once):
//   0 SpMV FP64            nnz*(8+4) + n*(8+8)
//   1 pre-smoother FP64    nnz*(8+4) + n*(8 f + 8 u + 4 P-row + 8 rs)
//   2 post-smoother FP64   nnz*(8+4) + n*(8 f + 8 d + 8 u + 8 u_out)
//   3 pre-smoother FP32    nnz*(4+4) + n*(4 f + 4 u + 4 P-row + 4 rs)
//   4 post-smoother FP32   nnz*(4+4) + n*(4*4)
// (values BF16 on levels >= bf16_from: 2 bytes instead of 4); the SELL
// form is built for the call where the level solves in a structured form.
// Structured forms (level 0: 4 coefficient arrays; level 1: 19 arrays of
// which the in-grid ones count), same vectors as above:
//   5 SpMV FP64 (level 0)           n*4*8 + n*(8+8)
//   6 pre-smoother FP32 (level 0)   n*4*4 + n*(4 f + 4 u + 4 rs)
//   7 post-smoother FP32 (level 0)  n*4*4 + n*4*4
//   8 pre-smoother FP32 (level 1)   nnz*4 + n*(4 f + 4 u + 4 P-row + 4 rs)
//   9 post-smoother FP32 (level 1)  nnz*4 + n*4*4
//  10 Chebyshev step FP32 (coarse level, SELL)  nnz*(4+4) + n*4*7
//  11 Chebyshev step FP64 (coarse level, SELL)  nnz*(8+4) + n*8*7
//     (d gathered, D^-1, r and u read and written, d' written)
// and 12: one whole V-cycle from level l in the solver's precision (bytes
// reported 0); the difference between levels l and l+1 is level l's share.
int time_kernel(Solver &s, int which, int l, int reps, float *ms, double *bytes)
{
    if (which == 12) {
        if (l < 0 || l >= s.nlevels || reps < 1) return HMFEM_E_ARG;
        cudaStream_t st = s.st;
        s.ctl_active = false;
        auto one = [&]() {
            return s.opt.precision == 1 ? cycle_t<float>(s, l, st, false, false)
                                        : cycle_t<double>(s, l, st, false, false);
        };
        HM_CHECK(one());
        cudaEvent_t e0, e1;
        HM_CUDA(cudaEventCreate(&e0));
        HM_CUDA(cudaEventCreate(&e1));
        HM_CUDA(cudaEventRecord(e0, st));
        for (int i = 0; i < reps; i++) HM_CHECK(one());
        HM_CUDA(cudaEventRecord(e1, st));
        HM_CUDA(cudaEventSynchronize(e1));
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms = t / reps;
        *bytes = 0;
        return HMFEM_OK;
    }
    if (l < 0 || l >= s.nlevels || reps < 1 || which < 0 || which > 11) return HMFEM_E_ARG;
    if (which >= 1 && l == s.nlevels - 1) return HMFEM_E_ARG;
    if (((which >= 3 && which <= 4) || (which >= 6 && which <= 10)) && s.opt.precision != 1)
        return HMFEM_E_ARG;
    if (which >= 5 && which <= 7 && !s.use_g7(l)) return HMFEM_E_ARG;
    if (which >= 8 && which <= 9 && (!s.use_g19(l) || s.use_bf16(l))) return HMFEM_E_ARG;
    if (which >= 10 && (!s.lv[l].cheb || s.use_bf16(l))) return HMFEM_E_ARG;
    Level &L = s.lv[l];
    cudaStream_t st = s.st;
    if (l < s.nlevels - 1) HM_CHECK(ensure_p(L, st));
    if (which <= 4 && !L.S.sptr) {
        HM_CHECK(csr_to_sell(L.A, L.S, st));
        if (s.opt.precision == 1) HM_CHECK(sell_fill_lowp(L.S, true, s.use_bf16(l), st));
    }
    const int n = L.A.n;
    const double nnz = (double)L.A.nnz;
    double *x = nullptr, *y = nullptr;
    x = (double *)dalloc(sizeof(double) * n);
    y = (double *)dalloc(sizeof(double) * n);
    if (!x || !y) { dfree(x); dfree(y); return HMFEM_E_CUDA; }
    HM_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
    float *xf = (float *)x, *yf = (float *)y;
    const double w = s.opt.omega;
    const int vb16 = s.use_bf16(l) ? 2 : 4;
    auto launch = [&]() {
        switch (which) {
        case 0:
            k_spmv_dot<<<nb(n), 256, 0, st>>>(L.S.sptr, L.S.col, L.S.val, n, x, y,
                                              s.ctl, s.part);
            break;
        case 1:
            k_pre<double, double><<<nb(n), 256, 0, st>>>(L.S.sptr, L.S.col, L.S.val, n,
                                                         x, L.ua, L.P.rowptr, y, nullptr);
            break;
        case 2:
            k_post<double, double, false><<<nb(n), 256, 0, st>>>(
                L.S.sptr, L.S.col, L.S.val, n, x, L.dsm, w, L.ua, y, nullptr, nullptr, 0);
            break;
        case 3:
            if (vb16 == 2)
                k_pre<float, __nv_bfloat16><<<nb(n), 256, 0, st>>>(
                    L.S.sptr, L.S.col, L.S.val16, n, xf, L.ua32, L.P.rowptr, yf, nullptr);
            else
                k_pre<float, float><<<nb(n), 256, 0, st>>>(
                    L.S.sptr, L.S.col, L.S.val32, n, xf, L.ua32, L.P.rowptr, yf, nullptr);
            break;
        case 5: g7_spmv_dot(L, x, y, s.ctl, s.part, st); break;
        case 6: g7_pre<float, float>(L, xf, L.ua32, yf, nullptr, st); break;
        case 7:
            g7_post<float, float, false>(L, xf, L.dsm32, (float)w, L.ua32, yf, nullptr,
                                         nullptr, 0, st);
            break;
        case 8: g19_pre<float, float>(L, xf, L.ua32, yf, nullptr, st); break;
        case 9: g19_post<float, float>(L, xf, L.dsm32, (float)w, L.ua32, yf, nullptr, st); break;
        case 10:
            k_cheb_step<float, float, 2><<<nb(n), 256, 0, st>>>(
                L.S.sptr, L.S.col, L.S.val32, n, L.f32, L.dsm32, 0.5f, 0.25f, xf, yf,
                L.rs32, L.ua32, 0, nullptr);
            break;
        case 11:
            k_cheb_step<double, double, 2><<<nb(n), 256, 0, st>>>(
                L.S.sptr, L.S.col, L.S.val, n, L.f, L.dsm, 0.5, 0.25, x, y, L.rs, L.ua, 0,
                nullptr);
            break;
        default:
            if (vb16 == 2)
                k_post<float, __nv_bfloat16, false><<<nb(n), 256, 0, st>>>(
                    L.S.sptr, L.S.col, L.S.val16, n, xf, L.dsm32, (float)w, L.ua32,
                    yf, nullptr, nullptr, 0);
            else
                k_post<float, float, false><<<nb(n), 256, 0, st>>>(
                    L.S.sptr, L.S.col, L.S.val32, n, xf, L.dsm32, (float)w, L.ua32,
                    yf, nullptr, nullptr, 0);
        }
    };
    // control block must not be in the finished state for case 0
    HM_CUDA(cudaMemsetAsync(s.ctl, 0, sizeof(Ctl), st));
    // x = 1 keeps (x, A x) > 0, so the fused dot never flags a breakdown
    k_fill_one<<<nb(n), 256, 0, st>>>(x, n);
    launch();
    cudaEvent_t e0, e1;
    HM_CUDA(cudaEventCreate(&e0));
    HM_CUDA(cudaEventCreate(&e1));
    HM_CUDA(cudaEventRecord(e0, st));
    for (int i = 0; i < reps; i++) launch();
    HM_CUDA(cudaEventRecord(e1, st));
    HM_CUDA(cudaEventSynchronize(e1));
    HM_LAUNCHED();
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    dfree(x);
    dfree(y);
    *ms = t / reps;
    switch (which) {
    case 0: *bytes = nnz * 12 + (double)n * 16; break;
    case 1: *bytes = nnz * 12 + (double)n * 28; break;
    case 2: *bytes = nnz * 12 + (double)n * 32; break;
    case 3: *bytes = nnz * (vb16 + 4) + (double)n * 16; break;
    case 4: *bytes = nnz * (vb16 + 4) + (double)n * 16; break;
    case 5: *bytes = (double)n * 48; break;
    case 6: *bytes = (double)n * 28; break;
    case 7: *bytes = (double)n * 32; break;
    case 8: *bytes = nnz * 4 + (double)n * 16; break;
    case 9: *bytes = nnz * 4 + (double)n * 16; break;
    case 10: *bytes = nnz * 8 + (double)n * 4 * 7; break;
    default: *bytes = nnz * 12 + (double)n * 8 * 7; break;
    }
    return HMFEM_OK;
}

}  // namespace hm
