// solver.cu -- the hmfem_* C-ABI: problem upload / assembly, AMG setup
// orchestration, the CG driver loop, flux reconstruction, inspection, and
// the reference's compute() / solve_linsys() entry points on top of them.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <cxxabi.h>

#include <algorithm>

#include "solver.cuh"
#include "cycle.cuh"

namespace hm {

// ---- small kernels used only here --------------------------------------

// Smoother diagonal: kind 0 Jacobi (1/a_ii, last stored diagonal entry as
// amg.h:159-166), kind 1 l1-Jacobi 1/(a_ii + sum_{j!=i} |a_ij|) in row
// order.
__global__ void k_smoother_diag(const int *__restrict__ rowptr,
                                const int *__restrict__ col,
                                const double *__restrict__ val, int n, int kind,
                                double *dsm, float *dsm32)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        double d = 0.0, t = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; k++) {
            if (col[k] == i) d = val[k];
            else t = dadd(t, fabs(val[k]));
        }
        double v = kind == 1 ? 1.0 / dadd(d, t) : 1.0 / d;
        dsm[i] = v;
        dsm32[i] = (float)v;
    }
}

int launch_smoother_diag(const Csr &A, int kind, double *dsm, float *dsm32,
                         cudaStream_t st)
{
    long b = ceil_div(A.n, 256);
    k_smoother_diag<<<(int)(b < 2368 ? (b > 0 ? b : 1) : 2368), 256, 0, st>>>(
        A.rowptr, A.col, A.val, A.n, kind, dsm, dsm32);
    HM_LAUNCHED();
    return HMFEM_OK;
}

// Explicit FP64 inverse of a small SPD level by Gauss-Jordan elimination
// (SPD, so no pivoting): the coarse solve then is a single dense mat-vec.
// Step k maps row i != k to r_i - r_ik (r_k / p) (column k: -r_ik / p) and
// row k to r_k / p (column k: 1 / p), p = r_kk; err = 1 on a non-positive
// pivot.
//
// kGjBlock steps per launch, reading one buffer and writing the other.
// Every CTA first takes the block's pivot rows through the block's steps in
// shared memory -- each becomes its normalised form r_k / p at its own step
// -- then each warp applies the steps in turn to its rows, one at a time in
// shared memory, from those normalised rows.  Entry by entry the operations and
// operands are those of the one-step-per-launch form; 272 launches become
// 17 at the coarse size of a 256^3 grid.
constexpr int kDenseMax = 512;
constexpr int kGjBlock = 16;
constexpr int kGjThreads = 256;

__global__ void k_dense_load(int n, const int *__restrict__ rowptr,
                             const int *__restrict__ col, const double *__restrict__ val,
                             double *M)
{
    const int i = blockIdx.y;
    for (int j = threadIdx.x; j < n; j += blockDim.x) M[(long)i * n + j] = 0.0;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = rowptr[i]; k < rowptr[i + 1]; k++) M[(long)i * n + col[k]] += val[k];
}

__global__ void __launch_bounds__(kGjThreads)
k_gj_block(int n, int k0, int nb, const double *__restrict__ src, double *__restrict__ dst,
           int *err)
{
    // [kGjBlock][n] the pivot rows, then their normalised forms; then one
    // row of n per warp
    extern __shared__ double panel[];
    __shared__ double c_sh[kGjBlock];
    for (int e = threadIdx.x; e < nb * n; e += blockDim.x)
        panel[e] = src[(long)k0 * n + e];
    __syncthreads();
    for (int s = 0; s < nb; s++) {
        const int k = k0 + s;
        double *rk = panel + (long)s * n;
        const double p = rk[k];
        const double pinv = 1.0 / (p > 0.0 ? p : 1.0);
        if (blockIdx.x == 0 && threadIdx.x == 0 && !(p > 0.0)) *err = 1;
        if (threadIdx.x > s && threadIdx.x < nb) c_sh[threadIdx.x] = panel[(long)threadIdx.x * n + k];
        __syncthreads();
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double nj = j == k ? pinv : rk[j] * pinv;
            for (int t = s + 1; t < nb; t++) {
                double *rt = panel + (long)t * n;
                const double c = c_sh[t];
                rt[j] = j == k ? c * -pinv : rt[j] - c * nj;
            }
            rk[j] = nj;
        }
        __syncthreads();
    }
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    double *row = panel + (long)kGjBlock * n + (long)(threadIdx.x >> 5) * n;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        for (int j = lane; j < n; j += 32) row[j] = src[(long)i * n + j];
        __syncwarp();
        for (int s = 0; s < nb; s++) {
            const int k = k0 + s;
            const double *nk = panel + (long)s * n;
            const double c = row[k], pinv = nk[k];
            __syncwarp();
            for (int j = lane; j < n; j += 32)
                row[j] = i == k ? nk[j] : j == k ? c * -pinv : row[j] - c * nk[j];
            __syncwarp();
        }
        for (int j = lane; j < n; j += 32) dst[(long)i * n + j] = row[j];
        __syncwarp();
    }
}

int dense_factor(const Csr &A, double *Lf, int *err, cudaStream_t st)
{
    const int n = A.n;
    if (n <= 0) return HMFEM_OK;
    if (n > kDenseMax) {
        set_last_error("dense coarse solve: level too large", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    double *tmp = (double *)dalloc(sizeof(double) * (size_t)n * n);
    if (!tmp) return HMFEM_E_CUDA;
    const int launches = (int)ceil_div(n, kGjBlock);
    // after the last launch the inverse must land in Lf: start in the other buffer
    double *a = (launches & 1) ? tmp : Lf, *b = (launches & 1) ? Lf : tmp;
    const int th = n < 128 ? 32 * (int)ceil_div(n, 32) : 128;
    k_dense_load<<<dim3(1, n), th, 0, st>>>(n, A.rowptr, A.col, A.val, a);
    HM_LAUNCHED();
    const size_t smem = sizeof(double) * (size_t)(kGjBlock + kGjThreads / 32) * n;
    HM_CUDA(cudaFuncSetAttribute(k_gj_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(double) * (kGjBlock + kGjThreads / 32) * kDenseMax)));
    const int blocks = (int)ceil_div((long)n * 32, kGjThreads);
    for (int k0 = 0; k0 < n; k0 += kGjBlock) {
        const int nb = n - k0 < kGjBlock ? n - k0 : kGjBlock;
        k_gj_block<<<blocks, kGjThreads, smem, st>>>(n, k0, nb, a, b, err);
        HM_LAUNCHED();
        double *t = a; a = b; b = t;
    }
    HM_CUDA(cudaStreamSynchronize(st));
    dfree(tmp);
    return HMFEM_OK;
}

__global__ void k_fill(double *p, long n, double v)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
        p[i] = v;
}

// ---- helpers -------------------------------------------------------------

static void free_csr(Csr &A)
{
    dfree(A.rowptr); dfree(A.col); dfree(A.val);
    A = Csr();
}

static void free_sell(Sell &S)
{
    dfree(S.sptr); dfree(S.col); dfree(S.val); dfree(S.val32); dfree(S.val16); dfree(S.pk);
    S = Sell();
}

// Frees everything built by setup on level l (keeps level 0's matrix).
static void free_level_setup(Level &L, bool keep_matrix)
{
    if (L.sel_ready) {  // a split still running on the side stream
        cudaEventSynchronize(L.sel_ready);
        cudaEventDestroy(L.sel_ready);
        L.sel_ready = nullptr;
    }
    dfree(L.split_work);
    if (!keep_matrix) free_csr(L.A);
    free_sell(L.S);
    dfree(L.dinv); dfree(L.dinv32); dfree(L.dsm); dfree(L.dsm32);
    dfree(L.sel); dfree(L.cid); dfree(L.pw); dfree(L.pw32); dfree(L.cpts);
    free_csr(L.P); free_csr(L.R);
    dfree(L.f); dfree(L.ua); dfree(L.ub); dfree(L.rs);
    dfree(L.f32); dfree(L.ua32); dfree(L.ub32); dfree(L.rs32);
    dfree(L.dx); dfree(L.dx32);
    dfree(L.color); dfree(L.crows); dfree(L.cslot); dfree(L.aval32); dfree(L.aval16);
    g7_free(L.g7);
    g19_free(L.g19);
    Csr a = L.A;
    L = Level();
    if (keep_matrix) L.A = a;
}

static void drop_graph(Solver &s)
{
    if (s.gexec) cudaGraphExecDestroy(s.gexec);
    if (s.graph) cudaGraphDestroy(s.graph);
    s.gexec = nullptr;
    s.graph = nullptr;
}

static void free_hierarchy(Solver &s, bool keep_l0)
{
    drop_graph(s);
    for (size_t l = 0; l < s.lv.size(); l++) free_level_setup(s.lv[l], keep_l0 && l == 0);
    if (!keep_l0) s.lv.clear();
    else s.lv.resize(s.lv.empty() ? 0 : 1);
    dfree(s.dense_L);
    s.dense_L = nullptr;
    s.direct_level = -1;
    s.nlevels = s.lv.size();
    s.setup_done = false;
    s.schur0_built = false;
}

static void free_vectors(Solver &s)
{
    dfree(s.b); dfree(s.x); dfree(s.r); dfree(s.s); dfree(s.v); dfree(s.z);
    s.b = s.x = s.r = s.s = s.v = s.z = nullptr;
}

template <class T> static T *alloc_n(long n)
{
    return (T *)dalloc(sizeof(T) * (n > 0 ? n : 1));
}

#define HM_ALLOC(p, T, n)                                                     \
    do {                                                                      \
        (p) = hm::alloc_n<T>(n);                                              \
        if (!(p)) {                                                           \
            hm::set_last_error("out of device memory", __FILE__, __LINE__);   \
            return HMFEM_E_CUDA;                                              \
        }                                                                     \
    } while (0)

// Copy n elements from host (mem 0) or device (mem 1) into a device buffer.
template <class T>
static int upload(T *dst, const T *src, long n, int mem, cudaStream_t st)
{
    if (n <= 0) return HMFEM_OK;
    HM_CUDA(cudaMemcpyAsync(dst, src, sizeof(T) * n,
                            mem ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                            st));
    return HMFEM_OK;
}

template <class T>
static int download(T *dst, const T *src, long n, int mem, cudaStream_t st)
{
    if (n <= 0) return HMFEM_OK;
    HM_CUDA(cudaMemcpyAsync(dst, src, sizeof(T) * n,
                            mem ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                            st));
    return HMFEM_OK;
}

// flag = 1 if the m 32-bit words at a and b differ anywhere
__global__ void k_words_differ(const unsigned *__restrict__ a, const unsigned *__restrict__ b,
                               long m, int *flag)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < m;
         i += (long)gridDim.x * blockDim.x)
        if (a[i] != b[i]) { *flag = 1; return; }
}

static int words_differ(const void *a, const void *b, long bytes, int *flag, cudaStream_t st)
{
    const long m = bytes / 4;
    if (m <= 0) return HMFEM_OK;
    long nb = ceil_div(m, 256);
    if (nb > 148L * 8) nb = 148L * 8;
    k_words_differ<<<(int)nb, 256, 0, st>>>((const unsigned *)a, (const unsigned *)b, m, flag);
    HM_LAUNCHED();
    return HMFEM_OK;
}

// Setup reuse: compare a candidate level-0 CSR (device arrays) with the
// one the hierarchy was built from; *same = bitwise identical.
static int same_level0(Solver &s, const int *rowptr, const int *col, const double *val,
                       bool *same)
{
    const Csr &A = s.lv[0].A;
    cudaStream_t st = s.st;
    HM_CUDA(cudaMemsetAsync(s.dwork, 0, sizeof(int), st));
    HM_CHECK(words_differ(rowptr, A.rowptr, sizeof(int) * ((long)A.n + 1), s.dwork, st));
    HM_CHECK(words_differ(col, A.col, sizeof(int) * A.nnz, s.dwork, st));
    HM_CHECK(words_differ(val, A.val, sizeof(double) * A.nnz, s.dwork, st));
    int flag = 1;
    HM_CUDA(cudaMemcpyAsync(&flag, s.dwork, sizeof(int), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    *same = flag == 0;
    return HMFEM_OK;
}

static bool can_reuse(const Solver &s, long n, long nnz)
{
    return s.opt.reuse_setup && s.setup_done && !s.have_grid && !s.lv.empty() &&
           s.lv[0].A.n == n && (nnz < 0 || s.lv[0].A.nnz == nnz);
}

static int new_level0(Solver &s, int n)
{
    s.l0_same = false;
    free_hierarchy(s, false);
    free_vectors(s);
    s.lv.resize(1);
    s.nlevels = 1;
    Level &L = s.lv[0];
    L.A.n = n;
    HM_ALLOC(L.A.rowptr, int, (long)n + 1);
    HM_ALLOC(s.b, double, n);
    HM_ALLOC(s.x, double, n);
    HM_ALLOC(s.r, double, n);
    HM_ALLOC(s.s, double, n);
    HM_ALLOC(s.v, double, n);
    HM_ALLOC(s.z, double, n);
    return HMFEM_OK;
}

// ---- setup ------------------------------------------------------------------

static int alloc_level_vectors(Solver &s, Level &L)
{
    const long n = L.A.n;
    HM_ALLOC(L.f, double, n);
    HM_ALLOC(L.ua, double, n);
    HM_ALLOC(L.ub, double, n);
    HM_ALLOC(L.rs, double, n);
    if (s.opt.precision == 1) {
        HM_ALLOC(L.f32, float, n);
        HM_ALLOC(L.ua32, float, n);
        HM_ALLOC(L.ub32, float, n);
        HM_ALLOC(L.rs32, float, n);
    }
    return HMFEM_OK;
}

int setup(Solver &s)
{
    if (s.lv.empty() || !s.lv[0].A.col) {
        set_last_error("no matrix: call hmfem_assemble / hmfem_set_matrix first",
                       __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    if (s.opt.reuse_setup && s.setup_done && s.l0_same) {
        s.l0_same = false;  // one reuse per matrix set
        s.last.setup_reused = 1;
        return HMFEM_OK;
    }
    s.last.setup_reused = 0;
    cudaStream_t st = s.st;
    HM_PHASE(nullptr, st);
    free_hierarchy(s, true);
    HM_PHASE("setup: free", st);
    s.lv.reserve(s.opt.max_levels + 1);
    // level loop (amg.h:1186-1213)
    int l = 0;
    long gcnt = s.lv[0].A.n;
    double rel = 0.0;
    // level 0's diagonal is checked for positivity (flag in dwork[8], read
    // with the last synchronisation of the setup); the Galerkin levels below
    // an SPD level 0 are SPD
    HM_CUDA(cudaMemsetAsync(s.dwork + 8, 0, sizeof(int), st));
    // the stencil form of an assembled level 0 first: the exact reduction's
    // Galerkin level reads its coefficients from it
    const bool low = s.opt.precision == 1;
    if (s.have_grid && s.opt.generic_setup == 0)
        HM_CHECK(g7_build(s.lv[0], s.nx, s.ny, s.nz, low, st, s.dwork));
    for (;;) {
        Level &L = s.lv[l];
        HM_ALLOC(L.dinv, double, L.A.n);
        HM_ALLOC(L.dinv32, float, L.A.n);
        HM_CHECK(launch_diag_inv(L.A, L.dinv, L.dinv32, st, l == 0 ? s.dwork + 8 : nullptr));
        if (!(l < s.opt.max_levels - 1 && gcnt > s.opt.min_coarse && rel < 1.0)) break;
        s.lv.emplace_back();
        const int grid3[3] = {s.nx, s.ny, s.nz};
        const bool stencil = l == 0 && s.have_grid && s.opt.generic_setup == 0;
        const bool schur = stencil && s.opt.schur0 && s.opt.precision == 1;
        HM_CHECK(amg_coarsen(s.lv[l], s.lv[l + 1], st, s.dwork,
                             stencil ? grid3 : nullptr, schur));
        if (schur) s.schur0_built = true;
        l++;
        long gold = gcnt;
        gcnt = s.lv[l].A.n;
        rel = (double)gcnt / (double)gold;
    }
    s.nlevels = l + 1;
    HM_PHASE("setup: hierarchy", st);
    if (s.schur0_built && !s.use_g7(0)) {
        // the reduction needs the stencil form of level 0 (a bitwise
        // symmetric 7-point matrix, which hmfem_assemble always produces)
        set_last_error("schur0: level 0 has no 7-point stencil form", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    // Chebyshev levels: cheb_from and below, above the coarsest
    for (int k = 0; k < s.nlevels; k++)
        s.lv[k].cheb = s.opt.cheb_from >= 1 && k >= s.opt.cheb_from && k < s.nlevels - 1;
    if (s.nlevels > 1 && s.lv[1].g19.v) {
        const bool smoothed = 1 < s.nlevels - 1 && s.opt.gs_from != 1 && !s.lv[1].cheb;
        if (s.use_g7(0) && smoothed)
            HM_CHECK(g19_lowp(s.lv[1].g19, s.lv[1].A.n, low && !s.use_bf16(1),
                              low && s.use_bf16(1), st));
        else
            g19_free(s.lv[1].g19);
    }
    // solve-phase formats and vectors
    for (int k = 0; k < s.nlevels; k++) {
        Level &L = s.lv[k];
        if (!s.use_g7(k) && !s.use_g19(k)) {
            HM_CHECK(csr_to_sell(L.A, L.S, st));
            if (low) HM_CHECK(sell_fill_lowp(L.S, true, s.use_bf16(k), st));
        }
        HM_ALLOC(L.dsm, double, L.A.n);
        HM_ALLOC(L.dsm32, float, L.A.n);
        // Chebyshev levels always use the l1 diagonal (its bound 1 on the
        // spectrum of D^-1 A fixes the Chebyshev interval)
        HM_CHECK(launch_smoother_diag(L.A, L.cheb ? 1 : s.opt.smoother, L.dsm, L.dsm32, st));
        HM_CHECK(alloc_level_vectors(s, L));
        if (L.cheb) {
            HM_ALLOC(L.dx, double, L.A.n);
            if (low) HM_ALLOC(L.dx32, float, L.A.n);
        }
    }
    HM_PHASE("setup: SELL + vectors", st);
    // dense coarse solve on the first level small enough
    s.direct_level = -1;
    if (s.opt.coarse_direct > 0) {
        for (int k = 0; k < s.nlevels; k++) {
            if (s.lv[k].A.n <= s.opt.coarse_direct && s.lv[k].A.n <= kDenseMax) {
                const long n = s.lv[k].A.n;
                HM_ALLOC(s.dense_L, double, n * n);
                HM_CUDA(cudaMemsetAsync(s.dwork, 0, sizeof(int), st));
                HM_CHECK(dense_factor(s.lv[k].A, s.dense_L, s.dwork, st));
                int err = 0;
                HM_CUDA(cudaMemcpyAsync(&err, s.dwork, sizeof(int), cudaMemcpyDeviceToHost, st));
                HM_CUDA(cudaStreamSynchronize(st));
                if (err) {  // not SPD: keep the reference's diagonal solve
                    dfree(s.dense_L);
                    s.dense_L = nullptr;
                } else {
                    s.direct_level = k;
                }
                HM_PHASE("setup: coarse inverse", st);
                break;
            }
        }
    }
    // multicolour Gauss-Seidel on the coarse levels above the coarse solve
    if (s.opt.gs_from >= 1) {
        const int stop = s.direct_level >= 0 ? s.direct_level : s.nlevels - 1;
        for (int k = s.opt.gs_from; k < stop; k++) {
            if (s.lv[k].cheb) continue;
            HM_CHECK(color_level(s.lv[k], st, s.dwork));
            if (s.lv[k].gs && s.opt.precision == 1)
                HM_CHECK(csr_fill_lowp(s.lv[k], s.use_bf16(k), st));
        }
        HM_PHASE("setup: colouring", st);
    }
    int nonpos = 0;
    HM_CUDA(cudaMemcpyAsync(&nonpos, s.dwork + 8, sizeof(int), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    if (nonpos) {
        char msg[160];
        snprintf(msg, sizeof(msg),
                 "matrix is not SPD: diagonal entry of row %d is not positive", nonpos - 1);
        set_last_error(msg, __FILE__, __LINE__);
        return HMFEM_E_BREAKDOWN;
    }
    s.setup_done = true;
    return HMFEM_OK;
}

// ---- solve ------------------------------------------------------------------

static int capture_iteration(Solver &s)
{
    drop_graph(s);
    cudaStream_t cs;
    HM_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    HM_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    const unsigned long long before = t_nlaunch;
    int rc = cg_iteration(s, cs);
    s.graph_kernels = t_nlaunch - before;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (rc != HMFEM_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    HM_CUDA(e);
    s.graph = g;
    HM_CUDA(cudaGraphInstantiate(&s.gexec, g, 0));
    return HMFEM_OK;
}

// the CG control block at the start of a solve
static int ctl_reset(Solver &s, cudaStream_t st)
{
    s.ctl_init = Ctl{};
    s.ctl_init.tol2 = s.opt.tol * s.opt.tol;
    s.ctl_init.max_iter = s.opt.max_iter;
    s.ctl_init.stop_rule = s.opt.stop_rule;
    HM_CUDA(cudaMemcpyAsync(s.ctl, &s.ctl_init, sizeof(Ctl), cudaMemcpyHostToDevice, st));
    HM_CUDA(cudaMemsetAsync(s.gsbar, 0, sizeof(unsigned) * 4, st));
    return HMFEM_OK;
}

static int finish_solve(Solver &s, double *x, int mem, cudaStream_t st, cudaEvent_t e0,
                        cudaEvent_t e1, hmfem_stats *out);

int solve(Solver &s, const double *b, double *x, int mem, hmfem_stats *out)
{
    if (!s.setup_done) HM_CHECK(setup(s));
    cudaStream_t st = s.st;
    const int n = s.lv[0].A.n;
    if (b) HM_CHECK(upload(s.b, b, n, mem, st));
    if (x) HM_CHECK(upload(s.x, (const double *)x, n, mem, st));
    else HM_CUDA(cudaMemsetAsync(s.x, 0, sizeof(double) * n, st));
    HM_CHECK(ctl_reset(s, st));
    cudaEvent_t e0, e1;
    HM_CUDA(cudaEventCreate(&e0));
    HM_CUDA(cudaEventCreate(&e1));
    HM_CUDA(cudaEventRecord(e0, st));
    s.ctl_active = true;
    HM_PHASE(nullptr, st);
    int rc = cg_init(s, st);
    HM_PHASE("solve: init", st);
    if (rc == HMFEM_OK && !s.gexec) rc = capture_iteration(s);
    s.ctl_active = false;
    if (rc != HMFEM_OK) return rc;
    // chunks of k iterations, one chunk kept queued ahead of the host check
    const int k = s.opt.check_every > 0 ? s.opt.check_every : 4;
    cudaEvent_t ev[2];
    HM_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    HM_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    int slot = 0, launched = 0;
    bool pending = false;
    for (;;) {
        for (int i = 0; i < k; i++) {
            HM_CUDA(cudaGraphLaunch(s.gexec, st));
            g_nlaunch += s.graph_kernels;
        }
        launched += k;
        HM_CUDA(cudaMemcpyAsync(&s.ctl_host[slot], s.ctl, sizeof(Ctl),
                                cudaMemcpyDeviceToHost, st));
        HM_CUDA(cudaEventRecord(ev[slot], st));
        if (pending) {
            HM_CUDA(cudaEventSynchronize(ev[slot ^ 1]));
            if (s.ctl_host[slot ^ 1].done) break;
        }
        pending = true;
        slot ^= 1;
        if (launched > s.opt.max_iter + 2 * k) break;
    }
    HM_CUDA(cudaStreamSynchronize(st));
    HM_PHASE("solve: iterations", st);
    cudaEventDestroy(ev[0]); cudaEventDestroy(ev[1]);
    return finish_solve(s, x, mem, st, e0, e1, out);
}

// The end of a solve: the final true residual, x back to the caller, the
// stats (and a message when the device reported a failure).  e0 marks the
// start of the solve on st; both events are destroyed here.
static int finish_solve(Solver &s, double *x, int mem, cudaStream_t st, cudaEvent_t e0,
                        cudaEvent_t e1, hmfem_stats *out)
{
    const int n = s.lv[0].A.n;
    HM_CHECK(cg_final_residual(s, st));
    HM_CUDA(cudaEventRecord(e1, st));
    Ctl ch;
    HM_CUDA(cudaMemcpyAsync(&ch, s.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
    if (x) HM_CHECK(download(x, (const double *)s.x, n, mem, st));
    HM_CUDA(cudaStreamSynchronize(st));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    s.last.iterations = ch.iters;
    s.last.levels = s.nlevels;
    s.last.status = ch.done ? ch.status : HMFEM_E_NOTCONV;
    s.last.relres = ch.bb > 0 ? sqrt(ch.trr / ch.bb) : sqrt(ch.trr);
    s.last.t_solve_ms = ms;
    if (s.opt.stop_rule == 0 && s.last.status == HMFEM_OK &&
        !(s.last.relres <= s.opt.tol))
        s.last.status = HMFEM_E_NOTCONV;
    if (s.last.status != HMFEM_OK) {
        // the device reported the outcome: give it a message of its own
        char msg[200];
        if (s.last.status == HMFEM_E_BREAKDOWN)
            snprintf(msg, sizeof(msg), "CG breakdown after %d iterations: (z, r) or "
                     "(s, A s) is NaN, infinite or zero", ch.iters);
        else if (s.last.status == HMFEM_E_TIMEOUT)
            snprintf(msg, sizeof(msg), "a bounded device wait gave up after %d iterations",
                     ch.iters);
        else
            snprintf(msg, sizeof(msg), "not converged: relres %.3e after %d iterations",
                     s.last.relres, ch.iters);
        set_last_error(msg, __FILE__, __LINE__);
    }
    if (out) *out = s.last;
    return s.last.status;
}

// ---- many solvers solved together -----------------------------------------
//
// Every member is set up on its own.  Then ONE CUDA graph solves them all,
// launched once: for each member a conditional WHILE node whose body is one
// CG iteration of that member (its V-cycle included) followed by a kernel
// that keeps the loop going while the member's control block is not done;
// done is set by the member's own kernels (converged, breakdown, or the
// iteration cap), so every member iterates exactly as long as it needs and
// its result is the one a solve on its own gives.  The WHILE nodes are
// independent, so the members' loops run side by side on the GPU.

__global__ void k_while_next(cudaGraphConditionalHandle h, const Ctl *ctl)
{
    if (threadIdx.x == 0) cudaGraphSetConditional(h, *(volatile const int *)&ctl->done ? 0u : 1u);
}

int batch_solve(Solver *const *ss, int m, double *const *x, int mem, hmfem_stats *out)
{
    if (m <= 0) return HMFEM_OK;
    cudaStream_t ms;
    HM_CUDA(cudaStreamCreateWithFlags(&ms, cudaStreamNonBlocking));
    std::vector<cudaEvent_t> ev(m), ev0(m);
    int rc = HMFEM_OK;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    std::vector<cudaStream_t> cs(m, nullptr);
    auto fail = [&](int r) { if (rc == HMFEM_OK) rc = r; };
    // ---- every member: x, control block, the CG start on its own stream
    for (int i = 0; i < m && rc == HMFEM_OK; i++) {
        Solver &s = *ss[i];
        set_alloc_context(s.st, s.cache);
        if (!s.setup_done) { fail(setup(s)); if (rc) break; }
        const int n = s.lv[0].A.n;
        if (x && x[i]) { fail(upload(s.x, (const double *)x[i], n, mem, s.st)); }
        else if (cudaMemsetAsync(s.x, 0, sizeof(double) * n, s.st) != cudaSuccess) fail(HMFEM_E_CUDA);
        if (rc) break;
        fail(ctl_reset(s, s.st));
        if (cudaEventCreate(&ev0[i]) != cudaSuccess) fail(HMFEM_E_CUDA);
        if (rc) break;
        cudaEventRecord(ev0[i], s.st);
        s.ctl_active = true;
        fail(cg_init(s, s.st));
        s.ctl_active = false;
        if (cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess) fail(HMFEM_E_CUDA);
        if (rc) break;
        cudaEventRecord(ev[i], s.st);
        if (cudaStreamWaitEvent(ms, ev[i], 0) != cudaSuccess) fail(HMFEM_E_CUDA);
    }
    // ---- one graph: a WHILE node per member
    std::vector<unsigned long long> body_kernels(m, 0);
    if (rc == HMFEM_OK && cudaGraphCreate(&graph, 0) != cudaSuccess) fail(HMFEM_E_CUDA);
    for (int i = 0; i < m && rc == HMFEM_OK; i++) {
        Solver &s = *ss[i];
        cudaGraphConditionalHandle h;
        if (cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault) !=
            cudaSuccess) {
            fail(HMFEM_E_CUDA);
            break;
        }
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        if (cudaGraphAddNode(&node, graph, nullptr, 0, &np) != cudaSuccess) {
            fail(HMFEM_E_CUDA);
            break;
        }
        cudaGraph_t body = np.conditional.phGraph_out[0];
        if (cudaStreamCreateWithFlags(&cs[i], cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamBeginCaptureToGraph(cs[i], body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            fail(HMFEM_E_CUDA);
            break;
        }
        const unsigned long long before = t_nlaunch;
        t_nopdl = 1;
        s.ctl_active = true;
        fail(cg_iteration(s, cs[i]));
        s.ctl_active = false;
        t_nopdl = 0;
        k_while_next<<<1, 32, 0, cs[i]>>>(h, s.ctl);
        HM_COUNT();
        body_kernels[i] = t_nlaunch - before;
        g_nlaunch -= body_kernels[i];  // counted per iteration below
        cudaGraph_t captured = nullptr;
        if (cudaStreamEndCapture(cs[i], &captured) != cudaSuccess) fail(HMFEM_E_CUDA);
    }
    if (rc == HMFEM_OK && cudaGraphInstantiate(&gexec, graph, 0) != cudaSuccess)
        fail(HMFEM_E_CUDA);
    // ---- one launch solves every member
    if (rc == HMFEM_OK) {
        if (cudaGraphLaunch(gexec, ms) != cudaSuccess) fail(HMFEM_E_CUDA);
        if (cudaStreamSynchronize(ms) != cudaSuccess) fail(HMFEM_E_CUDA);
    }
    // ---- every member: final residual, x, stats
    int worst = HMFEM_OK;
    if (rc == HMFEM_OK) {
        for (int i = 0; i < m; i++) {
            Solver &s = *ss[i];
            set_alloc_context(s.st, s.cache);
            cudaEvent_t e1;
            cudaEventCreate(&e1);
            // the member's stream after the whole replay
            cudaEvent_t after;
            cudaEventCreateWithFlags(&after, cudaEventDisableTiming);
            cudaEventRecord(after, ms);
            cudaStreamWaitEvent(s.st, after, 0);
            cudaEventDestroy(after);
            const int r = finish_solve(s, x ? x[i] : nullptr, mem, s.st, ev0[i], e1,
                                       out ? out + i : nullptr);
            ev0[i] = nullptr;
            g_nlaunch += (unsigned long long)(s.last.iterations + 1) * body_kernels[i];
            if (r != HMFEM_OK && worst == HMFEM_OK) worst = r;
        }
    }
    for (int i = 0; i < m; i++) {
        if (ev[i]) cudaEventDestroy(ev[i]);
        if (ev0[i]) cudaEventDestroy(ev0[i]);
        if (cs[i]) cudaStreamDestroy(cs[i]);
    }
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamSynchronize(ms);
    cudaStreamDestroy(ms);
    return rc != HMFEM_OK ? rc : worst;
}

// `iters` CG iterations from x = 0, launched without the graph, each
// kernel bracketed by CUDA events on the solver stream; per (kernel,
// level): launches and summed milliseconds.  The solver's x and r are
// overwritten (the next hmfem_solve starts from its own x).
int profile_iteration(Solver &s, int iters, hmfem_kernel_time *out, int cap, int *count)
{
    if (!s.setup_done) HM_CHECK(setup(s));
    cudaStream_t st = s.st;
    const int n = s.lv[0].A.n;
    HM_CUDA(cudaMemsetAsync(s.x, 0, sizeof(double) * n, st));
    HM_CHECK(ctl_reset(s, st));
    s.ctl_active = true;
    int rc = cg_init(s, st);
    std::vector<KRec> recs;
    recs.reserve(2048);
    t_kprof = &recs;
    for (int i = 0; i < iters && rc == HMFEM_OK; i++) rc = cg_iteration(s, st);
    t_kprof = nullptr;
    s.ctl_active = false;
    HM_CUDA(cudaStreamSynchronize(st));
    struct Agg { const void *fn; int level; int launches; double ms; };
    std::vector<Agg> agg;
    for (const KRec &r : recs) {
        float ms = 0;
        cudaEventElapsedTime(&ms, r.e0, r.e1);
        cudaEventDestroy(r.e0);
        cudaEventDestroy(r.e1);
        size_t q = 0;
        while (q < agg.size() && !(agg[q].fn == r.fn && agg[q].level == r.level)) q++;
        if (q == agg.size()) agg.push_back({r.fn, r.level, 0, 0.0});
        agg[q].launches++;
        agg[q].ms += ms;
    }
    HM_CUDA(cudaGetLastError());
    if (rc != HMFEM_OK) return rc;
    const int m = (int)agg.size() < cap ? (int)agg.size() : cap;
    for (int q = 0; q < m; q++) {
        const char *name = nullptr;
        if (cudaFuncGetName(&name, agg[q].fn) != cudaSuccess || !name) name = "?";
        int dst = 0;
        char *dem = abi::__cxa_demangle(name, nullptr, nullptr, &dst);
        snprintf(out[q].name, sizeof(out[q].name), "%s", dem && dst == 0 ? dem : name);
        free(dem);
        out[q].level = agg[q].level;
        out[q].launches = agg[q].launches;
        out[q].ms = agg[q].ms;
    }
    *count = (int)agg.size();
    return HMFEM_OK;
}

int assemble_coupled(Solver &s, const double *KI, const double *WI, const double *pw)
{
    if (!s.have_grid || s.lv.empty() || !s.lv[0].A.val) {
        set_last_error("the coupled matrix needs an assembled grid (hmfem_assemble)",
                       __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    free_hierarchy(s, true);
    Level &L = s.lv[0];
    // same sparsity (the exchange terms only touch the centre): row pointers
    // and columns stay, values and right-hand side are rewritten
    HM_CHECK(launch_assemble(s.nx, s.ny, s.nz, s.hx, s.hy, s.hz, s.visc, s.KX, s.KY,
                             s.KZ, s.bc, s.face, KI, WI, nullptr, pw, L.A.rowptr,
                             L.A.col, L.A.val, s.b, s.st));
    s.setup_done = false;
    s.l0_same = false;
    return HMFEM_OK;
}

}  // namespace hm

using hm::Solver;

// ============================================================================
// C-ABI
// ============================================================================
extern "C" {

void hmfem_default_options(hmfem_options *o)
{
    memset(o, 0, sizeof(*o));
    o->precision = 0;
    o->bf16_from = -1;
    o->smoother = 1;
    o->gs_from = 2;
    o->omega = 1.0;
    o->tol = 1e-10;
    o->stop_rule = 0;
    o->max_iter = 10000;
    o->max_levels = 16;
    o->min_coarse = 1;
    o->coarse_direct = 512;
    o->check_every = 2;
    o->gs_fused = 0;
    o->cheb_from = 2;
    o->cheb_degree = 4;
    o->schur0 = 0;
    o->verbose = 0;
}

int hmfem_create(hmfem_solver **out, const hmfem_options *opt)
{
    if (!out) return HMFEM_E_ARG;
    hmfem_solver *h = new hmfem_solver();
    Solver &s = h->s;
    hm::set_alloc_context(s.st, s.cache);
    if (opt) s.opt = *opt;
    else hmfem_default_options(&s.opt);
    if (s.opt.max_levels < 1 || s.opt.max_levels > 64 || s.opt.tol < 0 ||
        (s.opt.cheb_from >= 1 && (s.opt.cheb_degree < 2 || s.opt.cheb_degree > 9))) {
        delete h;
        hm::set_last_error("invalid options", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    cudaError_t e = cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        hm::set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
        delete h;
        return HMFEM_E_CUDA;
    }
    s.own_stream = true;
    s.cache = hm::alloc_cache_new();
    hm::set_alloc_context(s.st, s.cache);
    const char *ev = getenv("HMFEM_VERBOSE");
    if (s.opt.verbose || (ev && atoi(ev) > 0)) hm::g_verbose = 1;
    s.ctl = (hm::Ctl *)hm::dalloc(sizeof(hm::Ctl));
    s.part = (double *)hm::dalloc(sizeof(double) * hm::kRedBlocks * 2);
    s.dwork = (int *)hm::dalloc(sizeof(int) * 64);
    s.mm = (double *)hm::dalloc(sizeof(double) * 2);
    s.gsbar = (unsigned *)hm::dalloc(sizeof(unsigned) * 4);
    if (cudaMallocHost(&s.ctl_host, 2 * sizeof(hm::Ctl)) != cudaSuccess ||
        !s.ctl || !s.part || !s.dwork || !s.mm || !s.gsbar) {
        hm::set_last_error("out of memory", __FILE__, __LINE__);
        hmfem_destroy(h);
        return HMFEM_E_CUDA;
    }
    cudaMemset(s.ctl, 0, sizeof(hm::Ctl));
    cudaMemset(s.gsbar, 0, sizeof(unsigned) * 4);
    cudaDeviceSynchronize();
    *out = h;
    return HMFEM_OK;
}

int hmfem_destroy(hmfem_solver *h)
{
    if (!h) return HMFEM_OK;
    Solver &s = h->s;
    hm::set_alloc_context(s.st, s.cache);
    if (s.st) cudaStreamSynchronize(s.st);
    hm::karst_release(s);
    hm::free_hierarchy(s, false);
    hm::free_vectors(s);
    for (int i = 0; i < 3; i++) hm::dfree(s.Kown[i]);
    for (int f = 0; f < 6; f++) hm::dfree(s.face[f]);
    hm::dfree(s.ctl); hm::dfree(s.part); hm::dfree(s.dwork); hm::dfree(s.mm);
    hm::dfree(s.gsbar);
    hm::alloc_cache_release(s.cache);
    s.cache = nullptr;
    hm::set_alloc_context(s.st, nullptr);
    if (s.ctl_host) cudaFreeHost(s.ctl_host);
    if (s.st) cudaStreamSynchronize(s.st);
    if (s.own_stream && s.st) cudaStreamDestroy(s.st);
    // the thread's allocation context must not keep naming a dead stream
    hm::set_alloc_context(nullptr, nullptr);
    delete h;
    return HMFEM_OK;
}

int hmfem_set_stream(hmfem_solver *h, void *stream)
{
    if (!h) return HMFEM_E_ARG;
    Solver &s = h->s;
    hm::set_alloc_context(s.st, s.cache);
    cudaStreamSynchronize(s.st);
    if (s.own_stream) cudaStreamDestroy(s.st);
    if (stream) {
        s.st = (cudaStream_t)stream;
        s.own_stream = false;
    } else {
        cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking);
        s.own_stream = true;
    }
    return HMFEM_OK;
}

void *hmfem_get_stream(hmfem_solver *h) { return h ? (void *)h->s.st : nullptr; }

int hmfem_assemble(hmfem_solver *h, int nx, int ny, int nz, double hx,
                   double hy, double hz, double visc, const double *KX,
                   const double *KY, const double *KZ, const int bc_type[6],
                   const double bc_value[6], const double *const *face_vals,
                   int mem)
{
    if (!h || nx < 1 || ny < 1 || nz < 1 || !KX || !KY || !KZ || !bc_type)
        return HMFEM_E_ARG;
    for (int f = 0; f < 6; f++)
        if (bc_type[f] != 0 && bc_type[f] != 1) {
            hm::set_last_error("boundary types must be 0 (Dirichlet) or 1 (Neumann)",
                               __FILE__, __LINE__);
            return HMFEM_E_ARG;
        }
    long n = (long)nx * ny * nz;
    if (n > 2000000000L / 8) {
        hm::set_last_error("grid too large for 32-bit nonzero indices", __FILE__, __LINE__);
        return HMFEM_E_CAPACITY;
    }
    Solver &s = h->s;
    hm::set_alloc_context(s.st, s.cache);
    cudaStream_t st = s.st;
    HM_PHASE(nullptr, st);
    if (!s.have_grid || s.nx != nx || s.ny != ny || s.nz != nz || s.lv.empty() ||
        s.lv[0].A.n != n) {
        HM_CHECK(hm::new_level0(s, (int)n));
        for (int f = 0; f < 6; f++) { hm::dfree(s.face[f]); s.face[f] = nullptr; }
        for (int i = 0; i < 3; i++) { hm::dfree(s.Kown[i]); s.Kown[i] = nullptr; }
    } else {
        hm::free_hierarchy(s, true);
        hm::free_csr(s.lv[0].A);
        s.lv[0].A.n = (int)n;
        HM_ALLOC(s.lv[0].A.rowptr, int, n + 1);
    }
    s.have_grid = true;
    s.nx = nx; s.ny = ny; s.nz = nz;
    s.hx = hx; s.hy = hy; s.hz = hz; s.visc = visc;
    for (int f = 0; f < 6; f++) s.bc[f] = bc_type[f];
    // permeabilities: device pointers are used in place, host arrays copied
    // -- once when the caller passes the same array for several directions
    // (isotropic K, as the reference's Perm fields usually are)
    const double *K[3] = {KX, KY, KZ};
    const double *dK[3] = {KX, KY, KZ};
    for (int i = 0; i < 3; i++) {
        if (mem) {
            hm::dfree(s.Kown[i]);
            s.Kown[i] = nullptr;
            continue;
        }
        int same = -1;
        for (int j = 0; j < i; j++)
            if (K[j] == K[i]) same = j;
        if (same >= 0) {
            hm::dfree(s.Kown[i]);
            s.Kown[i] = nullptr;
            dK[i] = dK[same];
            continue;
        }
        if (!s.Kown[i]) HM_ALLOC(s.Kown[i], double, n);
        HM_CHECK(hm::upload(s.Kown[i], K[i], n, 0, st));
        dK[i] = s.Kown[i];
    }
    s.KX = dK[0];
    s.KY = dK[1];
    s.KZ = dK[2];
    // face values in the Bound layout (l,r: ny*nz; u,d: nx*nz; t,b: nx*ny)
    const long fsz[6] = {(long)ny * nz, (long)ny * nz, (long)nx * nz,
                         (long)nx * nz, (long)nx * ny, (long)nx * ny};
    for (int f = 0; f < 6; f++) {
        if (!s.face[f]) HM_ALLOC(s.face[f], double, fsz[f]);
        if (face_vals && face_vals[f]) {
            HM_CHECK(hm::upload(s.face[f], face_vals[f], fsz[f], mem, st));
        } else {
            double v = bc_value ? bc_value[f] : 0.0;
            hm::k_fill<<<(int)hm::ceil_div(fsz[f], 256) < 1024 ? (int)hm::ceil_div(fsz[f], 256) : 1024,
                         256, 0, st>>>(s.face[f], fsz[f], v);
            HM_LAUNCHED();
        }
    }
    hm::Level &L = s.lv[0];
    HM_PHASE("assemble: buffers + faces", st);
    HM_CHECK(hm::launch_l0_rowcounts(nx, ny, nz, L.A.rowptr, st));
    HM_CHECK(hm::rowptr_from_counts(L.A.rowptr, (int)n, st, &L.A.nnz));
    HM_ALLOC(L.A.col, int, L.A.nnz);
    HM_ALLOC(L.A.val, double, L.A.nnz);
    HM_PHASE("assemble: row pointers", st);
    HM_CUDA(cudaMemsetAsync(s.dwork, 0, sizeof(int), st));
    HM_CHECK(hm::launch_assemble(nx, ny, nz, hx, hy, hz, visc, s.KX, s.KY, s.KZ,
                                 s.bc, s.face, nullptr, nullptr, nullptr,
                                 nullptr, L.A.rowptr, L.A.col, L.A.val, s.b, st,
                                 s.dwork));
    int bad = 0;
    HM_CUDA(cudaMemcpyAsync(&bad, s.dwork, sizeof(int), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    HM_PHASE("assemble: TPFA kernel", st);
    s.setup_done = false;
    s.bad_matrix = bad != 0;
    if (bad) {
        // the matrix holds garbage: no setup, solve or fluxes until a valid
        // matrix is set
        char msg[160];
        snprintf(msg, sizeof(msg),
                 "permeability of cell %d is NaN, infinite or negative", bad - 1);
        hm::set_last_error(msg, __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    return HMFEM_OK;
}

int hmfem_set_matrix(hmfem_solver *h, int n, long nnz, const int *cnt,
                     const int *col, const double *ele, const double *b,
                     int mem)
{
    if (!h || n < 1 || nnz < 1 || !cnt || !col || !ele) return HMFEM_E_ARG;
    if (nnz > 2147483647L) return HMFEM_E_CAPACITY;
    Solver &s = h->s;
    s.bad_matrix = false;
    hm::set_alloc_context(s.st, s.cache);
    cudaStream_t st = s.st;
    if (hm::can_reuse(s, n, nnz)) {
        int *rp = nullptr, *cl = nullptr;
        double *vl = nullptr;
        HM_ALLOC(rp, int, (long)n + 1);
        HM_ALLOC(cl, int, nnz);
        HM_ALLOC(vl, double, nnz);
        HM_CHECK(hm::upload(rp, cnt, n, mem, st));
        long tot = 0;
        HM_CHECK(hm::rowptr_from_counts(rp, n, st, &tot));
        bool same = false;
        if (tot == nnz) {
            HM_CHECK(hm::upload(cl, col, nnz, mem, st));
            HM_CHECK(hm::upload(vl, ele, nnz, mem, st));
            HM_CHECK(hm::same_level0(s, rp, cl, vl, &same));
        }
        hm::dfree(rp); hm::dfree(cl); hm::dfree(vl);
        if (same) {
            if (b) HM_CHECK(hm::upload(s.b, b, n, mem, st));
            else HM_CUDA(cudaMemsetAsync(s.b, 0, sizeof(double) * n, st));
            HM_CUDA(cudaStreamSynchronize(st));
            s.l0_same = true;
            return HMFEM_OK;
        }
    }
    HM_CHECK(hm::new_level0(s, n));
    s.have_grid = false;
    // until the indices are validated the matrix must not be used
    s.bad_matrix = true;
    hm::Level &L = s.lv[0];
    HM_CHECK(hm::upload(L.A.rowptr, cnt, n, mem, st));
    int bad = 0;
    HM_CUDA(cudaMemsetAsync(s.dwork + 9, 0, sizeof(int), st));
    HM_CHECK(hm::launch_validate_counts(L.A.rowptr, n, s.dwork + 9, st));
    HM_CUDA(cudaMemcpyAsync(&bad, s.dwork + 9, sizeof(int), cudaMemcpyDeviceToHost, st));
    long tot = 0;
    HM_CHECK(hm::rowptr_from_counts(L.A.rowptr, n, st, &tot));  // synchronises
    if (bad) {
        hm::set_last_error("negative row count", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    if (tot != nnz) {
        hm::set_last_error("row counts do not add up to hdr[1]", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    L.A.nnz = nnz;
    HM_ALLOC(L.A.col, int, nnz);
    HM_ALLOC(L.A.val, double, nnz);
    HM_CHECK(hm::upload(L.A.col, col, nnz, mem, st));
    HM_CHECK(hm::launch_validate_cols(L.A.col, nnz, n, s.dwork + 9, st));
    HM_CUDA(cudaMemcpyAsync(&bad, s.dwork + 9, sizeof(int), cudaMemcpyDeviceToHost, st));
    HM_CHECK(hm::upload(L.A.val, ele, nnz, mem, st));
    if (b) HM_CHECK(hm::upload(s.b, b, n, mem, st));
    else HM_CUDA(cudaMemsetAsync(s.b, 0, sizeof(double) * n, st));
    HM_CUDA(cudaStreamSynchronize(st));
    if (bad) {
        hm::set_last_error("column index outside [0, n)", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    s.bad_matrix = false;
    return HMFEM_OK;
}

int hmfem_set_stencil(hmfem_solver *h, int nx, int ny, int nz,
                      const hmfem_ele *perm, const hmfem_ind *indcol,
                      const double *b, int mem)
{
    if (!h || nx < 1 || ny < 1 || nz < 1 || !perm || !indcol) return HMFEM_E_ARG;
    long n = (long)nx * ny * nz;
    Solver &s = h->s;
    s.bad_matrix = false;
    hm::set_alloc_context(s.st, s.cache);
    cudaStream_t st = s.st;
    if (hm::can_reuse(s, n, -1)) {
        // pack into scratch and compare with the matrix setup used
        const hmfem_ele *cp = perm;
        const hmfem_ind *ci = indcol;
        hmfem_ele *tp = nullptr;
        hmfem_ind *ti = nullptr;
        if (!mem) {
            HM_ALLOC(tp, hmfem_ele, n);
            HM_ALLOC(ti, hmfem_ind, n);
            HM_CHECK(hm::upload(tp, perm, n, 0, st));
            HM_CHECK(hm::upload(ti, indcol, n, 0, st));
            cp = tp;
            ci = ti;
        }
        int *rp = nullptr;
        HM_ALLOC(rp, int, n + 1);
        HM_CHECK(hm::launch_pack_stencil((int)n, cp, ci, rp, nullptr, nullptr, nullptr, 0, st));
        long nnz = 0;
        HM_CHECK(hm::rowptr_from_counts(rp, (int)n, st, &nnz));
        bool same = false;
        if (nnz == s.lv[0].A.nnz && nnz > 0) {
            int *cl = nullptr;
            double *vl = nullptr;
            HM_ALLOC(cl, int, nnz);
            HM_ALLOC(vl, double, nnz);
            HM_CHECK(hm::launch_pack_stencil((int)n, cp, ci, nullptr, rp, cl, vl, 1, st));
            HM_CHECK(hm::same_level0(s, rp, cl, vl, &same));
            hm::dfree(cl); hm::dfree(vl);
        }
        hm::dfree(rp); hm::dfree(tp); hm::dfree(ti);
        if (same) {
            if (b) HM_CHECK(hm::upload(s.b, b, n, mem, st));
            else HM_CUDA(cudaMemsetAsync(s.b, 0, sizeof(double) * n, st));
            HM_CUDA(cudaStreamSynchronize(st));
            s.l0_same = true;
            return HMFEM_OK;
        }
    }
    HM_CHECK(hm::new_level0(s, (int)n));
    s.have_grid = false;
    const hmfem_ele *dp = perm;
    const hmfem_ind *di = indcol;
    hmfem_ele *tp = nullptr;
    hmfem_ind *ti = nullptr;
    if (!mem) {
        HM_ALLOC(tp, hmfem_ele, n);
        HM_ALLOC(ti, hmfem_ind, n);
        HM_CHECK(hm::upload(tp, perm, n, 0, st));
        HM_CHECK(hm::upload(ti, indcol, n, 0, st));
        dp = tp;
        di = ti;
    }
    hm::Level &L = s.lv[0];
    s.bad_matrix = true;  // until the indices are validated
    int bad = 0;
    HM_CUDA(cudaMemsetAsync(s.dwork + 9, 0, sizeof(int), st));
    HM_CHECK(hm::launch_pack_stencil((int)n, dp, di, L.A.rowptr, nullptr, nullptr,
                                     nullptr, 0, st, s.dwork + 9));
    HM_CUDA(cudaMemcpyAsync(&bad, s.dwork + 9, sizeof(int), cudaMemcpyDeviceToHost, st));
    HM_CHECK(hm::rowptr_from_counts(L.A.rowptr, (int)n, st, &L.A.nnz));  // synchronises
    if (bad) {
        hm::dfree(tp); hm::dfree(ti);
        hm::set_last_error("stencil index outside [-1, n)", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    if (L.A.nnz == 0) {
        hm::dfree(tp); hm::dfree(ti);
        hm::set_last_error("no nonzero elements", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    HM_ALLOC(L.A.col, int, L.A.nnz);
    HM_ALLOC(L.A.val, double, L.A.nnz);
    HM_CHECK(hm::launch_pack_stencil((int)n, dp, di, nullptr, L.A.rowptr, L.A.col,
                                     L.A.val, 1, st));
    if (b) HM_CHECK(hm::upload(s.b, b, n, mem, st));
    else HM_CUDA(cudaMemsetAsync(s.b, 0, sizeof(double) * n, st));
    HM_CUDA(cudaStreamSynchronize(st));
    hm::dfree(tp);
    hm::dfree(ti);
    s.bad_matrix = false;
    return HMFEM_OK;
}

static int refuse_bad_matrix(const hm::Solver &s)
{
    if (!s.bad_matrix) return HMFEM_OK;
    hm::set_last_error("the last matrix assembled or set was rejected; assemble "
                       "or set a valid matrix first", __FILE__, __LINE__);
    return HMFEM_E_ARG;
}

int hmfem_setup(hmfem_solver *h)
{
    if (!h) return HMFEM_E_ARG;
    HM_CHECK(refuse_bad_matrix(h->s));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, h->s.st);
    hm::set_alloc_context(h->s.st, h->s.cache);
    int rc = hm::setup(h->s);
    cudaEventRecord(e1, h->s.st);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    h->s.last.t_setup_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

int hmfem_solve(hmfem_solver *h, const double *b, double *x, int mem,
                hmfem_stats *st)
{
    if (!h) return HMFEM_E_ARG;
    if (h->s.lv.empty()) return HMFEM_E_ARG;
    HM_CHECK(refuse_bad_matrix(h->s));
    hm::set_alloc_context(h->s.st, h->s.cache);
    return hm::solve(h->s, b, x, mem, st);
}

int hmfem_fluxes(hmfem_solver *h, const double *p, hmfem_ele *v, int mem,
                 double *divmin, double *divmax)
{
    if (!h || !p || !v) return HMFEM_E_ARG;
    Solver &s = h->s;
    HM_CHECK(refuse_bad_matrix(s));
    hm::set_alloc_context(s.st, s.cache);
    if (!s.have_grid) {
        hm::set_last_error("fluxes need the grid problem (hmfem_assemble)", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    cudaStream_t st = s.st;
    const long n = (long)s.nx * s.ny * s.nz;
    const double *dp = p;
    hmfem_ele *dv = v;
    if (!mem) {
        HM_CHECK(hm::upload(s.r, p, n, 0, st));
        dp = s.r;
        HM_ALLOC(dv, hmfem_ele, n);
        HM_CHECK(hm::upload(dv, v, n, 0, st));  // keeps the untouched c field
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    HM_CHECK(hm::launch_flux(s.nx, s.ny, s.nz, s.hx, s.hy, s.hz, s.visc, s.KX,
                             s.KY, s.KZ, s.bc, s.face, dp, dv, s.mm, st));
    cudaEventRecord(e1, st);
    double mm[2];
    HM_CUDA(cudaMemcpyAsync(mm, s.mm, sizeof(mm), cudaMemcpyDeviceToHost, st));
    if (!mem) HM_CHECK(hm::download(v, (const hmfem_ele *)dv, n, 0, st));
    HM_CUDA(cudaStreamSynchronize(st));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s.last.t_flux_ms = ms;
    s.last.divmin = mm[0];
    s.last.divmax = mm[1];
    if (divmin) *divmin = mm[0];
    if (divmax) *divmax = mm[1];
    if (!mem) hm::dfree(dv);
    return HMFEM_OK;
}

int hmfem_num_levels(hmfem_solver *h) { return h ? h->s.nlevels : 0; }

int hmfem_level_info(hmfem_solver *h, int l, int *n, long *nnz, long *pnnz)
{
    if (!h || l < 0 || l >= h->s.nlevels) return HMFEM_E_ARG;
    hm::Level &L = h->s.lv[l];
    hm::set_alloc_context(h->s.st, h->s.cache);
    if (l < h->s.nlevels - 1) HM_CHECK(hm::ensure_p(L, h->s.st));
    *n = L.A.n;
    *nnz = L.A.nnz;
    *pnnz = l < h->s.nlevels - 1 ? L.P.nnz : 0;
    return HMFEM_OK;
}

int hmfem_level_copy(hmfem_solver *h, int l, int *cnt, int *col, double *ele,
                     double *dinv, signed char *sel, int *pcnt, int *pcol)
{
    if (!h || l < 0 || l >= h->s.nlevels) return HMFEM_E_ARG;
    Solver &s = h->s;
    hm::set_alloc_context(s.st, s.cache);
    hm::Level &L = s.lv[l];
    cudaStream_t st = s.st;
    if (l < s.nlevels - 1) HM_CHECK(hm::ensure_p(L, st));
    const int n = L.A.n;
    std::vector<int> rp(n + 1);
    HM_CUDA(cudaMemcpyAsync(rp.data(), L.A.rowptr, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, st));
    if (col) HM_CUDA(cudaMemcpyAsync(col, L.A.col, sizeof(int) * L.A.nnz, cudaMemcpyDeviceToHost, st));
    if (ele) HM_CUDA(cudaMemcpyAsync(ele, L.A.val, sizeof(double) * L.A.nnz, cudaMemcpyDeviceToHost, st));
    if (dinv && L.dinv) HM_CUDA(cudaMemcpyAsync(dinv, L.dinv, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    std::vector<int> pr;
    if (l < s.nlevels - 1) {
        if (sel) HM_CUDA(cudaMemcpyAsync(sel, L.sel, n, cudaMemcpyDeviceToHost, st));
        pr.resize(n + 1);
        HM_CUDA(cudaMemcpyAsync(pr.data(), L.P.rowptr, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, st));
        if (pcol) HM_CUDA(cudaMemcpyAsync(pcol, L.P.col, sizeof(int) * L.P.nnz, cudaMemcpyDeviceToHost, st));
    }
    HM_CUDA(cudaStreamSynchronize(st));
    if (cnt) for (int i = 0; i < n; i++) cnt[i] = rp[i + 1] - rp[i];
    if (pcnt && !pr.empty()) for (int i = 0; i < n; i++) pcnt[i] = pr[i + 1] - pr[i];
    return HMFEM_OK;
}

int hmfem_vcycle(hmfem_solver *h, const double *f, double *u, int mem)
{
    if (!h || !f || !u) return HMFEM_E_ARG;
    Solver &s = h->s;
    hm::set_alloc_context(s.st, s.cache);
    if (!s.setup_done) HM_CHECK(hm::setup(s));
    cudaStream_t st = s.st;
    const int n = s.lv[0].A.n;
    // level-0 FP64 cycle reads r and writes z (or ua on a one-level cycle)
    HM_CHECK(hm::upload(s.r, f, n, mem, st));
    s.ctl_active = false;
    const bool top_coarse = s.nlevels == 1 || s.direct_level == 0;
    HM_CUDA(cudaMemsetAsync(s.gsbar, 0, sizeof(unsigned) * 4, st));
    HM_CHECK(hm::cycle_fp64(s, 0, st, false, false));
    HM_CHECK(hm::download(u, (const double *)(top_coarse ? s.lv[0].ua : s.z), n, mem, st));
    unsigned bar[4];
    HM_CUDA(cudaMemcpyAsync(bar, s.gsbar, sizeof(bar), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    if (bar[2]) {
        hm::set_last_error("Gauss-Seidel grid barrier timed out", __FILE__, __LINE__);
        return HMFEM_E_TIMEOUT;
    }
    return HMFEM_OK;
}

int hmfem_spmv(hmfem_solver *h, int level, const double *x, double *y, int mem)
{
    if (!h || level < 0 || !x || !y) return HMFEM_E_ARG;
    Solver &s = h->s;
    hm::set_alloc_context(s.st, s.cache);
    if (level > 0 && !s.setup_done) HM_CHECK(hm::setup(s));
    if (level >= (int)s.lv.size()) return HMFEM_E_ARG;
    cudaStream_t st = s.st;
    hm::Level &L = s.lv[level];
    const int n = L.A.n;
    double *dx = nullptr, *dy = nullptr;
    HM_ALLOC(dx, double, n);
    HM_ALLOC(dy, double, n);
    HM_CHECK(hm::upload(dx, x, n, mem, st));
    HM_CHECK(hm::level_spmv(s, level, dx, dy, st));
    HM_CHECK(hm::download(y, (const double *)dy, n, mem, st));
    HM_CUDA(cudaStreamSynchronize(st));
    hm::dfree(dx);
    hm::dfree(dy);
    return HMFEM_OK;
}

int hmfem_rhs(hmfem_solver *h, double *b, int mem)
{
    if (!h || !b || h->s.lv.empty()) return HMFEM_E_ARG;
    Solver &s = h->s;
    hm::set_alloc_context(s.st, s.cache);
    HM_CHECK(hm::download(b, (const double *)s.b, s.lv[0].A.n, mem, s.st));
    HM_CUDA(cudaStreamSynchronize(s.st));
    return HMFEM_OK;
}

int hmfem_last_stats(hmfem_solver *h, hmfem_stats *st)
{
    if (!h || !st) return HMFEM_E_ARG;
    *st = h->s.last;
    return HMFEM_OK;
}

int hmfem_batch_solve(hmfem_solver *const *solvers, int m, double *const *x, int mem,
                      hmfem_stats *st)
{
    if (m < 0 || (m > 0 && !solvers)) return HMFEM_E_ARG;
    std::vector<Solver *> ss(m);
    for (int i = 0; i < m; i++) {
        if (!solvers[i] || solvers[i]->s.lv.empty()) return HMFEM_E_ARG;
        for (int j = 0; j < i; j++)
            if (solvers[j] == solvers[i]) {
                hm::set_last_error("hmfem_batch_solve: a solver appears twice", __FILE__, __LINE__);
                return HMFEM_E_ARG;
            }
        HM_CHECK(refuse_bad_matrix(solvers[i]->s));
        ss[i] = &solvers[i]->s;
    }
    return hm::batch_solve(ss.data(), m, x, mem, st);
}

int hmfem_profile_iteration(hmfem_solver *h, int iters, hmfem_kernel_time *out, int cap,
                            int *count)
{
    if (!h || iters < 1 || !out || cap < 0 || !count) return HMFEM_E_ARG;
    HM_CHECK(refuse_bad_matrix(h->s));
    if (h->s.lv.empty()) return HMFEM_E_ARG;
    hm::set_alloc_context(h->s.st, h->s.cache);
    return hm::profile_iteration(h->s, iters, out, cap, count);
}

int hmfem_time_kernel(hmfem_solver *h, int which, int level, int reps,
                      float *ms, double *bytes)
{
    if (!h || !ms || !bytes) return HMFEM_E_ARG;
    hm::set_alloc_context(h->s.st, h->s.cache);
    if (!h->s.setup_done) HM_CHECK(hm::setup(h->s));
    return hm::time_kernel(h->s, which, level, reps, ms, bytes);
}

// ---- the reference bridge ---------------------------------------------------

__attribute__((weak)) int iter_amg;

static hmfem_solver *g_bridge = nullptr;

static void bridge_options(hmfem_options *o)
{
    hmfem_default_options(o);
    // compute.cpp:41-42: PCG eps 1e-8 on the preconditioned residual
    o->tol = 1e-8;
    o->stop_rule = 1;
    // the reservoir loop hands the same matrix again on every Picard
    // iteration (main.c:457-514): keep the hierarchy when it is unchanged
    o->reuse_setup = 1;
    const char *t = getenv("HMFEM_TOL");
    if (t) o->tol = atof(t);
    const char *r = getenv("HMFEM_STOP");
    if (r) o->stop_rule = atoi(r);
    const char *p = getenv("HMFEM_PRECISION");
    if (p) o->precision = atoi(p);
}

static int bridge_solver(hmfem_solver **h)
{
    if (!g_bridge) {
        hmfem_options o;
        bridge_options(&o);
        HM_CHECK(hmfem_create(&g_bridge, &o));
    }
    *h = g_bridge;
    return HMFEM_OK;
}

int compute(int *hdr, int *cnt, int *col, double *ele, double *b, double *x)
{
    hmfem_solver *h = nullptr;
    int rc = bridge_solver(&h);
    if (rc == HMFEM_OK) rc = hmfem_set_matrix(h, hdr[0], hdr[1], cnt, col, ele, b, 0);
    hmfem_stats st{};
    if (rc == HMFEM_OK) rc = hmfem_setup(h);
    if (rc == HMFEM_OK) rc = hmfem_solve(h, nullptr, x, 0, &st);
    if (rc != HMFEM_OK && rc != HMFEM_E_NOTCONV)
        fprintf(stderr, "hmfem_gpu compute: status %d: %s\n", rc, hmfem_last_error());
    // pcg.h iterations() counts the final, failing loop test as well
    iter_amg = st.iterations + 1;
    return 0;
}

void solve_linsys(hmfem_ele *perm, hmfem_ind *indcol, double *b, double *x,
                  hmfem_dim N)
{
    hmfem_solver *h = nullptr;
    int rc = bridge_solver(&h);
    if (rc == HMFEM_OK) rc = hmfem_set_stencil(h, N.x, N.y, N.z, perm, indcol, b, 0);
    if (rc == HMFEM_E_ARG && h && h->s.lv.size() == 1 && h->s.lv[0].A.nnz == 0) {
        // solve_linearsystem_AMG.c:92-96
        printf("ERROR: No nonzero elements. \n");
        exit(0);
    }
    hmfem_stats st{};
    if (rc == HMFEM_OK) rc = hmfem_setup(h);
    if (rc == HMFEM_OK) rc = hmfem_solve(h, nullptr, x, 0, &st);
    if (rc != HMFEM_OK && rc != HMFEM_E_NOTCONV)
        fprintf(stderr, "hmfem_gpu solve_linsys: status %d: %s\n", rc, hmfem_last_error());
    iter_amg = st.iterations + 1;
}

}  // extern "C"

// The hmfem application compiles its .c files with g++ (makefile:40-41), so
// its objects reference the C++ names; export those as well.
int compute_cxx(int *hdr, int *cnt, int *col, double *ele, double *b,
                double *x) __asm__("_Z7computePiS_S_PdS0_S0_");
int compute_cxx(int *hdr, int *cnt, int *col, double *ele, double *b, double *x)
{
    return compute(hdr, cnt, col, ele, b, x);
}
struct ELEstruct;
struct Index;
struct Dimension;
void solve_linsys_cxx(hmfem_ele *perm, hmfem_ind *indcol, double *b, double *x,
                      hmfem_dim N) __asm__("_Z12solve_linsysP9ELEstructP5IndexPdS3_9Dimension");
void solve_linsys_cxx(hmfem_ele *perm, hmfem_ind *indcol, double *b, double *x,
                      hmfem_dim N)
{
    solve_linsys(perm, indcol, b, x, N);
}

extern "C" unsigned long long hmfem_launch_count(void) { return hm::g_nlaunch.load(); }
