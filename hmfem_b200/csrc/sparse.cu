// sparse.cu -- scans, CSR -> SELL-32 conversion, diagonal extraction and the
// FP64 SELL SpMV.
#include <cstdlib>
#include <cub/device/device_scan.cuh>
#include <atomic>
#include <map>
#include <mutex>
#include <unordered_map>

#include "hm.cuh"

namespace hm {

// per host thread: solvers driven from several threads report their own
static thread_local char g_err[512];

void set_last_error(const char *msg, const char *file, int line)
{
    snprintf(g_err, sizeof(g_err), "%s (%s:%d)", msg, file, line);
}

int g_verbose = 0;
std::atomic<unsigned long long> g_nlaunch{0};
thread_local unsigned long long t_nlaunch = 0;

void phase_mark(const char *label, cudaStream_t st)
{
    static struct timespec last = {0, 0};
    cudaStreamSynchronize(st);
    struct timespec now;
    clock_gettime(CLOCK_MONOTONIC, &now);
    double ms = (now.tv_sec - last.tv_sec) * 1e3 + (now.tv_nsec - last.tv_nsec) * 1e-6;
    if (last.tv_sec != 0 && label) fprintf(stderr, "[hmfem] %-28s %9.3f ms\n", label, ms);
    last = now;
}

}  // namespace hm

extern "C" const char *hmfem_last_error(void) { return hm::g_err; }

namespace hm {

// Device memory comes from the stream-ordered pool of the current device
// with its release threshold raised, so the buffers a setup frees are handed
// back to the next setup without synchronising cudaMalloc / cudaFree calls.
// the allocation context is per host thread (one solver per thread)
static thread_local cudaStream_t g_astream = nullptr;
static std::atomic<unsigned> g_pool_ready{0};  // bit per device

// Per-solver cache of freed blocks keyed by exact size: a solver that sets
// up the same grid again gets every buffer back without touching the pool.
struct AllocCache {
    std::unordered_map<void *, size_t> live;
    std::multimap<size_t, void *> idle;
};
static thread_local AllocCache *g_cache = nullptr;

void set_alloc_stream(cudaStream_t st) { g_astream = st; }

void set_alloc_context(cudaStream_t st, AllocCache *c)
{
    g_astream = st;
    g_cache = c;
}

void get_alloc_context(cudaStream_t *st, AllocCache **c)
{
    *st = g_astream;
    *c = g_cache;
}

AllocCache *alloc_cache_new() { return new AllocCache(); }

void alloc_cache_release(AllocCache *c)
{
    if (!c) return;
    for (auto &kv : c->idle) cudaFreeAsync(kv.second, g_astream);
    for (auto &kv : c->live) cudaFreeAsync(kv.first, g_astream);
    if (g_cache == c) g_cache = nullptr;
    delete c;
}

static void *pool_alloc(size_t bytes);

// Blocks for a grid-stride kernel over n items: every block the SMs can
// hold at once for this kernel (its register / shared-memory occupancy), so
// the grid is one full wave; fewer when n is small; at most cap.
int occ_blocks(const void *kernel, long n, int threads, int cap)
{
    static std::mutex mu;
    static std::unordered_map<const void *, int> cache;
    static int nsm = 0;
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> g(mu);
        if (nsm == 0) {
            int dev = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            if (nsm <= 0) nsm = 148;
        }
        auto it = cache.find(kernel);
        if (it == cache.end()) {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) !=
                    cudaSuccess || per_sm < 1)
                per_sm = 1;
            cache[kernel] = per_sm;
        } else {
            per_sm = it->second;
        }
    }
    long b = ceil_div(n, threads);
    const long full = (long)nsm * per_sm;
    if (b > full) b = full;
    if (b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

void *dalloc(size_t bytes)
{
    bytes = bytes == 0 ? 256 : (bytes + 255) & ~(size_t)255;
    if (g_cache) {
        auto it = g_cache->idle.find(bytes);
        if (it != g_cache->idle.end()) {
            void *p = it->second;
            g_cache->idle.erase(it);
            g_cache->live[p] = bytes;
            return p;
        }
    }
    void *p = pool_alloc(bytes);
    if (p && g_cache) g_cache->live[p] = bytes;
    return p;
}

static void *pool_alloc(size_t bytes)
{
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 32 && !(g_pool_ready & (1u << dev))) {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            unsigned long long keep = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        g_pool_ready |= 1u << dev;
    }
    void *p = nullptr;
    if (bytes == 0) bytes = 16;
    if (cudaMallocAsync(&p, bytes, g_astream) != cudaSuccess) return nullptr;
    return p;
}

void dfree(void *p)
{
    if (!p) return;
    if (g_cache) {
        auto it = g_cache->live.find(p);
        if (it != g_cache->live.end()) {
            g_cache->idle.insert({it->second, p});
            g_cache->live.erase(it);
            return;
        }
    }
    cudaFreeAsync(p, g_astream);
}

int scan_exclusive(const int *in, int *out, int n, cudaStream_t st)
{
    size_t tmp = 0;
    HM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, n, st));
    void *t = dalloc(tmp);
    if (!t) { set_last_error("out of device memory (scan)", __FILE__, __LINE__); return HMFEM_E_CUDA; }
    cudaError_t e = cub::DeviceScan::ExclusiveSum(t, tmp, in, out, n, st);
    cudaStreamSynchronize(st);
    dfree(t);
    HM_CUDA(e);
    return HMFEM_OK;
}

// rowptr[0..n) holds counts on entry; on exit rowptr[0..n] is the exclusive
// scan with rowptr[n] = total, which is returned in *nnz_out.
int rowptr_from_counts(int *rowptr, int n, cudaStream_t st, long *nnz_out)
{
    int last = 0;
    if (n > 0)
        HM_CUDA(cudaMemcpyAsync(&last, rowptr + n - 1, sizeof(int),
                                cudaMemcpyDeviceToHost, st));
    HM_CHECK(scan_exclusive(rowptr, rowptr, n, st));
    int base = 0;
    if (n > 0)
        HM_CUDA(cudaMemcpyAsync(&base, rowptr + n - 1, sizeof(int),
                                cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    long tot = (long)base + last;
    if (tot > 2147483647L) {
        set_last_error("more than 2^31-1 nonzeros", __FILE__, __LINE__);
        return HMFEM_E_CAPACITY;
    }
    int t32 = (int)tot;
    HM_CUDA(cudaMemcpyAsync(rowptr + n, &t32, sizeof(int),
                            cudaMemcpyHostToDevice, st));
    HM_CUDA(cudaStreamSynchronize(st));
    *nnz_out = tot;
    return HMFEM_OK;
}

namespace {

__global__ void k_slice_len(const int *__restrict__ rowptr, int n, int nslices,
                            long long *slen)
{
    int lane = threadIdx.x & 31;
    for (long q = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
         q < nslices; q += ((long)gridDim.x * blockDim.x) >> 5) {
        long r = q * 32 + lane;
        int len = r < n ? rowptr[r + 1] - rowptr[r] : 0;
        for (int o = 16; o > 0; o >>= 1)
            len = max(len, __shfl_xor_sync(0xffffffffu, len, o));
        if (lane == 0) slen[q] = (long long)len * 32;
    }
}

__global__ void k_sell_fill(const int *__restrict__ rowptr,
                            const int *__restrict__ col,
                            const double *__restrict__ val, int n,
                            long nrows_pad, const long long *__restrict__ sptr,
                            int *scol, double *sval)
{
    for (long r = blockIdx.x * (long)blockDim.x + threadIdx.x; r < nrows_pad;
         r += (long)gridDim.x * blockDim.x) {
        long q = r >> 5;
        int lane = (int)(r & 31);
        long long base = sptr[q];
        int w = (int)((sptr[q + 1] - base) >> 5);
        int a = 0, len = 0;
        if (r < n) { a = rowptr[r]; len = rowptr[r + 1] - a; }
        int self = r < n ? (int)r : 0;
        for (int k = 0; k < w; k++) {
            long long o = base + (long long)k * 32 + lane;
            if (k < len) { scol[o] = col[a + k]; sval[o] = val[a + k]; }
            else { scol[o] = self; sval[o] = 0.0; }
        }
    }
}

__global__ void k_to_lowp(const double *__restrict__ v, long len, float *f32,
                          __nv_bfloat16 *b16)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < len;
         i += (long)gridDim.x * blockDim.x) {
        double x = v[i];
        if (f32) f32[i] = (float)x;
        if (b16) b16[i] = __float2bfloat16((float)x);
    }
}

// Packed BF16 entries (Sell::pk); *bad set when an offset does not fit.
__global__ void k_pack16(const long long *__restrict__ sptr, const int *__restrict__ scol,
                         const __nv_bfloat16 *__restrict__ v16, long nrows_pad,
                         unsigned *pk, int *bad)
{
    for (long r = blockIdx.x * (long)blockDim.x + threadIdx.x; r < nrows_pad;
         r += (long)gridDim.x * blockDim.x) {
        const long long base = sptr[r >> 5];
        const int w = (int)((sptr[(r >> 5) + 1] - base) >> 5);
        for (int k = 0; k < w; k++) {
            const long long o = base + (long long)k * 32 + (r & 31);
            long d = (long)scol[o] - r;
            if (d < -32768 || d > 32767) { *bad = 1; d = 0; }
            pk[o] = ((unsigned)(d & 0xffff) << 16) | (unsigned)__bfloat16_as_ushort(v16[o]);
        }
    }
}

// amg.h:159-166 / 1216-1225: the LAST stored diagonal entry wins.
__global__ void k_diag_inv(const int *__restrict__ rowptr,
                           const int *__restrict__ col,
                           const double *__restrict__ val, int n, double *dinv,
                           float *dinv32, int *bad)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        double d = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; k++)
            if (col[k] == i) d = val[k];
        // an SPD matrix has a positive diagonal: flag one row that has not
        // (zero, negative or NaN) as 1 + its index
        if (bad && !(d > 0.0)) atomicExch(bad, (int)(i + 1));
        double v = 1.0 / d;
        dinv[i] = v;
        if (dinv32) dinv32[i] = (float)v;
    }
}

// y = A x, one thread per row, row order kept (generic_operator.h:230-245).
__global__ void __launch_bounds__(256)
k_spmv(const long long *__restrict__ sptr, const int *__restrict__ scol,
       const double *__restrict__ sval, int n, const double *__restrict__ x,
       double *__restrict__ y)
{
    for (long r = blockIdx.x * (long)blockDim.x + threadIdx.x; r < n;
         r += (long)gridDim.x * blockDim.x) {
        long q = r >> 5;
        int lane = (int)(r & 31);
        long long base = sptr[q];
        int w = (int)((sptr[q + 1] - base) >> 5);
        double s = 0.0;
        for (int k = 0; k < w; k++) {
            long long o = base + (long long)k * 32 + lane;
            s = dadd(s, dmul(sval[o], x[scol[o]]));
        }
        y[r] = s;
    }
}

int nblocks(long n, int threads, long cap = 148L * 16)
{
    long b = ceil_div(n, threads);
    if (b < 1) b = 1;
    return (int)(b < cap ? b : cap);
}

}  // namespace

int csr_to_sell(const Csr &A, Sell &S, cudaStream_t st)
{
    S.n = A.n;
    S.nslices = (int)ceil_div(A.n, 32);
    S.sptr = (long long *)dalloc(sizeof(long long) * (S.nslices + 1));
    if (!S.sptr) { set_last_error("out of device memory (sell)", __FILE__, __LINE__); return HMFEM_E_CUDA; }
    k_slice_len<<<nblocks((long)S.nslices * 32, 256), 256, 0, st>>>(
        A.rowptr, A.n, S.nslices, S.sptr);
    HM_LAUNCHED();
    size_t tmp = 0;
    HM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, S.sptr, S.sptr,
                                          S.nslices + 1, st));
    void *t = dalloc(tmp);
    HM_CUDA(cudaMemsetAsync(S.sptr + S.nslices, 0, sizeof(long long), st));
    HM_CUDA(cub::DeviceScan::ExclusiveSum(t, tmp, S.sptr, S.sptr,
                                          S.nslices + 1, st));
    long long len = 0;
    HM_CUDA(cudaMemcpyAsync(&len, S.sptr + S.nslices, sizeof(long long),
                            cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    dfree(t);
    S.len = len;
    S.col = (int *)dalloc(sizeof(int) * (len > 0 ? len : 1));
    S.val = (double *)dalloc(sizeof(double) * (len > 0 ? len : 1));
    if (!S.col || !S.val) { set_last_error("out of device memory (sell)", __FILE__, __LINE__); return HMFEM_E_CUDA; }
    k_sell_fill<<<nblocks((long)S.nslices * 32, 256), 256, 0, st>>>(
        A.rowptr, A.col, A.val, A.n, (long)S.nslices * 32, S.sptr, S.col, S.val);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int sell_fill_lowp(Sell &S, bool f32, bool bf16, cudaStream_t st)
{
    if (f32 && !S.val32) S.val32 = (float *)dalloc(sizeof(float) * (S.len > 0 ? S.len : 1));
    if (bf16 && !S.val16) S.val16 = (__nv_bfloat16 *)dalloc(2 * (S.len > 0 ? S.len : 1));
    k_to_lowp<<<nblocks(S.len, 256), 256, 0, st>>>(S.val, S.len,
                                                   f32 ? S.val32 : nullptr,
                                                   bf16 ? S.val16 : nullptr);
    HM_LAUNCHED();
    // HMFEM_PACK16=0 keeps the col + val16 form (the packed one computes the
    // same terms in the same order: a check of the packing)
    const char *pe = getenv("HMFEM_PACK16");
    if (bf16 && !S.pk && S.len > 0 && !(pe && atoi(pe) == 0)) {
        S.pk = (unsigned *)dalloc(sizeof(unsigned) * S.len);
        int *bad = (int *)dalloc(sizeof(int));
        if (!S.pk || !bad) { dfree(S.pk); dfree(bad); S.pk = nullptr; return HMFEM_E_CUDA; }
        HM_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), st));
        k_pack16<<<nblocks((long)S.nslices * 32, 256), 256, 0, st>>>(
            S.sptr, S.col, S.val16, (long)S.nslices * 32, S.pk, bad);
        HM_LAUNCHED();
        int hb = 0;
        HM_CUDA(cudaMemcpyAsync(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
        HM_CUDA(cudaStreamSynchronize(st));
        dfree(bad);
        if (hb) {  // columns too far from their rows: the col + val16 form
            dfree(S.pk);
            S.pk = nullptr;
        }
    }
    return HMFEM_OK;
}

int csr_fill_lowp(Level &L, bool bf16, cudaStream_t st)
{
    const long len = L.A.nnz;
    if (!L.aval32) L.aval32 = (float *)dalloc(sizeof(float) * (len > 0 ? len : 1));
    if (bf16 && !L.aval16) L.aval16 = (__nv_bfloat16 *)dalloc(2 * (len > 0 ? len : 1));
    if (!L.aval32 || (bf16 && !L.aval16)) return HMFEM_E_CUDA;
    k_to_lowp<<<nblocks(len, 256), 256, 0, st>>>(L.A.val, len, L.aval32,
                                                 bf16 ? L.aval16 : nullptr);
    HM_LAUNCHED();
    return HMFEM_OK;
}

// Index validation of a caller's row-by-count matrix before any kernel
// indexes with it: a negative count flags bad[0] = 1, a column outside
// [0, n) bad[0] = 2 (the reference reads such indices unchecked).
__global__ void k_validate_counts(const int *__restrict__ cnt, int n, int *bad)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
        if (cnt[i] < 0) atomicExch(bad, 1);
}

__global__ void k_validate_cols(const int *__restrict__ col, long nnz, int n, int *bad)
{
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < nnz;
         k += (long)gridDim.x * blockDim.x) {
        const int c = col[k];
        if (c < 0 || c >= n) atomicExch(bad, 2);
    }
}

int launch_validate_counts(const int *cnt, int n, int *bad, cudaStream_t st)
{
    k_validate_counts<<<nblocks(n, 256), 256, 0, st>>>(cnt, n, bad);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int launch_validate_cols(const int *col, long nnz, int n, int *bad, cudaStream_t st)
{
    k_validate_cols<<<nblocks(nnz, 256), 256, 0, st>>>(col, nnz, n, bad);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int launch_diag_inv(const Csr &A, double *dinv, float *dinv32, cudaStream_t st,
                    int *bad)
{
    k_diag_inv<<<nblocks(A.n, 256), 256, 0, st>>>(A.rowptr, A.col, A.val, A.n,
                                                   dinv, dinv32, bad);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int launch_spmv(const Sell &S, const double *x, double *y, cudaStream_t st)
{
    k_spmv<<<nblocks(S.n, 256), 256, 0, st>>>(S.sptr, S.col, S.val, S.n, x, y);
    HM_LAUNCHED();
    return HMFEM_OK;
}

}  // namespace hm
