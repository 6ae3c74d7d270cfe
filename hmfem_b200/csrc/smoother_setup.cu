// smoother_setup.cu -- setup of the multicolour Gauss-Seidel smoother used on
// the coarse levels: a colouring and a SELL-32
// copy of the level with rows grouped by colour, so one colour is one
// coalesced, conflict-free kernel.
//
// The colouring is Jones-Plassmann with fixed pseudo-random priorities
// (a round per launch, double-buffered, so the result is deterministic and
// the oracle reproduces it exactly).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "hm.cuh"

namespace hm {

namespace {

constexpr int kTile = 256;
constexpr int kMaxColors = 63;

// Jones-Plassmann colouring, one round: a row still uncoloured (old < 0)
// whose (priority, index) key beats every uncoloured neighbour's takes the
// smallest colour not used by its coloured neighbours.  Reads `old`, writes
// `nw` (double-buffered rounds), so the result is order-independent.
__device__ __forceinline__ unsigned long long jp_key(int v)
{
    unsigned x = (unsigned)v;
    x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16;
    return ((unsigned long long)x << 32) | (unsigned)v;
}

__global__ void __launch_bounds__(kTile)
k_jp_round(const int *__restrict__ rowptr, const int *__restrict__ col, int n,
           const signed char *__restrict__ old, signed char *__restrict__ nw,
           int *left, int *ncol, int *err)
{
    for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < n;
         v += (long)gridDim.x * blockDim.x) {
        signed char cv = old[v];
        if (cv >= 0) { nw[v] = cv; continue; }
        const unsigned long long kv = jp_key((int)v);
        unsigned long long used = 0;
        bool ok = true;
        for (int k = rowptr[v]; k < rowptr[v + 1]; k++) {
            int u = col[k];
            if (u == v) continue;
            signed char c = old[u];
            if (c >= 0) used |= 1ull << c;
            else if (jp_key(u) > kv) { ok = false; break; }
        }
        if (!ok) { nw[v] = -1; continue; }
        int c = __ffsll((long long)~used) - 1;
        if (c < 0 || c >= kMaxColors) { atomicExch(err, 2); c = kMaxColors; }
        nw[v] = (signed char)c;
        atomicSub(left, 1);
        atomicMax(ncol, c + 1);
    }
}

__global__ void k_color_key(const signed char *__restrict__ color, int n,
                            int *key, int *row)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        key[i] = color[i];
        row[i] = (int)i;
    }
}

__global__ void k_color_hist(const signed char *__restrict__ color, int n,
                             int *cnt)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
        atomicAdd(cnt + color[i], 1);
}

// cperm[slot]: the rows of colour c occupy slots [dst[c], dst[c] + cnt[c]),
// padded with -1 up to dst[c+1] (a multiple of 32).
__global__ void k_cperm(const int *__restrict__ sorted_rows,
                        const long *__restrict__ src, const long *__restrict__ dst,
                        int ncolors, long nslots, int *cperm)
{
    for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < nslots;
         s += (long)gridDim.x * blockDim.x) {
        int c = 0;
        while (c + 1 < ncolors && dst[c + 1] <= s) c++;
        long k = s - dst[c];
        long cnt = src[c + 1] - src[c];
        cperm[s] = k < cnt ? sorted_rows[src[c] + k] : -1;
    }
}

__global__ void k_cslice_len(const int *__restrict__ rowptr,
                             const int *__restrict__ cperm, long nslices,
                             long long *slen)
{
    const int lane = threadIdx.x & 31;
    for (long q = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5; q < nslices;
         q += ((long)gridDim.x * blockDim.x) >> 5) {
        int r = cperm[q * 32 + lane];
        int len = r >= 0 ? rowptr[r + 1] - rowptr[r] : 0;
        for (int o = 16; o > 0; o >>= 1)
            len = max(len, __shfl_xor_sync(0xffffffffu, len, o));
        if (lane == 0) slen[q] = (long long)len * 32;
    }
}

__global__ void k_csell_fill(const int *__restrict__ rowptr,
                             const int *__restrict__ col,
                             const double *__restrict__ val,
                             const int *__restrict__ cperm, long nslots,
                             const long long *__restrict__ sptr, int *scol,
                             double *sval)
{
    for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < nslots;
         s += (long)gridDim.x * blockDim.x) {
        long q = s >> 5;
        int lane = (int)(s & 31);
        long long base = sptr[q];
        int w = (int)((sptr[q + 1] - base) >> 5);
        int r = cperm[s];
        int a = 0, len = 0;
        if (r >= 0) { a = rowptr[r]; len = rowptr[r + 1] - a; }
        for (int k = 0; k < w; k++) {
            long long o = base + (long long)k * 32 + lane;
            if (k < len) { scol[o] = col[a + k]; sval[o] = val[a + k]; }
            else { scol[o] = 0; sval[o] = 0.0; }
        }
    }
}

int nb(long n, int threads = 256, long cap = 148L * 16)
{
    long b = ceil_div(n, threads);
    if (b < 1) b = 1;
    return (int)(b < cap ? b : cap);
}

}  // namespace

int color_level(Level &L, cudaStream_t st, int *dwork)
{
    const int n = L.A.n;
    L.gs = false;
    if (n < 1) return HMFEM_OK;
    L.color = (signed char *)dalloc(n);
    signed char *tmpc = (signed char *)dalloc(n);
    if (!L.color || !tmpc) return HMFEM_E_CUDA;
    HM_CUDA(cudaMemsetAsync(L.color, 0xff, n, st));
    int h0[3] = {n, 0, 0};  // left, colours, error
    HM_CUDA(cudaMemcpyAsync(dwork, h0, sizeof(h0), cudaMemcpyHostToDevice, st));
    signed char *a = L.color, *b = tmpc;
    int h[3] = {n, 0, 0};
    for (int round = 0; round < 4096 && h[0] > 0; round++) {
        k_jp_round<<<nb(n), kTile, 0, st>>>(L.A.rowptr, L.A.col, n, a, b, dwork,
                                            dwork + 1, dwork + 2);
        HM_CUDA(cudaGetLastError());
        signed char *t = a; a = b; b = t;
        if ((round & 3) == 3 || round < 4) {
            HM_CUDA(cudaMemcpyAsync(h, dwork, sizeof(h), cudaMemcpyDeviceToHost, st));
            HM_CUDA(cudaStreamSynchronize(st));
        }
    }
    if (a != L.color) HM_CUDA(cudaMemcpyAsync(L.color, a, n, cudaMemcpyDeviceToDevice, st));
    HM_CUDA(cudaMemcpyAsync(h, dwork, sizeof(h), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    dfree(tmpc);
    if (h[0] > 0) {
        set_last_error("colouring did not finish", __FILE__, __LINE__);
        return HMFEM_E_TIMEOUT;
    }
    if (h[2] == 2) return HMFEM_OK;  // over 63 colours: keep l1-Jacobi here
    const int nc = h[1];
    // rows grouped by colour (stable: ascending within a colour)
    int *key = (int *)dalloc(sizeof(int) * n), *row = (int *)dalloc(sizeof(int) * n);
    int *skey = (int *)dalloc(sizeof(int) * n), *srow = (int *)dalloc(sizeof(int) * n);
    int *hist = (int *)dalloc(sizeof(int) * 64);
    if (!key || !row || !skey || !srow || !hist) return HMFEM_E_CUDA;
    k_color_key<<<nb(n), 256, 0, st>>>(L.color, n, key, row);
    HM_CUDA(cudaMemsetAsync(hist, 0, sizeof(int) * 64, st));
    k_color_hist<<<nb(n), 256, 0, st>>>(L.color, n, hist);
    {
        size_t tmp = 0;
        HM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, key, skey, row, srow, n, 0, 6, st));
        void *t = dalloc(tmp);
        HM_CUDA(cub::DeviceRadixSort::SortPairs(t, tmp, key, skey, row, srow, n, 0, 6, st));
        dfree(t);
    }
    int hh[64];
    HM_CUDA(cudaMemcpyAsync(hh, hist, sizeof(int) * 64, cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    std::vector<long> src(nc + 1), dst(nc + 1);
    src[0] = dst[0] = 0;
    for (int c = 0; c < nc; c++) {
        src[c + 1] = src[c] + hh[c];
        dst[c + 1] = dst[c] + ceil_div(hh[c], 32) * 32;
    }
    const long nslots = dst[nc];
    long *dsrc = (long *)dalloc(sizeof(long) * (nc + 1));
    long *ddst = (long *)dalloc(sizeof(long) * (nc + 1));
    L.cperm = (int *)dalloc(sizeof(int) * nslots);
    if (!dsrc || !ddst || !L.cperm) return HMFEM_E_CUDA;
    HM_CUDA(cudaMemcpyAsync(dsrc, src.data(), sizeof(long) * (nc + 1), cudaMemcpyHostToDevice, st));
    HM_CUDA(cudaMemcpyAsync(ddst, dst.data(), sizeof(long) * (nc + 1), cudaMemcpyHostToDevice, st));
    k_cperm<<<nb(nslots), 256, 0, st>>>(srow, dsrc, ddst, nc, nslots, L.cperm);
    HM_CUDA(cudaGetLastError());
    // SELL over the colour-ordered slots
    Sell &S = L.CS;
    S.n = (int)nslots;
    S.nslices = (int)(nslots / 32);
    S.sptr = (long long *)dalloc(sizeof(long long) * (S.nslices + 1));
    k_cslice_len<<<nb((long)S.nslices * 32), 256, 0, st>>>(L.A.rowptr, L.cperm,
                                                           S.nslices, S.sptr);
    HM_CUDA(cudaGetLastError());
    HM_CUDA(cudaMemsetAsync(S.sptr + S.nslices, 0, sizeof(long long), st));
    {
        size_t tmp = 0;
        HM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, S.sptr, S.sptr, S.nslices + 1, st));
        void *t = dalloc(tmp);
        HM_CUDA(cub::DeviceScan::ExclusiveSum(t, tmp, S.sptr, S.sptr, S.nslices + 1, st));
        dfree(t);
    }
    long long len = 0;
    HM_CUDA(cudaMemcpyAsync(&len, S.sptr + S.nslices, sizeof(long long), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    S.len = len;
    S.col = (int *)dalloc(sizeof(int) * (len > 0 ? len : 1));
    S.val = (double *)dalloc(sizeof(double) * (len > 0 ? len : 1));
    if (!S.col || !S.val) return HMFEM_E_CUDA;
    k_csell_fill<<<nb(nslots), 256, 0, st>>>(L.A.rowptr, L.A.col, L.A.val, L.cperm,
                                             nslots, S.sptr, S.col, S.val);
    HM_CUDA(cudaGetLastError());
    dfree(key); dfree(row); dfree(skey); dfree(srow); dfree(hist);
    dfree(dsrc); dfree(ddst);
    L.ncolors = nc;
    L.color_slot = dst;
    L.gs = true;
    return HMFEM_OK;
}

}  // namespace hm
