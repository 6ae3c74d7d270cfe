// smoother_setup.cu -- setup of the multicolour Gauss-Seidel smoother used on
// the coarse levels: a colouring and the list of rows grouped by colour, so
// one colour is one conflict-free kernel over the level's CSR rows.
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
        HM_LAUNCHED();
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
    HM_LAUNCHED();
    HM_CUDA(cudaMemsetAsync(hist, 0, sizeof(int) * 64, st));
    k_color_hist<<<nb(n), 256, 0, st>>>(L.color, n, hist);
    HM_LAUNCHED();
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
    std::vector<long> off(nc + 1);
    off[0] = 0;
    for (int c = 0; c < nc; c++) off[c + 1] = off[c] + hh[c];
    dfree(key); dfree(row); dfree(skey); dfree(hist);
    std::vector<int> off32(off.begin(), off.end());
    L.cslot = (int *)dalloc(sizeof(int) * (nc + 1));
    if (!L.cslot) return HMFEM_E_CUDA;
    HM_CUDA(cudaMemcpyAsync(L.cslot, off32.data(), sizeof(int) * (nc + 1),
                            cudaMemcpyHostToDevice, st));
    HM_CUDA(cudaStreamSynchronize(st));
    L.crows = srow;          // rows by colour, ascending within a colour
    L.ncolors = nc;
    L.color_slot = off;      // first row of each colour in crows (+ end)
    L.gs = true;
    return HMFEM_OK;
}

}  // namespace hm
