// amg_setup.cu -- one AMG coarsening step on the device, reproducing the
// reference's single-rank setup (toolbox/inverse_operator/amg.h) exactly:
//
//   C/F split   amg.h:1-32, 219-223   greedy maximal independent set in
//               natural row order (epsilon = 0: every stored entry strong)
//   P           amg.h:326-387         C row {self, 1}; F row: its C
//               neighbours in stored order, weight 1/count
//   numbering   amg.h:394-403         coarse id = rank of the C row
//   Galerkin    amg.h:408-582         (A P)^T, then ((A P)^T P)^T = P^T A P,
//               coarse rows column-ascending, values summed in the same
//               order as sparse_multiply_transpose, without FMA contraction,
//               so the hierarchy is bit-identical to the reference's.
//
// The greedy MIS is sequential by definition; here it runs as a
// dependency-driven wavefront: row v becomes F as soon as one lower
// neighbour is C and C once all lower neighbours are F, which is the same
// set the sequential sweep produces.  Row tiles are handed out in
// increasing order through an atomic ticket, so a tile only ever waits on
// tiles that are already resident; every wait is bounded.
#include <cub/device/device_radix_sort.cuh>

#include "hm.cuh"

namespace hm {

namespace {

constexpr int kMisTile = 256;
constexpr long long kMaxPolls = 1ll << 22;

__global__ void __launch_bounds__(kMisTile)
k_lfmis(const int *__restrict__ rowptr, const int *__restrict__ col, int n,
        signed char *sel, unsigned *ticket, int *err)
{
    __shared__ int s_tile;
    if (threadIdx.x == 0) s_tile = (int)atomicAdd(ticket, 1u);
    __syncthreads();
    long v = (long)s_tile * kMisTile + threadIdx.x;
    if (v >= n) return;
    volatile signed char *vs = sel;
    volatile int *verr = err;
    const int a = rowptr[v], e = rowptr[v + 1];
    long long polls = 0;
    for (;;) {
        bool anyC = false, allF = true;
        for (int k = a; k < e; k++) {
            int u = col[k];
            if (u >= v) continue;
            signed char t = vs[u];
            if (t == 1) { anyC = true; break; }
            if (t == 0) allF = false;
        }
        if (anyC) { vs[v] = 2; return; }
        if (allF) { vs[v] = 1; return; }
        if (++polls > kMaxPolls || *verr) { atomicExch(err, 1); return; }
        if (polls > 32) __nanosleep(64);
    }
}

__global__ void k_cflag(const signed char *__restrict__ sel, int n, int *flag)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
        flag[i] = sel[i] == 1 ? 1 : 0;
}

// P row counts (amg.h:332-346), then rows (amg.h:352-380) and weights.
__global__ void k_pcount(const int *__restrict__ rowptr,
                         const int *__restrict__ col,
                         const signed char *__restrict__ sel, int n, int *pcnt)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        int c = 0;
        if (sel[i] == 1) c = 1;
        else
            for (int k = rowptr[i]; k < rowptr[i + 1]; k++) c += sel[col[k]] == 1;
        pcnt[i] = c;
    }
}

__global__ void k_pfill(const int *__restrict__ rowptr,
                        const int *__restrict__ col,
                        const signed char *__restrict__ sel,
                        const int *__restrict__ cid, int n,
                        const int *__restrict__ prow, int *pcol, int *pown,
                        double *pw, float *pw32)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        int q = prow[i], c = prow[i + 1] - q;
        double w = 1.0 / (double)c;
        pw[i] = w;
        pw32[i] = (float)w;
        if (sel[i] == 1) { pcol[q] = cid[i]; pown[q] = (int)i; continue; }
        for (int k = rowptr[i]; k < rowptr[i + 1]; k++) {
            int j = col[k];
            if (sel[j] == 1) { pcol[q] = cid[j]; pown[q] = (int)i; q++; }
        }
    }
}

__global__ void k_hist(const int *__restrict__ key, long m, int *cnt)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < m;
         i += (long)gridDim.x * blockDim.x)
        atomicAdd(cnt + key[i], 1);
}

// ---- sparse union of rows: warp (or block) per output row -------------
//
// Candidates of an output row are generated in the reference's summation
// order; the distinct columns are sorted; each slot's value is the ordered
// sum of its candidates.  MODE 0 counts distinct columns, MODE 1 writes
// columns and values.
//
// STAGE 0: AP row i   = sum_{j in A(i)} a_ij * w_j * e_{P(j)}
// STAGE 1: Ac row e   = sum_{i in R(e), ascending} w_i * AP(i)
struct UnionArgs {
    int nrows;
    // outer rows: stage 0 -> A, stage 1 -> R
    const int *orow, *ocol;
    const double *oval;  // stage 0: A values; stage 1: unused
    const double *w;     // stage 0: P weight of column row; stage 1: of row i
    // inner rows: stage 0 -> P (cols), stage 1 -> AP (cols, vals)
    const int *irow, *icol;
    const double *ival;
    // output
    int *cnt;            // MODE 0
    const int *out_row;  // MODE 1
    int *out_col;
    double *out_val;
    int *long_rows, *n_long;  // rows over capacity (first pass)
    int *err;
};

template <int STAGE>
__device__ __forceinline__ int cand_count(const UnionArgs &A, int r)
{
    int m = 0;
    for (int k = A.orow[r]; k < A.orow[r + 1]; k++) {
        int j = A.ocol[k];
        m += A.irow[j + 1] - A.irow[j];
    }
    return m;
}

struct WarpG {
    __device__ int rank() const { return threadIdx.x & 31; }
    __device__ int size() const { return 32; }
    __device__ void sync() const { __syncwarp(); }
};
struct BlockG {
    __device__ int rank() const { return threadIdx.x; }
    __device__ int size() const { return blockDim.x; }
    __device__ void sync() const { __syncthreads(); }
};

// Gathers candidates of row r into cd/ct (generation order), sorts a copy
// in sb, compacts distinct columns to the front of sb; returns the count.
template <int STAGE, bool VALUES, class G>
__device__ int row_union(const G &g, const UnionArgs &A, int r, int m,
                         int *cd, double *ct, int *sb)
{
    // generation: walk the outer row in order; each outer entry expands
    // into a contiguous inner row.  Position of each inner entry = running
    // offset, computed serially per outer entry (rows are short).
    int base = 0;
    for (int k = A.orow[r]; k < A.orow[r + 1]; k++) {
        int j = A.ocol[k];
        int ib = A.irow[j], ie = A.irow[j + 1];
        double s = 0.0;
        if (VALUES) s = STAGE == 0 ? dmul(A.oval[k], A.w[j]) : A.w[j];
        for (int q = ib + g.rank(); q < ie; q += g.size()) {
            int d = A.icol[q];
            cd[base + q - ib] = d;
            sb[base + q - ib] = d;
            // stage 0: t = a_ij * p_jd with p_jd = w_j (amg.h:537)
            // stage 1: t = AP[i][d] * p_ie with p_ie = w_i (same line)
            if (VALUES) ct[base + q - ib] = STAGE == 0 ? s : dmul(A.ival[q], s);
        }
        base += ie - ib;
    }
    int mp = next_pow2(m);
    for (int q = m + g.rank(); q < mp; q += g.size()) sb[q] = 0x7fffffff;
    g.sync();
    if (g.size() == 32) warp_bitonic_sort(sb, mp);
    else block_bitonic_sort(sb, mp);
    // compact distinct values (one warp does it; others wait)
    __shared__ int s_u;
    int u = 0;
    if (g.size() == 32 || threadIdx.x < 32) {
        int lane = threadIdx.x & 31;
        for (int c0 = 0; c0 < m; c0 += 32) {
            int idx = c0 + lane;
            int x = idx < m ? sb[idx] : 0;
            bool head = idx < m && (idx == 0 || sb[idx - 1] != x);
            unsigned bal = __ballot_sync(0xffffffffu, head);
            int pos = u + __popc(bal & ((1u << lane) - 1));
            __syncwarp();
            if (head) sb[pos] = x;
            __syncwarp();
            u += __popc(bal);
        }
        if (g.size() != 32 && lane == 0) s_u = u;
    }
    if (g.size() != 32) {
        g.sync();
        u = s_u;
    }
    g.sync();
    return u;
}

template <int STAGE, int MODE, class G>
__device__ void union_row(const G &g, const UnionArgs &A, int r, int cap,
                          int *cd, double *ct, int *sb)
{
    int m = cand_count<STAGE>(A, r);
    if (m > cap) {
        // first (warp) pass only: defer to the block kernel
        if (g.rank() == 0 && MODE == 0) {
            int p = atomicAdd(A.n_long, 1);
            A.long_rows[p] = r;
        }
        return;
    }
    int u = row_union<STAGE, MODE == 1, G>(g, A, r, m, cd, ct, sb);
    if (MODE == 0) {
        if (g.rank() == 0) A.cnt[r] = u;
        g.sync();
        return;
    }
    int o = A.out_row[r];
    if (A.out_row[r + 1] - o != u) {
        if (g.rank() == 0) atomicExch(A.err, 2);
        return;
    }
    // lane-owns-slot accumulation in generation order (amg.h:531-546)
    for (int q = g.rank(); q < u; q += g.size()) {
        int d = sb[q];
        double acc = 0.0;
        bool first = true;
        for (int c = 0; c < m; c++) {
            if (cd[c] != d) continue;
            acc = first ? ct[c] : dadd(acc, ct[c]);
            first = false;
        }
        A.out_col[o + q] = d;
        A.out_val[o + q] = acc;
    }
    g.sync();
}

constexpr int kWarpCap = 1024;
constexpr int kWarpsPerBlock = 4;

template <int STAGE, int MODE>
__global__ void __launch_bounds__(32 * kWarpsPerBlock)
k_union_warp(UnionArgs A)
{
    extern __shared__ unsigned char smem[];
    int w = threadIdx.x >> 5;
    size_t per = kWarpCap * (sizeof(int) * 2 + (MODE == 1 ? sizeof(double) : 0));
    unsigned char *base = smem + per * w;
    int *cd = (int *)base;
    int *sb = cd + kWarpCap;
    double *ct = (double *)(sb + kWarpCap);
    WarpG g;
    for (long r = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
         r < A.nrows; r += ((long)gridDim.x * blockDim.x) >> 5)
        union_row<STAGE, MODE>(g, A, (int)r, kWarpCap, cd, ct, sb);
}

// Long rows: one block per row with the whole dynamic shared memory.
template <int STAGE, int MODE>
__global__ void __launch_bounds__(256)
k_union_block(UnionArgs A, const int *rows, int nrows, int cap)
{
    extern __shared__ unsigned char smem[];
    int *cd = (int *)smem;
    int *sb = cd + cap;
    double *ct = (double *)(sb + cap);
    BlockG g;
    for (int t = blockIdx.x; t < nrows; t += gridDim.x) {
        int r = rows[t];
        int m = cand_count<STAGE>(A, r);
        if (m > cap) {
            if (threadIdx.x == 0) atomicExch(A.err, 3);
            return;
        }
        int u = row_union<STAGE, MODE == 1, BlockG>(g, A, r, m, cd, ct, sb);
        if (MODE == 0) {
            if (threadIdx.x == 0) A.cnt[r] = u;
            __syncthreads();
            continue;
        }
        int o = A.out_row[r];
        for (int q = threadIdx.x; q < u; q += blockDim.x) {
            int d = sb[q];
            double acc = 0.0;
            bool first = true;
            for (int c = 0; c < m; c++) {
                if (cd[c] != d) continue;
                acc = first ? ct[c] : dadd(acc, ct[c]);
                first = false;
            }
            A.out_col[o + q] = d;
            A.out_val[o + q] = acc;
        }
        __syncthreads();
    }
}

int nblk(long n, int threads, long cap = 148L * 16)
{
    long b = ceil_div(n, threads);
    if (b < 1) b = 1;
    return (int)(b < cap ? b : cap);
}

// Runs count + fill of one sparse-union stage into `out` (rowptr, col, val).
template <int STAGE>
int run_union(UnionArgs A, Csr &out, int *dwork, cudaStream_t st)
{
    // dwork: [0] n_long, [1] err; long_rows separately
    int *long_rows = (int *)dalloc(sizeof(int) * (A.nrows > 0 ? A.nrows : 1));
    out.n = A.nrows;
    out.rowptr = (int *)dalloc(sizeof(int) * (A.nrows + 1));
    if (!long_rows || !out.rowptr) {
        set_last_error("out of device memory (RAP)", __FILE__, __LINE__);
        return HMFEM_E_CUDA;
    }
    HM_CUDA(cudaMemsetAsync(dwork, 0, 2 * sizeof(int), st));
    A.cnt = out.rowptr;
    A.long_rows = long_rows;
    A.n_long = dwork;
    A.err = dwork + 1;
    const int thr = 32 * kWarpsPerBlock;
    size_t smem0 = (size_t)kWarpsPerBlock * kWarpCap * 2 * sizeof(int);
    size_t smem1 = (size_t)kWarpsPerBlock * kWarpCap * (2 * sizeof(int) + sizeof(double));
    HM_CUDA(cudaFuncSetAttribute(k_union_warp<STAGE, 0>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem0));
    HM_CUDA(cudaFuncSetAttribute(k_union_warp<STAGE, 1>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1));
    k_union_warp<STAGE, 0><<<nblk((long)A.nrows * 32, thr, 148L * 64), thr, smem0, st>>>(A);
    HM_CUDA(cudaGetLastError());
    int h[2];
    HM_CUDA(cudaMemcpyAsync(h, dwork, sizeof(h), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    int nlong = h[0];
    // 16 B per candidate: 128 KB; a power of two so the padded sort stays
    // inside the column buffer
    const int bcap = 8 * 1024;
    size_t bsm = (size_t)bcap * (2 * sizeof(int) + sizeof(double));
    if (nlong > 0) {
        HM_CUDA(cudaFuncSetAttribute(k_union_block<STAGE, 0>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsm));
        HM_CUDA(cudaFuncSetAttribute(k_union_block<STAGE, 1>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsm));
        k_union_block<STAGE, 0><<<nblk(nlong, 1, 148L * 4), 256, bsm, st>>>(
            A, long_rows, nlong, bcap);
        HM_CUDA(cudaGetLastError());
    }
    HM_CHECK(rowptr_from_counts(out.rowptr, A.nrows, st, &out.nnz));
    out.col = (int *)dalloc(sizeof(int) * (out.nnz > 0 ? out.nnz : 1));
    out.val = (double *)dalloc(sizeof(double) * (out.nnz > 0 ? out.nnz : 1));
    if (!out.col || !out.val) {
        set_last_error("out of device memory (RAP)", __FILE__, __LINE__);
        return HMFEM_E_CUDA;
    }
    A.out_row = out.rowptr;
    A.out_col = out.col;
    A.out_val = out.val;
    k_union_warp<STAGE, 1><<<nblk((long)A.nrows * 32, thr, 148L * 64), thr, smem1, st>>>(A);
    HM_CUDA(cudaGetLastError());
    if (nlong > 0) {
        k_union_block<STAGE, 1><<<nblk(nlong, 1, 148L * 4), 256, bsm, st>>>(
            A, long_rows, nlong, bcap);
        HM_CUDA(cudaGetLastError());
    }
    HM_CUDA(cudaMemcpyAsync(h, dwork, sizeof(h), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    dfree(long_rows);
    if (h[1] != 0) {
        set_last_error(h[1] == 3 ? "sparse row over the setup capacity"
                                 : "inconsistent Galerkin row count",
                       __FILE__, __LINE__);
        return HMFEM_E_CAPACITY;
    }
    return HMFEM_OK;
}

}  // namespace

int amg_coarsen(Level &L, Level &C, cudaStream_t st, int *dwork)
{
    const int n = L.A.n;
    // ---- C/F split ----------------------------------------------------
    L.sel = (signed char *)dalloc(n > 0 ? n : 1);
    HM_CUDA(cudaMemsetAsync(L.sel, 0, n > 0 ? n : 1, st));
    HM_CUDA(cudaMemsetAsync(dwork, 0, 4 * sizeof(int), st));
    if (n > 0) {
        k_lfmis<<<(int)ceil_div(n, kMisTile), kMisTile, 0, st>>>(
            L.A.rowptr, L.A.col, n, L.sel, (unsigned *)(dwork + 2), dwork);
        HM_CUDA(cudaGetLastError());
    }
    int herr = 0;
    HM_CUDA(cudaMemcpyAsync(&herr, dwork, sizeof(int), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    if (herr) {
        set_last_error("C/F split wavefront gave up waiting", __FILE__, __LINE__);
        return HMFEM_E_TIMEOUT;
    }
    // ---- coarse numbering ---------------------------------------------
    L.cid = (int *)dalloc(sizeof(int) * (n + 1));
    k_cflag<<<nblk(n, 256), 256, 0, st>>>(L.sel, n, L.cid);
    HM_CUDA(cudaGetLastError());
    long nc = 0;
    HM_CHECK(rowptr_from_counts(L.cid, n, st, &nc));
    L.nc = (int)nc;
    // ---- P ---------------------------------------------------------------
    L.P.n = n;
    L.P.rowptr = (int *)dalloc(sizeof(int) * (n + 1));
    k_pcount<<<nblk(n, 256), 256, 0, st>>>(L.A.rowptr, L.A.col, L.sel, n, L.P.rowptr);
    HM_CUDA(cudaGetLastError());
    HM_CHECK(rowptr_from_counts(L.P.rowptr, n, st, &L.P.nnz));
    L.P.col = (int *)dalloc(sizeof(int) * (L.P.nnz > 0 ? L.P.nnz : 1));
    int *pown = (int *)dalloc(sizeof(int) * (L.P.nnz > 0 ? L.P.nnz : 1));
    L.pw = (double *)dalloc(sizeof(double) * (n > 0 ? n : 1));
    L.pw32 = (float *)dalloc(sizeof(float) * (n > 0 ? n : 1));
    k_pfill<<<nblk(n, 256), 256, 0, st>>>(L.A.rowptr, L.A.col, L.sel, L.cid, n,
                                          L.P.rowptr, L.P.col, pown, L.pw, L.pw32);
    HM_CUDA(cudaGetLastError());
    // ---- R = P^T, fine rows ascending (stable radix sort on coarse id) -
    L.R.n = L.nc;
    L.R.nnz = L.P.nnz;
    L.R.rowptr = (int *)dalloc(sizeof(int) * (L.nc + 1));
    L.R.col = (int *)dalloc(sizeof(int) * (L.P.nnz > 0 ? L.P.nnz : 1));
    int *keys_out = (int *)dalloc(sizeof(int) * (L.P.nnz > 0 ? L.P.nnz : 1));
    HM_CUDA(cudaMemsetAsync(L.R.rowptr, 0, sizeof(int) * (L.nc + 1), st));
    k_hist<<<nblk(L.P.nnz, 256), 256, 0, st>>>(L.P.col, L.P.nnz, L.R.rowptr);
    HM_CUDA(cudaGetLastError());
    long rn = 0;
    HM_CHECK(rowptr_from_counts(L.R.rowptr, L.nc, st, &rn));
    {
        size_t tmp = 0;
        int bits = 1;
        while ((1l << bits) < (long)L.nc + 1) bits++;
        HM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, L.P.col, keys_out,
                                                pown, L.R.col, (int)L.P.nnz, 0,
                                                bits, st));
        void *t = dalloc(tmp);
        HM_CUDA(cub::DeviceRadixSort::SortPairs(t, tmp, L.P.col, keys_out, pown,
                                                L.R.col, (int)L.P.nnz, 0, bits,
                                                st));
        HM_CUDA(cudaStreamSynchronize(st));
        dfree(t);
    }
    dfree(keys_out);
    dfree(pown);
    // ---- Galerkin product ---------------------------------------------
    Csr AP;
    UnionArgs a0{};
    a0.nrows = n;
    a0.orow = L.A.rowptr; a0.ocol = L.A.col; a0.oval = L.A.val; a0.w = L.pw;
    a0.irow = L.P.rowptr; a0.icol = L.P.col; a0.ival = nullptr;
    HM_CHECK(run_union<0>(a0, AP, dwork, st));
    UnionArgs a1{};
    a1.nrows = L.nc;
    a1.orow = L.R.rowptr; a1.ocol = L.R.col; a1.oval = nullptr; a1.w = L.pw;
    a1.irow = AP.rowptr; a1.icol = AP.col; a1.ival = AP.val;
    HM_CHECK(run_union<1>(a1, C.A, dwork, st));
    HM_CUDA(cudaStreamSynchronize(st));
    dfree(AP.rowptr); dfree(AP.col); dfree(AP.val);
    return HMFEM_OK;
}

}  // namespace hm
