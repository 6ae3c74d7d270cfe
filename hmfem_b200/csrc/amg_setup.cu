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
#include <cub/device/device_scan.cuh>

#include "grid19.cuh"
#include <stdlib.h>

#include "hm.cuh"

namespace hm {

constexpr long long kMaxPolls = 1ll << 22;

// The poll limit of the splits' bounded waits: kMaxPolls, or lower when the
// environment sets HMFEM_TEST_POLL_LIMIT (a test makes the wait run out and
// checks that the call returns HMFEM_E_TIMEOUT and the next one succeeds).
long long split_poll_limit()
{
    const char *e = getenv("HMFEM_TEST_POLL_LIMIT");
    if (!e || !*e) return kMaxPolls;
    long long v = atoll(e);
    return v < 0 ? 0 : (v < kMaxPolls ? v : kMaxPolls);
}

namespace {

constexpr int kMisTile = 1024;

// The greedy split in natural order (node_selection, amg.h:1-226 with
// eps = 0): row v is C when every lower neighbour is F, F as soon as one is
// C -- the lexicographically first maximal independent set, so any order of
// evaluation that respects these dependencies gives the reference's split.
// Tiles of kMisTile rows are handed out in start order (ticket); a row
// waits (bounded) only on lower rows, i.e. on its own tile or on tiles that
// started earlier, so every wait ends.  Decisions inside the tile are
// exchanged through shared memory (most dependencies are short-range), and
// written to global memory for the tiles after it.
__global__ void __launch_bounds__(kMisTile)
k_lfmis(const int *__restrict__ rowptr, const int *__restrict__ col, int n,
        signed char *sel, unsigned *ticket, int *err, long long max_polls)
{
    __shared__ int s_tile;
    __shared__ signed char s_sel[kMisTile];
    if (threadIdx.x == 0) s_tile = (int)atomicAdd(ticket, 1u);
    s_sel[threadIdx.x] = 0;
    __syncthreads();
    const long base = (long)s_tile * kMisTile;
    const long v = base + threadIdx.x;
    if (v >= n) return;
    volatile signed char *vs = sel;
    volatile signed char *ss = s_sel;
    volatile int *verr = err;
    const int a = rowptr[v], e = rowptr[v + 1];
    long long polls = 0;
    for (;;) {
        bool anyC = false, allF = true, far = false;
        for (int k = a; k < e; k++) {
            int u = col[k];
            if (u >= v) continue;
            const bool in_tile = u >= base;
            signed char t = in_tile ? ss[u - base] : vs[u];
            if (t == 1) { anyC = true; break; }
            if (t == 0) {
                allF = false;
                far |= !in_tile;
            }
        }
        if (anyC || allF) {
            const signed char d = anyC ? 2 : 1;
            ss[threadIdx.x] = d;
            vs[v] = d;
            return;
        }
        if (++polls > max_polls || *verr) { atomicExch(err, 1); return; }
        if (far && polls > 32) __nanosleep(64);   // waiting on an earlier tile
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

// ---- Galerkin products: sparse union of rows ---------------------------
//
// One output row is the union of several inner rows scaled by outer
// entries:
//   STAGE 0:  AP row i  = sum_{j in A(i), stored order}   a_ij w_j * P(j)
//   STAGE 1:  Ac row e  = sum_{i in R(e), ascending}       w_i * AP(i)
// (w = the P weight 1/|P row|).  Candidates are generated in exactly the
// order sparse_multiply_transpose adds them (amg.h:520-546), tagged with
// their generation index g, and sorted by (column, g); each run of equal
// columns is then summed in g order with non-contracted adds, so every
// value is bit-identical to the reference's.
//
// Pass A counts candidates per row (an upper bound of the row length);
// pass B writes distinct columns and sums into a padded buffer (a warp per
// row, sized by the row's candidate count; long rows fall through to wider
// tiers); pass C compacts the padded rows into CSR.
struct UnionArgs {
    int nrows;
    const int *orow, *ocol;  // outer rows: stage 0 A, stage 1 R
    const double *oval;      // stage 0: A values
    const double *w;         // P weight per fine row
    const int *irow, *icol;  // inner rows: stage 0 P, stage 1 AP
    const double *ival;      // stage 1: AP values
    const long long *cptr;   // candidate offsets (pass A scan)
    int *ucnt;               // distinct columns per row
    int *pcol;               // padded output
    double *pval;
    int *list[2], *nlist[2]; // rows deferred to the next tier
    int *err;
};

template <int STAGE>
__global__ void k_cand_count(UnionArgs A, long long *ccnt)
{
    for (long r = blockIdx.x * (long)blockDim.x + threadIdx.x; r < A.nrows;
         r += (long)gridDim.x * blockDim.x) {
        long long m = 0;
        for (int k = A.orow[r]; k < A.orow[r + 1]; k++) {
            int j = A.ocol[k];
            m += A.irow[j + 1] - A.irow[j];
        }
        ccnt[r] = m;
    }
}

__device__ __forceinline__ int key_col(unsigned long long k) { return (int)(k >> 32); }
__device__ __forceinline__ int key_gen(unsigned long long k) { return (int)(k & 0xffffffffu); }

// Bitonic sort of m (power of two) 64-bit keys in shared memory by a group
// of `gs` threads with rank `gr`.
template <bool BLOCK>
__device__ void sort_keys(unsigned long long *a, int m, int gr, int gs)
{
    for (int k = 2; k <= m; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = gr; i < m; i += gs) {
                int ixj = i ^ j;
                if (ixj > i) {
                    unsigned long long x = a[i], y = a[ixj];
                    if ((x > y) == ((i & k) == 0)) { a[i] = y; a[ixj] = x; }
                }
            }
            if (BLOCK) __syncthreads(); else __syncwarp();
        }
}

// Generates the candidates of row r into keys/vals (group-parallel over the
// outer entries: each thread expands one outer entry's inner row).
template <int STAGE, bool BLOCK>
__device__ void gen_row(const UnionArgs &A, int r, unsigned long long *keys,
                        double *vals, int gr, int gs, int *s_scan)
{
    const int ob = A.orow[r], oe = A.orow[r + 1];
    int base = 0;
    for (int c0 = ob; c0 < oe; c0 += gs) {
        int k = c0 + gr;
        bool ok = k < oe;
        int j = ok ? A.ocol[k] : 0;
        int ib = ok ? A.irow[j] : 0;
        int len = ok ? A.irow[j + 1] - ib : 0;
        double s = 0.0;
        if (ok) s = STAGE == 0 ? dmul(A.oval[k], A.w[j]) : A.w[j];
        // exclusive scan of len over the group
        int off, tot;
        if (!BLOCK) {
            int lane = gr;
            int x = len;
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            off = x - len;
            tot = __shfl_sync(0xffffffffu, x, 31);
        } else {
            s_scan[gr] = len;
            __syncthreads();
            if (gr == 0) {
                int t = 0;
                for (int q = 0; q < gs; q++) { int v = s_scan[q]; s_scan[q] = t; t += v; }
                s_scan[gs] = t;
            }
            __syncthreads();
            off = s_scan[gr];
            tot = s_scan[gs];
            __syncthreads();
        }
        for (int q = 0; q < len; q++) {
            int g = base + off + q;
            int d = A.icol[ib + q];
            keys[g] = ((unsigned long long)(unsigned)d << 32) | (unsigned)g;
            // stage 0: t = a_ij * p_jd (p_jd = w_j); stage 1: t = AP[i][d] * w_i
            vals[g] = STAGE == 0 ? s : dmul(A.ival[ib + q], s);
        }
        base += tot;
    }
}

// Distinct columns + ordered sums of sorted keys[0..m) into the padded
// output at o; returns the number of distinct columns.  Done by one warp
// (lane = gr & 31), chunk by chunk.
__device__ int reduce_runs(const UnionArgs &A, const unsigned long long *keys,
                           const double *vals, int m, long long o)
{
    const int lane = threadIdx.x & 31;
    int u = 0;
    for (int c0 = 0; c0 < m; c0 += 32) {
        int idx = c0 + lane;
        bool head = false;
        int col = 0;
        if (idx < m) {
            col = key_col(keys[idx]);
            head = idx == 0 || key_col(keys[idx - 1]) != col;
        }
        unsigned bal = __ballot_sync(0xffffffffu, head);
        if (head) {
            int pos = u + __popc(bal & ((1u << lane) - 1));
            double acc = vals[key_gen(keys[idx])];
            for (int t = idx + 1; t < m && key_col(keys[t]) == col; t++)
                acc = dadd(acc, vals[key_gen(keys[t])]);
            A.pcol[o + pos] = col;
            A.pval[o + pos] = acc;
        }
        u += __popc(bal);
    }
    return u;
}

// Warp per row; rows with more candidates than CAP go to list[tier].
template <int STAGE, int CAP, int WPB>
__global__ void __launch_bounds__(32 * WPB)
k_union_warp(UnionArgs A, const int *rows, const int *nrows_dev, int tier)
{
    __shared__ unsigned long long s_keys[WPB][CAP];
    __shared__ double s_vals[WPB][CAP];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long *keys = s_keys[w];
    double *vals = s_vals[w];
    const long nr = rows ? *nrows_dev : A.nrows;
    for (long t = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5; t < nr;
         t += ((long)gridDim.x * blockDim.x) >> 5) {
        const int r = rows ? rows[t] : (int)t;
        const long long o = A.cptr[r];
        const int m = (int)(A.cptr[r + 1] - o);
        if (m > CAP) {
            if (lane == 0) A.list[tier][atomicAdd(A.nlist[tier], 1)] = r;
            continue;
        }
        gen_row<STAGE, false>(A, r, keys, vals, lane, 32, nullptr);
        const int mp = next_pow2(m);
        for (int q = m + lane; q < mp; q += 32) keys[q] = ~0ull;
        __syncwarp();
        sort_keys<false>(keys, mp, lane, 32);
        int u = reduce_runs(A, keys, vals, m, o);
        if (lane == 0) A.ucnt[r] = u;
        __syncwarp();
    }
}

// Warp per row with a shared-memory hash table: candidates are walked in
// generation order, 32 at a time; lanes holding the same column in a chunk
// are grouped (match_any) and the group's lowest lane adds their values to
// the column's slot in lane (= generation) order, so every sum keeps the
// reference's order.  Only the distinct columns are sorted at the end.
// The table is sized for distinct columns, not candidates: a row whose
// distinct count passes HCAP/2 is abandoned (nothing written yet) and goes
// to list[tier]; as at most 32 keys enter per chunk, the load stays below
// HCAP - 32 and every probe sequence ends.
template <int STAGE, int HCAP>
__global__ void __launch_bounds__(128)
k_union_hash(UnionArgs A, const int *rows, const int *nrows_dev, int tier)
{
    extern __shared__ __align__(16) unsigned char s_raw[];
    struct WarpMem {
        int key[HCAP];
        double val[HCAP];
        unsigned long long sorted[HCAP / 2];
        double cv[32];
        int off[33], ib[32];
        double sc[32];
    };
    static_assert(sizeof(WarpMem) % 8 == 0, "alignment");
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpMem &M = ((WarpMem *)s_raw)[w];
    const long nr = rows ? *nrows_dev : A.nrows;
    for (long t = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5; t < nr;
         t += ((long)gridDim.x * blockDim.x) >> 5) {
        const int r = rows ? rows[t] : (int)t;
        const long long o = A.cptr[r];
        for (int q = lane; q < HCAP; q += 32) M.key[q] = -1;
        __syncwarp();
        const int ob = A.orow[r], oe = A.orow[r + 1];
        int ndist = 0;
        bool full = false;
        for (int c0 = ob; c0 < oe && !full; c0 += 32) {
            // this group's outer entries: inner row start, length, scale
            const int k = c0 + lane;
            const bool ok = k < oe;
            const int j = ok ? A.ocol[k] : 0;
            const int ib = ok ? A.irow[j] : 0;
            const int len = ok ? A.irow[j + 1] - ib : 0;
            double sc = 0.0;
            if (ok) sc = STAGE == 0 ? dmul(A.oval[k], A.w[j]) : A.w[j];
            int x = len;
            for (int d = 1; d < 32; d <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, x, d);
                if (lane >= d) x += y;
            }
            M.off[lane] = x - len;
            M.ib[lane] = ib;
            M.sc[lane] = sc;
            const int tot = __shfl_sync(0xffffffffu, x, 31);
            const int nk = min(32, oe - c0);
            __syncwarp();
            for (int g0 = 0; g0 < tot && !full; g0 += 32) {
                const int g = g0 + lane;
                const bool on = g < tot;
                int col = -1;
                double tv = 0.0;
                if (on) {
                    int lo = 0, hi = nk - 1;  // largest kk with off[kk] <= g
                    while (lo < hi) {
                        int mid = (lo + hi + 1) >> 1;
                        if (M.off[mid] <= g) lo = mid; else hi = mid - 1;
                    }
                    const int q = M.ib[lo] + (g - M.off[lo]);
                    col = A.icol[q];
                    // stage 0: a_ij * p_jd (= w_j); stage 1: AP[i][d] * w_i
                    tv = STAGE == 0 ? M.sc[lo] : dmul(A.ival[q], M.sc[lo]);
                }
                M.cv[lane] = tv;
                const unsigned grp = __match_any_sync(0xffffffffu, col);
                __syncwarp();
                bool fresh = false;
                if (on && lane == __ffs(grp) - 1) {
                    unsigned h = ((unsigned)col * 2654435761u) & (HCAP - 1);
                    for (;;) {
                        int prev = atomicCAS(&M.key[h], -1, col);
                        if (prev == -1) { fresh = true; break; }
                        if (prev == col) break;
                        h = (h + 1) & (HCAP - 1);
                    }
                    unsigned mm = grp;
                    double acc = fresh ? M.cv[__ffs(mm) - 1] : dadd(M.val[h], M.cv[__ffs(mm) - 1]);
                    mm &= mm - 1;
                    while (mm) {
                        acc = dadd(acc, M.cv[__ffs(mm) - 1]);
                        mm &= mm - 1;
                    }
                    M.val[h] = acc;
                }
                ndist += __popc(__ballot_sync(0xffffffffu, fresh));
                full = ndist > HCAP / 2;
                __syncwarp();
            }
        }
        if (full) {  // too many distinct columns for this tier
            if (lane == 0) A.list[tier][atomicAdd(A.nlist[tier], 1)] = r;
            continue;
        }
        // distinct columns, sorted
        int u = 0;
        for (int q0 = 0; q0 < HCAP; q0 += 32) {
            const int q = q0 + lane;
            const int kq = M.key[q];
            const bool occ = kq >= 0;
            const unsigned bal = __ballot_sync(0xffffffffu, occ);
            if (occ)
                M.sorted[u + __popc(bal & ((1u << lane) - 1))] =
                    ((unsigned long long)(unsigned)kq << 32) | (unsigned)q;
            u += __popc(bal);
        }
        __syncwarp();
        const int up = next_pow2(u);
        for (int q = u + lane; q < up; q += 32) M.sorted[q] = ~0ull;
        __syncwarp();
        sort_keys<false>(M.sorted, up, lane, 32);
        for (int q = lane; q < u; q += 32) {
            const unsigned long long kk = M.sorted[q];
            A.pcol[o + q] = key_col(kk);
            A.pval[o + q] = M.val[key_gen(kk)];
        }
        if (lane == 0) A.ucnt[r] = u;
        __syncwarp();
    }
}

template <int STAGE, int HCAP>
size_t hash_smem()
{
    return 4 * (sizeof(int) * HCAP + sizeof(double) * HCAP + 8 * (HCAP / 2) +
                8 * 32 + 4 * 33 + 4 * 32 + 8 * 32 + 4);
}

// Block per row for the longest rows (dynamic shared memory, cap entries).
template <int STAGE>
__global__ void __launch_bounds__(256)
k_union_block(UnionArgs A, const int *rows, const int *nrows_dev, int cap)
{
    extern __shared__ unsigned long long s_dyn[];
    __shared__ int s_scan[257];
    unsigned long long *keys = s_dyn;
    double *vals = (double *)(s_dyn + cap);
    const long nr = *nrows_dev;
    for (long t = blockIdx.x; t < nr; t += gridDim.x) {
        const int r = rows[t];
        const long long o = A.cptr[r];
        const int m = (int)(A.cptr[r + 1] - o);
        if (m > cap) {
            if (threadIdx.x == 0) atomicExch(A.err, 3);
            return;
        }
        gen_row<STAGE, true>(A, r, keys, vals, threadIdx.x, blockDim.x, s_scan);
        const int mp = next_pow2(m);
        for (int q = m + threadIdx.x; q < mp; q += blockDim.x) keys[q] = ~0ull;
        __syncthreads();
        sort_keys<true>(keys, mp, threadIdx.x, blockDim.x);
        if (threadIdx.x < 32) {
            int u = reduce_runs(A, keys, vals, m, o);
            if (threadIdx.x == 0) A.ucnt[r] = u;
        }
        __syncthreads();
    }
}

__global__ void k_compact(const long long *__restrict__ cptr,
                          const int *__restrict__ rowptr, int n,
                          const int *__restrict__ pcol,
                          const double *__restrict__ pval, int *col,
                          double *val)
{
    // a warp per row: rows are short and contiguous
    const int lane = threadIdx.x & 31;
    for (long r = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5; r < n;
         r += ((long)gridDim.x * blockDim.x) >> 5) {
        const long long src = cptr[r];
        const int dst = rowptr[r], len = rowptr[r + 1] - dst;
        for (int q = lane; q < len; q += 32) {
            col[dst + q] = pcol[src + q];
            val[dst + q] = pval[src + q];
        }
    }
}

int nblk(long n, int threads, long cap = 148L * 16)
{
    long b = ceil_div(n, threads);
    if (b < 1) b = 1;
    return (int)(b < cap ? b : cap);
}

// Runs passes A-C of one Galerkin stage into `out`.
template <int STAGE>
int run_union(UnionArgs A, Csr &out, int *dwork, cudaStream_t st)
{
    const int n = A.nrows;
    out.n = n;
    long long *cptr = (long long *)dalloc(sizeof(long long) * (n + 1));
    out.rowptr = (int *)dalloc(sizeof(int) * (n + 1));
    int *lists = (int *)dalloc(sizeof(int) * 2 * (n > 0 ? n : 1));
    if (!cptr || !out.rowptr || !lists) {
        set_last_error("out of device memory (RAP)", __FILE__, __LINE__);
        return HMFEM_E_CUDA;
    }
    // pass A
    k_cand_count<STAGE><<<nblk(n, 256), 256, 0, st>>>(A, cptr);
    HM_LAUNCHED();
    HM_CUDA(cudaMemsetAsync(cptr + n, 0, sizeof(long long), st));
    {
        size_t tmp = 0;
        HM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, cptr, cptr, n + 1, st));
        void *t = dalloc(tmp);
        HM_CUDA(cub::DeviceScan::ExclusiveSum(t, tmp, cptr, cptr, n + 1, st));
        dfree(t);
    }
    long long mtot = 0;
    HM_CUDA(cudaMemcpyAsync(&mtot, cptr + n, sizeof(long long), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    A.cptr = cptr;
    A.pcol = (int *)dalloc(sizeof(int) * (mtot > 0 ? mtot : 1));
    A.pval = (double *)dalloc(sizeof(double) * (mtot > 0 ? mtot : 1));
    if (!A.pcol || !A.pval) {
        set_last_error("out of device memory (RAP)", __FILE__, __LINE__);
        return HMFEM_E_CUDA;
    }
    A.ucnt = out.rowptr;
    A.list[0] = lists;
    A.list[1] = lists + n;
    A.nlist[0] = dwork;
    A.nlist[1] = dwork + 1;
    A.err = dwork + 2;
    HM_CUDA(cudaMemsetAsync(dwork, 0, 3 * sizeof(int), st));
    // pass B: three tiers (<= 64 distinct columns, <= 512, <= 4096
    // candidates)
    {
        auto k0 = k_union_hash<STAGE, 128>;
        auto k1 = k_union_hash<STAGE, 1024>;
        const size_t m0 = hash_smem<STAGE, 128>(), m1 = hash_smem<STAGE, 1024>();
        HM_CUDA(cudaFuncSetAttribute(k0, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m0));
        HM_CUDA(cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m1));
        k0<<<nblk((long)n * 32, 128, 148L * 64), 128, m0, st>>>(A, nullptr, nullptr, 0);
        HM_LAUNCHED();
        k1<<<148 * 4, 128, m1, st>>>(A, A.list[0], A.nlist[0], 1);
        HM_LAUNCHED();
    }
    const int bcap = 4096;  // 16 B per candidate: 64 KB
    const size_t bsm = (size_t)bcap * 16;
    HM_CUDA(cudaFuncSetAttribute(k_union_block<STAGE>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsm));
    k_union_block<STAGE><<<148 * 2, 256, bsm, st>>>(A, A.list[1], A.nlist[1], bcap);
    HM_LAUNCHED();
    // pass C
    HM_CHECK(rowptr_from_counts(out.rowptr, n, st, &out.nnz));
    int herr = 0;
    HM_CUDA(cudaMemcpyAsync(&herr, A.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    if (herr) {
        set_last_error("sparse row over the Galerkin-product capacity", __FILE__, __LINE__);
        return HMFEM_E_CAPACITY;
    }
    out.col = (int *)dalloc(sizeof(int) * (out.nnz > 0 ? out.nnz : 1));
    out.val = (double *)dalloc(sizeof(double) * (out.nnz > 0 ? out.nnz : 1));
    if (!out.col || !out.val) {
        set_last_error("out of device memory (RAP)", __FILE__, __LINE__);
        return HMFEM_E_CUDA;
    }
    k_compact<<<nblk((long)n * 32, 256, 148L * 32), 256, 0, st>>>(
        cptr, out.rowptr, n, A.pcol, A.pval, out.col, out.val);
    HM_LAUNCHED();
    dfree(A.pcol);
    dfree(A.pval);
    dfree(cptr);
    dfree(lists);
    return HMFEM_OK;
}

}  // namespace

// P rows (amg.h:332-346), their entries (amg.h:352-380) and weights from
// the level's split and coarse ids; *pown: the fine row of every entry
// (for the transpose), freed by the caller, or nullptr not to keep it.
int build_p(Level &L, cudaStream_t st, int **pown_out)
{
    const int n = L.A.n;
    L.P.n = n;
    L.P.rowptr = (int *)dalloc(sizeof(int) * (n + 1));
    if (!L.P.rowptr) return HMFEM_E_CUDA;
    k_pcount<<<nblk(n, 256), 256, 0, st>>>(L.A.rowptr, L.A.col, L.sel, n, L.P.rowptr);
    HM_LAUNCHED();
    HM_CHECK(rowptr_from_counts(L.P.rowptr, n, st, &L.P.nnz));
    L.P.col = (int *)dalloc(sizeof(int) * (L.P.nnz > 0 ? L.P.nnz : 1));
    int *pown = (int *)dalloc(sizeof(int) * (L.P.nnz > 0 ? L.P.nnz : 1));
    L.pw = (double *)dalloc(sizeof(double) * (n > 0 ? n : 1));
    L.pw32 = (float *)dalloc(sizeof(float) * (n > 0 ? n : 1));
    if (!L.P.col || !pown || !L.pw || !L.pw32) {
        dfree(pown);
        set_last_error("out of device memory (P)", __FILE__, __LINE__);
        return HMFEM_E_CUDA;
    }
    k_pfill<<<nblk(n, 256), 256, 0, st>>>(L.A.rowptr, L.A.col, L.sel, L.cid, n,
                                          L.P.rowptr, L.P.col, pown, L.pw, L.pw32);
    HM_LAUNCHED();
    L.p_deferred = false;
    if (pown_out) *pown_out = pown;
    else dfree(pown);
    return HMFEM_OK;
}

int ensure_p(Level &L, cudaStream_t st)
{
    if (!L.p_deferred) return HMFEM_OK;
    HM_CHECK(build_p(L, st, nullptr));
    HM_CUDA(cudaStreamSynchronize(st));
    return HMFEM_OK;
}

// Per host thread: the stream that forms level 1's split while level 0's
// Galerkin product runs (the split depends only on the grid's shape).  Its
// kernels are a latency-bound wavefront of small launches, so the stream
// has the highest priority: their blocks are scheduled between the
// bandwidth-bound blocks of the main stream instead of after them.
static cudaStream_t side_stream()
{
    static thread_local cudaStream_t t_side = nullptr;
    if (!t_side) {
        int least = 0, greatest = 0;
        cudaDeviceGetStreamPriorityRange(&least, &greatest);
        cudaStreamCreateWithPriority(&t_side, cudaStreamNonBlocking, greatest);
    }
    return t_side;
}

int amg_coarsen(Level &L, Level &C, cudaStream_t st, int *dwork,
                const int *grid3, bool schur)
{
    const int n = L.A.n;
    // ---- C/F split ----------------------------------------------------
    HM_CUDA(cudaMemsetAsync(dwork, 0, 4 * sizeof(int), st));
    int *wave = nullptr, *wave_err = nullptr;  // the level-1 split's work and error word
    if (L.sel_split) {  // formed on the side stream while the level above coarsened
        HM_CUDA(cudaStreamWaitEvent(st, L.sel_ready, 0));
        cudaEventDestroy(L.sel_ready);
        L.sel_ready = nullptr;
        wave = L.split_work;
        wave_err = L.split_err;
        L.split_work = L.split_err = nullptr;
    } else {
        L.sel = (signed char *)dalloc(n > 0 ? n : 1);
        HM_CUDA(cudaMemsetAsync(L.sel, 0, n > 0 ? n : 1, st));
        if (grid3) {
            HM_CHECK(stencil_parity_split(grid3[0], grid3[1], grid3[2], L.sel, st));
        } else if (L.g19.nx > 0) {
            const long wi = stencil19_split_work_ints(L.g19.nx, L.g19.ny, L.g19.nz);
            wave = (int *)dalloc(sizeof(int) * wi);
            if (!wave) return HMFEM_E_CUDA;
            wave_err = wave + wi - 1;
            const int rc = stencil19_split(L.g19.nx, L.g19.ny, L.g19.nz, L.sel, wave, st);
            if (rc != HMFEM_OK) {
                cudaStreamSynchronize(st);
                dfree(wave);
                return rc;
            }
        } else if (n > 0) {
            k_lfmis<<<(int)ceil_div(n, kMisTile), kMisTile, 0, st>>>(
                L.A.rowptr, L.A.col, n, L.sel, (unsigned *)(dwork + 2), dwork,
                split_poll_limit());
            HM_LAUNCHED();
        }
    }
    int herr[2] = {0, 0};
    HM_CUDA(cudaMemcpyAsync(&herr[0], dwork, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (wave_err)
        HM_CUDA(cudaMemcpyAsync(&herr[1], wave_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    dfree(wave);
    HM_PHASE("  C/F split", st);
    if (herr[0] || herr[1]) {
        set_last_error("C/F split wavefront gave up waiting", __FILE__, __LINE__);
        return HMFEM_E_TIMEOUT;
    }
    // ---- coarse numbering ---------------------------------------------
    L.cid = (int *)dalloc(sizeof(int) * (n + 1));
    k_cflag<<<nblk(n, 256), 256, 0, st>>>(L.sel, n, L.cid);
    HM_LAUNCHED();
    long nc = 0;
    HM_CHECK(rowptr_from_counts(L.cid, n, st, &nc));
    HM_PHASE("  coarse ids", st);
    L.nc = (int)nc;
    // the next level's split from the 19-offset structure, on the side
    // stream, overlapping the rest of this level's coarsening
    if (grid3 && g19_applies(grid3[0], grid3[1], grid3[2]) && nc > 0) {
        C.sel = (signed char *)dalloc(nc);
        const long wi = stencil19_split_work_ints(grid3[0], grid3[1], grid3[2]);
        C.split_work = (int *)dalloc(sizeof(int) * wi);
        if (!C.sel || !C.split_work) return HMFEM_E_CUDA;
        C.split_err = C.split_work + wi - 1;
        cudaEvent_t allocated;
        HM_CUDA(cudaEventCreateWithFlags(&allocated, cudaEventDisableTiming));
        HM_CUDA(cudaEventRecord(allocated, st));
        cudaStream_t side = side_stream();
        HM_CUDA(cudaStreamWaitEvent(side, allocated, 0));
        cudaEventDestroy(allocated);
        HM_CHECK(stencil19_split(grid3[0], grid3[1], grid3[2], C.sel, C.split_work, side));
        HM_CUDA(cudaEventCreateWithFlags(&C.sel_ready, cudaEventDisableTiming));
        HM_CUDA(cudaEventRecord(C.sel_ready, side));
        C.sel_split = true;
    }
    // ---- P and R = P^T (fine rows ascending) ----------------------------
    if (grid3 && schur) {
        // the exact reduction transfers level 0 without P, R or the P
        // weights: the reference's P is formed only when it is asked for
        // (ensure_p: the hierarchy export)
        L.P = Csr();
        L.R = Csr();
        L.p_deferred = true;
    } else {
        int *pown = nullptr;
        HM_CHECK(build_p(L, st, &pown));
        L.R.n = L.nc;
        L.R.nnz = L.P.nnz;
        L.R.rowptr = (int *)dalloc(sizeof(int) * (L.nc + 1));
        L.R.col = (int *)dalloc(sizeof(int) * (L.P.nnz > 0 ? L.P.nnz : 1));
        bool done = false;
        if (grid3) {
            HM_CHECK(stencil_parity_R(grid3[0], grid3[1], grid3[2], L.cid, L.nc, L.R, st));
            done = true;
        } else if (L.g19.nx > 0) {
            HM_CHECK(g19_transpose(L, L.R, st, &done));
        }
        if (done) {
            dfree(pown);
        } else {  // stable radix sort on the coarse id
            int *keys_out = (int *)dalloc(sizeof(int) * (L.P.nnz > 0 ? L.P.nnz : 1));
            HM_CUDA(cudaMemsetAsync(L.R.rowptr, 0, sizeof(int) * (L.nc + 1), st));
            k_hist<<<nblk(L.P.nnz, 256), 256, 0, st>>>(L.P.col, L.P.nnz, L.R.rowptr);
            HM_LAUNCHED();
            long rn = 0;
            HM_CHECK(rowptr_from_counts(L.R.rowptr, L.nc, st, &rn));
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
            dfree(keys_out);
            dfree(pown);
        }
    }
    if (L.g19.nx > 0) HM_CHECK(g19_cpts(L, st));  // for the product
    HM_PHASE("  P and R", st);
    // ---- Galerkin product ---------------------------------------------
    if (grid3) {
        double *g19v = nullptr;
        if (g19_applies(grid3[0], grid3[1], grid3[2])) {
            const long long m = slice_len(L.nc, kQ19);
            g19v = (double *)dalloc(sizeof(double) * m);
            if (!g19v) return HMFEM_E_CUDA;
            HM_CUDA(cudaMemsetAsync(g19v, 0, sizeof(double) * m, st));  // last slice's tail
            C.g19.nx = grid3[0];
            C.g19.ny = grid3[1];
            C.g19.nz = grid3[2];
            C.g19.v = g19v;
        }
        HM_CHECK(stencil_galerkin(grid3[0], grid3[1], grid3[2], L, C.A, g19v, st, schur));
        HM_PHASE("  P^T A P (stencil)", st);
        return HMFEM_OK;
    }
    if (L.g19.nx > 0) {  // level 1 of a parity split: from its 19-offset structure
        bool done = false;
        HM_CHECK(galerkin19(L, C.A, st, &done));
        if (done) {
            HM_PHASE("  P^T A P (19-point)", st);
            return HMFEM_OK;
        }
    }
    Csr AP;
    UnionArgs a0{};
    a0.nrows = n;
    a0.orow = L.A.rowptr; a0.ocol = L.A.col; a0.oval = L.A.val; a0.w = L.pw;
    a0.irow = L.P.rowptr; a0.icol = L.P.col; a0.ival = nullptr;
    HM_CHECK(run_union<0>(a0, AP, dwork, st));
    HM_PHASE("  A P", st);
    UnionArgs a1{};
    a1.nrows = L.nc;
    a1.orow = L.R.rowptr; a1.ocol = L.R.col; a1.oval = nullptr; a1.w = L.pw;
    a1.irow = AP.rowptr; a1.icol = AP.col; a1.ival = AP.val;
    HM_CHECK(run_union<1>(a1, C.A, dwork, st));
    HM_PHASE("  P^T (A P)", st);
    HM_CUDA(cudaStreamSynchronize(st));
    dfree(AP.rowptr); dfree(AP.col); dfree(AP.val);
    return HMFEM_OK;
}

}  // namespace hm
