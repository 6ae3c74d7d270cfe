// rap19.cu -- the Galerkin product P^T A P of a level with the 19-offset
// structure (Grid19: the level below the parity split of a 7-point grid),
// formed from that structure instead of by the generic sparse union.
//
// The level's rows are the even cells (i+j+k even) of the fine nx*ny*nz
// grid, row r = fine index s >> 1 (nx even).  Every row stores the in-grid
// offsets of the 19-point set in ascending column order (grid19.cuh), and
// its C/F split (amg.h:1-32, every stored entry strong) is an independent
// set of that graph.  P is the reference's (amg.h:326-387): a C row maps to
// itself, an F row to each of its C neighbours with weight w = 1/count.  So
//
//   (A P)(i, k)   = sum over the entries j of row i, in stored order, with
//                   k in P(j) -- j = k, or j an F neighbour of k -- of
//                   a_ij * w_j;
//   (P^T A P)(e, k) = sum over i in R(e) = {c_e} + the F neighbours of the
//                   C cell c_e, ascending, of (A P)(i, k) * w_i;
//
// the order sparse_multiply_transpose adds them in (amg.h:520-546), first
// term as is and the rest with round-to-nearest adds: bit-identical to the
// generic kernels of amg_setup.cu (and to the reference).
//
// The columns of (A P)(i) are C cells within fine L1 distance 4 of i (85
// candidate offsets), those of a coarse row within distance 6 of c_e (231
// offsets).  An independent set of the 19-offset graph holds at most 19
// cells of the first ball and 45 of the second (maximum independent sets of
// those balls), which sizes the padded rows.  A row over either size, or a
// level whose stored pattern is not the 19-offset one, makes the caller fall
// back to the generic product.
#include <utility>

#include "grid19.cuh"
#include "hm.cuh"

namespace hm {

namespace {

constexpr int kB4 = 85, kB6 = 231;
constexpr int kCap0 = 20;   // (A P) row: at most 19 C cells
constexpr int kCap1 = 48;   // coarse row: at most 45
constexpr int kCentre = 9;  // q19 of offset 0

__host__ __device__ constexpr int iabs(int v) { return v < 0 ? -v : v; }

// the n-th offset with |dx|+|dy|+|dz| <= R and dx+dy+dz even, in ascending
// (dz, dy, dx) order, which is ascending fine index for every in-grid pair;
// axis 0 x, 1 y, 2 z
__host__ __device__ constexpr int ball_pos(int R, int n, int axis)
{
    int c = 0;
    for (int dz = -R; dz <= R; dz++)
        for (int dy = -R; dy <= R; dy++)
            for (int dx = -R; dx <= R; dx++) {
                if (iabs(dx) + iabs(dy) + iabs(dz) > R || ((dx + dy + dz) & 1)) continue;
                if (c == n) return axis == 0 ? dx : axis == 1 ? dy : dz;
                c++;
            }
    return 1 << 20;
}

struct G19L {
    int nx, ny, nz, hx;  // fine grid, hx = nx / 2 (fine cells < 2^31)
    int nxy;
};

// fine coordinates and index of level row r
__device__ __forceinline__ int row_cell(const G19L &g, int r, int &x, int &y, int &z)
{
    const unsigned t = (unsigned)r / (unsigned)g.hx;
    const unsigned zz = t / (unsigned)g.ny;
    y = (int)(t - zz * (unsigned)g.ny);
    z = (int)zz;
    const int par = (y + z) & 1;
    x = 2 * (r - (int)t * g.hx) + par;
    return 2 * r + par;
}

__device__ __forceinline__ bool in_grid3(const G19L &g, int x, int y, int z)
{
    return (unsigned)x < (unsigned)g.nx && (unsigned)y < (unsigned)g.ny &&
           (unsigned)z < (unsigned)g.nz;
}

__host__ __device__ constexpr int q19_lin32(int q, int nx, int nxy)
{
    return q19x(q) + q19y(q) * nx + q19z(q) * nxy;
}

// ---- stage 0: (A P) rows, one thread per level row ----------------------

struct Row0 {
    double t[kQ19];   // a_ij * w_j per stored offset q (0 where absent)
    double tf[kQ19];  // t where q's cell is F, else -0.0
    double w;         // the row's own P weight
    unsigned fm;      // q: in grid and F
    unsigned cm[3];   // ball-4 offsets: in grid and C
};

// The ball-4 offsets with the same (dy, dz) are a run of m + 1 offsets,
// dx = -m, -m+2, .., m (m = 4 - |dy| - |dz|), i.e. m + 1 consecutive level
// rows; runs are numbered in (dz, dy) order, and run R starts at ball index
// run_first(R).
__host__ __device__ constexpr int run_dz(int R)
{
    int c = 0;
    for (int dz = -4; dz <= 4; dz++)
        for (int dy = -4; dy <= 4; dy++) {
            if (iabs(dy) + iabs(dz) > 4) continue;
            if (c == R) return dz;
            c++;
        }
    return 99;
}
__host__ __device__ constexpr int run_dy(int R)
{
    int c = 0;
    for (int dz = -4; dz <= 4; dz++)
        for (int dy = -4; dy <= 4; dy++) {
            if (iabs(dy) + iabs(dz) > 4) continue;
            if (c == R) return dy;
            c++;
        }
    return 99;
}
__host__ __device__ constexpr int ball4_index(int dx, int dy, int dz)
{
    for (int P = 0; P < kB4; P++)
        if (ball_pos(4, P, 0) == dx && ball_pos(4, P, 1) == dy && ball_pos(4, P, 2) == dz)
            return P;
    return -1;
}
constexpr int kRuns = 41;

// C flags of the run: bits of the level's C-flag words (word -1 and the
// word past the end are padding), masked by the x range of this row
template <int R>
__device__ __forceinline__ void load_run(const G19L &g, int y, int z, int s, unsigned ve,
                                         unsigned vo, const unsigned *__restrict__ cbits,
                                         Row0 &Rw)
{
    constexpr int dy = run_dy(R), dz = run_dz(R), m = 4 - iabs(dy) - iabs(dz);
    constexpr int P0 = ball4_index(-m, dy, dz);
    static_assert(P0 >= 0, "run start");
    if ((unsigned)(y + dy) >= (unsigned)g.ny || (unsigned)(z + dz) >= (unsigned)g.nz) return;
    const int b0 = (s - m + dy * g.nx + dz * g.nxy) >> 1;  // >= -2
    const int wi = b0 >> 5;
    const unsigned bits = __funnelshift_r(cbits[wi], cbits[wi + 1], (unsigned)b0 & 31u);
    // x range: ve bit k is dx = -4 + 2k, vo bit k is dx = -3 + 2k
    const unsigned xm = (m & 1) ? (vo >> ((3 - m) / 2)) : (ve >> ((4 - m) / 2));
    const unsigned run = bits & xm & ((1u << (m + 1)) - 1u);
    Rw.cm[P0 >> 5] |= run << (P0 & 31);
    if constexpr ((P0 & 31) + m + 1 > 32) Rw.cm[(P0 >> 5) + 1] |= run >> (32 - (P0 & 31));
}

template <int... R>
__device__ __forceinline__ void load_runs(const G19L &g, int y, int z, int s, unsigned ve,
                                          unsigned vo, const unsigned *__restrict__ cbits,
                                          Row0 &Rw, std::integer_sequence<int, R...>)
{
    (load_run<R>(g, y, z, s, ve, vo, cbits, Rw), ...);
}

// F flags of the stored offsets: in grid and not C
template <int... Q>
__device__ __forceinline__ unsigned f_flags(unsigned pm, const Row0 &Rw,
                                            std::integer_sequence<int, Q...>)
{
    unsigned fm = 0;
    ((fm |= ((pm >> Q) & ~(Rw.cm[ball4_index(q19x(Q), q19y(Q), q19z(Q)) >> 5] >>
                           (ball4_index(q19x(Q), q19y(Q), q19z(Q)) & 31)) & 1u) << Q), ...);
    return fm;
}

// stored offset Q reaches ball-4 offset P through q19 offset pair_q2(P, Q)
// (or -1): Q's cell j is P's cell k (pair_q2 = the centre) or j's
// neighbour
__host__ __device__ constexpr int pair_q2(int P, int Q)
{
    return q19_of(ball_pos(4, P, 0) - q19x(Q), ball_pos(4, P, 1) - q19y(Q),
                  ball_pos(4, P, 2) - q19z(Q));
}
// the Q that reach P through an F cell j
__host__ __device__ constexpr unsigned fmask_of(int P)
{
    unsigned m = 0;
    for (int Q = 0; Q < kQ19; Q++) {
        const int q2 = pair_q2(P, Q);
        if (q2 >= 0 && q2 != kCentre) m |= 1u << Q;
    }
    return m;
}

// Every sum starts from -0.0, and a term that does not apply is -0.0 too:
// x + (-0.0) = x exactly for every x, so the first applying term enters as
// is and the rest are added in order, as in the generic kernels.
template <int P, int Q>
__device__ __forceinline__ void fold_q(const Row0 &R, double &acc)
{
    constexpr int q2 = pair_q2(P, Q);
    if constexpr (q2 == kCentre) acc = dadd(acc, R.t[Q]);  // j = k, a C cell
    else if constexpr (q2 >= 0) acc = dadd(acc, R.tf[Q]);  // j F
}

template <int P, int... Q>
__device__ __forceinline__ void fold_p(const Row0 &R, int &u, long o, unsigned char *op,
                                       double *ov, std::integer_sequence<int, Q...>)
{
    if (!((R.cm[P >> 5] >> (P & 31)) & 1u)) return;
    double acc = -0.0;
    (fold_q<P, Q>(R, acc), ...);
    // a C cell in the 19-point ball always has a term (itself); others one
    // per F neighbour of theirs in row i
    constexpr bool centre = q19_of(ball_pos(4, P, 0), ball_pos(4, P, 1), ball_pos(4, P, 2)) >= 0;
    constexpr unsigned fm = fmask_of(P);
    if (centre || (R.fm & fm)) {
        if (u < kCap0) {  // stored times w_i, the factor of the second stage
            op[o + u] = (unsigned char)P;
            ov[o + u] = dmul(acc, R.w);
        }
        u++;
    }
}

template <int... P>
__device__ __forceinline__ void fold_all(const Row0 &R, int &u, long o, unsigned char *op,
                                         double *ov, std::integer_sequence<int, P...>)
{
    (fold_p<P>(R, u, o, op, ov, std::make_integer_sequence<int, kQ19>{}), ...);
}

__global__ void __launch_bounds__(128, 5)
k_g19_ap(G19L g, int n, const int *__restrict__ rowptr, const double *__restrict__ val,
         const unsigned *__restrict__ cbits, const double *__restrict__ pw,
         int *__restrict__ ucnt, unsigned char *__restrict__ op, double *__restrict__ ov,
         int *err)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        int x, y, z;
        const int s = row_cell(g, r, x, y, z);
        unsigned pm = 0;
#pragma unroll
        for (int q = 0; q < kQ19; q++)
            pm |= (unsigned)in_grid3(g, x + q19x(q), y + q19y(q), z + q19z(q)) << q;
        const int rb = rowptr[r];
        if (rowptr[r + 1] - rb != __popc(pm)) {  // not the 19-offset pattern
            atomicExch(err, 1);
            ucnt[r] = 0;
            continue;
        }
        Row0 R;
        R.cm[0] = R.cm[1] = R.cm[2] = 0;
        R.w = pw[r];
#pragma unroll
        for (int q = 0; q < kQ19; q++) {
            R.t[q] = 0.0;
            if ((pm >> q) & 1u) {
                const int j = (s + q19_lin32(q, g.nx, g.nxy)) >> 1;
                R.t[q] = dmul(val[rb + __popc(pm & ((1u << q) - 1))], pw[j]);
            }
        }
        unsigned ve = 0, vo = 0;
#pragma unroll
        for (int k = 0; k < 5; k++) ve |= (unsigned)((unsigned)(x - 4 + 2 * k) < (unsigned)g.nx) << k;
#pragma unroll
        for (int k = 0; k < 4; k++) vo |= (unsigned)((unsigned)(x - 3 + 2 * k) < (unsigned)g.nx) << k;
        load_runs(g, y, z, s, ve, vo, cbits, R, std::make_integer_sequence<int, kRuns>{});
        R.fm = f_flags(pm, R, std::make_integer_sequence<int, kQ19>{});
#pragma unroll
        for (int q = 0; q < kQ19; q++) R.tf[q] = ((R.fm >> q) & 1u) ? R.t[q] : -0.0;
        int u = 0;
        fold_all(R, u, (long)r * kCap0, op, ov, std::make_integer_sequence<int, kB4>{});
        if (u > kCap0) atomicExch(err, 2);
        constexpr int pc = ball4_index(0, 0, 0);
        const unsigned is_c = (R.cm[pc >> 5] >> (pc & 31)) & 1u;
        ucnt[r] = (u < kCap0 ? u : kCap0) | (int)(is_c << 8);
    }
}

// C flags as bits: bit r % 32 of word r / 32 is row r's; words up to nw
__global__ void k_cbits(const signed char *__restrict__ sel, int n, int nw, unsigned *bits)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nw * 32;
         r += gridDim.x * blockDim.x) {
        const unsigned b = __ballot_sync(0xffffffffu, r < n && sel[r] == 1);
        if ((threadIdx.x & 31) == 0) bits[r >> 5] = b;
    }
}

// ---- stage 1: coarse rows, one warp per row ---------------------------------

// Offset tables of the second stage (built on the host): the ball-6 slot of
// q19 offset q plus ball-4 offset P, and each ball-6 offset.
struct T6 {
    unsigned char map[kQ19 * kB4];
    signed char pos[kB6][3];
};

constexpr int kWarps1 = 8;

// The terms of a coarse row, in order (the rows of R(e) ascending, each
// row's entries), are taken 32 at a time; lanes whose terms go to the same
// slot are grouped and the group's lowest lane adds them in lane order, so
// every slot's sum keeps the order.
__global__ void __launch_bounds__(32 * kWarps1)
k_g19_ptap(G19L g, T6 tb, const int *__restrict__ cpts, int nc,
           const int *__restrict__ cid, const int *__restrict__ ucnt0,
           const unsigned char *__restrict__ op, const double *__restrict__ ov,
           int *__restrict__ ucnt1, int *__restrict__ pcol, double *__restrict__ pval, int *err)
{
    __shared__ unsigned char s_map[kQ19 * kB4];
    __shared__ int s_lin[kB6];
    __shared__ double s_acc[kWarps1][kB6];
    __shared__ double s_v[kWarps1][32];
    __shared__ unsigned s_has[kWarps1][8];  // slots holding a value
    for (int q = threadIdx.x; q < kQ19 * kB4; q += blockDim.x) s_map[q] = tb.map[q];
    for (int q = threadIdx.x; q < kB6; q += blockDim.x)
        s_lin[q] = tb.pos[q][0] + tb.pos[q][1] * g.nx + tb.pos[q][2] * g.nxy;
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *acc = s_acc[w];
    double *sv = s_v[w];
    unsigned *has = s_has[w];
    for (long e = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5; e < nc;
         e += ((long)gridDim.x * blockDim.x) >> 5) {
        int x, y, z;
        const int s = row_cell(g, cpts[e], x, y, z);
        // R(e): the C cell itself and its F neighbours, ascending; lane q
        // holds offset q's row and its (A P) length (bit 8 of ucnt0: a C row)
        int ri = 0;
        int ul = 0;
        if (lane < kQ19 && in_grid3(g, x + q19x(lane), y + q19y(lane), z + q19z(lane))) {
            ri = (s + q19_lin32(lane, g.nx, g.nxy)) >> 1;
            const int uf = ucnt0[ri];
            if (lane == kCentre || !(uf & 256)) ul = uf & 255;
        }
        int inc = ul;  // inclusive scan: the terms of rows 0..lane
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= d) inc += t;
        }
        const int total = __shfl_sync(0xffffffffu, inc, 31);
        if (lane < 8) has[lane] = 0;
        __syncwarp();
        for (int k0 = 0; k0 < total; k0 += 32) {
            const int k = k0 + lane;
            // term k's row: the number of rows whose terms end at or before k
            int q = 0;
#pragma unroll
            for (int b = 16; b > 0; b >>= 1)
                if (__shfl_sync(0xffffffffu, inc, q + b - 1) <= k) q += b;
            const int first = __shfl_sync(0xffffffffu, inc, q) - __shfl_sync(0xffffffffu, ul, q);
            const int iq = __shfl_sync(0xffffffffu, ri, q);
            int sl = -1 - lane;  // distinct for lanes past the end
            double v = 0.0;
            if (k < total) {
                const long at = (long)iq * kCap0 + (k - first);
                sl = s_map[q * kB4 + op[at]];
                v = ov[at];
            }
            sv[lane] = v;
            const unsigned grp = __match_any_sync(0xffffffffu, sl);
            __syncwarp();
            if (k < total && lane == __ffs(grp) - 1) {
                const unsigned bit = 1u << (sl & 31);
                double a = (has[sl >> 5] & bit) ? dadd(acc[sl], v) : v;
                for (unsigned m = grp & (grp - 1); m; m &= m - 1) a = dadd(a, sv[__ffs(m) - 1]);
                acc[sl] = a;
                atomicOr(&has[sl >> 5], bit);
            }
            __syncwarp();
        }
        // emit the slots in order (ascending column)
        int u = 0;
        const long o = e * kCap1;
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const unsigned hw = has[r];
            const int p = r * 32 + lane;
            if ((hw >> lane) & 1u) {
                const int k = u + __popc(hw & ((1u << lane) - 1));
                if (k < kCap1) {
                    pcol[o + k] = cid[(s + s_lin[p]) >> 1];
                    pval[o + k] = acc[p];
                }
            }
            u += __popc(hw);
        }
        if (lane == 0) {
            if (u > kCap1) atomicExch(err, 2);
            ucnt1[e] = u < kCap1 ? u : kCap1;
        }
        __syncwarp();
    }
}

__global__ void k_cpts(const signed char *__restrict__ sel, const int *__restrict__ cid,
                       long n, int *cpts)
{
    for (long r = blockIdx.x * (long)blockDim.x + threadIdx.x; r < n;
         r += (long)gridDim.x * blockDim.x)
        if (sel[r] == 1) cpts[cid[r]] = (int)r;
}

__global__ void k_compact_rows(const int *__restrict__ rowptr, int n, int stride,
                               const int *__restrict__ pcol, const double *__restrict__ pval,
                               int *col, double *val)
{
    const int lane = threadIdx.x & 31;
    for (long r = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5; r < n;
         r += ((long)gridDim.x * blockDim.x) >> 5) {
        const int dst = rowptr[r], len = rowptr[r + 1] - dst;
        for (int q = lane; q < len; q += 32) {
            col[dst + q] = pcol[r * (long)stride + q];
            val[dst + q] = pval[r * (long)stride + q];
        }
    }
}

// R = P^T of the level: coarse row e lists its C row and that row's F
// neighbours, ascending (the rows whose P holds e).  A thread per level row;
// C rows only.
// (every row's stored length is checked against the 19-offset pattern)
__global__ void k_g19_rcount(G19L g, int n, const int *__restrict__ rowptr,
                             const signed char *__restrict__ sel,
                             const int *__restrict__ cid, int *cnt, int *bad)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        int x, y, z;
        const int s = row_cell(g, r, x, y, z);
        unsigned pm = 0;
#pragma unroll
        for (int q = 0; q < kQ19; q++)
            pm |= (unsigned)in_grid3(g, x + q19x(q), y + q19y(q), z + q19z(q)) << q;
        if (rowptr[r + 1] - rowptr[r] != __popc(pm)) *bad = 1;
        if (sel[r] != 1) continue;
        int c = 0;
#pragma unroll
        for (int q = 0; q < kQ19; q++)
            if (q == kCentre ||
                (in_grid3(g, x + q19x(q), y + q19y(q), z + q19z(q)) &&
                 sel[(s + q19_lin32(q, g.nx, g.nxy)) >> 1] == 2))
                c++;
        cnt[cid[r]] = c;
    }
}

__global__ void k_g19_rfill(G19L g, int n, const signed char *__restrict__ sel,
                            const int *__restrict__ cid, const int *__restrict__ rrow, int *rcol)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        if (sel[r] != 1) continue;
        int x, y, z;
        const int s = row_cell(g, r, x, y, z);
        int o = rrow[cid[r]];
#pragma unroll
        for (int q = 0; q < kQ19; q++) {
            if (q == kCentre) {
                rcol[o++] = r;
                continue;
            }
            if (!in_grid3(g, x + q19x(q), y + q19y(q), z + q19z(q))) continue;
            const int j = (s + q19_lin32(q, g.nx, g.nxy)) >> 1;
            if (sel[j] == 2) rcol[o++] = j;
        }
    }
}

T6 make_t6()
{
    T6 t;
    int idx[13][13][13];
    for (int a = 0; a < 13; a++)
        for (int b = 0; b < 13; b++)
            for (int c = 0; c < 13; c++) idx[a][b][c] = -1;
    for (int p = 0; p < kB6; p++) {
        const int dx = ball_pos(6, p, 0), dy = ball_pos(6, p, 1), dz = ball_pos(6, p, 2);
        t.pos[p][0] = (signed char)dx;
        t.pos[p][1] = (signed char)dy;
        t.pos[p][2] = (signed char)dz;
        idx[dz + 6][dy + 6][dx + 6] = p;
    }
    for (int q = 0; q < kQ19; q++)
        for (int P = 0; P < kB4; P++) {
            const int dx = q19x(q) + ball_pos(4, P, 0), dy = q19y(q) + ball_pos(4, P, 1),
                      dz = q19z(q) + ball_pos(4, P, 2);
            t.map[q * kB4 + P] = (unsigned char)idx[dz + 6][dy + 6][dx + 6];
        }
    return t;
}

int blocks_for(long n, int threads, long cap = 148L * 16)
{
    long b = ceil_div(n, threads);
    if (b < 1) b = 1;
    return (int)(b < cap ? b : cap);
}

}  // namespace

int g19_transpose(const Level &L, Csr &R, cudaStream_t st, bool *done)
{
    *done = false;
    const Grid19 &gg = L.g19;
    if (gg.nx <= 0 || (gg.nx & 1) || gg.nx < 4 || gg.ny < 4) return HMFEM_OK;
    if ((long)gg.nx * gg.ny * gg.nz > (1l << 30)) return HMFEM_OK;
    const G19L g{gg.nx, gg.ny, gg.nz, gg.nx / 2, gg.nx * gg.ny};
    const long n = L.A.n;
    if (n != (long)g.hx * g.ny * g.nz || L.nc < 1) return HMFEM_OK;
    int *bad = (int *)dalloc(sizeof(int));
    if (!bad) return HMFEM_E_CUDA;
    HM_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), st));
    HM_CUDA(cudaMemsetAsync(R.rowptr, 0, sizeof(int) * ((long)L.nc + 1), st));
    k_g19_rcount<<<blocks_for(n, 256), 256, 0, st>>>(g, (int)n, L.A.rowptr, L.sel, L.cid,
                                                      R.rowptr, bad);
    HM_LAUNCHED();
    int hbad = 0;
    HM_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    long nnz = 0;
    HM_CHECK(rowptr_from_counts(R.rowptr, L.nc, st, &nnz));  // synchronises
    dfree(bad);
    // not this structure: the radix sort forms R
    if (hbad || nnz != L.P.nnz) return HMFEM_OK;
    k_g19_rfill<<<blocks_for(n, 256), 256, 0, st>>>(g, (int)n, L.sel, L.cid, R.rowptr, R.col);
    HM_LAUNCHED();
    *done = true;
    return HMFEM_OK;
}

int g19_cpts(Level &L, cudaStream_t st)
{
    dfree(L.cpts);
    L.cpts = (int *)dalloc(sizeof(int) * (L.nc > 0 ? L.nc : 1));
    if (!L.cpts) return HMFEM_E_CUDA;
    k_cpts<<<blocks_for(L.A.n, 256), 256, 0, st>>>(L.sel, L.cid, L.A.n, L.cpts);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int galerkin19(const Level &L, Csr &out, cudaStream_t st, bool *done)
{
    *done = false;
    const Grid19 &gg = L.g19;
    if (gg.nx <= 0 || (gg.nx & 1) || gg.nx < 4 || gg.ny < 4) return HMFEM_OK;
    if ((long)gg.nx * gg.ny * gg.nz > (1l << 30)) return HMFEM_OK;  // 32-bit indices
    const G19L g{gg.nx, gg.ny, gg.nz, gg.nx / 2, gg.nx * gg.ny};
    const long n = L.A.n, nc = L.nc;
    if (n != (long)g.hx * g.ny * g.nz || nc < 1 || !L.cpts) return HMFEM_OK;
    int *ucnt0 = (int *)dalloc(sizeof(int) * n);
    unsigned char *op = (unsigned char *)dalloc((size_t)n * kCap0);
    double *ov = (double *)dalloc(sizeof(double) * n * kCap0);
    const int *cpts = L.cpts;
    int *pcol = (int *)dalloc(sizeof(int) * nc * kCap1);
    double *pval = (double *)dalloc(sizeof(double) * nc * kCap1);
    int *err = (int *)dalloc(sizeof(int));
    const int nw = (int)((n - 1) / 32 + 2);  // C-flag words, and one word of padding
    unsigned *cb = (unsigned *)dalloc(sizeof(unsigned) * (nw + 1));
    out.n = (int)nc;
    out.rowptr = (int *)dalloc(sizeof(int) * (nc + 1));
    auto release = [&]() {
        dfree(ucnt0); dfree(op); dfree(ov); dfree(pcol); dfree(pval); dfree(err);
        dfree(cb);
    };
    if (!ucnt0 || !op || !ov || !pcol || !pval || !err || !cb || !out.rowptr) {
        release();
        set_last_error("out of device memory (19-point RAP)", __FILE__, __LINE__);
        return HMFEM_E_CUDA;
    }
    HM_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    HM_CUDA(cudaMemsetAsync(cb, 0, sizeof(unsigned), st));  // word -1
    k_cbits<<<blocks_for((long)nw * 32, 256), 256, 0, st>>>(L.sel, (int)n, nw, cb + 1);
    HM_LAUNCHED();
    k_g19_ap<<<occ_blocks((const void *)k_g19_ap, n, 128, 148 * 16), 128, 0, st>>>(
        g, (int)n, L.A.rowptr, L.A.val, cb + 1, L.pw, ucnt0, op, ov, err);
    HM_LAUNCHED();
    HM_PHASE("    (A P) rows", st);
    static const T6 tb = make_t6();
    k_g19_ptap<<<occ_blocks((const void *)k_g19_ptap, nc * 32, 32 * kWarps1, 148 * 8),
                 32 * kWarps1, 0, st>>>(g, tb, cpts, (int)nc, L.cid, ucnt0, op, ov,
                                        out.rowptr, pcol, pval, err);
    HM_LAUNCHED();
    HM_PHASE("    coarse rows", st);
    int herr = 0;
    HM_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    HM_CHECK(rowptr_from_counts(out.rowptr, (int)nc, st, &out.nnz));  // synchronises
    if (herr) {  // not this structure after all: the generic product runs
        release();
        dfree(out.rowptr);
        out = Csr();
        return HMFEM_OK;
    }
    out.col = (int *)dalloc(sizeof(int) * (out.nnz > 0 ? out.nnz : 1));
    out.val = (double *)dalloc(sizeof(double) * (out.nnz > 0 ? out.nnz : 1));
    if (!out.col || !out.val) {
        release();
        set_last_error("out of device memory (19-point RAP)", __FILE__, __LINE__);
        return HMFEM_E_CUDA;
    }
    k_compact_rows<<<blocks_for(nc * 32, 256, 148L * 32), 256, 0, st>>>(
        out.rowptr, (int)nc, kCap1, pcol, pval, out.col, out.val);
    HM_LAUNCHED();
    release();
    *done = true;
    return HMFEM_OK;
}

}  // namespace hm
