// hm.cuh -- solver data structures and launcher prototypes shared by the
// hmfem B200 translation units.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

namespace hm {

// Compressed rows: rowptr[n+1], col/val[nnz].  Rows keep the producer's
// column order (level 0: d,l,c,r,u,t,b as solve_linsys packs it; coarse
// levels: ascending, as new_triple_product leaves them).
struct Csr {
    int n = 0;
    long nnz = 0;
    int *rowptr = nullptr;
    int *col = nullptr;
    double *val = nullptr;
};

// SELL-32: slices of 32 rows, each padded to its longest row; element k of
// row r lives at sptr[r/32] + k*32 + r%32 (warp-coalesced).  Padding has
// col = the row itself (or 0 past n) and value 0.
struct Sell {
    int n = 0;
    int nslices = 0;
    long len = 0;             // padded entries
    long long *sptr = nullptr;  // nslices+1
    int *col = nullptr;
    double *val = nullptr;    // FP64 values
    float *val32 = nullptr;   // FP32 copy (mixed-precision V-cycle)
    __nv_bfloat16 *val16 = nullptr;  // BF16 copy (coarse levels)
    // BF16 levels whose every column is within +-32767 of its row: one
    // 32-bit word per entry, the column offset (int16) in the high half and
    // the BF16 bits in the low half (2/3 of the bytes of col + val16)
    unsigned *pk = nullptr;
};

// Solve-phase forms of the two finest levels of a matrix assembled on the
// device (stencil_cycle.cu).  Both keep their coefficients slice-interleaved
// like SELL-32 without column indices: the coefficients of rows 32t..32t+31
// form one contiguous block, coefficient k of row r at
// (r / 32) * K * 32 + k * 32 + r % 32, so a warp reads one stream.
//
// Level 0 (K = 4): the 7-point stencil as a_cc and the couplings to the +x,
// +y, +z neighbours (0 where absent); the coupling to -x is the -x
// neighbour's +x one, and so on (the matrix is checked to be bitwise
// symmetric first).
struct Grid7 {
    int nx = 0, ny = 0, nz = 0;
    double *cf = nullptr;
    float *cf32 = nullptr;
};

// Level 1 of the parity split (K = 19; nx even, nx >= 4, ny >= 4): even
// cell s has coarse id s >> 1; coefficient q (grid19.cuh) of a row is 0
// where that neighbour is outside the grid.
struct Grid19 {
    int nx = 0, ny = 0, nz = 0;
    double *v = nullptr;
    float *v32 = nullptr;
    __nv_bfloat16 *v16 = nullptr;
};

// index of coefficient k of row r in a slice-interleaved array of K per row
__host__ __device__ __forceinline__ long long slice_at(long long r, int k, int K)
{
    return (r >> 5) * (32LL * K) + k * 32 + (r & 31);
}
__host__ __device__ __forceinline__ long long slice_len(long long n, int K)
{
    return ((n + 31) >> 5) * 32LL * K;
}

struct Level {
    Csr A;
    Grid7 g7;      // set on level 0 when the structured form applies
    Grid19 g19;    // set on level 1 when the structured form applies
    Sell S;
    double *dinv = nullptr;   // 1 / last stored diagonal entry (amg.h:1195)
    float *dinv32 = nullptr;
    double *dsm = nullptr;    // smoother diagonal inverse (Jacobi or l1)
    float *dsm32 = nullptr;
    // transfer to level+1 (absent on the coarsest)
    signed char *sel = nullptr;  // 1 = C, 2 = F
    bool sel_split = false;           // sel formed early on a side stream,
    cudaEvent_t sel_ready = nullptr;  // complete once this event is
    int *split_work = nullptr;        // that split's flags, ticket, error word
    int *split_err = nullptr;         // (freed once the split is consumed)
    int *cid = nullptr;          // coarse id of C rows (prefix count)
    int nc = 0;
    Csr P;                    // P rows: coarse ids in the fine row's order
    double *pw = nullptr;     // 1 / pcnt per fine row (the P weights)
    float *pw32 = nullptr;
    Csr R;                    // P^T rows: fine ids ascending
    bool p_deferred = false;  // P not formed (level 0 of the exact reduction)
    int *cpts = nullptr;      // 19-offset level: the row of each coarse row (setup)
    // V-cycle vectors (FP64 and FP32 sets)
    double *f = nullptr, *ua = nullptr, *ub = nullptr, *rs = nullptr;
    float *f32 = nullptr, *ua32 = nullptr, *ub32 = nullptr, *rs32 = nullptr;
    // Chebyshev smoother (levels >= cheb_from): second search direction
    bool cheb = false;
    double *dx = nullptr;
    float *dx32 = nullptr;
    // multicolour Gauss-Seidel smoother (levels >= gs_from)
    bool gs = false;
    int ncolors = 0;
    signed char *color = nullptr;     // Jones-Plassmann colouring
    int *crows = nullptr;             // rows grouped by colour
    std::vector<long> color_slot;     // first row of each colour in crows
    int *cslot = nullptr;             // the same offsets on the device
    float *aval32 = nullptr;          // CSR values in FP32 / BF16 (GS levels)
    __nv_bfloat16 *aval16 = nullptr;
};

// Device-resident CG state; kernels read the scalars they need from here,
// so an iteration runs without host round trips.
struct Ctl {
    double sigma, sigma_last, sigma_first, tau, alpha, beta;
    double rr, bb, trr, tol2, rz_old;
    int done, check, iters, status, max_iter, stop_rule, nrep, pad;
    unsigned tickets[16];
};

// reduction slots (tickets[] index + partial buffer row)
enum { RED_TAU = 0, RED_RR, RED_SIGMA, RED_TRR, RED_BB, RED_A, RED_B, RED_C,
       RED_SLOTS };

// ---- launchers (all enqueue on `st`) ---------------------------------
// assembly / flux (assemble.cu)
int launch_l0_rowcounts(int nx, int ny, int nz, int *cnt, cudaStream_t st);
int launch_assemble(int nx, int ny, int nz, double hx, double hy, double hz,
                    double visc, const double *KX, const double *KY,
                    const double *KZ, const int bc[6], double *const face[6],
                    const double *KI, const double *WI, const double *pc,
                    const double *pw, const int *rowptr, int *col, double *val,
                    double *b, cudaStream_t st, int *bad = nullptr);
int launch_exchange_rhs(int nx, int ny, int nz, double hx, double hy, double hz,
                        double visc, const double *KX, const double *KY,
                        const double *KZ, const int bc[6], double *const face[6],
                        int m, const int *own, const int *ecell, const double *pc,
                        const double *KI, const double *WI, const double *pw,
                        double *b, cudaStream_t st);
int launch_pack_stencil(int n, const hmfem_ele *perm, const hmfem_ind *ind,
                        int *cnt, const int *rowptr, int *col, double *val,
                        int pass, cudaStream_t st, int *bad = nullptr);
int launch_flux(int nx, int ny, int nz, double hx, double hy, double hz,
                double visc, const double *KX, const double *KY,
                const double *KZ, const int bc[6], double *const face[6],
                const double *p, hmfem_ele *v, double *mm, cudaStream_t st);

// sparse utilities (sparse.cu)
int scan_exclusive(const int *in, int *out, int n, cudaStream_t st);
int rowptr_from_counts(int *rowptr, int n, cudaStream_t st, long *nnz_out);
int csr_to_sell(const Csr &A, Sell &S, cudaStream_t st);
int sell_fill_lowp(Sell &S, bool f32, bool bf16, cudaStream_t st);
struct Level;
int csr_fill_lowp(Level &L, bool bf16, cudaStream_t st);
int launch_diag_inv(const Csr &A, double *dinv, float *dinv32, cudaStream_t st,
                    int *bad = nullptr);
int launch_validate_counts(const int *cnt, int n, int *bad, cudaStream_t st);
int launch_validate_cols(const int *col, long nnz, int n, int *bad, cudaStream_t st);
int launch_spmv(const Sell &S, const double *x, double *y, cudaStream_t st);

// AMG setup (amg_setup.cu)
// grid3 (nx, ny, nz) marks a level-0 matrix assembled on the device: its
// split and Galerkin product then come from the 7-point structure
// (rap_stencil.cu), bit-identical to the generic kernels.
int amg_coarsen(Level &L, Level &C, cudaStream_t st, int *err_dev,
                const int *grid3 = nullptr, bool schur = false);
// the reference's P of a level whose setup left it out (p_deferred)
int ensure_p(Level &L, cudaStream_t st);
int stencil_parity_split(int nx, int ny, int nz, signed char *sel, cudaStream_t st);
// R = P^T of the parity split (rowptr / col allocated by the caller, R.nnz
// set to P's nnz)
int stencil_parity_R(int nx, int ny, int nz, const int *cid, int nc, Csr &R, cudaStream_t st);
// level 1 of a parity split (nx even, nx, ny >= 4): its greedy C/F split
// from the 19-offset structure, the x-row wavefront in one launch; work
// holds stencil19_split_work_ints(nx, ny, nz) ints (8-byte aligned), the
// last one the error word (1 when a bounded wait gave up)
long stencil19_split_work_ints(int nx, int ny, int nz);
int stencil19_split(int nx, int ny, int nz, signed char *sel, int *work, cudaStream_t st);
// the poll limit of the splits' bounded waits (HMFEM_TEST_POLL_LIMIT lowers it)
long long split_poll_limit();
// schur: the exact red-black reduction's level 1 instead of the Galerkin
// product with the averaging interpolation (same rows and columns)
int stencil_galerkin(int nx, int ny, int nz, const Level &L, Csr &out,
                     double *g19v, cudaStream_t st, bool schur = false);
// P^T A P of a level with the 19-offset structure (L.g19 set: level 1 of a
// parity split) from that structure, bit-identical to the generic product;
// *done false (and out untouched) when the level does not have it
int galerkin19(const Level &L, Csr &out, cudaStream_t st, bool *done);
// R = P^T of such a level from its structure (R.rowptr / R.col allocated by
// the caller, P formed); *done false when the level does not have it
int g19_transpose(const Level &L, Csr &R, cudaStream_t st, bool *done);
// L.cpts of such a level (its C rows in coarse-id order, for galerkin19)
int g19_cpts(Level &L, cudaStream_t st);
// colouring + rows grouped by colour; returns HMFEM_OK with L.gs = false
// when the level needs more than 63 colours
int color_level(Level &L, cudaStream_t st, int *dwork);
// structured solve-phase forms (stencil_cycle.cu): g7_build fills L.g7 from
// the assembled CSR and returns HMFEM_OK with L.g7.c == nullptr when the
// matrix is not bitwise symmetric; g19 values come from stencil_galerkin.
int g7_build(Level &L, int nx, int ny, int nz, bool f32, cudaStream_t st, int *dwork);
void g7_free(Grid7 &g);
bool g19_applies(int nx, int ny, int nz);
int g19_lowp(Grid19 &g, int n, bool f32, bool bf16, cudaStream_t st);
void g19_free(Grid19 &g);

// cycle + CG (cycle.cu)
struct Solver;
// seeded: the level-0 smoother's first iterate was written by the producer
// of the right-hand side (the CG kernels); otherwise the cycle writes it
int cycle_fp64(Solver &s, int l, cudaStream_t st, bool dot_into_sigma, bool seeded);
int cycle_fp32(Solver &s, int l, cudaStream_t st, bool dot_into_sigma, bool seeded);

int occ_blocks(const void *kernel, long n, int threads, int cap);
void *dalloc(size_t bytes);
void dfree(void *p);
void set_alloc_stream(cudaStream_t st);  // stream that orders dalloc/dfree
struct AllocCache;                       // per-solver exact-size block cache
void set_alloc_context(cudaStream_t st, AllocCache *c);
void get_alloc_context(cudaStream_t *st, AllocCache **c);
AllocCache *alloc_cache_new();
void alloc_cache_release(AllocCache *c);

}  // namespace hm
