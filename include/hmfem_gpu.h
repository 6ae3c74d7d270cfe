/*
 * hmfem_gpu.h -- C-ABI of the B200 (sm_100a) pressure solver for hmfem.
 *
 * Three layers, all plain C types (pointers, sizes, status codes):
 *
 *  1. The reference's own bridge, same names and argument meaning, so the
 *     hmfem application links against this library instead of compute.cpp:
 *       compute       -- replaces compute.cpp:7-51 (declared functions.h:53)
 *       solve_linsys  -- replaces solve_linearsystem_AMG.c:37-157
 *                        (declared functions.h:54)
 *     The application compiles its .c files with g++ (makefile:40-41), so
 *     both symbols are also exported under their C++ names.
 *
 *  2. The reference's device layer (toolbox/lib/toolbox.cu:22-608, declared
 *     in device_pcg.h:1-9, device_amg.h:1-10, device_generic_operator.h:7-10,
 *     device_binary_operator.h:7-9, device_communicator.h:5-8), the fifteen
 *     _device_* entry points with their signatures, so toolbox host code that
 *     drives device_vector / device_amg_solver / device_conjugate_gradient
 *     links unchanged.  They run synchronously on the legacy default stream,
 *     as the reference's do.
 *
 *  3. hmfem_* : the status-returning API (no counterpart in the reference,
 *     which prints CUDA errors and continues, toolbox.h:21-26): assembly from
 *     permeabilities on the device, AMG setup on the device, PCG / flexible
 *     CG, flux reconstruction, hierarchy inspection.
 *
 * Memory kinds: functions taking `int mem` accept host pointers (mem = 0;
 * the library copies in and out) or device pointers (mem = 1; the caller's
 * CUDA allocations on the current device).
 */
#ifndef HMFEM_GPU_H
#define HMFEM_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------- */
#define HMFEM_OK 0
#define HMFEM_E_NOTCONV 1   /* iteration cap reached before the tolerance */
#define HMFEM_E_BREAKDOWN 2 /* non-finite or zero curvature in CG */
#define HMFEM_E_CUDA 3      /* a CUDA runtime call failed */
#define HMFEM_E_ARG 4       /* invalid argument / state */
#define HMFEM_E_TIMEOUT 5   /* a bounded device wait gave up */
#define HMFEM_E_CAPACITY 6  /* a sparse row exceeded the setup kernels' limit */

/* ---- reference data layouts (structs.h) ------------------------------ */
/* ELE, structs.h:7-17: per-cell face coefficients u,d,l,r, centre c, t,b */
typedef struct { double u, d, l, r, c, t, b; } hmfem_ele;
/* IND, structs.h:38-48: matrix column per face, -1 = boundary (RHS) */
typedef struct { int c, u, d, l, r, t, b; } hmfem_ind;
/* Dim, structs.h:84-95 */
typedef struct { int x, y, z, xy, t, px, pz, py; } hmfem_dim;

/* ---- layer 1: the reference bridge ------------------------------------ */
/* compute.cpp:7-51.  hdr[0] = rows, hdr[1] = nnz; cnt/col/ele row-by-count;
 * b read-only; x = initial guess in, solution out.  AMG (16 levels, min 1
 * node, epsilon 0) + PCG with the reference's stopping rule at 1e-8 unless
 * HMFEM_TOL / HMFEM_STOP override it.  Returns 0 like the reference; the
 * iteration count goes to iter_amg.  Errors: see hmfem_last_error(). */
int compute(int *hdr, int *cnt, int *col, double *ele, double *b, double *x);
/* solve_linearsystem_AMG.c:37-157: packs the AoS stencil on the device in
 * the reference's row order (d,l,c,r,u,t,b) and solves as compute() does. */
void solve_linsys(hmfem_ele *perm, hmfem_ind *indcol, double *b, double *x,
                  hmfem_dim N);
/* variables.h:63 -- defined weakly here; the application's definition wins */
extern int iter_amg;

/* ---- layer 2: the reference device layer (toolbox.cu) --------------- */
void _device_add_scale(double *x, double *y, double s, unsigned int m);   /* toolbox.cu:22-33  x += s y */
void _device_sub_scale(double *x, double *y, double s, unsigned int m);   /* toolbox.cu:52-63  x -= s y */
void _device_scale_add(double *x, double *y, double s, unsigned int m);   /* toolbox.cu:82-93  x = s x + y */
void _device_vector_product(double *x, double *y, double *z, unsigned int n,
                            unsigned int m);                              /* toolbox.cu:102-143 z[0..m) partials */
void _device_linear_operator(int *cnt, int *dsp, int *col, double *ele, int l,
                             int m, int n, double *u, double *v);         /* toolbox.cu:150-240 SELL-32 v = A u */
void _device_jacobi(int *cnt, int *dsp, int *col, double *ele, int l, int n,
                    double *f, double *u, double *v);                     /* toolbox.cu:249-347 v = f - A u */
void _device_set_mul(double *x, double *y, double *z, double omega,
                     unsigned int m);                                     /* toolbox.cu:356-377 x = w y z */
void _device_add_mul(double *x, double *y, double *z, double omega,
                     unsigned int m);                                     /* toolbox.cu:386-407 x += w y z */
void _device_diagonal_solver(double *x, double *y, double *z,
                             unsigned int m);                             /* toolbox.cu:415-435 x = y z */
void _device_com_snd(double *x, double *svec, int *rcom, unsigned int n);  /* toolbox.cu:443-464 svec = x[rcom] */
void _device_com_rcv(double *x, double *rvec, int *rcom, unsigned int n);  /* toolbox.cu:472-506 x[rcom] += rvec */
void _device_sub(double *x, double *y, unsigned int m);                   /* toolbox.cu:513-532 y -= x */
void _device_add(double *x, double *y, unsigned int m);                   /* toolbox.cu:539-558 y += x */
void _device_rsb(double *x, double *y, unsigned int m);                   /* toolbox.cu:565-584 y = x - y */
void _device_matrix_conversion(int *acnt, int *adsp, int *acol, double *aele,
                               int *tdsp, int *tcol, double *tele, int n); /* toolbox.cu:586-608 CSR -> SELL-32 */

/* ---- layer 3: status-returning API ------------------------------------ */
typedef struct hmfem_solver hmfem_solver;

typedef struct {
    int precision;     /* 0: FP64 V-cycle inside PCG (the plain drop-in);
                          1: FP32 V-cycle (coarse values BF16 from level
                          `bf16_from`) inside FP64 flexible CG */
    int bf16_from;     /* first level stored in BF16 (precision 1); <0 = none */
    int smoother;      /* 0: damped Jacobi with 1/a_ii (device_amg.h design);
                          1: l1-Jacobi, 1/(a_ii + sum_j!=i |a_ij|) (default:
                          SPD preconditioner for any SPD matrix) */
    int gs_from;       /* levels >= gs_from (below the coarse solve) use a
                          multicolour Gauss-Seidel smoother instead: forward
                          sweep over Jones-Plassmann colours before the
                          restriction, backward sweep after the
                          prolongation; < 0 disables (default 2) */
    double omega;      /* Jacobi weight (compute.cpp:35 passes 1.0) */
    double tol;        /* stopping tolerance */
    int stop_rule;     /* 0: true residual ||b-Ax||/||b|| <= tol;
                          1: reference rule (pcg.h:57) sigma/sigma0 <= tol^2 */
    int max_iter;      /* CG iteration cap (compute.cpp:42: 10000) */
    int max_levels;    /* compute.cpp:36: 16 */
    int min_coarse;    /* compute.cpp:37: 1 */
    int coarse_direct; /* solve the first level with <= this many rows
                          (at most 512) exactly (explicit FP64 inverse,
                          default 512); 0 =
                          the reference's diagonal solve on the coarsest
                          level (amg.h:1353-1364) */
    int check_every;   /* host polls convergence every k iterations */
    int generic_setup; /* 1: coarsen an assembled level 0 with the generic
                          kernels and solve every level on SELL-32 (default
                          0: level 0 from its 7-point structure, levels 0-1
                          solved in structured forms; identical results) */
    int gs_fused;      /* 1: one cooperative launch per Gauss-Seidel sweep
                          (grid barrier between colours); 0 (default): one
                          launch per colour (identical results) */
    int cheb_from;     /* levels >= cheb_from (below the coarse solve) are
                          smoothed by `cheb_degree` Chebyshev steps in
                          D_l1^-1 A over [1/30, 1] instead (takes precedence
                          over gs_from; default 2; < 1 disables) */
    int cheb_degree;   /* 2..9 (default 4) */
    int reuse_setup;   /* 1: hmfem_set_matrix / hmfem_set_stencil compare
                          the new level-0 matrix with the current one on
                          the device and, when it is bitwise identical,
                          keep the whole hierarchy (the next hmfem_setup is
                          a no-op) -- the reference's Picard loop re-runs
                          the AMG setup on an unchanged matrix (main.c:
                          457-514).  Default 0; compute / solve_linsys set
                          it. */
    int schur0;        /* 1 (with precision 1 on an assembled grid): level 1
                          is the Schur complement A_CC - A_CF A_FF^-1 A_FC
                          of level 0's red-black split instead of the
                          Galerkin product with the reference's averaging
                          interpolation (same rows and columns, so every
                          coarser level keeps the reference's structure),
                          and the V-cycle reduces level 0 exactly: no
                          level-0 smoothing, one restriction and one
                          prolongation pass.  Default 0. */
    int verbose;
} hmfem_options;

typedef struct {
    int iterations;
    int levels;
    int status;
    double relres;        /* final true ||b - A x|| / ||b|| (FP64) */
    double t_assemble_ms, t_setup_ms, t_solve_ms, t_flux_ms;
    double divmin, divmax; /* divvel_pontual min/max |div u| */
    int setup_reused;      /* 1: the last hmfem_setup kept the hierarchy */
} hmfem_stats;

void hmfem_default_options(hmfem_options *opt);
int hmfem_create(hmfem_solver **s, const hmfem_options *opt);
int hmfem_destroy(hmfem_solver *s);
/* Work on a caller stream (cudaStream_t passed as void*); NULL = the
 * solver's own non-blocking stream. */
int hmfem_set_stream(hmfem_solver *s, void *stream);
void *hmfem_get_stream(hmfem_solver *s);
const char *hmfem_last_error(void);

/* TPFA assembly from permeabilities (permeabilities.c:196-492 and
 * set_source_term.c:9-223 on the device).  K arrays are n = nx*ny*nz cells,
 * s = i + j nx + k nx ny.  Faces l,r,u,d,t,b; bc_type 0 Dirichlet, 1
 * Neumann; face_vals[f] (nullable) are per-face arrays in the Bound layout,
 * else bc_value[f] everywhere.  No well or conduit exchange terms: the
 * coupled reservoir / conduit run adds them (hmfem_picard, hmfem_karst.h). */
int hmfem_assemble(hmfem_solver *s, int nx, int ny, int nz, double hx,
                   double hy, double hz, double visc, const double *KX,
                   const double *KY, const double *KZ, const int bc_type[6],
                   const double bc_value[6], const double *const *face_vals,
                   int mem);
/* A general symmetric matrix in the reference's row-by-count form. */
int hmfem_set_matrix(hmfem_solver *s, int n, long nnz, const int *cnt,
                     const int *col, const double *ele, const double *b,
                     int mem);
/* AoS stencil + index arrays as solve_linsys receives them. */
int hmfem_set_stencil(hmfem_solver *s, int nx, int ny, int nz,
                      const hmfem_ele *perm, const hmfem_ind *indcol,
                      const double *b, int mem);
/* AMG hierarchy on the device (structure bit-exact with amg.h). */
int hmfem_setup(hmfem_solver *s);
/* Solve A x = b; x = initial guess in, solution out.  A b passed here
 * replaces the solver's right-hand side; b NULL solves with the current one
 * (the assembled or set right-hand side, or the last b passed here). */
int hmfem_solve(hmfem_solver *s, const double *b, double *x, int mem,
                hmfem_stats *st);
/* Face fluxes (flux_reconstruction.c:9-279) into n ELE (c untouched) and the
 * divvel_pontual min/max.  Needs hmfem_assemble. */
int hmfem_fluxes(hmfem_solver *s, const double *p, hmfem_ele *v, int mem,
                 double *divmin, double *divmax);
/* Inspection for parity tests. */
int hmfem_num_levels(hmfem_solver *s);
int hmfem_level_info(hmfem_solver *s, int l, int *n, long *nnz, long *pnnz);
int hmfem_level_copy(hmfem_solver *s, int l, int *cnt, int *col, double *ele,
                     double *dinv, signed char *sel, int *pcnt, int *pcol);
int hmfem_vcycle(hmfem_solver *s, const double *f, double *u, int mem);
int hmfem_spmv(hmfem_solver *s, int level, const double *x, double *y,
               int mem);
int hmfem_rhs(hmfem_solver *s, double *b, int mem);
int hmfem_last_stats(hmfem_solver *s, hmfem_stats *st);
/* Measurement: mean duration of `reps` launches of one solve-phase kernel
 * on level l (0 SpMV FP64, 1/2 pre/post smoother FP64, 3/4 pre/post
 * smoother FP32) timed with CUDA events on the solver stream, and its
 * algorithmic bytes per launch. */
int hmfem_time_kernel(hmfem_solver *s, int which, int level, int reps,
                      float *ms, double *bytes);

/* Many set-up solvers solved together (batched uneven instances): one
 * CUDA graph holds one CG iteration of every solver, each on a branch of
 * its own, and is replayed until every solver has converged; a converged
 * solver's kernels return at once, so each stops at its own tolerance and
 * gives the result it gives solved alone.  x[i]: solver i's initial guess
 * in, solution out (NULL array or entry: zero guess, nothing copied back);
 * st[i] (nullable) its stats.  Returns the first failing status. */
int hmfem_batch_solve(hmfem_solver *const *solvers, int m, double *const *x,
                      int mem, hmfem_stats *st);

/* Measurement: `iters` CG iterations from x = 0 launched one kernel at a
 * time (no graph), each bracketed by CUDA events on the solver stream;
 * out[0..min(count, cap)) gets, per kernel and level (-1 = the CG's
 * level-0 vector work), the launches and their summed duration.  *count =
 * the number of (kernel, level) pairs.  Overwrites the solver's x. */
typedef struct {
    char name[96];
    int level;
    int launches;
    double ms;
} hmfem_kernel_time;
int hmfem_profile_iteration(hmfem_solver *s, int iters, hmfem_kernel_time *out,
                            int cap, int *count);

/* Number of this library's kernels launched so far in the process
 * (graph replays included): a measurement aid. */
unsigned long long hmfem_launch_count(void);

/* Flux reconstruction that allocates nothing.  No counterpart in the
 * reference.  For callers that cannot let a library allocate device memory
 * (their device memory is already reserved by their own or a framework's
 * caching allocator, or they run where allocation is not permitted): the
 * same fluxes and divvel_pontual bounds as hmfem_fluxes, with constant
 * boundary values per face, from device arrays K*, p and into device v
 * (c untouched); divmin/divmax are host doubles.  All scratch lives in one
 * fixed __device__ array inside the library, so every boundary face must
 * have at most HMFEM_NOALLOC_MAX_FACE cells (else HMFEM_E_CAPACITY).  The
 * array is shared by all calls on a device and keeps the last call's
 * contents: calls that overlap on the GPU race.  The first call on a device
 * looks the array's address up (once, also when several host threads call
 * at the same time); make it before any stream capture.  The call reads the
 * bounds back to the host, so it returns after its work on the stream is done.
 * stream: cudaStream_t as void*, NULL = the legacy default stream. */
#define HMFEM_NOALLOC_MAX_FACE 262144
int hmfem_fluxes_noalloc(int nx, int ny, int nz, double hx, double hy,
                         double hz, double visc, const double *KX,
                         const double *KY, const double *KZ,
                         const int bc_type[6], const double bc_value[6],
                         const double *p, hmfem_ele *v, double *divmin,
                         double *divmax, void *stream);

#ifdef __cplusplus
}
#endif
#endif
