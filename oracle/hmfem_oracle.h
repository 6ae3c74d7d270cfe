/*
 * hmfem_oracle.h -- CPU restatement of hmfem's pressure-solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the correctness oracle: plain C, single
 * threaded, following the reference algorithm step by step (each function
 * cites the reference file:line it restates).  Only tests/, the smoke check
 * and the bench's cpu_baseline leg may load it, and only as the checker or
 * the timed CPU baseline.  The GPU product path never calls into it.
 *
 * Parity pinning: this restatement is checked against fixtures produced by
 * the reference's own sources (compiled by oracle/Makefile into oracle/_ref/
 * from the reference tree) -- see tests/golden/make_golden.py.
 */
#ifndef HMFEM_ORACLE_H
#define HMFEM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Layout-identical to the reference's ELE (structs.h:7-17) and IND
 * (structs.h:38-48). */
typedef struct { double u, d, l, r, c, t, b; } or_ele;
typedef struct { int c, u, d, l, r, t, b; } or_ind;

/* Face order used for boundary descriptions everywhere in this project:
 * 0=l (x-), 1=r (x+), 2=u (y+), 3=d (y-), 4=t (z+), 5=b (z-) -- the order of
 * val_bound[1..6] in main.c:140-145 / set_boundaries.c:8-40.
 * bc_type: 0 = Dirichlet, 1 = Neumann (main.c:347-350). */

/* Face-value arrays, one per face, indexed like the reference's Bound
 * (pyzindex for l/r, pxzindex for u/d, pxyindex for t/b;
 * solve_linearsystem_AMG.c:22-35). */
typedef struct { const double *l, *r, *u, *d, *t, *b; } or_bound;

/* permeabilities.c:188-193 */
double or_hm(double a, double b);

/* permeabilities.c:196-492 (permeabilidade_arestas). KI/WI may be NULL (0). */
void or_assemble(int nx, int ny, int nz, double hx, double hy, double hz,
                 double visc, const double *KX, const double *KY,
                 const double *KZ, const int bc_type[6], const double *KI,
                 const double *WI, or_ele *perm, or_ind *indcol);

/* set_source_term.c:9-223 (source_term). b must be zero-initialised by the
 * caller (reservoir.c:15).  KI/WI/pc/pw may be NULL (0). */
void or_source_term(int nx, int ny, int nz, double hx, double hy, double hz,
                    double visc, const or_bound *B, const int bc_type[6],
                    const or_ele *perm, const double *KI, const double *WI,
                    const double *pc, const double *pw, double *b);

/* solve_linearsystem_AMG.c:37-157: AoS stencil -> count/col/ele (row order
 * d,l,c,r,u,t,b).  Returns nnz; cnt/col/ele may be NULL for a count pass. */
long or_pack_csr(int n, const or_ele *perm, const or_ind *indcol, int *cnt,
                 int *col, double *ele);

/* One AMG level (toolbox/inverse_operator/amg.h:1099-1239). */
typedef struct {
    int n;
    long nnz;
    int *cnt, *col;       /* row counts, row-concatenated columns */
    double *ele;          /* values */
    double *dinv;         /* 1 / (last stored diagonal entry) */
    double *dl1inv;       /* 1 / (a_ii + sum_{j!=i} |a_ij|), row order: the
                             l1-Jacobi diagonal (not in the reference) */
    signed char *color;   /* greedy natural-order colouring (not in the
                             reference) and its number of colours */
    int ncolors;
    /* transfer to the next level (absent on the coarsest level) */
    char *sel;            /* 1 = C, 2 = F (amg.h:1-32) */
    long pnnz;
    int *pcnt, *pcol;     /* P rows: coarse ids */
    double *pele;         /* 1 / pcnt (amg.h:326-387) */
} or_level;

#define OR_MAX_LEVELS 32
typedef struct {
    int nlevels;          /* levels 0..nlevels-1; coarsest = nlevels-1 */
    or_level lv[OR_MAX_LEVELS];
} or_hierarchy;

/* amg_solver ctor, amg.h:1135-1239 with parallel_coarsening (amg.h:37-223),
 * parallel_interpolation (amg.h:228-406) and new_triple_product
 * (amg.h:408-582), single rank.  The fine matrix is copied. */
int or_amg_setup(int n, const int *cnt, const int *col, const double *ele,
                 int max_level, int max_size, double eps, or_hierarchy *H);
void or_amg_free(or_hierarchy *H);

/* One V-cycle u = C f.
 * smoother 0: the NOMPI Gauss-Seidel branch (amg.h:1315-1322, 759-784,
 *             930-961), the path compute.cpp runs.
 * smoother 1: the device design's damped Jacobi (device_amg.h:11-43,
 *             396-411), with omega.
 * smoother 2: the same cycle with the l1-Jacobi diagonal (dl1inv): an SPD
 *             preconditioner for any SPD matrix.
 * smoother 10+g: l1-Jacobi on levels < g, multicolour Gauss-Seidel (forward
 *             pre-sweep over colours 0..C-1 from zero, backward post-sweep)
 *             on levels >= g;
 * smoother 100+10g+t: as 10+g on levels [g, t) only;
 * smoother 200+10c+K: l1-Jacobi on levels < c, Chebyshev of degree K
 *             (2..9) in D_l1^-1 A over [1/30, 1] on levels >= c -- the GPU
 *             solver's default with c = 2, K = 3. */
void or_vcycle(const or_hierarchy *H, int smoother, double omega,
               const double *f, double *u);

/* y = A x on level 0 layout (generic_operator.h:212-247). */
void or_spmv(int n, const int *cnt, const int *col, const double *ele,
             const double *x, double *y);

/* PCG (pcg.h:13-76).  stop 0: the reference's test on the preconditioned
 * residual, sigma/sigma0 <= eps^2.  stop 1: true residual
 * ||b - A x|| / ||b|| <= eps, recomputed from x every iteration (used for
 * parity runs).  x is the initial guess in, the solution out.  Returns the
 * iteration count as pcg.h's iterations(); *relres receives the final true
 * relative residual. */
int or_pcg(const or_hierarchy *H, int smoother, double omega, const double *b,
           double *x, double eps, int max_it, int stop, double *relres);

/* compute.cpp:7-51 with a configurable tolerance/stop rule. */
int or_compute(const int *hdr, const int *cnt, const int *col,
               const double *ele, const double *b, double *x, double eps,
               int stop, int *iters, double *relres);

/* flux_reconstruction.c:9-279 (fluxos) and :281-319 (divvel_pontual).
 * v[s].c is left untouched.  divmin/divmax may be NULL. */
void or_fluxes(int nx, int ny, int nz, double hx, double hy, double hz,
               const double *p, const or_ele *perm, const or_bound *B,
               const int bc_type[6], or_ele *v, double *divmin,
               double *divmax);

/* Accessors for ctypes users: heap-allocated hierarchy, level sizes, and a
 * copy-out of one level (sel/pcnt/pcol/pele untouched on the coarsest). */
or_hierarchy *or_amg_create(int n, const int *cnt, const int *col,
                            const double *ele, int max_level, int max_size,
                            double eps);
void or_amg_destroy(or_hierarchy *H);
int or_amg_nlevels(const or_hierarchy *H);
int or_level_info(const or_hierarchy *H, int l, int *n, long *nnz,
                  long *pnnz);
int or_level_copy(const or_hierarchy *H, int l, int *cnt, int *col,
                  double *ele, double *dinv, char *sel, int *pcnt, int *pcol,
                  double *pele);

/* ---- the coupled conduit model (karst.c, main.c:383-557) --------------- */

/* A conduit set as main.c:197-280 reads it from data_<nk>_<type>.dat.
 * Per-conduit arrays have nk entries; the per-end tables cont/ccont are
 * [f*nk + j] (f = 0 left end, 1 right end); the per-fracture tables are
 * [b*nk + j] for b < max_brechas, beta already R^4 - 1 (main.c:256).
 * pos: 1 = conduit along x, 2 = along y, 3 = along z.  bound: 0 Dirichlet,
 * 1 Neumann, 3 nonlinear Robin (permeabilities.c:826-858).  Same layout as
 * hmfem_karst in include/hmfem_karst.h. */
typedef struct {
    int nk, max_brechas;
    const int *len, *sxi, *syi, *szi, *pos;
    const double *Kc;
    const int *bound_l, *bound_r;
    const double *cont, *ccont;
    const double *kindex, *area;
    const int *n_brechas;
    const double *beta, *cb;
    const int *brechas;
} or_karst;

/* The 3-D side the conduit terms read (the matrix faces of the coupled
 * system, K and the last reservoir pressure). */
typedef struct {
    int nx, ny, nz;
    double hx, hy, hz, visc, rho;
    const double *KX, *KY, *KZ;
    const or_ele *perm;
    const double *p_old;
} or_kgrid;

/* Conduit state; matrices are [i*nk + j] with mmax rows (pc[i][j] of
 * main.c), ucR/ucL are [b*nk + j]. */
typedef struct {
    int mmax;
    double *kl, *kr, *kc, *kic, *paux, *pc, *pc_old, *ucR, *ucL;
} or_kstate;

/* 0 when the set is usable on an nx x ny x nz grid, else -1: a conduit
 * leaves the grid, a fracture sits on the last element, a Robin end has no
 * reservoir cell beyond it, or a Robin right end of a z conduit (the
 * reference leaves its source term undefined, set_source_term.c:368-404). */
int or_karst_check(const or_karst *K, int nx, int ny, int nz);
/* 3-D cell of conduit j, element i (main.c:416-448). */
int or_karst_cell(const or_karst *K, int j, int i, int nx, int ny);
/* permeabilities.c:795-867 (permeabilidade_karst) for conduit j. */
void or_karst_keff(const or_karst *K, const or_kgrid *G, or_kstate *S, int j);
/* set_source_term.c:256-414 (source_term1d) for conduit j into f (len). */
void or_source_term1d(const or_karst *K, const or_kgrid *G, or_kstate *S,
                      int j, double *f);
/* The tridiagonal conduit system solve_linearsystem_AMG.c:200-294 builds
 * (row i: -kl[i] x[i-1] + kc[i] x[i] - kr[i] x[i+1] = f[i]) solved by the
 * Thomas algorithm; kl/kc/kr are read with stride `stride`. */
void or_thomas(int m, const double *kl, const double *kc, const double *kr,
               int stride, const double *f, double *x);
/* karst.c:8-40 (conduit): keff, source term and solve of every conduit.
 * solver 0: Thomas; 1: compute() (AMG-PCG, 1e-8, pcg.h rule) as the
 * reference does (compute.cpp:40-45). */
void or_conduit(const or_karst *K, const or_kgrid *G, or_kstate *S,
                int solver);
/* flux_reconstruction.c:322-496 (fluxo1d) into ucl/ucr ([i*nk + j]). */
void or_fluxo1d(const or_karst *K, const or_kgrid *G, const or_kstate *S,
                double *ucl, double *ucr);

/* The coupled Picard loop of main.c:383-489 and the conduit/well balances
 * of main.c:523-593.  The 3-D solves run this oracle's AMG-PCG (compute.cpp
 * settings) to solve_eps with stop rule solve_stop (or_pcg); conduit_solver
 * as or_conduit.  WI/pw (nullable) are the well index and well pressure.
 * Outputs: p (n), pc (mmax*nk), and when non-NULL ucl/ucr (mmax*nk), v (n
 * 3-D face fluxes), out[0..2] = {error, Q well, mean p} and
 * qk[3*nk] = {Qc1d, Qc3d, Qcb} per conduit.  Returns the Picard iteration
 * count, or -1 when or_karst_check fails. */
int or_picard(const or_karst *K, int nx, int ny, int nz, double hx, double hy,
              double hz, double visc, double rho, const double *KX,
              const double *KY, const double *KZ, const int bc_type[6],
              const double val6[6], const double *WI, const double *pw,
              double tol, int iter_max, double solve_eps, int solve_stop,
              int conduit_solver, double *p, double *pc, double *ucl,
              double *ucr, or_ele *v, double *out, double *qk);

#ifdef __cplusplus
}
#endif
#endif
