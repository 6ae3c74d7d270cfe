/*
 * hmfem_karst.h -- the coupled reservoir / karst-conduit model on the device.
 *
 * The reference couples the 3-D Darcy reservoir with 1-D conduits (karst
 * channels) by a Picard loop in its application (main.c:383-489): every
 * iteration solves the reservoir with the conduit pressures in the exchange
 * term (reservoir.c:8-57), then every conduit's tridiagonal system with the
 * new reservoir pressure (karst.c:8-40), until the reservoir pressure stops
 * changing.  hmfem_picard runs that whole loop on the GPU: the coupled 3-D
 * matrix is set up once (its values do not change between iterations; the
 * reference re-runs the AMG setup each time), the exchange right-hand side
 * is patched in place, the 3-D solve warm-starts from the previous
 * pressure, and all conduits are solved in one batched Thomas launch.
 *
 * Conduit layout mirrors the reference's data file data_<nk>_<type>.dat as
 * main.c:197-280 reads it.  Matrices of per-conduit-element values use the
 * reference's pc[i][j] layout flattened row-major: [i * number_karst + j],
 * i < max(len) (entries past a conduit's length are zero).  All pointers in
 * hmfem_karst are host pointers.
 */
#ifndef HMFEM_KARST_H
#define HMFEM_KARST_H

#include "hmfem_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int number_karst;          /* conduits (main.c:164) */
    int max_brechas;           /* rows of the fracture tables (main.c:245-250) */
    const int *len;            /* M[j].s: elements of conduit j */
    const int *sxi, *syi, *szi;/* M[j].sxi/syi/szi: reservoir cell of element 0 */
    const int *pos;            /* M[j].pos: 1 along x, 2 along y, 3 along z */
    const double *Kc;          /* conduit permeability (main.c:225-227) */
    const int *bound_l;        /* BoundKarst->l: 0 Dirichlet, 1 Neumann, */
    const int *bound_r;        /*   3 nonlinear Robin (permeabilities.c:826) */
    const double *cont;        /* cont_karst[f][j] at [f*nk + j]; f 0 left, 1 right */
    const double *ccont;       /* C_contorno[f][j] at [f*nk + j] */
    const double *karst_index; /* karst_index[j] (exchange coefficient) */
    const double *area;        /* Ac[j]: conduit cross-section */
    const int *n_brechas;      /* fractures per conduit */
    const double *beta;        /* [b*nk + j], already R^4 - 1 (main.c:256) */
    const double *cbrecha;     /* C[b][j] at [b*nk + j] */
    const int *brechas;        /* element index of fracture b of conduit j */
} hmfem_karst;

/* main.c:197-280: reads data_<nk>_<type>.dat (whitespace-separated; ints
 * as fscanf %i reads them).  Arrays are allocated by the library; release
 * them with hmfem_karst_release.  Returns HMFEM_E_ARG on a missing file or a
 * short read. */
int hmfem_karst_read(const char *path, int number_karst, hmfem_karst *out);
void hmfem_karst_release(hmfem_karst *k);

/* HMFEM_OK when the set can run on an nx*ny*nz grid, else HMFEM_E_ARG with
 * the reason in hmfem_last_error(): a conduit leaving the grid, a position
 * code outside 1..3, an end code outside {0, 1, 3}, a fracture on the last
 * element, a nonlinear Robin end with no reservoir cell beyond it, or a
 * Robin right end of a z conduit (the reference leaves that source term
 * undefined, set_source_term.c:368-404). */
int hmfem_karst_check(const hmfem_karst *k, int nx, int ny, int nz);

typedef struct {
    double rho;     /* fluid density in the fracture and Robin terms (main.c:127: 1000) */
    double tol;     /* Picard tolerance on ||p - p_old|| / ||p|| (main.c:118: 1e-8) */
    int iter_max;   /* Picard iteration cap (main.c:119: 1000) */
} hmfem_picard_options;

void hmfem_picard_default_options(hmfem_picard_options *o);

typedef struct {
    int iterations;        /* Picard iterations (main.c's iter) */
    int status;            /* HMFEM_OK, or HMFEM_E_NOTCONV at iter_max */
    double error;          /* the last relative reservoir change; the
                              reference's loop test keeps only this entry
                              of error1[] (main.c:480-486) */
    int cg_iterations;     /* summed over every 3-D solve */
    int setups;            /* AMG setups run (uncoupled + coupled matrix) */
    double q_well;         /* sum (WI/mu)(pw - p) (main.c:523-526) */
    double p_mean;         /* mean reservoir pressure (main.c:529) */
    double t_setup_ms;     /* both assemblies + both AMG setups + the first
                              solve + conduit setup */
    double t_loop_ms;      /* first conduit solve + the Picard loop */
    double t_total_ms;
} hmfem_picard_stats;

/* The coupled run of main.c:383-489 on solver s (its options choose the 3-D
 * solve: precision, tolerance, stop rule).  Grid, K, boundary arguments as
 * hmfem_assemble (bc types 0/1, constant face values bc_value).  WI / pw
 * (nullable, n cells each) are the well index and well pressure; the first
 * reservoir solve runs without them and without conduit exchange, as the
 * reference's does (main.c:393).  p (n) receives the reservoir pressure,
 * pc (max(len) * number_karst, nullable) the conduit pressures.  mem as in
 * hmfem_gpu.h for K, WI, pw, p and pc.  Returns HMFEM_OK, HMFEM_E_NOTCONV
 * when iter_max was reached, or an error. */
int hmfem_picard(hmfem_solver *s, const hmfem_karst *k, int nx, int ny,
                 int nz, double hx, double hy, double hz, double visc,
                 const double *KX, const double *KY, const double *KZ,
                 const int bc_type[6], const double bc_value[6],
                 const double *WI, const double *pw,
                 const hmfem_picard_options *opt, double *p, double *pc,
                 int mem, hmfem_picard_stats *st);

/* After hmfem_picard: the conduit fluxes of flux_reconstruction.c:322-496
 * (fluxo1d) into ucl / ucr (max(len) * number_karst each, nullable) and the
 * per-conduit balances of main.c:566-593 into qk (3 * number_karst,
 * nullable): Qc1d[j], Qc3d[j], Qcb[j].  mem for ucl, ucr, qk.  The
 * reservoir face fluxes come from hmfem_fluxes on the same solver. */
int hmfem_picard_fluxes(hmfem_solver *s, double *ucl, double *ucr,
                        double *qk, int mem);

/* One conduit() call (karst.c:8-40) on given state, for parity tests:
 * reservoir pressure p_old (n), conduit pressures of the previous
 * iteration pc_old ([i*nk + j]) and fracture velocities ucR / ucL
 * ([b*nk + j]; in: the previous values, out: updated) -> pc, and the
 * conduit matrix keff l/r/c.  All arrays host (mem 0) or device (mem 1);
 * kl/kr/kc nullable. */
int hmfem_conduit_step(const hmfem_karst *k, int nx, int ny, int nz,
                       double hx, double hy, double hz, double visc,
                       double rho, const double *KX, const double *KY,
                       const double *KZ, const double *p_old,
                       const double *pc_old, double *ucR, double *ucL,
                       double *pc, double *kl, double *kr, double *kc,
                       int mem);

#ifdef __cplusplus
}
#endif
#endif
