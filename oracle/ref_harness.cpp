/*
 * ref_harness.cpp -- drives the reference's OWN sources (compiled from the
 * hmfem tree by oracle/Makefile, never copied) so that the C restatement in
 * hmfem_oracle.c can be pinned against them and so that the reference CPU
 * path can be timed as a baseline.
 *
 * TEST INFRASTRUCTURE ONLY.  Output goes to oracle/_ref/ (git-ignored).
 *
 * What is the reference's code here: permeabilidade_arestas, create_boundary,
 * source_term, solve_linsys (AoS -> CSR packing), fluxos, and the toolbox's
 * amg_solver / conjugate_gradient / linear_operator / vector_product
 * templates.  What is this harness's: the globals the application's main.c
 * would define, a compute() that replaces compute.cpp so the tolerance and
 * stopping rule can be chosen, and extern "C" wrappers for ctypes.
 */
#define NOMPI
#include <sys/time.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <sstream>
#include <fstream>
#include <string>
#include <iostream>
#include <algorithm>
/* amg_solver keeps its hierarchy private; the harness reads it for the
 * structure dumps. */
#define private public
#include "toolbox/toolbox.h"
#undef private
#include "structs.h"
#include "functions.h"
#include "hmfem_oracle.h"

#include "app_globals.h"

static double now()
{
    timeval t;
    gettimeofday(&t, 0);
    return t.tv_sec + 1e-6 * t.tv_usec;
}

/* ---- compute() replacement ------------------------------------------- */
/* mode 0: capture the CSR that solve_linsys hands over;
 * mode 1: the reference conjugate_gradient (pcg.h stop rule);
 * mode 2: same operators, loop stopped on the true residual. */
static int g_mode = 1;
static double g_eps = 1e-8;
static std::vector<int> g_cnt, g_col;
static std::vector<double> g_ele;
static double g_setup_s, g_solve_s, g_relres;

static double true_relres(linear_operator<int, double> &lin,
                          const vector<double> &b, const vector<double> &x)
{
    vector<double> r(b.size());
    lin(x, r);
    double rr = 0, bb = 0;
    for (size_t i = 0; i < b.size(); i++) {
        double d = b[i] - r[i];
        rr += d * d;
        bb += b[i] * b[i];
    }
    return bb > 0 ? sqrt(rr / bb) : sqrt(rr);
}

int compute(int *_hdr, int *_cnt, int *_col, double *_ele, double *_b, double *_x)
{
    int n = _hdr[0], nnz = _hdr[1];
    if (g_mode == 0) {
        g_cnt.assign(_cnt, _cnt + n);
        g_col.assign(_col, _col + nnz);
        g_ele.assign(_ele, _ele + nnz);
        return 0;
    }
    vector<int> col(_col, _col + nnz), cnt(_cnt, _cnt + n), nod(n);
    vector<double> ele(_ele, _ele + nnz), b(_b, _b + n), x(_x, _x + n);
    for (int i = 0; i < n; i++) nod[i] = i;
    communicator<int, double> com(nod);
    linear_operator<int, double> lin(cnt, col, ele);
    vector_product<int, double> sca(com);
    double t0 = now();
    /* compute.cpp:35-38 */
    amg_solver<int, double> amg(nod, cnt, col, ele, 16, 1, 0.0, 1.0, true);
    double t1 = now();
    if (g_mode == 1) {
        conjugate_gradient<int, double> cg(lin, amg, sca, g_eps, 10000, false);
        cg(b, x);
        iter_amg = cg.iterations();
    } else {
        /* pcg.h:33-76 with the test replaced by ||b-Ax||/||b|| <= eps */
        vector<double> alpha(1, 1.0), beta(1, 0.0), sigma(1, 0.0),
            sigma_last(1, 0.0), tau(1, 0.0);
        vector<double> r(b), s(x), w(n);
        lin(s, w);
        sub_scale(r, w, alpha);
        amg(r, w);
        sca(w, r, sigma);
        if (sigma[0] < 0.0) sigma[0] = fabs(sigma[0]);
        scale_add(s, w, beta);
        sigma_last[0] = sigma[0];
        int loop = 0;
        double rel = true_relres(lin, b, x);
        while (++loop < 10000 && rel > g_eps) {
            lin(s, w);
            sca(s, w, tau);
            if (tau[0] < 0.0) tau[0] = fabs(tau[0]);
            alpha[0] = sigma[0] / tau[0];
            add_scale(x, s, alpha);
            sub_scale(r, w, alpha);
            amg(r, w);
            sca(w, r, sigma);
            if (sigma[0] < 0.0) sigma[0] = fabs(sigma[0]);
            beta[0] = sigma[0] / sigma_last[0];
            scale_add(s, w, beta);
            sigma_last[0] = sigma[0];
            rel = true_relres(lin, b, x);
        }
        iter_amg = loop;
    }
    double t2 = now();
    g_setup_s = t1 - t0;
    g_solve_s = t2 - t1;
    g_relres = true_relres(lin, b, x);
    for (int i = 0; i < n; i++) _x[i] = x[i];
    return 0;
}

/* ---- extern "C" wrappers ------------------------------------------------ */
static void set_grid(int nx, int ny, int nz, double hx, double hy, double hz,
                     const int bc[6], double visc)
{
    N.x = nx; N.y = ny; N.z = nz; N.xy = nx * ny; N.t = nx * ny * nz;
    h.x = hx; h.y = hy; h.z = hz;
    I.x = hx * nx; I.y = hy * ny; I.z = hz * nz;
    boundary.l = bc[0]; boundary.r = bc[1]; boundary.u = bc[2];
    boundary.d = bc[3]; boundary.t = bc[4]; boundary.b = bc[5];
    viscosidade = visc;
}

static Bound *make_bound(const double val6[6])
{
    Bound *Bd = (Bound *)malloc(sizeof(Bound));
    Bd->l = create_vector(N.t); Bd->r = create_vector(N.t);
    Bd->u = create_vector(N.t); Bd->d = create_vector(N.t);
    Bd->t = create_vector(N.t); Bd->b = create_vector(N.t);
    /* val_bound[1..6] = L, R, U, D, T, B (main.c:140-152) */
    double vb[7] = {0, val6[0], val6[1], val6[2], val6[3], val6[4], val6[5]};
    create_boundary(vb, Bd, N, boundary);
    return Bd;
}

static void free_bound(Bound *Bd)
{
    free(Bd->l); free(Bd->r); free(Bd->u); free(Bd->d); free(Bd->t); free(Bd->b);
    free(Bd);
}

extern "C" {

/* Assembly + RHS through permeabilidade_arestas and source_term.
 * bc: l,r,u,d,t,b types; val6: l,r,u,d,t,b constant face values. */
int ref_assemble(int nx, int ny, int nz, double hx, double hy, double hz,
                 double visc, const double *KX, const double *KY,
                 const double *KZ, const int *bc, const double *val6,
                 ELE *perm_out, IND *ind_out, double *b_out)
{
    set_grid(nx, ny, nz, hx, hy, hz, bc, visc);
    Perm K;
    K.X = (double *)KX; K.Y = (double *)KY; K.Z = (double *)KZ;
    Bound *Bd = make_bound(val6);
    double *zero = create_vector(N.t);
    for (int s = 0; s < N.t; s++) {
        ind_out[s].c = ind_out[s].u = ind_out[s].d = ind_out[s].l = -1;
        ind_out[s].r = ind_out[s].t = ind_out[s].b = -1;
        b_out[s] = 0.0;
    }
    permeabilidade_arestas(&K, perm_out, ind_out, h, N, boundary, zero, zero,
                           viscosidade);
    source_term(Bd, perm_out, h, N, boundary, zero, zero, zero, zero,
                viscosidade, b_out);
    free(zero);
    free_bound(Bd);
    return 0;
}

/* solve_linsys packing; returns nnz, then ref_packed copies it out. */
long ref_pack(int nx, int ny, int nz, ELE *perm_in, IND *ind_in)
{
    N.x = nx; N.y = ny; N.z = nz; N.xy = nx * ny; N.t = nx * ny * nz;
    g_mode = 0;
    std::vector<double> b(N.t, 0.0), x(N.t, 0.0);
    solve_linsys(perm_in, ind_in, b.data(), x.data(), N);
    return (long)g_col.size();
}

void ref_packed(int *cnt, int *col, double *ele)
{
    for (size_t i = 0; i < g_cnt.size(); i++) cnt[i] = g_cnt[i];
    for (size_t i = 0; i < g_col.size(); i++) { col[i] = g_col[i]; ele[i] = g_ele[i]; }
}

/* AMG-PCG through compute(); stop 1 = pcg.h rule, 2 = true residual. */
int ref_compute(int n, long nnz, const int *cnt, const int *col,
                const double *ele, const double *b, double *x, double eps,
                int stop, double *setup_s, double *solve_s, double *relres)
{
    int hdr[2] = {n, (int)nnz};
    g_mode = stop;
    g_eps = eps;
    compute(hdr, (int *)cnt, (int *)col, (double *)ele, (double *)b, x);
    if (setup_s) *setup_s = g_setup_s;
    if (solve_s) *solve_s = g_solve_s;
    if (relres) *relres = g_relres;
    return iter_amg;
}

/* Hierarchy dump: the reference amg_solver is kept between calls. */
static amg_solver<int, double> *g_amg;
static std::vector<int> g_nod, g_hcnt, g_hcol;
static std::vector<double> g_hele;
static std::vector<std::vector<char> > g_sel;

int ref_amg_build(int n, long nnz, const int *cnt, const int *col,
                  const double *ele)
{
    delete g_amg;
    g_nod.resize(n);
    for (int i = 0; i < n; i++) g_nod[i] = i;
    g_hcnt.assign(cnt, cnt + n);
    g_hcol.assign(col, col + nnz);
    g_hele.assign(ele, ele + nnz);
    g_amg = new amg_solver<int, double>(g_nod, g_hcnt, g_hcol, g_hele, 16, 1,
                                        0.0, 1.0, true);
    /* C/F split per level: re-run the reference coarsening on each level. */
    g_sel.assign(g_amg->_level, std::vector<char>());
    for (int l = 0; l < g_amg->_level; l++) {
        vector<double> adia;
        vector<char> abou, acox;
        communicator<int, double> com;
        com.assign(g_amg->_anod[l]);
        parallel_coarsening<int, double> coarsening;
        coarsening(g_amg->_anod[l], g_amg->_acnt[l], g_amg->_acol[l],
                   g_amg->_aele[l], adia, abou, g_sel[l], acox, com, 0.0);
    }
    return g_amg->_level + 1;
}

/* sizes of level l: rows, nnz, P nnz */
int ref_amg_level(int l, int *n, long *nnz, long *pnnz)
{
    if (!g_amg || l > g_amg->_level) return -1;
    *n = (int)g_amg->_acnt[l].size();
    *nnz = (long)g_amg->_acol[l].size();
    *pnnz = l < g_amg->_level ? (long)g_amg->_rcol[l].size() : 0;
    return 0;
}

int ref_amg_copy(int l, int *cnt, int *col, double *ele, double *dinv,
                 char *sel, int *pcnt, int *pcol, double *pele)
{
    if (!g_amg || l > g_amg->_level) return -1;
    auto &A = *g_amg;
    for (size_t i = 0; i < A._acnt[l].size(); i++) cnt[i] = A._acnt[l][i];
    for (size_t i = 0; i < A._acol[l].size(); i++) { col[i] = A._acol[l][i]; ele[i] = A._aele[l][i]; }
    for (size_t i = 0; i < A._adia[l].size(); i++) dinv[i] = A._adia[l][i];
    if (l < A._level) {
        for (size_t i = 0; i < g_sel[l].size(); i++) sel[i] = g_sel[l][i];
        for (size_t i = 0; i < A._rcnt[l].size(); i++) pcnt[i] = A._rcnt[l][i];
        for (size_t i = 0; i < A._rcol[l].size(); i++) { pcol[i] = A._rcol[l][i]; pele[i] = A._rele[l][i]; }
    }
    return 0;
}

/* one application of the reference V-cycle, u = C f */
int ref_amg_apply(const double *f, double *u)
{
    if (!g_amg) return -1;
    int n = (int)g_hcnt.size();
    vector<double> ff(f, f + n), uu(n, 0.0);
    (*g_amg)(ff, uu);
    for (int i = 0; i < n; i++) u[i] = uu[i];
    return 0;
}

void ref_amg_free()
{
    delete g_amg;
    g_amg = 0;
}

/* fluxos + divvel_pontual; v_out is n ELE. */
int ref_fluxes(int nx, int ny, int nz, double hx, double hy, double hz,
               const int *bc, const double *val6, const double *p,
               ELE *perm_in, ELE *v_out)
{
    set_grid(nx, ny, nz, hx, hy, hz, bc, viscosidade);
    Bound *Bd = make_bound(val6);
    fluxos((double *)p, perm_in, v_out, Bd, h, N);
    free_bound(Bd);
    return 0;
}

/* Whole reference CPU path for one problem, as reservoir() + fluxos run it:
 * assembly, RHS, CSR packing + AMG-PCG (true-residual stop), flux.  times:
 * [assemble, setup, solve, flux, total]. */
int ref_solve_all(int nx, int ny, int nz, double hx, double hy, double hz,
                  double visc, const double *KX, const double *KY,
                  const double *KZ, const int *bc, const double *val6,
                  double eps, double *p_out, ELE *v_out, double *times,
                  double *relres)
{
    double t0 = now();
    set_grid(nx, ny, nz, hx, hy, hz, bc, visc);
    ELE *pm = (ELE *)calloc(N.t + 1, sizeof(ELE));
    IND *ic = (IND *)malloc((N.t + 1) * sizeof(IND));
    double *b = create_vector(N.t);
    ref_assemble(nx, ny, nz, hx, hy, hz, visc, KX, KY, KZ, bc, val6, pm, ic, b);
    double t1 = now();
    for (int s = 0; s < N.t; s++) p_out[s] = 0.0;
    g_mode = 2;
    g_eps = eps;
    solve_linsys(pm, ic, b, p_out, N);
    double t2 = now();
    fluxos(p_out, pm, v_out, B = make_bound(val6), h, N);
    free_bound(B);
    B = 0;
    double t3 = now();
    if (times) {
        times[0] = t1 - t0;
        times[1] = g_setup_s;
        times[2] = g_solve_s;
        times[3] = t3 - t2;
        times[4] = t3 - t0;
    }
    if (relres) *relres = g_relres;
    free(pm); free(ic); free(b);
    return iter_amg;
}

/* ---- the same path in steps (the timed reference arm) -------------------
 * ref_solve_all's work split so that a caller can time it in parts: the
 * assembly with the CSR packing, the AMG setup with the CG start, CG
 * iterations in chunks, the fluxes.  The CG is the loop of compute() mode
 * 2 above (pcg.h:33-76 with the true-residual test), so a job's result is
 * ref_solve_all's.  One job per process (the reference's globals). */
struct RefJob {
    int nx, ny, nz, bc[6];
    double hx, hy, hz, visc, eps, val6[6];
    const double *KX, *KY, *KZ;
    ELE *pm;
    IND *ic;
    double *b, *p;
    vector<int> cnt, col, nod;
    vector<double> ele, bv, x, r, s, w;
    amg_solver<int, double> *amg;
    linear_operator<int, double> *lin;
    communicator<int, double> *com;
    vector_product<int, double> *sca;
    vector<double> alpha, beta, sigma, sigma_last, tau;
    int loop, done;
    double rel, t_asm, t_setup, t_solve, t_flux;
};

void *ref_job_new(int nx, int ny, int nz, double hx, double hy, double hz, double visc,
                  const double *KX, const double *KY, const double *KZ, const int *bc,
                  const double *val6, double eps)
{
    RefJob *j = new RefJob();
    j->nx = nx; j->ny = ny; j->nz = nz; j->hx = hx; j->hy = hy; j->hz = hz;
    j->visc = visc; j->eps = eps;
    for (int f = 0; f < 6; f++) { j->bc[f] = bc[f]; j->val6[f] = val6[f]; }
    j->KX = KX; j->KY = KY; j->KZ = KZ;
    return j;
}

/* assembly + RHS (permeabilidade_arestas, source_term) and solve_linsys's
 * CSR packing (captured by compute() mode 0) */
int ref_job_assemble(void *job)
{
    RefJob *j = (RefJob *)job;
    double t0 = now();
    const long n = (long)j->nx * j->ny * j->nz;
    j->pm = (ELE *)calloc(n + 1, sizeof(ELE));
    j->ic = (IND *)malloc((n + 1) * sizeof(IND));
    j->b = create_vector((int)n);
    j->p = create_vector((int)n);
    ref_assemble(j->nx, j->ny, j->nz, j->hx, j->hy, j->hz, j->visc, j->KX, j->KY, j->KZ,
                 j->bc, j->val6, j->pm, j->ic, j->b);
    g_mode = 0;
    solve_linsys(j->pm, j->ic, j->b, j->p, N);
    g_mode = 1;
    j->cnt.swap(g_cnt);
    j->col.swap(g_col);
    j->ele.swap(g_ele);
    j->t_asm = now() - t0;
    return 0;
}

/* amg_solver (compute.cpp:35-38) and the CG start (pcg.h:33-52) */
int ref_job_setup(void *job)
{
    RefJob *j = (RefJob *)job;
    double t0 = now();
    const int n = (int)j->cnt.size();
    j->nod.resize(n);
    for (int i = 0; i < n; i++) j->nod[i] = i;
    j->bv.assign(j->b, j->b + n);
    j->x.assign(n, 0.0);
    j->com = new communicator<int, double>(j->nod);
    j->lin = new linear_operator<int, double>(j->cnt, j->col, j->ele);
    j->sca = new vector_product<int, double>(*j->com);
    j->amg = new amg_solver<int, double>(j->nod, j->cnt, j->col, j->ele, 16, 1, 0.0, 1.0, true);
    double t1 = now();
    j->alpha.assign(1, 1.0); j->beta.assign(1, 0.0); j->sigma.assign(1, 0.0);
    j->sigma_last.assign(1, 0.0); j->tau.assign(1, 0.0);
    j->r = j->bv;
    j->s = j->x;
    j->w.assign(n, 0.0);
    (*j->lin)(j->s, j->w);
    sub_scale(j->r, j->w, j->alpha);
    (*j->amg)(j->r, j->w);
    (*j->sca)(j->w, j->r, j->sigma);
    if (j->sigma[0] < 0.0) j->sigma[0] = fabs(j->sigma[0]);
    scale_add(j->s, j->w, j->beta);
    j->sigma_last[0] = j->sigma[0];
    j->loop = 0;
    j->rel = true_relres(*j->lin, j->bv, j->x);
    j->done = !(j->rel > j->eps);
    j->t_setup = t1 - t0;
    j->t_solve = now() - t1;
    return 0;
}

/* up to k CG iterations (k < 0: to convergence); returns 1 once converged */
int ref_job_iterate(void *job, int k)
{
    RefJob *j = (RefJob *)job;
    double t0 = now();
    for (int it = 0; !j->done && (k < 0 || it < k); it++) {
        if (!(++j->loop < 10000)) { j->done = 1; break; }
        (*j->lin)(j->s, j->w);
        (*j->sca)(j->s, j->w, j->tau);
        if (j->tau[0] < 0.0) j->tau[0] = fabs(j->tau[0]);
        j->alpha[0] = j->sigma[0] / j->tau[0];
        add_scale(j->x, j->s, j->alpha);
        sub_scale(j->r, j->w, j->alpha);
        (*j->amg)(j->r, j->w);
        (*j->sca)(j->w, j->r, j->sigma);
        if (j->sigma[0] < 0.0) j->sigma[0] = fabs(j->sigma[0]);
        j->beta[0] = j->sigma[0] / j->sigma_last[0];
        scale_add(j->s, j->w, j->beta);
        j->sigma_last[0] = j->sigma[0];
        j->rel = true_relres(*j->lin, j->bv, j->x);
        if (!(j->rel > j->eps)) j->done = 1;
    }
    j->t_solve += now() - t0;
    return j->done;
}

/* a new stopping tolerance: iterate() then continues the same CG to it */
void ref_job_set_eps(void *job, double eps)
{
    RefJob *j = (RefJob *)job;
    j->eps = eps;
    j->done = !(j->rel > eps);
}

/* fluxos + divvel_pontual of the job's pressure into v (n ELE, may be NULL:
 * then the job keeps its own) */
int ref_job_flux(void *job, ELE *v_out)
{
    RefJob *j = (RefJob *)job;
    double t0 = now();
    const int n = (int)j->x.size();
    for (int i = 0; i < n; i++) j->p[i] = j->x[i];
    ELE *v = v_out ? v_out : (ELE *)calloc(n + 1, sizeof(ELE));
    set_grid(j->nx, j->ny, j->nz, j->hx, j->hy, j->hz, j->bc, j->visc);
    Bound *Bd = make_bound(j->val6);
    fluxos(j->p, j->pm, v, Bd, h, N);
    free_bound(Bd);
    if (!v_out) free(v);
    j->t_flux = now() - t0;
    return 0;
}

/* p_out (n), times [assemble, setup, solve, flux, total]; returns the
 * iteration count (compute() mode 2's) */
int ref_job_result(void *job, double *p_out, double *times, double *relres)
{
    RefJob *j = (RefJob *)job;
    if (p_out) for (size_t i = 0; i < j->x.size(); i++) p_out[i] = j->x[i];
    if (times) {
        times[0] = j->t_asm; times[1] = j->t_setup; times[2] = j->t_solve;
        times[3] = j->t_flux;
        times[4] = j->t_asm + j->t_setup + j->t_solve + j->t_flux;
    }
    if (relres) *relres = j->rel;
    return j->loop;
}

void ref_job_free(void *job)
{
    RefJob *j = (RefJob *)job;
    delete j->amg; delete j->lin; delete j->sca; delete j->com;
    free(j->pm); free(j->ic); free(j->b); free(j->p);
    delete j;
}

}  // extern "C"

/* ---- the coupled conduit model ------------------------------------------ */
/* Sets the conduit globals that main.c:197-307 would read from the data file
 * (an or_karst has the data file's layout, see hmfem_oracle.h). */
static void karst_globals(const or_karst *k)
{
    const int nk = k->nk;
    number_karst = nk;
    M = (DimK *)malloc((nk + 1) * sizeof(DimK));
    Mmax = 0;
    for (int j = 0; j < nk; j++) {
        M[j].s = k->len[j]; M[j].sxi = k->sxi[j]; M[j].syi = k->syi[j];
        M[j].szi = k->szi[j]; M[j].pos = k->pos[j];
        if (M[j].s > Mmax) Mmax = M[j].s;
    }
    Kc = create_vector(nk);
    BoundKarst = (FACEK *)malloc(sizeof(FACEK));
    BoundKarst->l = create_int(nk);
    BoundKarst->r = create_int(nk);
    cont_karst = create_matrix(2, nk);
    C_contorno = create_matrix(2, nk);
    n_brechas = create_int(nk);
    hs = create_vector(nk);
    for (int j = 0; j < nk; j++) {
        Kc[j] = k->Kc[j];
        BoundKarst->l[j] = k->bound_l[j];
        BoundKarst->r[j] = k->bound_r[j];
        for (int f = 0; f < 2; f++) {
            cont_karst[f][j] = k->cont[f * nk + j];
            C_contorno[f][j] = k->ccont[f * nk + j];
        }
        n_brechas[j] = k->n_brechas[j];
        hs[j] = M[j].pos == 1 ? h.x : M[j].pos == 2 ? h.y : h.z;
    }
    const int mb = k->max_brechas;
    ::beta = create_matrix(mb, nk);
    C = create_matrix(mb, nk);
    brechas = create_matrix_int(mb, nk);
    for (int b = 0; b < mb; b++)
        for (int j = 0; j < nk; j++) {
            ::beta[b][j] = k->beta[b * nk + j];
            C[b][j] = k->cb[b * nk + j];
            brechas[b][j] = k->brechas[b * nk + j];
        }
    ucL_old = create_matrix(mb, nk);
    ucR_old = create_matrix(mb, nk);
    pc = create_matrix(Mmax, nk);
    pc_old = create_matrix(Mmax, nk);
    indcol1 = (IND *)malloc((Mmax + 1) * sizeof(IND));
    uc = (ELEK *)malloc((Mmax + 1) * sizeof(ELEK));
    uc->l = create_matrix(Mmax, nk);
    uc->r = create_matrix(Mmax, nk);
    uc->c = create_matrix(Mmax, nk);
}

static int karst_cell(int j, int i)
{
    int x = M[j].sxi, y = M[j].syi, z = M[j].szi;
    if (M[j].pos == 1) x += i;
    else if (M[j].pos == 2) y += i;
    else z += i;
    return pindex(x, y, z, N);
}

/* main.c:102-113 */
static double rel_change(const double *y, const double *y_old, int n)
{
    double s1 = 0, s2 = 0;
    for (int i = 0; i < n; i++) {
        s1 = s1 + (y[i] - y_old[i]) * (y[i] - y_old[i]);
        s2 = s2 + y[i] * y[i];
    }
    return sqrt(s1) / sqrt(s2);
}

extern "C" {

/* One conduit() call of the reference (karst.c:8-40 through
 * permeabilidade_karst, source_term1d and solve_linsys_1d) on given state:
 * p_old / perm / K of the 3-D side, paux, KI_c, pc_old and the fracture
 * velocities ucR/ucL (in: previous, out: updated).  Matrices [i*nk + j]
 * (mmax rows), fracture tables [b*nk + j].  Outputs keff (kl, kr, kc), the
 * source term f of each conduit ([i*nk + j]) and pc.  The 1-D solves go
 * through compute() with the pcg.h rule at eps. */
int ref_conduit_step(const or_karst *k, int nx, int ny, int nz, double hx,
                     double hy, double hz, double visc, double rho_,
                     const double *KX, const double *KY, const double *KZ,
                     ELE *perm_in, const double *p_old, const double *paux,
                     const double *kic, const double *pcold_in, double *ucR_io,
                     double *ucL_io, double *kl, double *kr, double *kc,
                     double *f_out, double *pc_out, double eps)
{
    N.x = nx; N.y = ny; N.z = nz; N.xy = nx * ny; N.t = nx * ny * nz;
    h.x = hx; h.y = hy; h.z = hz;
    viscosidade = visc;
    rho = rho_;
    karst_globals(k);
    const int nk = k->nk, mb = k->max_brechas;
    Perm Kp;
    Kp.X = (double *)KX; Kp.Y = (double *)KY; Kp.Z = (double *)KZ;
    Kp.S = create_matrix(Mmax, nk);
    double **KI_c = create_matrix(Mmax, nk), **p_aux = create_matrix(Mmax, nk);
    for (int j = 0; j < nk; j++)
        for (int i = 0; i < Mmax; i++) {
            Kp.S[i][j] = Kc[j];
            KI_c[i][j] = kic[i * nk + j];
            p_aux[i][j] = paux[i * nk + j];
            pc_old[i][j] = pcold_in[i * nk + j];
        }
    for (int b = 0; b < mb; b++)
        for (int j = 0; j < nk; j++) {
            ucR_old[b][j] = ucR_io[b * nk + j];
            ucL_old[b][j] = ucL_io[b * nk + j];
        }
    ELEK keff;
    keff.l = create_matrix(Mmax, nk);
    keff.r = create_matrix(Mmax, nk);
    keff.c = create_matrix(Mmax, nk);
    g_mode = 1;
    g_eps = eps;
    /* the source terms by themselves first (they update the fracture
     * velocities), then conduit() from the same starting state */
    for (int j = 0; j < nk; j++) {
        std::vector<double> f(M[j].s + 2, 0.0);
        permeabilidade_karst(&Kp, &keff, indcol1, hs, M, BoundKarst, viscosidade, KI_c, j);
        source_term1d(&keff, hs, M, BoundKarst, cont_karst, KI_c, p_aux, &Kp,
                      perm_in, (double *)p_old, j, f.data());
        for (int i = 0; i < M[j].s; i++) f_out[i * nk + j] = f[i];
    }
    for (int b = 0; b < mb; b++)
        for (int j = 0; j < nk; j++) {
            ucR_old[b][j] = ucR_io[b * nk + j];
            ucL_old[b][j] = ucL_io[b * nk + j];
        }
    conduit(p_aux, cont_karst, KI_c, viscosidade, M, hs, indcol1, BoundKarst,
            &keff, &Kp, perm_in, (double *)p_old, pc);
    for (int j = 0; j < nk; j++)
        for (int i = 0; i < M[j].s; i++) {
            kl[i * nk + j] = keff.l[i][j];
            kr[i * nk + j] = keff.r[i][j];
            kc[i * nk + j] = keff.c[i][j];
            pc_out[i * nk + j] = pc[i][j];
        }
    for (int b = 0; b < mb; b++)
        for (int j = 0; j < nk; j++) {
            ucR_io[b * nk + j] = ucR_old[b][j];
            ucL_io[b * nk + j] = ucL_old[b][j];
        }
    return 0;
}

/* The reference's coupled run: main.c:383-489 (restated loop around the
 * reference's own reservoir() and conduit()), then fluxo1d / fluxos and the
 * balances of main.c:523-593.  Every solve goes through compute() with the
 * pcg.h stop rule at eps (compute.cpp uses 1e-8).  Same outputs as
 * or_picard; times[0] = the run (s), times[1] = compute() calls. */
int ref_picard(const or_karst *k, int nx, int ny, int nz, double hx, double hy,
               double hz, double visc, double rho_, const double *KX,
               const double *KY, const double *KZ, const int *bc,
               const double *val6, const double *WI_in, const double *pw_in,
               double tol, int iter_max, double eps, double *p_out,
               double *pc_out, double *ucl, double *ucr, ELE *v_out,
               double *out, double *qk, double *times)
{
    double t0 = now();
    set_grid(nx, ny, nz, hx, hy, hz, bc, visc);
    rho = rho_;
    karst_globals(k);
    const int nk = k->nk;
    Perm Kp;
    Kp.X = create_vector(N.t); Kp.Y = create_vector(N.t); Kp.Z = create_vector(N.t);
    for (int s = 0; s < N.t; s++) { Kp.X[s] = KX[s]; Kp.Y[s] = KY[s]; Kp.Z[s] = KZ[s]; }
    Kp.S = create_matrix(Mmax, nk);
    for (int j = 0; j < nk; j++)
        for (int i = 0; i < Mmax; i++) Kp.S[i][j] = Kc[j];   /* permeabilities.c:46-51 */
    double *WI = create_vector(N.t), *KI = create_vector(N.t), *pw = create_vector(N.t);
    if (pw_in) for (int s = 0; s < N.t; s++) pw[s] = pw_in[s];
    Bound *Bd = make_bound(val6);
    ELE *pm = (ELE *)calloc(N.t + 1, sizeof(ELE));
    IND *ic = (IND *)malloc((N.t + 1) * sizeof(IND));
    for (int s = 0; s < N.t; s++) {
        ic[s].c = ic[s].u = ic[s].d = ic[s].l = -1;
        ic[s].r = ic[s].t = ic[s].b = -1;
    }
    double *p = create_vector(N.t), *p_old = create_vector(N.t);
    g_mode = 1;
    g_eps = eps;
    int ncompute = 0;
    reservoir(N, &Kp, WI, KI, pc_old, ic, Bd, pm, h, boundary, viscosidade, pw, M, p);
    ncompute++;
    for (int s = 0; s < N.t; s++) p_old[s] = p[s];
    if (WI_in) for (int s = 0; s < N.t; s++) WI[s] = WI_in[s];
    double **KI_c = create_matrix(Mmax, nk), **p_aux = create_matrix(Mmax, nk);
    for (int j = 0; j < nk; j++)
        for (int i = 0; i < M[j].s; i++) {
            int aux = karst_cell(j, i);
            KI[aux] = k->kindex[j];
            KI_c[i][j] = k->kindex[j] / (k->area[j] * hs[j]);
            p_aux[i][j] = p_old[aux];
            Kp.S[i][j] = Kc[j];
        }
    ELEK keff;
    keff.l = create_matrix(Mmax, nk);
    keff.r = create_matrix(Mmax, nk);
    keff.c = create_matrix(Mmax, nk);
    conduit(p_aux, cont_karst, KI_c, viscosidade, M, hs, indcol1, BoundKarst,
            &keff, &Kp, pm, p_old, pc);
    ncompute += nk;
    double error = 1;
    int iter = 0;
    while (iter < iter_max && error > tol) {
        for (int i = 0; i < Mmax; i++)
            for (int j = 0; j < nk; j++) pc_old[i][j] = pc[i][j];
        reservoir(N, &Kp, WI, KI, pc_old, ic, Bd, pm, h, boundary, viscosidade, pw, M, p);
        error = rel_change(p, p_old, N.t);
        for (int s = 0; s < N.t; s++) p_old[s] = p[s];
        for (int j = 0; j < nk; j++)
            for (int i = 0; i < M[j].s; i++) p_aux[i][j] = p_old[karst_cell(j, i)];
        conduit(p_aux, cont_karst, KI_c, viscosidade, M, hs, indcol1, BoundKarst,
                &keff, &Kp, pm, p_old, pc);
        ncompute += 1 + nk;
        iter++;
    }
    double t1 = now();
    fluxo1d(pc, &keff, uc, hs, M, cont_karst, BoundKarst, &Kp, pm, p_old);
    if (v_out) fluxos(p, pm, v_out, Bd, h, N);
    for (int s = 0; s < N.t; s++) p_out[s] = p[s];
    for (int i = 0; i < Mmax; i++)
        for (int j = 0; j < nk; j++) {
            bool in = i < M[j].s;
            pc_out[i * nk + j] = in ? pc[i][j] : 0.0;
            if (ucl) ucl[i * nk + j] = in ? uc->l[i][j] : 0.0;
            if (ucr) ucr[i * nk + j] = in ? uc->r[i][j] : 0.0;
        }
    if (out) {
        double Q = 0.0, pm_ = 0.0;
        for (int s = 0; s < N.t; s++) {
            Q = Q + (WI[s] / viscosidade) * (pw[s] - p[s]);
            pm_ = pm_ + p[s];
        }
        out[0] = error;
        out[1] = Q;
        out[2] = pm_ / N.t;
    }
    if (qk)
        for (int j = 0; j < nk; j++) {
            double qc = 0.0, q3 = 0.0;
            for (int i = 0; i < M[j].s; i++) {
                int aux = karst_cell(j, i);
                qc = qc + (-KI[aux] / viscosidade) * (pc[i][j] - p[aux]) * hs[j];
                q3 = q3 + (KI[aux] / viscosidade) * (pc[i][j] - p[aux]);
            }
            qk[j] = qc;
            qk[nk + j] = q3;
            qk[2 * nk + j] = uc->l[0][j] * k->area[j] + uc->r[M[j].s - 1][j] * k->area[j];
        }
    if (times) { times[0] = t1 - t0; times[1] = ncompute; }
    free_bound(Bd);
    free(pm); free(ic); free(p); free(p_old); free(WI); free(KI); free(pw);
    free(Kp.X); free(Kp.Y); free(Kp.Z);
    return iter;
}

}  // extern "C"

/* ---- the reference's result writers (posprocessing_output.c, vtk.c) ------ */
extern "C" {

/* save_pressure / save_flux / vts_StructuredGrid_file into directory dir
 * (the reference's dirname): pressure_reservoir.dat, flux_reservoir.dat,
 * campos.vts. */
int ref_save_grid(const char *dir, int nx, int ny, int nz, double hx, double hy,
                  double hz, double *p, ELE *v)
{
    N.x = nx; N.y = ny; N.z = nz; N.xy = nx * ny; N.t = nx * ny * nz;
    h.x = hx; h.y = hy; h.z = hz;
    dirname = dir;
    if (p) save_pressure(p, N, h);
    if (v) save_flux(v, N, h);
    if (p && v) vts_StructuredGrid_file(v, p, N, h);
    return 0;
}

/* save_pressure_1d / save_flux_1d into dir for a conduit set; pc, ucl, ucr
 * in the [i*nk + j] layout. */
int ref_save_karst(const char *dir, const or_karst *k, double hx, double hy,
                   double hz, const double *pcf, const double *ucl,
                   const double *ucr)
{
    h.x = hx; h.y = hy; h.z = hz;
    dirname = dir;
    karst_globals(k);
    const int nk = k->nk;
    for (int i = 0; i < Mmax; i++)
        for (int j = 0; j < nk; j++) {
            pc[i][j] = pcf[i * nk + j];
            uc->l[i][j] = ucl[i * nk + j];
            uc->r[i][j] = ucr[i * nk + j];
        }
    save_pressure_1d(pc, M, hs, h);
    save_flux_1d(uc, M, hs, h);
    return 0;
}

}  // extern "C"

/* ---- the reference's permeability readers (permeabilities.c) ------------- */
extern "C" {

/* variant 0 read_set_perm_field, 1 read_layer_perm_field (layer), 2
 * gaussian_permfield (geological grid ngx^3 through nxg/nyg/nzg); the
 * simulation grid nx*ny*nz on Ix*Iy*Iz with h = I/N as main.c:163-165. */
int ref_read_perm(int variant, const char *path, int layer_, int ng, int nx, int ny,
                  int nz, double Ix, double Iy, double Iz, double *KX, double *KY,
                  double *KZ)
{
    N.x = nx; N.y = ny; N.z = nz; N.xy = nx * ny; N.t = nx * ny * nz;
    I.x = Ix; I.y = Iy; I.z = Iz;
    h.x = I.x / N.x; h.y = I.y / N.y; h.z = I.z / N.z;
    fn = path;
    layer = layer_;
    nxg = nyg = nzg = ng;
    Perm K;
    K.X = KX; K.Y = KY; K.Z = KZ;
    if (variant == 0) read_set_perm_field(&K, N, h, I);
    else if (variant == 1) read_layer_perm_field(&K, N, h, I);
    else gaussian_permfield(&K, N, h, I);
    return 0;
}

}  // extern "C"
