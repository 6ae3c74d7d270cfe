/*
 * hmfem_oracle.c -- CPU restatement of hmfem's pressure-solve path.
 *
 * TEST INFRASTRUCTURE ONLY (the correctness oracle and the CPU "port"
 * baseline).  Never linked into, loaded by or called from the GPU product
 * library.  Every function restates a reference routine; the citation is the
 * file:line in the hmfem tree (toolbox paths relative to the tree root).
 *
 * Floating-point expressions keep the reference's evaluation order so that
 * assembly, setup and transfer results are bit-identical to the reference
 * compiled with the same flags (no FMA contraction: -ffp-contract=off).
 */
#include "hmfem_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IDX(i, j, k) ((i) + (j) * nx + (k) * nxy)

double or_hm(double a, double b) { return 2 * a * b / (a + b); }

/* permeabilities.c:196-492 */
void or_assemble(int nx, int ny, int nz, double hx, double hy, double hz,
                 double visc, const double *KX, const double *KY,
                 const double *KZ, const int bc_type[6], const double *KI,
                 const double *WI, or_ele *perm, or_ind *indcol)
{
    const int nxy = nx * ny;
    int i, j, k, s;
    /* interior faces (permeabilities.c:214-293) */
    for (k = 0; k < nz; k++)
        for (j = 0; j < ny; j++)
            for (i = 0; i < nx; i++) {
                s = IDX(i, j, k);
                if (j < ny - 1) {
                    perm[s].u = or_hm(KY[s], KY[s + nx]);
                    perm[s].u = perm[s].u / (hy * hy * visc);
                    indcol[s].u = s + nx;
                }
                if (i < nx - 1) {
                    perm[s].r = or_hm(KX[s], KX[s + 1]);
                    perm[s].r = perm[s].r / (hx * hx * visc);
                    indcol[s].r = s + 1;
                }
                if (j > 0) {
                    perm[s].d = or_hm(KY[s], KY[s - nx]);
                    perm[s].d = perm[s].d / (hy * hy * visc);
                    indcol[s].d = s - nx;
                }
                if (i > 0) {
                    perm[s].l = or_hm(KX[s], KX[s - 1]);
                    perm[s].l = perm[s].l / (hx * hx * visc);
                    indcol[s].l = s - 1;
                }
                if (k < nz - 1) {
                    perm[s].t = or_hm(KZ[s], KZ[s + nxy]);
                    perm[s].t = perm[s].t / (hz * hz * visc);
                    indcol[s].t = s + nxy;
                }
                if (k > 0) {
                    perm[s].b = or_hm(KZ[s], KZ[s - nxy]);
                    perm[s].b = perm[s].b / (hz * hz * visc);
                    indcol[s].b = s - nxy;
                }
            }
    /* boundary faces (permeabilities.c:297-477): Dirichlet 2K/(h^2 mu),
     * Neumann 0; both go to the right-hand side (indcol = -1). */
    for (k = 0; k < nz; k++)
        for (j = 0; j < ny; j++) {
            s = IDX(0, j, k);
            perm[s].l = bc_type[0] == 0 ? 2.0 * KX[s] / (hx * hx * visc) : 0;
            indcol[s].l = -1;
            s = IDX(nx - 1, j, k);
            perm[s].r = bc_type[1] == 0 ? 2.0 * KX[s] / (hx * hx * visc) : 0;
            indcol[s].r = -1;
        }
    if (bc_type[0] == 1 && bc_type[1] == 1 && bc_type[2] == 1 &&
        bc_type[3] == 1 && bc_type[4] == 1 && bc_type[5] == 1) {
        /* all-Neumann: one Dirichlet face pins the pressure
         * (permeabilities.c:327-333) */
        s = IDX(0, ny - 1, nz / 2);
        perm[s].l = 2.0 * KX[s] / (hx * hx * visc);
        indcol[s].l = -1;
    }
    for (k = 0; k < nz; k++)
        for (i = 0; i < nx; i++) {
            s = IDX(i, 0, k);
            perm[s].d = bc_type[3] == 0 ? 2.0 * KY[s] / (hy * hy * visc) : 0;
            indcol[s].d = -1;
            s = IDX(i, ny - 1, k);
            perm[s].u = bc_type[2] == 0 ? 2.0 * KY[s] / (hy * hy * visc) : 0;
            indcol[s].u = -1;
        }
    for (j = 0; j < ny; j++)
        for (i = 0; i < nx; i++) {
            s = IDX(i, j, nz - 1);
            perm[s].t = bc_type[4] == 0 ? 2.0 * KZ[s] / (hz * hz * visc) : 0;
            indcol[s].t = -1;
            s = IDX(i, j, 0);
            perm[s].b = bc_type[5] == 0 ? 2.0 * KZ[s] / (hz * hz * visc) : 0;
            indcol[s].b = -1;
        }
    /* centre (permeabilities.c:480-489) */
    for (s = 0; s < nx * ny * nz; s++) {
        double ki = KI ? KI[s] : 0.0, wi = WI ? WI[s] : 0.0;
        perm[s].c = perm[s].l + perm[s].r + perm[s].u + perm[s].d +
                    perm[s].t + perm[s].b + ki / (visc * hx * hy * hz) +
                    wi / (visc * hx * hy * hz);
        indcol[s].c = s;
    }
}

/* set_source_term.c:9-223; faces in the reference's interface order
 * L, R, D, U, T, B. */
void or_source_term(int nx, int ny, int nz, double hx, double hy, double hz,
                    double visc, const or_bound *B, const int bc_type[6],
                    const or_ele *perm, const double *KI, const double *WI,
                    const double *pc, const double *pw, double *b)
{
    const int nxy = nx * ny;
    int i, j, k, s;
    for (j = 0; j < ny; j++)
        for (k = 0; k < nz; k++) {
            s = IDX(0, j, k);
            int l = k * ny + j;
            if (bc_type[0] == 0) b[s] = b[s] + (perm[s].l) * B->l[l];
            if (bc_type[0] == 1) b[s] = b[s] + B->l[l] / hx;
        }
    if (bc_type[0] == 1 && bc_type[1] == 1 && bc_type[2] == 1 &&
        bc_type[3] == 1 && bc_type[4] == 1 && bc_type[5] == 1) {
        s = IDX(0, ny - 1, nz / 2);
        b[s] = b[s] + (perm[s].l) * 1.0;
    }
    for (j = 0; j < ny; j++)
        for (k = 0; k < nz; k++) {
            s = IDX(nx - 1, j, k);
            int l = k * ny + j;
            if (bc_type[1] == 0) b[s] = b[s] + perm[s].r * B->r[l];
            if (bc_type[1] == 1) b[s] = b[s] - B->r[l] / hx;
        }
    for (i = 0; i < nx; i++)
        for (k = 0; k < nz; k++) {
            s = IDX(i, 0, k);
            int l = k * nx + i;
            if (bc_type[3] == 0) b[s] = b[s] + perm[s].d * B->d[l];
            if (bc_type[3] == 1) b[s] = b[s] + B->d[l] / hy;
        }
    for (i = 0; i < nx; i++)
        for (k = 0; k < nz; k++) {
            s = IDX(i, ny - 1, k);
            int l = k * nx + i;
            if (bc_type[2] == 0) b[s] = b[s] + perm[s].u * B->u[l];
            if (bc_type[2] == 1) b[s] = b[s] - B->u[l] / hy;
        }
    for (i = 0; i < nx; i++)
        for (j = 0; j < ny; j++) {
            s = IDX(i, j, nz - 1);
            int l = j * nx + i;
            if (bc_type[4] == 0) b[s] = b[s] + perm[s].t * B->t[l];
            if (bc_type[4] == 1) b[s] = b[s] - B->t[l] / hz;
        }
    for (i = 0; i < nx; i++)
        for (j = 0; j < ny; j++) {
            s = IDX(i, j, 0);
            int l = j * nx + i;
            if (bc_type[5] == 0) b[s] = b[s] + perm[s].b * B->b[l];
            if (bc_type[5] == 1) b[s] = b[s] + B->b[l] / hz;
        }
    /* sources (set_source_term.c:206-220) */
    double Ve = hx * hy * hz;
    for (s = 0; s < nx * ny * nz; s++) {
        double ki = KI ? KI[s] : 0.0, wi = WI ? WI[s] : 0.0;
        double pcs = pc ? pc[s] : 0.0, pws = pw ? pw[s] : 0.0;
        b[s] = b[s] + (ki * pcs) / (visc * Ve) + (wi * pws) / (visc * Ve);
    }
}

/* solve_linearsystem_AMG.c:55-141 */
long or_pack_csr(int n, const or_ele *perm, const or_ind *indcol, int *cnt,
                 int *col, double *ele)
{
    long l = 0;
    for (int s = 0; s < n; s++) {
        int c = 0;
#define PUT(f, v)                                                            \
    if (indcol[s].f != -1) {                                                 \
        if (col) { col[l] = indcol[s].f; ele[l] = (v); }                     \
        l++; c++;                                                            \
    }
        PUT(d, -perm[s].d)
        PUT(l, -perm[s].l)
        PUT(c, perm[s].c)
        PUT(r, -perm[s].r)
        PUT(u, -perm[s].u)
        PUT(t, -perm[s].t)
        PUT(b, -perm[s].b)
#undef PUT
        if (cnt) cnt[s] = c;
    }
    return l;
}

/* ---------------------------------------------------------------- AMG -- */

static long *offsets(int n, const int *cnt)
{
    long *dsp = (long *)malloc(sizeof(long) * (n + 1));
    dsp[0] = 0;
    for (int i = 0; i < n; i++) dsp[i + 1] = dsp[i] + cnt[i];
    return dsp;
}

/* node_selection (toolbox.h / amg.h:1-32) for one rank: bou = true. */
static void node_select(char sel, int n, const int *cnt, const long *dsp,
                        const int *col, const char *cox, char *asel)
{
    for (int i = 0; i < n; i++) {
        if (asel[i] != sel) continue;
        if (sel == 0) asel[i] = 1; /* master (C) node */
        for (long j = dsp[i]; j < dsp[i] + cnt[i]; j++) {
            int c = col[j];
            if (asel[c] != 0) continue;
            for (long k = dsp[c]; k < dsp[c] + cnt[c]; k++)
                if (col[k] == i && cox[k] != 0) { asel[c] = 2; break; }
        }
    }
}

/* sparse_multiply_transpose (amg.h:408-563, the active #else branch):
 * C = (A B)^T with B having `bcols` columns.  Columns of each C row come out
 * ascending (A's row index). */
static void spmt(int arows, const int *acnt, const int *acol,
                 const double *aele, int brows, const int *bcnt,
                 const int *bcol, const double *bele, int bcols, int **ccnt_o,
                 int **ccol_o, double **cele_o, long *csize_o)
{
    long *bdsp = offsets(brows, bcnt);
    int *ccnt = (int *)calloc(bcols > 0 ? bcols : 1, sizeof(int));
    int *clst = (int *)malloc(sizeof(int) * (bcols > 0 ? bcols : 1));
    for (int i = 0; i < bcols; i++) clst[i] = -1;
    long csize = 0, m = 0;
    for (int i = 0; i < arows; i++)
        for (int j = 0; j < acnt[i]; j++) {
            int c = acol[m++];
            for (long k = bdsp[c]; k < bdsp[c] + bcnt[c]; k++) {
                int d = bcol[k];
                if (clst[d] != i) { clst[d] = i; ccnt[d]++; csize++; }
            }
        }
    for (int i = 0; i < bcols; i++) clst[i] = -1;
    long *cdsp = (long *)malloc(sizeof(long) * (bcols > 0 ? bcols : 1));
    for (long t = 0, i = 0; i < bcols; i++) { cdsp[i] = t; t += ccnt[i]; }
    int *ccol = (int *)malloc(sizeof(int) * (csize > 0 ? csize : 1));
    double *cele = (double *)malloc(sizeof(double) * (csize > 0 ? csize : 1));
    m = 0;
    for (int i = 0; i < arows; i++)
        for (int j = 0; j < acnt[i]; j++) {
            int c = acol[m];
            double s = aele[m];
            m++;
            for (long k = bdsp[c]; k < bdsp[c] + bcnt[c]; k++) {
                int d = bcol[k];
                long e = cdsp[d];
                double t = s * bele[k];
                if (clst[d] != i) {
                    clst[d] = i;
                    ccol[e] = i;
                    cele[e] = t;
                    cdsp[d] = e + 1;
                } else {
                    cele[e - 1] += t;
                }
            }
        }
    free(bdsp); free(clst); free(cdsp);
    *ccnt_o = ccnt; *ccol_o = ccol; *cele_o = cele; *csize_o = csize;
}

/* Colouring for the multicolour Gauss-Seidel smoother (project setup, no
 * reference counterpart): Jones-Plassmann rounds with fixed pseudo-random
 * priorities.  In each round every uncoloured row whose (priority, index)
 * key exceeds those of all its uncoloured neighbours takes the smallest
 * colour not used by its already-coloured neighbours; those rows form an
 * independent set, so a round's result does not depend on the order the
 * rows are visited in (the GPU visits them in parallel). */
static unsigned jp_prio(unsigned x)
{
    x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16;
    return x;
}

static unsigned long long jp_key(int v)
{
    return ((unsigned long long)jp_prio((unsigned)v) << 32) | (unsigned)v;
}

static int greedy_colour(or_level *A)
{
    const int n = A->n;
    A->color = (signed char *)malloc(n > 0 ? n : 1);
    signed char *nw = (signed char *)malloc(n > 0 ? n : 1);
    long *dsp = offsets(n, A->cnt);
    for (int i = 0; i < n; i++) A->color[i] = -1;
    int left = n, nc = 0;
    while (left > 0) {
        for (int v = 0; v < n; v++) {
            nw[v] = A->color[v];
            if (A->color[v] >= 0) continue;
            unsigned long long used = 0, kv = jp_key(v);
            int ok = 1;
            for (long j = dsp[v]; j < dsp[v + 1]; j++) {
                int u = A->col[j];
                if (u == v) continue;
                signed char c = A->color[u];
                if (c >= 0) used |= 1ull << c;
                else if (jp_key(u) > kv) { ok = 0; break; }
            }
            if (!ok) continue;
            int k = 0;
            while (k < 63 && (used & (1ull << k))) k++;
            nw[v] = (signed char)k;
        }
        for (int v = 0; v < n; v++) {
            if (A->color[v] < 0 && nw[v] >= 0) {
                left--;
                if (nw[v] + 1 > nc) nc = nw[v] + 1;
            }
            A->color[v] = nw[v];
        }
    }
    free(nw);
    free(dsp);
    return nc;
}

/* l1-Jacobi diagonal: a_ii + sum over the other stored entries of |a_ij|,
 * accumulated in row order (project smoother, no reference counterpart). */
static double *l1_inverse(const or_level *A, const double *dia)
{
    double *d = (double *)malloc(sizeof(double) * (A->n > 0 ? A->n : 1));
    long m = 0;
    for (int i = 0; i < A->n; i++) {
        double t = 0.0;
        for (int j = 0; j < A->cnt[i]; j++, m++)
            if (A->col[m] != i) t = t + fabs(A->ele[m]);
        d[i] = 1.0 / (dia[i] + t);
    }
    return d;
}

/* One coarsening step: parallel_coarsening (amg.h:37-223), then
 * parallel_interpolation (amg.h:228-406), then new_triple_product
 * (amg.h:567-582), for a single rank (no interface nodes). */
static void coarsen_level(double eps, or_level *A, or_level *Cn)
{
    int n = A->n;
    long *dsp = offsets(n, A->cnt);
    /* diagonal: last stored diagonal entry (amg.h:159-166) */
    double *dia = (double *)calloc(n, sizeof(double));
    for (int i = 0; i < n; i++)
        for (long j = dsp[i]; j < dsp[i] + A->cnt[i]; j++)
            if (A->col[j] == i) dia[i] = A->ele[j];
    /* strength (amg.h:167-193): |a_ij| >= |eps a_ii| */
    char *cox = (char *)malloc(A->nnz > 0 ? A->nnz : 1);
    for (int i = 0; i < n; i++) {
        double sda = fabs(eps * dia[i]);
        for (long j = dsp[i]; j < dsp[i] + A->cnt[i]; j++)
            cox[j] = fabs(A->ele[j]) >= sda ? 1 : 0;
    }
    /* phases (b) and (c) (amg.h:219-223) */
    char *sel = (char *)calloc(n, 1);
    node_select(1, n, A->cnt, dsp, A->col, cox, sel);
    node_select(0, n, A->cnt, dsp, A->col, cox, sel);
    A->sel = sel;
    /* interpolation (amg.h:326-387) */
    int *pcnt = (int *)calloc(n, sizeof(int));
    for (int i = 0; i < n; i++) {
        if (sel[i] == 1) { pcnt[i] = 1; continue; }
        for (long j = dsp[i]; j < dsp[i] + A->cnt[i]; j++)
            if (sel[A->col[j]] == 1 && cox[j] != 0) pcnt[i]++;
    }
    long pnnz = 0;
    for (int i = 0; i < n; i++) pnnz += pcnt[i];
    int *pcol = (int *)malloc(sizeof(int) * (pnnz > 0 ? pnnz : 1));
    double *pele = (double *)malloc(sizeof(double) * (pnnz > 0 ? pnnz : 1));
    long m = 0;
    for (int i = 0; i < n; i++) {
        if (sel[i] == 1) { pcol[m] = i; pele[m] = 1.0; m++; continue; }
        for (long j = dsp[i]; j < dsp[i] + A->cnt[i]; j++)
            if (sel[A->col[j]] == 1 && cox[j] != 0) {
                pcol[m] = A->col[j];
                pele[m] = 1.0 / pcnt[i];
                m++;
            }
    }
    /* coarse numbering: ascending order of the fine ids that appear in P
     * (amg.h:394-403, binary_sort_copy + unique_resize) */
    int *cid = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    for (int i = 0; i < n; i++) cid[i] = 0;
    for (long q = 0; q < pnnz; q++) cid[pcol[q]] = 1;
    int nc = 0;
    for (int i = 0; i < n; i++) { int a = cid[i]; cid[i] = a ? nc : -1; nc += a; }
    for (long q = 0; q < pnnz; q++) pcol[q] = cid[pcol[q]];
    A->pcnt = pcnt; A->pcol = pcol; A->pele = pele; A->pnnz = pnnz;
    /* Galerkin product P^T A P as two (X P)^T passes (amg.h:567-582) */
    int *tcnt, *tcol; double *tele; long tsize;
    spmt(n, A->cnt, A->col, A->ele, n, pcnt, pcol, pele, nc, &tcnt, &tcol,
         &tele, &tsize);
    int *ccnt, *ccol; double *cele; long csize;
    spmt(nc, tcnt, tcol, tele, n, pcnt, pcol, pele, nc, &ccnt, &ccol, &cele,
         &csize);
    free(tcnt); free(tcol); free(tele);
    Cn->n = nc; Cn->nnz = csize; Cn->cnt = ccnt; Cn->col = ccol; Cn->ele = cele;
    /* 1/diag on this level (amg.h:1195) */
    A->dinv = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
    for (int i = 0; i < n; i++) A->dinv[i] = 1.0 / dia[i];
    A->dl1inv = l1_inverse(A, dia);
    A->ncolors = greedy_colour(A);
    free(dia); free(cox); free(cid); free(dsp);
}

int or_amg_setup(int n, const int *cnt, const int *col, const double *ele,
                 int max_level, int max_size, double eps, or_hierarchy *H)
{
    memset(H, 0, sizeof(*H));
    if (max_level > OR_MAX_LEVELS) max_level = OR_MAX_LEVELS;
    or_level *L0 = &H->lv[0];
    long nnz = 0;
    for (int i = 0; i < n; i++) nnz += cnt[i];
    L0->n = n; L0->nnz = nnz;
    L0->cnt = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    L0->col = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    L0->ele = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
    memcpy(L0->cnt, cnt, sizeof(int) * n);
    memcpy(L0->col, col, sizeof(int) * nnz);
    memcpy(L0->ele, ele, sizeof(double) * nnz);
    /* level loop (amg.h:1188-1213) */
    int l = 0, gcnt = n;
    double rel = 0.0;
    while (l < max_level - 1 && gcnt > max_size && rel < 1.0) {
        coarsen_level(eps, &H->lv[l], &H->lv[l + 1]);
        l++;
        int gold = gcnt;
        gcnt = H->lv[l].n;
        rel = (double)gcnt / (double)gold;
    }
    /* coarsest level: 1/diag (amg.h:1214-1226) */
    or_level *C = &H->lv[l];
    C->dinv = (double *)malloc(sizeof(double) * (C->n > 0 ? C->n : 1));
    double *cd = (double *)calloc(C->n > 0 ? C->n : 1, sizeof(double));
    for (long t = 0, i = 0; i < C->n; i++) {
        for (int j = 0; j < C->cnt[i]; j++, t++)
            if (C->col[t] == i) cd[i] = C->ele[t];
        C->dinv[i] = 1.0 / cd[i];
    }
    C->dl1inv = l1_inverse(C, cd);
    free(cd);
    H->nlevels = l + 1;
    return H->nlevels;
}

void or_amg_free(or_hierarchy *H)
{
    for (int l = 0; l < H->nlevels; l++) {
        or_level *A = &H->lv[l];
        free(A->cnt); free(A->col); free(A->ele); free(A->dinv); free(A->dl1inv);
        free(A->color);
        free(A->sel); free(A->pcnt); free(A->pcol); free(A->pele);
    }
    memset(H, 0, sizeof(*H));
}

int or_level_info(const or_hierarchy *H, int l, int *n, long *nnz, long *pnnz)
{
    if (l < 0 || l >= H->nlevels) return -1;
    *n = H->lv[l].n;
    *nnz = H->lv[l].nnz;
    *pnnz = l < H->nlevels - 1 ? H->lv[l].pnnz : 0;
    return 0;
}

or_hierarchy *or_amg_create(int n, const int *cnt, const int *col,
                            const double *ele, int max_level, int max_size,
                            double eps)
{
    or_hierarchy *H = (or_hierarchy *)malloc(sizeof(or_hierarchy));
    or_amg_setup(n, cnt, col, ele, max_level, max_size, eps, H);
    return H;
}

void or_amg_destroy(or_hierarchy *H)
{
    if (!H) return;
    or_amg_free(H);
    free(H);
}

int or_amg_nlevels(const or_hierarchy *H) { return H->nlevels; }

int or_level_copy(const or_hierarchy *H, int l, int *cnt, int *col,
                  double *ele, double *dinv, char *sel, int *pcnt, int *pcol,
                  double *pele)
{
    if (l < 0 || l >= H->nlevels) return -1;
    const or_level *A = &H->lv[l];
    memcpy(cnt, A->cnt, sizeof(int) * A->n);
    memcpy(col, A->col, sizeof(int) * A->nnz);
    memcpy(ele, A->ele, sizeof(double) * A->nnz);
    memcpy(dinv, A->dinv, sizeof(double) * A->n);
    if (l < H->nlevels - 1) {
        memcpy(sel, A->sel, A->n);
        memcpy(pcnt, A->pcnt, sizeof(int) * A->n);
        memcpy(pcol, A->pcol, sizeof(int) * A->pnnz);
        memcpy(pele, A->pele, sizeof(double) * A->pnnz);
    }
    return 0;
}

/* generic_operator.h:212-247 */
void or_spmv(int n, const int *cnt, const int *col, const double *ele,
             const double *x, double *y)
{
    long m = 0;
    for (int i = 0; i < n; i++) {
        double s = 0.0;
        for (int j = 0; j < cnt[i]; j++, m++) s += ele[m] * x[col[m]];
        y[i] = s;
    }
}

/* simple_restriction (generic_operator.h:68-129): s = P^T u with 1/c */
static void restrict_simple(const or_level *A, int nc, const double *u,
                            double *s)
{
    for (int i = 0; i < nc; i++) s[i] = 0.0;
    long m = 0;
    for (int i = 0; i < A->n; i++) {
        int c = A->pcnt[i];
        if (c == 0) continue;
        double t = c == 1 ? u[i] : u[i] / (double)c;
        for (int j = 0; j < c; j++) s[A->pcol[m++]] += t;
    }
}

/* simple_prolongation (generic_operator.h:7-66): s = P u (average) */
static void prolong_simple(const or_level *A, const double *u, double *s)
{
    long m = 0;
    for (int i = 0; i < A->n; i++) {
        int c = A->pcnt[i];
        if (c == 0) continue;
        if (c == 1) { s[i] = u[A->pcol[m++]]; continue; }
        double t = u[A->pcol[m++]];
        for (int j = 1; j < c; j++) t += u[A->pcol[m++]];
        s[i] = t / (double)c;
    }
}

typedef struct { double *u, *f, *s, *r; } or_work;

/* One colour of a Gauss-Seidel sweep: rows of colour c, each
 * u_i += (f_i - sum_j a_ij u_j) / a_ii with the sum in row order. */
/* sum_j a_ij x_j for the coarse-level smoother in the order the GPU forms
 * it with eight threads per row: thread g sums entries g, g+8, g+16, ...
 * of the row in order, then the eight partial sums are combined pairwise
 * by offsets 4, 2, 1 and thread 0's value is used. */
static double row_dot8(const or_level *A, long m0, int cnt, const double *x)
{
    double p[8], q[8];
    for (int g = 0; g < 8; g++) {
        double t = 0.0;
        for (int k = g; k < cnt; k += 8) t += A->ele[m0 + k] * x[A->col[m0 + k]];
        p[g] = t;
    }
    for (int o = 4; o > 0; o >>= 1) {
        for (int g = 0; g < 8; g++) q[g] = p[g] + p[g ^ o];
        for (int g = 0; g < 8; g++) p[g] = q[g];
    }
    return p[0];
}

/* One colour of a Gauss-Seidel sweep: rows of colour c, each
 * u_i += (f_i - sum_j a_ij u_j) / a_ii. */
static void gs_colour(const or_level *A, int c, const double *f, double *u)
{
    long m = 0;
    for (int i = 0; i < A->n; i++) {
        if (A->color[i] == c) {
            double t = f[i] - row_dot8(A, m, A->cnt[i], u);
            u[i] += t * A->dinv[i];
        }
        m += A->cnt[i];
    }
}

/* Chebyshev smoothing (project smoother for the coarse levels, no
 * reference counterpart): K steps of the Chebyshev iteration (Saad,
 * Iterative Methods for Sparse Linear Systems, alg. 12.1) on D^-1 A with D
 * the l1 diagonal, over the interval [1/30, 1] -- 1 bounds the spectrum of
 * D^-1 A by Gershgorin (d_i = a_ii + sum_j!=i |a_ij|).  Coefficients:
 * theta = (hi+lo)/2, delta = (hi-lo)/2, sigma = theta/delta, rho_0 =
 * 1/sigma, rho_k = 1/(2 sigma - rho_{k-1}), c1_k = rho_k rho_{k-1}, c2_k =
 * 2 rho_k / delta.  The GPU computes the same doubles on its host. */
#define OR_CHEB_LO (1.0 / 30.0)
#define OR_CHEB_HI 1.0

static void cheb_coeffs(int K, double *ith, double *c1, double *c2)
{
    const double th = (OR_CHEB_HI + OR_CHEB_LO) / 2, de = (OR_CHEB_HI - OR_CHEB_LO) / 2;
    const double sg = th / de;
    double rho = 1.0 / sg;
    *ith = 1.0 / th;
    for (int k = 1; k < K; k++) {
        const double rn = 1.0 / (2.0 * sg - rho);
        c1[k] = rn * rho;
        c2[k] = 2.0 * rn / de;
        rho = rn;
    }
}

/* Steps k = 1..K-1 after the first direction d (= d0) is formed: per step
 * q = sum_j a_ij d_j (row order, from 0); r = r - D^-1 q; d' = c1 d + c2 r;
 * u = u + d' (first step: u = d0 + d' from zero, (u + d0) + d' otherwise).
 * first_r0: the pre-smoother forms r0 = D^-1 f inside its first step. */
static void cheb_steps(const or_level *A, int K, int from_zero, const double *f,
                       double *u, double *r, double *d, double *dn)
{
    double ith, c1[10], c2[10];
    cheb_coeffs(K, &ith, c1, c2);
    const int n = A->n;
    const double *dv = A->dl1inv;
    for (int k = 1; k < K; k++) {
        long m = 0;
        for (int i = 0; i < n; i++) {
            double q = 0.0;
            for (int j = 0; j < A->cnt[i]; j++, m++) q += A->ele[m] * d[A->col[m]];
            const double rp = (k == 1 && from_zero) ? dv[i] * f[i] : r[i];
            const double rn = rp - dv[i] * q;
            const double dd = c1[k] * d[i] + c2[k] * rn;
            if (k == 1) u[i] = from_zero ? d[i] + dd : (u[i] + d[i]) + dd;
            else u[i] = u[i] + dd;
            r[i] = rn;
            dn[i] = dd;
        }
        memcpy(d, dn, sizeof(double) * n);
    }
}

static void mg(const or_hierarchy *H, or_work *W, int l, int smoother,
               double omega)
{
    const or_level *A = &H->lv[l];
    int n = A->n;
    double *u = W[l].u, *f = W[l].f, *s = W[l].s, *r = W[l].r;
    if (l == H->nlevels - 1) {
        /* diagonal_solver (amg.h:1074-1097) */
        for (int i = 0; i < n; i++) u[i] = A->dinv[i] * f[i];
        return;
    }
    /* smoother 10+g: GS on levels >= g; 100+10g+t: GS on levels [g, t) */
    const int gs_from = smoother >= 100 ? (smoother / 10) % 10
                        : smoother >= 10 ? smoother - 10 : 1 << 30;
    const int gs_to = smoother >= 100 ? smoother % 10 : 1 << 30;
    const int use_gs = l >= gs_from && l < gs_to && smoother < 200;
    /* smoother 200+10c+K: Chebyshev of degree K on levels >= c, l1-Jacobi
     * below */
    const int use_cheb = smoother >= 200 && smoother < 300 && l >= (smoother / 10) % 10;
    const int cheb_k = smoother % 10;
    double *cd = NULL, *cdn = NULL;
    if (use_cheb) {
        cd = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
        cdn = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
    }
    if (use_cheb) {
        double ith, c1[10], c2[10];
        cheb_coeffs(cheb_k, &ith, c1, c2);
        for (int i = 0; i < n; i++) cd[i] = ith * f[i] * A->dl1inv[i];
        cheb_steps(A, cheb_k, 1, f, u, r, cd, cdn);
        long m = 0;
        for (int i = 0; i < n; i++) {
            double t = f[i];
            for (int j = 0; j < A->cnt[i]; j++, m++) t -= A->ele[m] * u[A->col[m]];
            r[i] = t;
        }
    } else if (use_gs) {
        /* multicolour Gauss-Seidel, forward over colours from zero, then the
         * residual (the GPU smoother on coarse levels; no reference
         * counterpart -- the reference's own GS is lexicographic) */
        for (int i = 0; i < n; i++) u[i] = 0.0;
        for (int c = 0; c < A->ncolors; c++) gs_colour(A, c, f, u);
        long m = 0;
        for (int i = 0; i < n; i++) {
            r[i] = f[i] - row_dot8(A, m, A->cnt[i], u);
            m += A->cnt[i];
        }
    } else if (smoother == 0) {
        /* gauss_seidel_f 3-arg (amg.h:759-784) */
        for (int i = 0; i < n; i++) r[i] = f[i];
        long m = 0;
        for (int i = 0; i < n; i++) {
            double t = A->dinv[i] * r[i];
            u[i] = t;
            for (int j = 0; j < A->cnt[i]; j++, m++) r[A->col[m]] -= A->ele[m] * t;
        }
    } else {
        /* device_jacobi 3-arg (device_amg.h:35-42): u = w D^-1 f; r = f - A u */
        const double *dv = smoother != 1 ? A->dl1inv : A->dinv;
        for (int i = 0; i < n; i++) u[i] = omega * f[i] * dv[i];
        long m = 0;
        for (int i = 0; i < n; i++) {
            double t = f[i];
            for (int j = 0; j < A->cnt[i]; j++, m++) t -= A->ele[m] * u[A->col[m]];
            r[i] = t;
        }
    }
    restrict_simple(A, H->lv[l + 1].n, r, W[l + 1].f);
    mg(H, W, l + 1, smoother, omega);
    prolong_simple(A, W[l + 1].u, s);
    if (use_cheb) {
        double ith, c1[10], c2[10];
        cheb_coeffs(cheb_k, &ith, c1, c2);
        for (int i = 0; i < n; i++) u[i] += s[i];
        long m = 0;
        for (int i = 0; i < n; i++) {
            double t = f[i];
            for (int j = 0; j < A->cnt[i]; j++, m++) t -= A->ele[m] * u[A->col[m]];
            r[i] = A->dl1inv[i] * t;
            cd[i] = ith * t * A->dl1inv[i];
        }
        cheb_steps(A, cheb_k, 0, f, u, r, cd, cdn);
        free(cd);
        free(cdn);
    } else if (use_gs) {
        for (int i = 0; i < n; i++) u[i] += s[i];
        for (int c = A->ncolors - 1; c >= 0; c--) gs_colour(A, c, f, u);
    } else if (smoother == 0) {
        /* gauss_seidel_b 3-arg (amg.h:930-961) */
        for (int i = 0; i < n; i++) u[i] += s[i];
        long m = A->nnz;
        for (int i = n - 1; i >= 0; i--) {
            double t = f[i];
            for (int j = 0; j < A->cnt[i]; j++) {
                m--;
                t -= A->ele[m] * u[A->col[m]];
            }
            u[i] += t * A->dinv[i];
        }
    } else {
        /* add, then device_jacobi 2-arg (device_amg.h:27-34, 411-412) */
        for (int i = 0; i < n; i++) u[i] += s[i];
        long m = 0;
        for (int i = 0; i < n; i++) {
            double t = f[i];
            for (int j = 0; j < A->cnt[i]; j++, m++) t -= A->ele[m] * u[A->col[m]];
            r[i] = t;
        }
        const double *dv = smoother != 1 ? A->dl1inv : A->dinv;
        for (int i = 0; i < n; i++) u[i] += omega * r[i] * dv[i];
    }
}

static or_work *work_alloc(const or_hierarchy *H)
{
    or_work *W = (or_work *)calloc(H->nlevels, sizeof(or_work));
    for (int l = 0; l < H->nlevels; l++) {
        int n = H->lv[l].n > 0 ? H->lv[l].n : 1;
        W[l].u = (double *)calloc(n, sizeof(double));
        W[l].f = (double *)calloc(n, sizeof(double));
        W[l].s = (double *)calloc(n, sizeof(double));
        W[l].r = (double *)calloc(n, sizeof(double));
    }
    return W;
}

static void work_free(const or_hierarchy *H, or_work *W)
{
    for (int l = 0; l < H->nlevels; l++) {
        free(W[l].u); free(W[l].f); free(W[l].s); free(W[l].r);
    }
    free(W);
}

void or_vcycle(const or_hierarchy *H, int smoother, double omega,
               const double *f, double *u)
{
    or_work *W = work_alloc(H);
    memcpy(W[0].f, f, sizeof(double) * H->lv[0].n);
    mg(H, W, 0, smoother, omega);
    memcpy(u, W[0].u, sizeof(double) * H->lv[0].n);
    work_free(H, W);
}

static double dot(int n, const double *x, const double *y)
{
    double s = 0.0;
    for (int i = 0; i < n; i++) s += x[i] * y[i];
    return s;
}

static double true_relres(const or_level *A, const double *b, const double *x,
                          double *tmp)
{
    or_spmv(A->n, A->cnt, A->col, A->ele, x, tmp);
    double rr = 0.0, bb = 0.0;
    for (int i = 0; i < A->n; i++) {
        double d = b[i] - tmp[i];
        rr += d * d;
        bb += b[i] * b[i];
    }
    return bb > 0 ? sqrt(rr / bb) : sqrt(rr);
}

/* conjugate_gradient::operator() (pcg.h:33-76) */
int or_pcg(const or_hierarchy *H, int smoother, double omega, const double *b,
           double *x, double eps, int max_it, int stop, double *relres)
{
    const or_level *A = &H->lv[0];
    int n = A->n;
    or_work *W = work_alloc(H);
    double *r = (double *)malloc(sizeof(double) * n);
    double *s = (double *)malloc(sizeof(double) * n);
    double *v = (double *)malloc(sizeof(double) * n);
    double *tmp = (double *)malloc(sizeof(double) * n);
    memcpy(r, b, sizeof(double) * n);
    memcpy(s, x, sizeof(double) * n);
    or_spmv(n, A->cnt, A->col, A->ele, s, v);
    for (int i = 0; i < n; i++) r[i] -= v[i] * 1.0;
#define PREC(rin, vout)                                                      \
    do {                                                                     \
        memcpy(W[0].f, rin, sizeof(double) * n);                             \
        mg(H, W, 0, smoother, omega);                                        \
        memcpy(vout, W[0].u, sizeof(double) * n);                            \
    } while (0)
    PREC(r, v);
    double sigma = dot(n, v, r);
    if (sigma < 0.0) sigma = fabs(sigma);
    for (int i = 0; i < n; i++) s[i] = s[i] * 0.0 + v[i];
    double sigma_last = sigma, sigma_first = sigma;
    if (sigma == 0.0) sigma_first = 1.0;
    double tau = sigma / sigma_first;
    double rel = stop == 1 ? true_relres(A, b, x, tmp) : 0.0;
    int loop = 0;
    while (++loop < max_it &&
           (stop == 1 ? rel > eps : tau > eps * eps)) {
        or_spmv(n, A->cnt, A->col, A->ele, s, v);
        tau = dot(n, s, v);
        if (tau < 0.0) tau = fabs(tau);
        double alpha = sigma / tau;
        for (int i = 0; i < n; i++) x[i] += s[i] * alpha;
        for (int i = 0; i < n; i++) r[i] -= v[i] * alpha;
        PREC(r, v);
        sigma = dot(n, v, r);
        if (sigma < 0.0) sigma = fabs(sigma);
        double beta = sigma / sigma_last;
        for (int i = 0; i < n; i++) s[i] = s[i] * beta + v[i];
        sigma_last = sigma;
        tau = sigma / sigma_first;
        if (stop == 1) rel = true_relres(A, b, x, tmp);
    }
#undef PREC
    if (relres) *relres = true_relres(A, b, x, tmp);
    free(r); free(s); free(v); free(tmp);
    work_free(H, W);
    return loop;
}

/* compute.cpp:7-51 (epsilon 0, omega 1, 16 levels, min 1 node, GS) */
int or_compute(const int *hdr, const int *cnt, const int *col,
               const double *ele, const double *b, double *x, double eps,
               int stop, int *iters, double *relres)
{
    or_hierarchy H;
    or_amg_setup(hdr[0], cnt, col, ele, 16, 1, 0.0, &H);
    int it = or_pcg(&H, 0, 1.0, b, x, eps, 10000, stop, relres);
    if (iters) *iters = it;
    or_amg_free(&H);
    return 0;
}

/* flux_reconstruction.c:9-319 */
void or_fluxes(int nx, int ny, int nz, double hx, double hy, double hz,
               const double *p, const or_ele *perm, const or_bound *B,
               const int bc_type[6], or_ele *v, double *divmin,
               double *divmax)
{
    const int nxy = nx * ny;
    int i, j, k, s;
    for (k = 0; k < nz; k++)
        for (j = 0; j < ny; j++)
            for (i = 0; i < nx; i++) {
                s = IDX(i, j, k);
                if (j < ny - 1) v[s].u = hy * perm[s].u * (p[s] - p[s + nx]);
                if (i < nx - 1) v[s].r = hx * perm[s].r * (p[s] - p[s + 1]);
                if (j > 0) v[s].d = hy * perm[s].d * (p[s] - p[s - nx]);
                if (i > 0) v[s].l = hx * perm[s].l * (p[s] - p[s - 1]);
                if (k < nz - 1) v[s].t = hz * perm[s].t * (p[s] - p[s + nxy]);
                if (k > 0) v[s].b = hz * perm[s].b * (p[s] - p[s - nxy]);
            }
    for (j = 0; j < ny; j++)
        for (k = 0; k < nz; k++) {
            int l = k * ny + j;
            s = IDX(0, j, k);
            v[s].l = bc_type[0] == 0 ? hx * perm[s].l * (p[s] - B->l[l]) : -B->l[l];
            s = IDX(nx - 1, j, k);
            v[s].r = bc_type[1] == 0 ? hx * perm[s].r * (p[s] - B->r[l]) : B->r[l];
        }
    for (i = 0; i < nx; i++)
        for (k = 0; k < nz; k++) {
            int l = k * nx + i;
            s = IDX(i, 0, k);
            v[s].d = bc_type[3] == 0 ? hy * perm[s].d * (p[s] - B->d[l]) : -B->d[l];
            s = IDX(i, ny - 1, k);
            v[s].u = bc_type[2] == 0 ? hy * perm[s].u * (p[s] - B->u[l]) : B->u[l];
        }
    for (i = 0; i < nx; i++)
        for (j = 0; j < ny; j++) {
            int l = j * nx + i;
            s = IDX(i, j, nz - 1);
            v[s].t = bc_type[4] == 0 ? hz * perm[s].t * (p[s] - B->t[l]) : B->t[l];
            s = IDX(i, j, 0);
            v[s].b = bc_type[5] == 0 ? hz * perm[s].b * (p[s] - B->b[l]) : -B->b[l];
        }
    /* divvel_pontual (flux_reconstruction.c:281-319) */
    double mx = 0.0, mn = 100.0;
    for (s = 0; s < nx * ny * nz; s++) {
        double dv = v[s].r / hx + v[s].l / hx + v[s].d / hy + v[s].u / hy +
                    v[s].b / hz + v[s].t / hz;
        if (fabs(dv) > mx) mx = fabs(dv);
        if (fabs(dv) < mn) mn = fabs(dv);
    }
    if (divmin) *divmin = mn;
    if (divmax) *divmax = mx;
}

/* ==== the coupled conduit model ========================================== */

/* main.c:416-448: element i of conduit j steps along its axis from
 * (sxi, syi, szi). */
int or_karst_cell(const or_karst *K, int j, int i, int nx, int ny)
{
    int x = K->sxi[j], y = K->syi[j], z = K->szi[j];
    if (K->pos[j] == 1) x += i;
    else if (K->pos[j] == 2) y += i;
    else z += i;
    return x + y * nx + z * nx * ny;
}

int or_karst_check(const or_karst *K, int nx, int ny, int nz)
{
    for (int j = 0; j < K->nk; j++) {
        int m = K->len[j], p = K->pos[j];
        int x = K->sxi[j], y = K->syi[j], z = K->szi[j];
        if (p < 1 || p > 3 || m < 1) return -1;
        int n_ax = p == 1 ? nx : p == 2 ? ny : nz;
        int a0 = p == 1 ? x : p == 2 ? y : z;
        if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) return -1;
        if (a0 + m > n_ax) return -1;
        for (int f = 0; f < 2; f++) {
            int bt = f ? K->bound_r[j] : K->bound_l[j];
            if (bt != 0 && bt != 1 && bt != 3) return -1;
            if (bt != 3) continue;
            if (f == 0 && a0 < 1) return -1;
            if (f == 1 && (a0 + m >= n_ax || p == 3)) return -1;
        }
        if (K->n_brechas[j] < 0 || K->n_brechas[j] > K->max_brechas) return -1;
        for (int b = 0; b < K->n_brechas[j]; b++) {
            int s = K->brechas[b * K->nk + j];
            if (s < 0 || s + 1 >= m) return -1;
        }
    }
    return 0;
}

#define KM(a, i, j) ((a)[(i) * nk + (j)])

/* permeabilities.c:795-867 */
void or_karst_keff(const or_karst *K, const or_kgrid *G, or_kstate *S, int j)
{
    const int nk = K->nk, m = K->len[j];
    const double hs = K->pos[j] == 1 ? G->hx : K->pos[j] == 2 ? G->hy : G->hz;
    const double ks = K->Kc[j], visc = G->visc;
    int i;
    for (i = 0; i < m - 1; i++) {
        KM(S->kr, i, j) = or_hm(ks, ks);
        KM(S->kr, i, j) = KM(S->kr, i, j) / (hs * hs * visc);
    }
    for (i = 1; i < m; i++) {
        KM(S->kl, i, j) = or_hm(ks, ks);
        KM(S->kl, i, j) = KM(S->kl, i, j) / (hs * hs * visc);
    }
    if (K->bound_l[j] == 0) KM(S->kl, 0, j) = 2 * (ks) / (hs * hs * visc);
    if (K->bound_l[j] == 1) KM(S->kl, 0, j) = 0;
    if (K->bound_l[j] == 3) KM(S->kl, 0, j) = 2 * ks / (visc * hs * hs);
    if (K->bound_r[j] == 0) KM(S->kr, m - 1, j) = 2 * (ks) / (hs * hs * visc);
    if (K->bound_r[j] == 1) KM(S->kr, m - 1, j) = 0;
    if (K->bound_r[j] == 3) KM(S->kr, m - 1, j) = 2 * ks / (visc * hs * hs);
    for (i = 0; i < m; i++)
        KM(S->kc, i, j) = KM(S->kl, i, j) + KM(S->kr, i, j) + KM(S->kic, i, j) / visc;
}

/* The nonlinear Robin end term of set_source_term.c:298-404 and
 * flux_reconstruction.c:398-486: the reservoir flux u through the face
 * between the cell beyond the end (s) and the end cell (saux), and the
 * K-weighted mean pressure lm of the two. */
static void robin_end(const or_karst *K, const or_kgrid *G, int j, int right,
                      double *u, double *lm)
{
    const int nx = G->nx, ny = G->ny, nxy = nx * ny, m = K->len[j];
    int x = K->sxi[j], y = K->syi[j], z = K->szi[j], s, saux;
    const double *p = G->p_old;
    const double *KK;
    double face, hh;
    if (K->pos[j] == 1) {
        s = right ? IDX(x + m, y, z) : IDX(x - 1, y, z);
        saux = right ? IDX(x + m - 1, y, z) : IDX(x, y, z);
        face = right ? G->perm[s].l : G->perm[s].r;
        KK = G->KX; hh = G->hx;
    } else if (K->pos[j] == 2) {
        s = right ? IDX(x, y + m, z) : IDX(x, y - 1, z);
        saux = right ? IDX(x, y + m - 1, z) : IDX(x, y, z);
        face = right ? G->perm[s].d : G->perm[s].u;
        KK = G->KY; hh = G->hy;
    } else {
        s = right ? IDX(x, y, z + m) : IDX(x, y, z - 1);
        saux = right ? IDX(x, y, z + m - 1) : IDX(x, y, z);
        face = right ? G->perm[s].b : G->perm[s].t;
        KK = G->KZ; hh = G->hz;
    }
    (void)ny;
    *u = hh * face * (p[s] - p[saux]);
    *lm = (KK[s] * p[s] + KK[saux] * p[saux]) / (KK[s] + KK[saux]);
}

/* set_source_term.c:256-414 */
void or_source_term1d(const or_karst *K, const or_kgrid *G, or_kstate *S,
                      int j, double *f)
{
    const int nk = K->nk, m = K->len[j];
    const double hs = K->pos[j] == 1 ? G->hx : K->pos[j] == 2 ? G->hy : G->hz;
    const double visc = G->visc, rho = G->rho, ks = K->Kc[j];
    int i;
    for (i = 0; i < m; i++)
        f[i] = (KM(S->kic, i, j) * KM(S->paux, i, j)) / visc;
    /* fractures (set_source_term.c:272-295) */
    for (i = 0; i < K->n_brechas[j]; i++) {
        int s = K->brechas[i * nk + j];
        double cR = or_hm(ks, ks), R;
        double *ucr = &S->ucR[i * nk + j], *ucl = &S->ucL[i * nk + j];
        double cb = K->cb[i * nk + j], be = K->beta[i * nk + j];
        if (*ucr < 0) R = -cb * be;
        else R = cb * be;
        double uR = (cR / (visc * hs)) *
                    (KM(S->pc_old, s, j) - KM(S->pc_old, s + 1, j) - rho * *ucr * *ucr * R);
        double uL = (cR / (visc * hs)) *
                    (KM(S->pc_old, s + 1, j) - KM(S->pc_old, s, j) + rho * *ucl * *ucl * R);
        *ucr = uR;
        *ucl = uL;
        f[s] = f[s] + (cR / (visc * hs)) * (rho * uR * uR * R);
        f[s + 1] = f[s + 1] - (cR / (visc * hs)) * (rho * uL * uL * R);
    }
    const double c0 = K->cont[j], c1 = K->cont[nk + j];
    /* left end (set_source_term.c:302-366) */
    if (K->bound_l[j] == 0) f[0] = f[0] + (KM(S->kl, 0, j)) * c0;
    if (K->bound_l[j] == 1) f[0] = f[0] + c0 / (hs);
    if (K->bound_l[j] == 3) {
        double u, lm, c;
        robin_end(K, G, j, 0, &u, &lm);
        if (u < 0) c = -K->ccont[j] * (c0 - 1);
        else c = K->ccont[j] * (c0 - 1);
        double font = -lm + rho * u * u * c;
        f[0] = f[0] - 2 * ks / (visc * hs * hs) * font;
    }
    /* right end (set_source_term.c:368-410) */
    if (K->bound_r[j] == 0) f[m - 1] = f[m - 1] + KM(S->kr, m - 1, j) * c1;
    if (K->bound_r[j] == 1) f[m - 1] = f[m - 1] - c1 / (hs);
    if (K->bound_r[j] == 3) {
        double u, lm, c;
        robin_end(K, G, j, 1, &u, &lm);
        if (u < 0) c = -K->ccont[nk + j] * (c1 - 1);
        else c = K->ccont[nk + j] * (c1 - 1);
        double font = -lm + rho * u * u * c;
        f[m - 1] = f[m - 1] - font * 2 * ks / (visc * hs * hs);
    }
}

void or_thomas(int m, const double *kl, const double *kc, const double *kr,
               int stride, const double *f, double *x)
{
    /* forward sweep: q[i] = r[i] / w[i] kept in x[], g[i] in a scratch;
     * w[i] = c[i] - l[i] q[i-1], g[i] = (f[i] + l[i] g[i-1]) / w[i] */
    double *g = (double *)malloc(sizeof(double) * (m > 0 ? m : 1));
    double w = kc[0];
    g[0] = f[0] / w;
    for (int i = 1; i < m; i++) {
        double q = kr[(i - 1) * stride] / w;
        x[i - 1] = q;
        double l = kl[i * stride];
        w = kc[i * stride] - l * q;
        g[i] = (f[i] + l * g[i - 1]) / w;
    }
    /* back substitution: x[i] = g[i] + q[i] x[i+1] */
    double nxt = g[m - 1];
    x[m - 1] = nxt;
    for (int i = m - 2; i >= 0; i--) {
        nxt = g[i] + x[i] * nxt;
        x[i] = nxt;
    }
    free(g);
}

/* solve_linearsystem_AMG.c:200-294: the conduit system in count/col/ele
 * form (l, c, r per row) handed to compute(). */
static void conduit_compute(const or_karst *K, const or_kstate *S, int j,
                            const double *f, double *x)
{
    const int nk = K->nk, m = K->len[j];
    int *cnt = (int *)malloc(sizeof(int) * m);
    int *col = (int *)malloc(sizeof(int) * 3 * m);
    double *ele = (double *)malloc(sizeof(double) * 3 * m);
    int l = 0;
    for (int s = 0; s < m; s++) {
        cnt[s] = 1 + (s > 0) + (s < m - 1);
        if (s > 0) { col[l] = s - 1; ele[l] = -KM(S->kl, s, j); l++; }
        col[l] = s; ele[l] = KM(S->kc, s, j); l++;
        if (s < m - 1) { col[l] = s + 1; ele[l] = -KM(S->kr, s, j); l++; }
    }
    int hdr[2] = {m, l};
    for (int s = 0; s < m; s++) x[s] = 0.0;
    or_compute(hdr, cnt, col, ele, f, x, 1e-8, 0, NULL, NULL);
    free(cnt); free(col); free(ele);
}

/* karst.c:8-40 */
void or_conduit(const or_karst *K, const or_kgrid *G, or_kstate *S,
                int solver)
{
    const int nk = K->nk;
    double *f = (double *)malloc(sizeof(double) * (S->mmax + 1));
    double *x = (double *)malloc(sizeof(double) * (S->mmax + 1));
    for (int j = 0; j < nk; j++) {
        const int m = K->len[j];
        or_karst_keff(K, G, S, j);
        or_source_term1d(K, G, S, j, f);
        if (solver == 1) conduit_compute(K, S, j, f, x);
        else or_thomas(m, &S->kl[j], &S->kc[j], &S->kr[j], nk, f, x);
        for (int i = 0; i < m; i++) KM(S->pc, i, j) = x[i];
    }
    free(f);
    free(x);
}

/* flux_reconstruction.c:322-496 */
void or_fluxo1d(const or_karst *K, const or_kgrid *G, const or_kstate *S,
                double *ucl, double *ucr)
{
    const int nk = K->nk;
    const double visc = G->visc, rho = G->rho;
    for (int j = 0; j < nk; j++) {
        const int m = K->len[j];
        const double hs = K->pos[j] == 1 ? G->hx : K->pos[j] == 2 ? G->hy : G->hz;
        const double ks = K->Kc[j];
        const double *x = S->pc;
        int i;
        for (i = 0; i < m - 1; i++)
            KM(ucr, i, j) = hs * KM(S->kr, i, j) * (KM(x, i, j) - KM(x, i + 1, j));
        for (i = 1; i < m; i++)
            KM(ucl, i, j) = hs * KM(S->kl, i, j) * (KM(x, i, j) - KM(x, i - 1, j));
        for (i = 0; i < K->n_brechas[j]; i++) {
            double c, cb = K->cb[i * nk + j], be = K->beta[i * nk + j];
            double ur = S->ucR[i * nk + j], ul = S->ucL[i * nk + j];
            if (ur < 0) c = -cb * be;
            else c = cb * be;
            int s = K->brechas[i * nk + j];
            double cR = or_hm(ks, ks);
            KM(ucr, s, j) = (cR / (visc * hs)) *
                            (KM(x, s, j) - KM(x, s + 1, j) - 0.5 * rho * ur * ur * c);
            KM(ucl, s + 1, j) = (cR / (visc * hs)) *
                                (KM(x, s + 1, j) - KM(x, s, j) + 0.5 * rho * ul * ul * c);
        }
        const double c0 = K->cont[j], c1 = K->cont[nk + j];
        if (K->bound_l[j] == 0) KM(ucl, 0, j) = hs * KM(S->kl, 0, j) * (KM(x, 0, j) - c0);
        /* the Neumann left end takes cont_karst[1] (flux_reconstruction.c:372-376) */
        if (K->bound_l[j] == 1) KM(ucl, 0, j) = -c1;
        if (K->bound_l[j] == 3) {
            double u, lm, c;
            robin_end(K, G, j, 0, &u, &lm);
            if (u < 0) c = -K->ccont[j] * (c0 - 1);
            else c = K->ccont[j] * (c0 - 1);
            KM(ucl, 0, j) = (2 * ks) / (visc * hs) * (KM(x, 0, j) - lm + rho * u * u * c);
        }
        if (K->bound_r[j] == 0)
            KM(ucr, m - 1, j) = hs * KM(S->kr, m - 1, j) * (KM(x, m - 1, j) - c1);
        if (K->bound_r[j] == 1) KM(ucr, m - 1, j) = c1;
        if (K->bound_r[j] == 3) {
            double u, lm, c;
            robin_end(K, G, j, 1, &u, &lm);
            if (u < 0) c = -K->ccont[nk + j] * (c1 - 1);
            else c = K->ccont[nk + j] * (c1 - 1);
            KM(ucr, m - 1, j) = (2 * ks) / (visc * hs) * (KM(x, m - 1, j) - lm + rho * u * u * c);
        }
    }
}

/* main.c:102-113 (erro_relativo) */
static double rel_change(int n, const double *y, const double *y_old)
{
    double s1 = 0, s2 = 0;
    for (int i = 0; i < n; i++) {
        s1 = s1 + (y[i] - y_old[i]) * (y[i] - y_old[i]);
        s2 = s2 + y[i] * y[i];
    }
    return sqrt(s1) / sqrt(s2);
}

/* reservoir.c:8-57 with the hierarchy kept: the matrix of the coupled
 * system does not change between Picard iterations, only pc_aux in the
 * right-hand side (set_source_term.c:206-220). */
static void reservoir_rhs(const or_karst *K, int nx, int ny, int nz, double hx,
                          double hy, double hz, double visc, const or_bound *B,
                          const int bc[6], const or_ele *perm, const double *KI,
                          const double *WI, const double *pw,
                          const double *pc_old, double *pcaux, double *b)
{
    const int n = nx * ny * nz, nk = K->nk;
    for (int s = 0; s < n; s++) pcaux[s] = 0.0;
    for (int j = 0; j < nk; j++)
        for (int i = 0; i < K->len[j]; i++)
            pcaux[or_karst_cell(K, j, i, nx, ny)] = KM(pc_old, i, j);
    for (int s = 0; s < n; s++) b[s] = 0.0;
    or_source_term(nx, ny, nz, hx, hy, hz, visc, B, bc, perm, KI, WI, pcaux,
                   pw, b);
}

int or_picard(const or_karst *K, int nx, int ny, int nz, double hx, double hy,
              double hz, double visc, double rho, const double *KX,
              const double *KY, const double *KZ, const int bc_type[6],
              const double val6[6], const double *WI, const double *pw,
              double tol, int iter_max, double solve_eps, int solve_stop,
              int conduit_solver, double *p, double *pc, double *ucl,
              double *ucr, or_ele *v, double *out, double *qk)
{
    if (or_karst_check(K, nx, ny, nz) != 0) return -1;
    const int n = nx * ny * nz, nk = K->nk;
    int mmax = 0;
    for (int j = 0; j < nk; j++) if (K->len[j] > mmax) mmax = K->len[j];
    const long mm = (long)mmax * nk;
    const long bb = (long)(K->max_brechas > 0 ? K->max_brechas : 1) * nk;
    or_kstate S;
    S.mmax = mmax;
    S.kl = (double *)calloc(mm, sizeof(double));
    S.kr = (double *)calloc(mm, sizeof(double));
    S.kc = (double *)calloc(mm, sizeof(double));
    S.kic = (double *)calloc(mm, sizeof(double));
    S.paux = (double *)calloc(mm, sizeof(double));
    S.pc = pc;
    S.pc_old = (double *)calloc(mm, sizeof(double));
    S.ucR = (double *)calloc(bb, sizeof(double));
    S.ucL = (double *)calloc(bb, sizeof(double));
    for (long q = 0; q < mm; q++) pc[q] = 0.0;
    /* constant boundary values (main.c:140-152, set_boundaries.c) */
    double *fv[6];
    const long fsz[6] = {(long)ny * nz, (long)ny * nz, (long)nx * nz,
                         (long)nx * nz, (long)nx * ny, (long)nx * ny};
    for (int f = 0; f < 6; f++) {
        fv[f] = (double *)malloc(sizeof(double) * fsz[f]);
        for (long q = 0; q < fsz[f]; q++) fv[f][q] = val6[f];
    }
    or_bound B = {fv[0], fv[1], fv[2], fv[3], fv[4], fv[5]};
    or_ele *perm = (or_ele *)calloc(n, sizeof(or_ele));
    or_ind *ind = (or_ind *)malloc(sizeof(or_ind) * n);
    double *b = (double *)malloc(sizeof(double) * n);
    double *pcaux = (double *)malloc(sizeof(double) * n);
    double *p_old = (double *)malloc(sizeof(double) * n);
    double *KI = (double *)calloc(n, sizeof(double));
    int *cnt = (int *)malloc(sizeof(int) * n);
    int *col = (int *)malloc(sizeof(int) * 7L * n);
    double *ele = (double *)malloc(sizeof(double) * 7L * n);
    or_hierarchy H;
    double rr;

    /* first reservoir solve: no well, no conduit exchange (main.c:393) */
    or_assemble(nx, ny, nz, hx, hy, hz, visc, KX, KY, KZ, bc_type, NULL, NULL,
                perm, ind);
    reservoir_rhs(K, nx, ny, nz, hx, hy, hz, visc, &B, bc_type, perm, NULL,
                  NULL, pw, S.pc_old, pcaux, b);
    or_pack_csr(n, perm, ind, cnt, col, ele);
    for (int s = 0; s < n; s++) p[s] = 0.0;
    or_amg_setup(n, cnt, col, ele, 16, 1, 0.0, &H);
    or_pcg(&H, 0, 1.0, b, p, solve_eps, 10000, solve_stop, &rr);
    or_amg_free(&H);
    memcpy(p_old, p, sizeof(double) * n);

    /* karst index, KI_c, p_aux (main.c:410-449) */
    for (int j = 0; j < nk; j++) {
        const double hs = K->pos[j] == 1 ? hx : K->pos[j] == 2 ? hy : hz;
        for (int i = 0; i < K->len[j]; i++) {
            int c = or_karst_cell(K, j, i, nx, ny);
            KI[c] = K->kindex[j];
            KM(S.kic, i, j) = K->kindex[j] / (K->area[j] * hs);
            KM(S.paux, i, j) = p_old[c];
        }
    }
    /* the coupled matrix (reservoir.c:51 with KI and WI) */
    or_assemble(nx, ny, nz, hx, hy, hz, visc, KX, KY, KZ, bc_type, KI, WI,
                perm, ind);
    or_pack_csr(n, perm, ind, cnt, col, ele);
    or_amg_setup(n, cnt, col, ele, 16, 1, 0.0, &H);
    or_kgrid G = {nx, ny, nz, hx, hy, hz, visc, rho, KX, KY, KZ, perm, p_old};
    /* conduit() before the loop (main.c:452) reads the matrix faces of the
     * first (uncoupled) call, which equal the coupled ones: KI and WI only
     * enter the centre */
    or_conduit(K, &G, &S, conduit_solver);

    double error = 1.0;
    int iter = 0;
    while (iter < iter_max && error > tol) {
        memcpy(S.pc_old, pc, sizeof(double) * mm);
        reservoir_rhs(K, nx, ny, nz, hx, hy, hz, visc, &B, bc_type, perm, KI,
                      WI, pw, S.pc_old, pcaux, b);
        or_pcg(&H, 0, 1.0, b, p, solve_eps, 10000, solve_stop, &rr);
        /* main.c:480-486 keeps the last entry, the reservoir change */
        error = rel_change(n, p, p_old);
        memcpy(p_old, p, sizeof(double) * n);
        for (int j = 0; j < nk; j++)
            for (int i = 0; i < K->len[j]; i++)
                KM(S.paux, i, j) = p_old[or_karst_cell(K, j, i, nx, ny)];
        or_conduit(K, &G, &S, conduit_solver);
        iter++;
    }
    or_amg_free(&H);

    double *ul = ucl ? ucl : (double *)calloc(mm, sizeof(double));
    double *ur = ucr ? ucr : (double *)calloc(mm, sizeof(double));
    for (long q = 0; q < mm; q++) { ul[q] = 0.0; ur[q] = 0.0; }
    or_fluxo1d(K, &G, &S, ul, ur);
    if (v) or_fluxes(nx, ny, nz, hx, hy, hz, p, perm, &B, bc_type, v, NULL, NULL);
    /* balances (main.c:523-529, 566-593) */
    if (out) {
        double Q = 0.0, pm = 0.0;
        for (int s = 0; s < n; s++) {
            double wi = WI ? WI[s] : 0.0, pws = pw ? pw[s] : 0.0;
            Q = Q + (wi / visc) * (pws - p[s]);
            pm = pm + p[s];
        }
        out[0] = error;
        out[1] = Q;
        out[2] = pm / n;
    }
    if (qk)
        for (int j = 0; j < nk; j++) {
            const double hs = K->pos[j] == 1 ? hx : K->pos[j] == 2 ? hy : hz;
            double qc = 0.0, q3 = 0.0;
            for (int i = 0; i < K->len[j]; i++) {
                int c = or_karst_cell(K, j, i, nx, ny);
                qc = qc + (-KI[c] / visc) * (KM(pc, i, j) - p[c]) * hs;
                q3 = q3 + (KI[c] / visc) * (KM(pc, i, j) - p[c]);
            }
            qk[j] = qc;
            qk[nk + j] = q3;
            qk[2 * nk + j] = KM(ul, 0, j) * K->area[j] + KM(ur, K->len[j] - 1, j) * K->area[j];
        }
    if (!ucl) free(ul);
    if (!ucr) free(ur);
    for (int f = 0; f < 6; f++) free(fv[f]);
    free(S.kl); free(S.kr); free(S.kc); free(S.kic); free(S.paux);
    free(S.pc_old); free(S.ucR); free(S.ucL);
    free(perm); free(ind); free(b); free(pcaux); free(p_old); free(KI);
    free(cnt); free(col); free(ele);
    return iter;
}
#undef KM
