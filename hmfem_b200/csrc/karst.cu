// karst.cu -- the coupled reservoir / karst-conduit model on the device:
// conduit sets (main.c:197-280), the batched conduit solve of karst.c:8-40
// (permeabilidade_karst, source_term1d, the tridiagonal solve), the conduit
// fluxes (fluxo1d) and the Picard driver of main.c:383-489.
//
// A conduit system is a few hundred unknowns at most and the reference has
// at most a few dozen conduits, so each conduit is one thread running the
// reference's operations in order; what the GPU buys is that the whole
// coupled loop stays on the device next to the 3-D solve.  Every conduit
// expression keeps the reference's operand order and rounding (__dmul_rn /
// __dadd_rn / __dsub_rn / __ddiv_rn, no FMA contraction), so keff, the
// source terms, the Thomas solve and the fluxes are bit-identical to a C
// evaluation of the same expressions.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <unordered_map>
#include <vector>

#include "solver.cuh"
#include "../../include/hmfem_karst.h"

namespace hm {

namespace {

__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// hm(), permeabilities.c:188-193: 2*a*b/(a+b)
__device__ __forceinline__ double hmean(double a, double b)
{
    return ddiv(dmul(dmul(2.0, a), b), dadd(a, b));
}

// Device view of a conduit set.  Per conduit j: elements off[j] ..
// off[j] + len[j] - 1 of the element arrays, fractures boff[j] ..
// boff[j] + nb[j] - 1 of the fracture arrays.
struct KDev {
    int nk;
    const int *len, *off, *pos, *cell0, *step, *bl, *br, *nb, *boff;
    const int *rob;     // 4 per conduit: (s, saux) beyond the left end, (s, saux) beyond the right
    const int *bel;     // fracture -> element within its conduit
    const int *ecell;   // element -> reservoir cell
    const int *econd;   // element -> conduit
    const double *hs, *Kc, *kic, *kidx, *area, *cont, *ccont;  // cont/ccont: [f*nk + j]
    const double *beta, *cb;
    double *ucR, *ucL;                                 // fracture velocities
    double *kl, *kr, *kc, *pc, *pc_old, *g, *q;        // per element
    double *ucl, *ucr;                                 // conduit fluxes per element
};

struct Axis {
    const double *KX, *KY, *KZ;
    double hx, hy, hz;
};

// permeabilities.c:795-867 for every conduit (one thread each)
__global__ void k_karst_keff(KDev d, double visc)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= d.nk) return;
    const int m = d.len[j], o = d.off[j];
    const double hs = d.hs[j], ks = d.Kc[j];
    const double inner = ddiv(hmean(ks, ks), dmul(dmul(hs, hs), visc));
    for (int i = 0; i < m - 1; i++) d.kr[o + i] = inner;
    for (int i = 1; i < m; i++) d.kl[o + i] = inner;
    const double dir = ddiv(dmul(2.0, ks), dmul(dmul(hs, hs), visc));   // 2*(S)/(hs*hs*mu)
    const double rob = ddiv(dmul(2.0, ks), dmul(dmul(visc, hs), hs));   // 2*S/(mu*hs*hs)
    const int bl = d.bl[j], br = d.br[j];
    d.kl[o] = bl == 0 ? dir : (bl == 1 ? 0.0 : rob);
    d.kr[o + m - 1] = br == 0 ? dir : (br == 1 ? 0.0 : rob);
    const double ex = ddiv(d.kic[j], visc);
    for (int i = 0; i < m; i++) d.kc[o + i] = dadd(dadd(d.kl[o + i], d.kr[o + i]), ex);
}

// The nonlinear Robin end (set_source_term.c:298-404, flux_reconstruction.c:
// 398-486): flux u through the face between the reservoir cell beyond the
// end (s) and the end cell (saux), and their K-weighted mean pressure lm.
// The face coefficient is perm[s] of that face, hm(K[s], K[saux]) / (h^2 mu).
__device__ void robin_end(const KDev &d, int j, int right, const double *__restrict__ p,
                          const Axis &ax, double visc, double *u, double *lm)
{
    const int s = d.rob[4 * j + 2 * right], saux = d.rob[4 * j + 2 * right + 1];
    const int pos = d.pos[j];
    const double *KK = pos == 1 ? ax.KX : (pos == 2 ? ax.KY : ax.KZ);
    const double hh = pos == 1 ? ax.hx : (pos == 2 ? ax.hy : ax.hz);
    const double ks = KK[s], ka = KK[saux], ps = p[s], pa = p[saux];
    const double face = ddiv(hmean(ks, ka), dmul(dmul(hh, hh), visc));
    *u = dmul(dmul(hh, face), dsub(ps, pa));
    *lm = ddiv(dadd(dmul(ks, ps), dmul(ka, pa)), dadd(ks, ka));
}

// karst.c:8-40 for every conduit (one thread each): source_term1d
// (set_source_term.c:256-414) into g, then the tridiagonal system of
// solve_linearsystem_AMG.c:200-294 (row i: -kl x[i-1] + kc x[i] - kr x[i+1])
// by the Thomas algorithm into pc.  p is the reservoir pressure p_old.
__global__ void k_conduit(KDev d, const double *__restrict__ p, Axis ax, double visc,
                          double rho)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= d.nk) return;
    const int m = d.len[j], o = d.off[j], c0 = d.cell0[j], st = d.step[j];
    const double hs = d.hs[j], ks = d.Kc[j], kic = d.kic[j];
    double *f = d.g + o;
    for (int i = 0; i < m; i++) f[i] = ddiv(dmul(kic, p[c0 + i * st]), visc);
    // fractures (set_source_term.c:272-295)
    const double cf = ddiv(hmean(ks, ks), dmul(visc, hs));
    for (int b = 0; b < d.nb[j]; b++) {
        const int t = d.boff[j] + b, s = d.bel[t];
        const double ur = d.ucR[t], ul = d.ucL[t];
        const double cbe = dmul(d.cb[t], d.beta[t]);
        const double R = ur < 0 ? -cbe : cbe;
        const double a0 = d.pc_old[o + s], a1 = d.pc_old[o + s + 1];
        const double uR = dmul(cf, dsub(dsub(a0, a1), dmul(dmul(dmul(rho, ur), ur), R)));
        const double uL = dmul(cf, dadd(dsub(a1, a0), dmul(dmul(dmul(rho, ul), ul), R)));
        d.ucR[t] = uR;
        d.ucL[t] = uL;
        f[s] = dadd(f[s], dmul(cf, dmul(dmul(dmul(rho, uR), uR), R)));
        f[s + 1] = dsub(f[s + 1], dmul(cf, dmul(dmul(dmul(rho, uL), uL), R)));
    }
    const int nk = d.nk;
    const double cl = d.cont[j], cr = d.cont[nk + j];
    // left end (set_source_term.c:302-366)
    const int bl = d.bl[j];
    if (bl == 0) f[0] = dadd(f[0], dmul(d.kl[o], cl));
    else if (bl == 1) f[0] = dadd(f[0], ddiv(cl, hs));
    else {
        double u, lm;
        robin_end(d, j, 0, p, ax, visc, &u, &lm);
        const double cv = dmul(d.ccont[j], dsub(cl, 1.0));
        const double c = u < 0 ? -cv : cv;
        const double font = dadd(-lm, dmul(dmul(dmul(rho, u), u), c));
        f[0] = dsub(f[0], dmul(ddiv(dmul(2.0, ks), dmul(dmul(visc, hs), hs)), font));
    }
    // right end (set_source_term.c:368-410)
    const int br = d.br[j];
    if (br == 0) f[m - 1] = dadd(f[m - 1], dmul(d.kr[o + m - 1], cr));
    else if (br == 1) f[m - 1] = dsub(f[m - 1], ddiv(cr, hs));
    else {
        double u, lm;
        robin_end(d, j, 1, p, ax, visc, &u, &lm);
        const double cv = dmul(d.ccont[nk + j], dsub(cr, 1.0));
        const double c = u < 0 ? -cv : cv;
        const double font = dadd(-lm, dmul(dmul(dmul(rho, u), u), c));
        f[m - 1] = dsub(f[m - 1], ddiv(dmul(dmul(font, 2.0), ks), dmul(dmul(visc, hs), hs)));
    }
    // Thomas: forward elimination in place (f becomes g), q[i] = r[i] / w[i],
    // w[i] = c[i] - l[i] q[i-1], g[i] = (f[i] + l[i] g[i-1]) / w[i]; then
    // x[i] = g[i] + q[i] x[i+1]
    const double *kl = d.kl + o, *kc = d.kc + o, *kr = d.kr + o;
    double *q = d.q + o, *x = d.pc + o;
    double w = kc[0];
    f[0] = ddiv(f[0], w);
    for (int i = 1; i < m; i++) {
        const double qi = ddiv(kr[i - 1], w);
        q[i - 1] = qi;
        const double l = kl[i];
        w = dsub(kc[i], dmul(l, qi));
        f[i] = ddiv(dadd(f[i], dmul(l, f[i - 1])), w);
    }
    double nxt = f[m - 1];
    x[m - 1] = nxt;
    for (int i = m - 2; i >= 0; i--) {
        nxt = dadd(f[i], dmul(q[i], nxt));
        x[i] = nxt;
    }
}

// flux_reconstruction.c:322-496 (fluxo1d) for every conduit; p is p_old.
__global__ void k_fluxo1d(KDev d, const double *__restrict__ p, Axis ax, double visc,
                          double rho)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= d.nk) return;
    const int m = d.len[j], o = d.off[j], nk = d.nk;
    const double hs = d.hs[j], ks = d.Kc[j];
    const double *x = d.pc + o;
    double *ucl = d.ucl + o, *ucr = d.ucr + o;
    for (int i = 0; i < m; i++) { ucl[i] = 0.0; ucr[i] = 0.0; }
    for (int i = 0; i < m - 1; i++) ucr[i] = dmul(dmul(hs, d.kr[o + i]), dsub(x[i], x[i + 1]));
    for (int i = 1; i < m; i++) ucl[i] = dmul(dmul(hs, d.kl[o + i]), dsub(x[i], x[i - 1]));
    const double cf = ddiv(hmean(ks, ks), dmul(visc, hs));
    const double hr = dmul(0.5, rho);
    for (int b = 0; b < d.nb[j]; b++) {
        const int t = d.boff[j] + b, s = d.bel[t];
        const double ur = d.ucR[t], ul = d.ucL[t];
        const double cbe = dmul(d.cb[t], d.beta[t]);
        const double c = ur < 0 ? -cbe : cbe;
        ucr[s] = dmul(cf, dsub(dsub(x[s], x[s + 1]), dmul(dmul(dmul(hr, ur), ur), c)));
        ucl[s + 1] = dmul(cf, dadd(dsub(x[s + 1], x[s]), dmul(dmul(dmul(hr, ul), ul), c)));
    }
    const double cl = d.cont[j], cr = d.cont[nk + j];
    const double g2 = ddiv(dmul(2.0, ks), dmul(visc, hs));
    const int bl = d.bl[j], br = d.br[j];
    if (bl == 0) ucl[0] = dmul(dmul(hs, d.kl[o]), dsub(x[0], cl));
    else if (bl == 1) ucl[0] = -cr;   // cont_karst[1], as flux_reconstruction.c:372-376 reads it
    else {
        double u, lm;
        robin_end(d, j, 0, p, ax, visc, &u, &lm);
        const double cv = dmul(d.ccont[j], dsub(cl, 1.0));
        const double c = u < 0 ? -cv : cv;
        ucl[0] = dmul(g2, dadd(dsub(x[0], lm), dmul(dmul(dmul(rho, u), u), c)));
    }
    if (br == 0) ucr[m - 1] = dmul(dmul(hs, d.kr[o + m - 1]), dsub(x[m - 1], cr));
    else if (br == 1) ucr[m - 1] = cr;
    else {
        double u, lm;
        robin_end(d, j, 1, p, ax, visc, &u, &lm);
        const double cv = dmul(d.ccont[nk + j], dsub(cr, 1.0));
        const double c = u < 0 ? -cv : cv;
        ucr[m - 1] = dmul(g2, dadd(dsub(x[m - 1], lm), dmul(dmul(dmul(rho, u), u), c)));
    }
}

// main.c:566-593 per conduit, in the reference's summation order:
// Qc1d = sum (-KI/mu)(pc - p) hs, Qc3d = sum (KI/mu)(pc - p),
// Qcb = ucl[0] Ac + ucr[last] Ac; qk is [3 * nk].
__global__ void k_karst_balance(KDev d, const double *__restrict__ p,
                                const double *__restrict__ KI, double visc, double *qk)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= d.nk) return;
    const int m = d.len[j], o = d.off[j], nk = d.nk;
    const double hs = d.hs[j];
    double qc = 0.0, q3 = 0.0;
    for (int i = 0; i < m; i++) {
        const int c = d.ecell[o + i];
        const double dp = dsub(d.pc[o + i], p[c]);
        qc = dadd(qc, dmul(dmul(ddiv(-KI[c], visc), dp), hs));
        q3 = dadd(q3, dmul(ddiv(KI[c], visc), dp));
    }
    qk[j] = qc;
    qk[nk + j] = q3;
    qk[2 * nk + j] = dadd(dmul(d.ucl[o], d.area[j]), dmul(d.ucr[o + m - 1], d.area[j]));
}

// KI[cell] = karst_index of the conduit that owns the cell (main.c:416-448:
// the last conduit element mapped to a cell wins)
__global__ void k_scatter_ki(KDev d, int nown, const int *__restrict__ own, double *KI)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nown; t += gridDim.x * blockDim.x) {
        const int e = own[t];
        KI[d.ecell[e]] = d.kidx[d.econd[e]];
    }
}

// element arrays <-> the reference's [i * nk + j] matrices (zero past len)
__global__ void k_elem_to_ref(KDev d, int mmax, const double *__restrict__ e, double *out)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= mmax * d.nk) return;
    const int i = t / d.nk, j = t % d.nk;
    out[t] = i < d.len[j] ? e[d.off[j] + i] : 0.0;
}

__global__ void k_ref_to_elem(KDev d, int mmax, const double *__restrict__ in, double *e)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= mmax * d.nk) return;
    const int i = t / d.nk, j = t % d.nk;
    if (i < d.len[j]) e[d.off[j] + i] = in[t];
}

// fracture arrays <-> the reference's [b * nk + j] tables (entries past a
// conduit's fracture count are left as they are, as the reference leaves
// ucR_old / ucL_old there)
__global__ void k_frac_to_ref(KDev d, int mb, const double *__restrict__ e, double *out)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= mb * d.nk) return;
    const int b = t / d.nk, j = t % d.nk;
    if (b < d.nb[j]) out[t] = e[d.boff[j] + b];
}

__global__ void k_ref_to_frac(KDev d, int mb, const double *__restrict__ in, double *e)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= mb * d.nk) return;
    const int b = t / d.nk, j = t % d.nk;
    if (b < d.nb[j]) e[d.boff[j] + b] = in[t];
}

// Two sums over the reservoir in a fixed order (deterministic): mode 0
// ||a - b||^2 and ||a||^2 (erro_relativo, main.c:102-113); mode 1
// sum (WI/mu)(pw - a) and sum a (main.c:523-529; w = WI, b = pw, nullable).
constexpr int kRedBlocks = 296, kRedThreads = 256;

__global__ void __launch_bounds__(kRedThreads)
k_pair_sums(int mode, long n, const double *__restrict__ a, const double *__restrict__ b,
            const double *__restrict__ w, double visc, double *part)
{
    double s0 = 0.0, s1 = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        const double ai = a[i];
        if (mode == 0) {
            const double dd = dsub(ai, b[i]);
            s0 = dadd(s0, dmul(dd, dd));
            s1 = dadd(s1, dmul(ai, ai));
        } else {
            if (w) s0 = dadd(s0, dmul(ddiv(w[i], visc), dsub(b ? b[i] : 0.0, ai)));
            s1 = dadd(s1, ai);
        }
    }
    __shared__ double sh[2][kRedThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
        s0 = dadd(s0, __shfl_xor_sync(0xffffffffu, s0, o));
        s1 = dadd(s1, __shfl_xor_sync(0xffffffffu, s1, o));
    }
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = s0;
        sh[1][threadIdx.x >> 5] = s1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int k = 0; k < kRedThreads / 32; k++) {
            t0 = dadd(t0, sh[0][k]);
            t1 = dadd(t1, sh[1][k]);
        }
        part[2 * blockIdx.x] = t0;
        part[2 * blockIdx.x + 1] = t1;
    }
}

__global__ void k_pair_final(const double *__restrict__ part, int nb, double *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double t0 = 0.0, t1 = 0.0;
    for (int k = 0; k < nb; k++) {
        t0 = dadd(t0, part[2 * k]);
        t1 = dadd(t1, part[2 * k + 1]);
    }
    out[0] = t0;
    out[1] = t1;
}

// ---- host side --------------------------------------------------------------

// Validates k for an nx*ny*nz grid (the conditions of hmfem_karst_check).
int karst_check(const hmfem_karst *k, int nx, int ny, int nz)
{
    char msg[256];
    auto bad = [&](const char *why, int j) {
        snprintf(msg, sizeof(msg), "conduit %d: %s", j, why);
        set_last_error(msg, __FILE__, __LINE__);
        return HMFEM_E_ARG;
    };
    if (!k || k->number_karst < 0 || k->max_brechas < 0) {
        set_last_error("no conduit set", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    const int nk = k->number_karst;
    if (nk > 0 && (!k->len || !k->sxi || !k->syi || !k->szi || !k->pos || !k->Kc ||
                   !k->bound_l || !k->bound_r || !k->cont || !k->ccont ||
                   !k->karst_index || !k->area || !k->n_brechas)) {
        set_last_error("conduit set with a missing array", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    if (k->max_brechas > 0 && (!k->beta || !k->cbrecha || !k->brechas)) {
        set_last_error("conduit set with a missing fracture table", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    for (int j = 0; j < nk; j++) {
        const int m = k->len[j], p = k->pos[j];
        const int x = k->sxi[j], y = k->syi[j], z = k->szi[j];
        if (p < 1 || p > 3) return bad("position code must be 1, 2 or 3", j);
        if (m < 1) return bad("needs at least one element", j);
        if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz)
            return bad("starts outside the grid", j);
        const int nax = p == 1 ? nx : (p == 2 ? ny : nz);
        const int a0 = p == 1 ? x : (p == 2 ? y : z);
        if ((long)a0 + m > nax) return bad("leaves the grid", j);
        for (int f = 0; f < 2; f++) {
            const int bt = f ? k->bound_r[j] : k->bound_l[j];
            if (bt != 0 && bt != 1 && bt != 3)
                return bad("end condition must be 0, 1 or 3", j);
            if (bt != 3) continue;
            if (f == 0 && a0 < 1) return bad("Robin left end has no reservoir cell before it", j);
            if (f == 1 && (long)a0 + m >= nax)
                return bad("Robin right end has no reservoir cell after it", j);
            if (f == 1 && p == 3)
                return bad("Robin right end of a z conduit (source term undefined in the reference)", j);
        }
        const int nb = k->n_brechas[j];
        if (nb < 0 || nb > k->max_brechas) return bad("fracture count outside 0..max_brechas", j);
        for (int b = 0; b < nb; b++) {
            const int s = k->brechas[b * nk + j];
            if (s < 0 || s + 1 >= m) return bad("fracture outside elements 0..len-2", j);
        }
    }
    return HMFEM_OK;
}

// Host image of a conduit set: one int block and one double block in the
// order KDev points into them, plus the sizes.
struct KHost {
    int nk = 0, mtot = 0, btot = 0, mmax = 0, nown = 0, mbt = 0;
    std::vector<int> iv;
    std::vector<double> dv;
    // offsets
    int i_len, i_off, i_pos, i_cell0, i_step, i_bl, i_br, i_nb, i_boff, i_rob, i_bel,
        i_ecell, i_econd, i_own;
    int d_hs, d_Kc, d_kic, d_kidx, d_area, d_cont, d_ccont, d_beta, d_cb;
};

void karst_host(const hmfem_karst *k, int nx, int ny, double hx, double hy, double hz,
                KHost &H)
{
    const int nk = k->number_karst;
    H.nk = nk;
    H.mbt = k->max_brechas;
    std::vector<int> off(nk), boff(nk);
    for (int j = 0; j < nk; j++) {
        off[j] = H.mtot;
        boff[j] = H.btot;
        H.mtot += k->len[j];
        H.btot += k->n_brechas[j];
        if (k->len[j] > H.mmax) H.mmax = k->len[j];
    }
    const long nxy = (long)nx * ny;
    auto cell = [&](int x, int y, int z) { return (int)(x + (long)y * nx + (long)z * nxy); };
    std::vector<int> ecell(H.mtot), econd(H.mtot);
    std::unordered_map<int, int> last;  // cell -> last element mapped to it
    for (int j = 0; j < nk; j++) {
        const int p = k->pos[j];
        for (int i = 0; i < k->len[j]; i++) {
            const int c = cell(k->sxi[j] + (p == 1 ? i : 0), k->syi[j] + (p == 2 ? i : 0),
                               k->szi[j] + (p == 3 ? i : 0));
            ecell[off[j] + i] = c;
            econd[off[j] + i] = j;
            last[c] = off[j] + i;
        }
    }
    std::vector<int> own;
    for (int e = 0; e < H.mtot; e++)
        if (last[ecell[e]] == e) own.push_back(e);
    H.nown = (int)own.size();
    std::vector<int> &iv = H.iv;
    auto put = [&](const int *a, int n) {
        int o = (int)iv.size();
        iv.insert(iv.end(), a, a + n);
        return o;
    };
    std::vector<int> cell0(nk), step(nk), rob(4 * (size_t)nk, -1), bel(H.btot);
    for (int j = 0; j < nk; j++) {
        const int p = k->pos[j], m = k->len[j];
        const int x = k->sxi[j], y = k->syi[j], z = k->szi[j];
        cell0[j] = cell(x, y, z);
        step[j] = p == 1 ? 1 : (p == 2 ? nx : (int)nxy);
        if (k->bound_l[j] == 3) {   // cell before the start, first element
            rob[4 * j] = cell0[j] - step[j];
            rob[4 * j + 1] = cell0[j];
        }
        if (k->bound_r[j] == 3) {   // cell after the end, last element
            rob[4 * j + 2] = cell0[j] + m * step[j];
            rob[4 * j + 3] = cell0[j] + (m - 1) * step[j];
        }
        for (int b = 0; b < k->n_brechas[j]; b++) bel[boff[j] + b] = k->brechas[b * nk + j];
    }
    H.i_len = put(k->len, nk);
    H.i_off = put(off.data(), nk);
    H.i_pos = put(k->pos, nk);
    H.i_cell0 = put(cell0.data(), nk);
    H.i_step = put(step.data(), nk);
    H.i_bl = put(k->bound_l, nk);
    H.i_br = put(k->bound_r, nk);
    H.i_nb = put(k->n_brechas, nk);
    H.i_boff = put(boff.data(), nk);
    H.i_rob = put(rob.data(), 4 * nk);
    H.i_bel = put(bel.data(), H.btot);
    H.i_ecell = put(ecell.data(), H.mtot);
    H.i_econd = put(econd.data(), H.mtot);
    H.i_own = put(own.data(), H.nown);
    std::vector<double> &dv = H.dv;
    auto putd = [&](const double *a, int n) {
        int o = (int)dv.size();
        dv.insert(dv.end(), a, a + n);
        return o;
    };
    std::vector<double> hs(nk), kic(nk), beta(H.btot), cb(H.btot);
    for (int j = 0; j < nk; j++) {
        hs[j] = k->pos[j] == 1 ? hx : (k->pos[j] == 2 ? hy : hz);
        kic[j] = k->karst_index[j] / (k->area[j] * hs[j]);   // main.c:422
        for (int b = 0; b < k->n_brechas[j]; b++) {
            beta[boff[j] + b] = k->beta[b * nk + j];
            cb[boff[j] + b] = k->cbrecha[b * nk + j];
        }
    }
    H.d_hs = putd(hs.data(), nk);
    H.d_Kc = putd(k->Kc, nk);
    H.d_kic = putd(kic.data(), nk);
    H.d_kidx = putd(k->karst_index, nk);
    H.d_area = putd(k->area, nk);
    H.d_cont = putd(k->cont, 2 * nk);
    H.d_ccont = putd(k->ccont, 2 * nk);
    H.d_beta = putd(beta.data(), H.btot);
    H.d_cb = putd(cb.data(), H.btot);
}

// Points d into device copies ib / db of H's blocks and into the mutable
// block mut: ucR, ucL (btot each) then kl, kr, kc, pc, pc_old, g, q, ucl,
// ucr (mtot each).
KDev karst_view(const KHost &H, const int *ib, const double *db, double *mut)
{
    KDev d;
    d.nk = H.nk;
    d.len = ib + H.i_len; d.off = ib + H.i_off; d.pos = ib + H.i_pos;
    d.cell0 = ib + H.i_cell0; d.step = ib + H.i_step; d.bl = ib + H.i_bl;
    d.br = ib + H.i_br; d.nb = ib + H.i_nb; d.boff = ib + H.i_boff;
    d.rob = ib + H.i_rob; d.bel = ib + H.i_bel; d.ecell = ib + H.i_ecell;
    d.econd = ib + H.i_econd;
    d.hs = db + H.d_hs; d.Kc = db + H.d_Kc; d.kic = db + H.d_kic;
    d.kidx = db + H.d_kidx; d.area = db + H.d_area; d.cont = db + H.d_cont;
    d.ccont = db + H.d_ccont; d.beta = db + H.d_beta; d.cb = db + H.d_cb;
    const long b = H.btot > 0 ? H.btot : 1, m = H.mtot > 0 ? H.mtot : 1;
    d.ucR = mut; d.ucL = mut + b;
    double *e = mut + 2 * b;
    d.kl = e; d.kr = e + m; d.kc = e + 2 * m; d.pc = e + 3 * m; d.pc_old = e + 4 * m;
    d.g = e + 5 * m; d.q = e + 6 * m; d.ucl = e + 7 * m; d.ucr = e + 8 * m;
    return d;
}

long karst_mut_len(const KHost &H)
{
    const long b = H.btot > 0 ? H.btot : 1, m = H.mtot > 0 ? H.mtot : 1;
    return 2 * b + 9 * m;
}

int grid1(long n, int th) { return (int)((n + th - 1) / th > 0 ? (n + th - 1) / th : 1); }

}  // namespace

// Picard state kept on the solver between hmfem_picard and
// hmfem_picard_fluxes.
struct KarstRun {
    KHost H;
    KDev d{};
    int *ib = nullptr;
    double *db = nullptr, *mut = nullptr;
    double *KI = nullptr, *WIown = nullptr, *pwown = nullptr;
    const double *WI = nullptr, *pw = nullptr;
    double *p = nullptr, *p_old = nullptr, *part = nullptr, *sums = nullptr;
    double *ref = nullptr;   // max(len) * nk staging for the reference layout
    double *qk = nullptr;    // 3 * nk
    double visc = 1, rho = 1000;
    Axis ax{};
    bool done = false;
};

void karst_release(Solver &s)
{
    KarstRun *R = s.karst;
    if (!R) return;
    dfree(R->ib); dfree(R->db); dfree(R->mut); dfree(R->KI);
    dfree(R->WIown); dfree(R->pwown); dfree(R->p); dfree(R->p_old);
    dfree(R->part); dfree(R->sums); dfree(R->ref); dfree(R->qk);
    delete R;
    s.karst = nullptr;
}

}  // namespace hm

using hm::KarstRun;
using hm::Solver;

#define KA_ALLOC(p, T, n)                                                      \
    do {                                                                       \
        (p) = (T *)hm::dalloc(sizeof(T) * (size_t)((n) > 0 ? (n) : 1));        \
        if (!(p)) {                                                            \
            hm::set_last_error("out of device memory", __FILE__, __LINE__);    \
            return HMFEM_E_CUDA;                                               \
        }                                                                      \
    } while (0)

static int karst_sums(KarstRun &R, int mode, long n, const double *a, const double *b,
                      const double *w, double out[2], cudaStream_t st)
{
    hm::k_pair_sums<<<hm::kRedBlocks, hm::kRedThreads, 0, st>>>(mode, n, a, b, w, R.visc,
                                                              R.part);
    HM_LAUNCHED();
    hm::k_pair_final<<<1, 32, 0, st>>>(R.part, hm::kRedBlocks, R.sums);
    HM_LAUNCHED();
    HM_CUDA(cudaMemcpyAsync(out, R.sums, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    return HMFEM_OK;
}

extern "C" {

int hmfem_karst_read(const char *path, int number_karst, hmfem_karst *out)
{
    if (!path || !out || number_karst < 0) return HMFEM_E_ARG;
    memset(out, 0, sizeof(*out));
    FILE *f = fopen(path, "r");
    if (!f) {
        hm::set_last_error("cannot open the conduit data file", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    const int nk = number_karst;
    auto ints = [&](int n) { return (int *)calloc(n > 0 ? n : 1, sizeof(int)); };
    auto dbls = [&](int n) { return (double *)calloc(n > 0 ? n : 1, sizeof(double)); };
    int *len = ints(nk), *sxi = ints(nk), *syi = ints(nk), *szi = ints(nk), *pos = ints(nk);
    int *bl = ints(nk), *br = ints(nk), *nb = ints(nk);
    double *Kc = dbls(nk), *cont = dbls(2 * nk), *ccont = dbls(2 * nk);
    double *kidx = dbls(nk), *area = dbls(nk);
    bool ok = true;
    // main.c:209-243, field by field in file order
    int *iblk[5] = {len, sxi, syi, szi, pos};
    for (int a = 0; a < 5 && ok; a++)
        for (int i = 0; i < nk && ok; i++) ok = fscanf(f, "%i", &iblk[a][i]) == 1;
    for (int i = 0; i < nk && ok; i++) ok = fscanf(f, "%lf", &Kc[i]) == 1;
    for (int i = 0; i < nk && ok; i++) ok = fscanf(f, "%i", &bl[i]) == 1;
    for (int i = 0; i < nk && ok; i++) ok = fscanf(f, "%i", &br[i]) == 1;
    for (int i = 0; i < 2 * nk && ok; i++) ok = fscanf(f, "%lf", &cont[i]) == 1;
    for (int i = 0; i < 2 * nk && ok; i++) ok = fscanf(f, "%lf", &ccont[i]) == 1;
    for (int i = 0; i < nk && ok; i++) ok = fscanf(f, "%lf", &kidx[i]) == 1;
    for (int i = 0; i < nk && ok; i++) ok = fscanf(f, "%lf", &area[i]) == 1;
    for (int i = 0; i < nk && ok; i++) ok = fscanf(f, "%i", &nb[i]) == 1;
    int mb = -1;  // main.c:245-250
    for (int i = 0; i < nk; i++)
        if (nb[i] >= mb) mb = nb[i];
    if (mb < 0) mb = 0;
    double *beta = dbls(mb * nk), *cb = dbls(mb * nk);
    int *brc = ints(mb * nk);
    for (int i = 0; i < mb * nk && ok; i++) {
        ok = fscanf(f, "%lf", &beta[i]) == 1;
        beta[i] = beta[i] - 1;  // main.c:256: beta = R^4 - 1
    }
    for (int i = 0; i < mb * nk && ok; i++) ok = fscanf(f, "%lf", &cb[i]) == 1;
    for (int i = 0; i < mb * nk && ok; i++) ok = fscanf(f, "%d", &brc[i]) == 1;
    fclose(f);
    out->number_karst = nk;
    out->max_brechas = mb;
    out->len = len; out->sxi = sxi; out->syi = syi; out->szi = szi; out->pos = pos;
    out->Kc = Kc; out->bound_l = bl; out->bound_r = br; out->cont = cont;
    out->ccont = ccont; out->karst_index = kidx; out->area = area;
    out->n_brechas = nb; out->beta = beta; out->cbrecha = cb; out->brechas = brc;
    if (!ok) {
        hmfem_karst_release(out);
        hm::set_last_error("short conduit data file", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    return HMFEM_OK;
}

void hmfem_karst_release(hmfem_karst *k)
{
    if (!k) return;
    const void *ps[] = {k->len, k->sxi, k->syi, k->szi, k->pos, k->Kc, k->bound_l,
                        k->bound_r, k->cont, k->ccont, k->karst_index, k->area,
                        k->n_brechas, k->beta, k->cbrecha, k->brechas};
    for (const void *p : ps) free((void *)p);
    memset(k, 0, sizeof(*k));
}

int hmfem_karst_check(const hmfem_karst *k, int nx, int ny, int nz)
{
    if (nx < 1 || ny < 1 || nz < 1) return HMFEM_E_ARG;
    return hm::karst_check(k, nx, ny, nz);
}

void hmfem_picard_default_options(hmfem_picard_options *o)
{
    if (!o) return;
    o->rho = 1000.0;     // main.c:127
    o->tol = 1e-8;       // main.c:118
    o->iter_max = 1000;  // main.c:119
}

int hmfem_picard(hmfem_solver *h, const hmfem_karst *k, int nx, int ny, int nz,
                 double hx, double hy, double hz, double visc, const double *KX,
                 const double *KY, const double *KZ, const int bc_type[6],
                 const double bc_value[6], const double *WI, const double *pw,
                 const hmfem_picard_options *opt, double *p, double *pc, int mem,
                 hmfem_picard_stats *out)
{
    if (!h || !k || !p || nx < 1 || ny < 1 || nz < 1) return HMFEM_E_ARG;
    HM_CHECK(hm::karst_check(k, nx, ny, nz));
    hmfem_picard_options o;
    hmfem_picard_default_options(&o);
    if (opt) o = *opt;
    Solver &s = h->s;
    hmfem_picard_stats ps;
    memset(&ps, 0, sizeof(ps));
    cudaStream_t st = s.st;
    const long n = (long)nx * ny * nz;
    cudaEvent_t ev[3];
    for (auto &e : ev) HM_CUDA(cudaEventCreate(&e));
    HM_CUDA(cudaEventRecord(ev[0], st));

    // (1) the uncoupled reservoir: no well, no exchange (main.c:393)
    HM_CHECK(hmfem_assemble(h, nx, ny, nz, hx, hy, hz, visc, KX, KY, KZ, bc_type,
                            bc_value, nullptr, mem));
    hm::set_alloc_context(s.st, s.cache);
    hm::karst_release(s);
    s.karst = new KarstRun();
    KarstRun &R = *s.karst;
    R.visc = visc;
    R.rho = o.rho;
    R.ax = hm::Axis{s.KX, s.KY, s.KZ, hx, hy, hz};
    hm::karst_host(k, nx, ny, hx, hy, hz, R.H);
    const hm::KHost &H = R.H;
    KA_ALLOC(R.ib, int, (long)H.iv.size());
    KA_ALLOC(R.db, double, (long)H.dv.size());
    KA_ALLOC(R.mut, double, hm::karst_mut_len(H));
    KA_ALLOC(R.KI, double, n);
    KA_ALLOC(R.p, double, n);
    KA_ALLOC(R.p_old, double, n);
    KA_ALLOC(R.part, double, 2 * hm::kRedBlocks);
    KA_ALLOC(R.sums, double, 2);
    KA_ALLOC(R.ref, double, (long)H.mmax * H.nk);
    KA_ALLOC(R.qk, double, 3L * H.nk);
    if (!H.iv.empty())
        HM_CUDA(cudaMemcpyAsync(R.ib, H.iv.data(), sizeof(int) * H.iv.size(),
                                cudaMemcpyHostToDevice, st));
    if (!H.dv.empty())
        HM_CUDA(cudaMemcpyAsync(R.db, H.dv.data(), sizeof(double) * H.dv.size(),
                                cudaMemcpyHostToDevice, st));
    HM_CUDA(cudaMemsetAsync(R.mut, 0, sizeof(double) * hm::karst_mut_len(H), st));
    HM_CUDA(cudaMemsetAsync(R.KI, 0, sizeof(double) * n, st));
    HM_CUDA(cudaMemsetAsync(R.p, 0, sizeof(double) * n, st));
    R.d = hm::karst_view(H, R.ib, R.db, R.mut);

    HM_CHECK(hm::setup(s));
    ps.setups = 1;
    hmfem_stats cs;
    int rc = hm::solve(s, nullptr, R.p, 1, &cs);
    if (rc != HMFEM_OK && rc != HMFEM_E_NOTCONV) return rc;
    ps.cg_iterations += cs.iterations;
    HM_CUDA(cudaMemcpyAsync(R.p_old, R.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));

    // (2) karst index of the conduit cells, well arrays (main.c:399-449)
    if (H.nown > 0) {
        hm::k_scatter_ki<<<hm::grid1(H.nown, 128), 128, 0, st>>>(R.d, H.nown,
                                                                 R.ib + H.i_own, R.KI);
        HM_LAUNCHED();
    }
    if (WI && !mem) {
        KA_ALLOC(R.WIown, double, n);
        HM_CUDA(cudaMemcpyAsync(R.WIown, WI, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        R.WI = R.WIown;
    } else {
        R.WI = WI;
    }
    if (pw && !mem) {
        KA_ALLOC(R.pwown, double, n);
        HM_CUDA(cudaMemcpyAsync(R.pwown, pw, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        R.pw = R.pwown;
    } else {
        R.pw = pw;
    }

    // (3) the coupled matrix: its values stay fixed for the whole loop, so
    // one setup serves every iteration
    HM_CHECK(hm::assemble_coupled(s, R.KI, R.WI, R.pw));
    HM_CHECK(hm::setup(s));
    ps.setups = 2;
    HM_CUDA(cudaEventRecord(ev[1], st));

    // (4) conduit() before the loop (main.c:452)
    const int nk = H.nk, cth = 64, cgrid = hm::grid1(nk, cth);
    if (nk > 0) {
        hm::k_karst_keff<<<cgrid, cth, 0, st>>>(R.d, visc);
        HM_LAUNCHED();
        hm::k_conduit<<<cgrid, cth, 0, st>>>(R.d, R.p_old, R.ax, visc, R.rho);
        HM_LAUNCHED();
    }

    // (5) the Picard loop (main.c:460-489)
    double err = 1.0;
    int iter = 0;
    while (iter < o.iter_max && err > o.tol) {
        if (H.mtot > 0)
            HM_CUDA(cudaMemcpyAsync(R.d.pc_old, R.d.pc, sizeof(double) * H.mtot,
                                    cudaMemcpyDeviceToDevice, st));
        HM_CHECK(hm::launch_exchange_rhs(nx, ny, nz, hx, hy, hz, visc, s.KX, s.KY, s.KZ,
                                         s.bc, s.face, H.nown, R.ib + H.i_own,
                                         R.d.ecell, R.d.pc_old, R.KI, R.WI, R.pw, s.b, st));
        rc = hm::solve(s, nullptr, R.p, 1, &cs);  // warm start from the last p
        if (rc != HMFEM_OK && rc != HMFEM_E_NOTCONV) return rc;
        ps.cg_iterations += cs.iterations;
        double sums[2];
        HM_CHECK(karst_sums(R, 0, n, R.p, R.p_old, nullptr, sums, st));
        err = sqrt(sums[0]) / sqrt(sums[1]);
        HM_CUDA(cudaMemcpyAsync(R.p_old, R.p, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                st));
        if (nk > 0) {
            hm::k_conduit<<<cgrid, cth, 0, st>>>(R.d, R.p_old, R.ax, visc, R.rho);
            HM_LAUNCHED();
        }
        iter++;
    }
    HM_CUDA(cudaEventRecord(ev[2], st));

    // (6) results and balances
    HM_CUDA(cudaMemcpyAsync(p, R.p, sizeof(double) * n,
                            mem ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    if (pc && nk > 0) {
        const long mm = (long)H.mmax * nk;
        hm::k_elem_to_ref<<<hm::grid1(mm, 128), 128, 0, st>>>(R.d, H.mmax, R.d.pc, R.ref);
        HM_LAUNCHED();
        HM_CUDA(cudaMemcpyAsync(pc, R.ref, sizeof(double) * mm,
                                mem ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    }
    double bal[2];
    HM_CHECK(karst_sums(R, 1, n, R.p, R.pw, R.WI, bal, st));
    R.done = true;
    float t01 = 0, t12 = 0;
    cudaEventElapsedTime(&t01, ev[0], ev[1]);
    cudaEventElapsedTime(&t12, ev[1], ev[2]);
    for (auto &e : ev) cudaEventDestroy(e);
    ps.iterations = iter;
    ps.error = err;
    ps.status = err > o.tol ? HMFEM_E_NOTCONV : HMFEM_OK;
    ps.q_well = bal[0];
    ps.p_mean = bal[1] / (double)n;
    ps.t_setup_ms = t01;
    ps.t_loop_ms = t12;
    ps.t_total_ms = t01 + t12;
    if (out) *out = ps;
    return ps.status;
}

int hmfem_picard_fluxes(hmfem_solver *h, double *ucl, double *ucr, double *qk, int mem)
{
    if (!h) return HMFEM_E_ARG;
    Solver &s = h->s;
    KarstRun *R = s.karst;
    if (!R || !R->done) {
        hm::set_last_error("conduit fluxes need a finished hmfem_picard run", __FILE__,
                           __LINE__);
        return HMFEM_E_ARG;
    }
    hm::set_alloc_context(s.st, s.cache);
    cudaStream_t st = s.st;
    const hm::KHost &H = R->H;
    const int nk = H.nk, cth = 64, cgrid = hm::grid1(nk, cth);
    if (nk == 0) return HMFEM_OK;
    const cudaMemcpyKind kind = mem ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    hm::k_fluxo1d<<<cgrid, cth, 0, st>>>(R->d, R->p_old, R->ax, R->visc, R->rho);
    HM_LAUNCHED();
    const long mm = (long)H.mmax * nk;
    double *const outs[2] = {ucl, ucr};
    double *const src[2] = {R->d.ucl, R->d.ucr};
    for (int a = 0; a < 2; a++) {
        if (!outs[a]) continue;
        hm::k_elem_to_ref<<<hm::grid1(mm, 128), 128, 0, st>>>(R->d, H.mmax, src[a], R->ref);
        HM_LAUNCHED();
        HM_CUDA(cudaMemcpyAsync(outs[a], R->ref, sizeof(double) * mm, kind, st));
        HM_CUDA(cudaStreamSynchronize(st));  // R->ref is reused
    }
    if (qk) {
        hm::k_karst_balance<<<cgrid, cth, 0, st>>>(R->d, R->p_old, R->KI, R->visc, R->qk);
        HM_LAUNCHED();
        HM_CUDA(cudaMemcpyAsync(qk, R->qk, sizeof(double) * 3 * nk, kind, st));
    }
    HM_CUDA(cudaStreamSynchronize(st));
    return HMFEM_OK;
}

int hmfem_conduit_step(const hmfem_karst *k, int nx, int ny, int nz, double hx, double hy,
                       double hz, double visc, double rho, const double *KX,
                       const double *KY, const double *KZ, const double *p_old,
                       const double *pc_old, double *ucR, double *ucL, double *pc,
                       double *kl, double *kr, double *kc, int mem)
{
    if (!k || !KX || !KY || !KZ || !p_old || !pc_old || !pc || nx < 1 || ny < 1 || nz < 1)
        return HMFEM_E_ARG;
    HM_CHECK(hm::karst_check(k, nx, ny, nz));
    if (k->max_brechas > 0 && (!ucR || !ucL)) return HMFEM_E_ARG;
    hm::KHost H;
    hm::karst_host(k, nx, ny, hx, hy, hz, H);
    const long n = (long)nx * ny * nz;
    const int nk = H.nk;
    const long mm = (long)H.mmax * nk, mb = (long)H.mbt * nk;
    cudaStream_t st;
    HM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    // device buffers: one block (this entry point serves parity checks)
    const long nK = mem ? 0 : 4 * n;
    const long tot = nK + (long)H.dv.size() + hm::karst_mut_len(H) + mm + mb + 1;
    double *buf = nullptr;
    int *ib = nullptr;
    cudaError_t e1 = cudaMalloc(&buf, sizeof(double) * tot);
    cudaError_t e2 = cudaMalloc(&ib, sizeof(int) * (H.iv.size() + 1));
    int rc = HMFEM_OK;
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
        hm::set_last_error("out of device memory", __FILE__, __LINE__);
        rc = HMFEM_E_CUDA;
    }
    if (rc == HMFEM_OK) {
        const cudaMemcpyKind in = mem ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        const cudaMemcpyKind outk = mem ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        double *cur = buf;
        const double *dK[3] = {KX, KY, KZ}, *dp = p_old;
        if (!mem) {
            const double *hK[3] = {KX, KY, KZ};
            for (int a = 0; a < 3; a++) {
                cudaMemcpyAsync(cur, hK[a], sizeof(double) * n, in, st);
                dK[a] = cur;
                cur += n;
            }
            cudaMemcpyAsync(cur, p_old, sizeof(double) * n, in, st);
            dp = cur;
            cur += n;
        }
        double *db = cur;
        cur += H.dv.size();
        double *mut = cur;
        cur += hm::karst_mut_len(H);
        double *stage = cur;
        cur += mm;
        double *fstage = cur;
        if (!H.iv.empty())
            cudaMemcpyAsync(ib, H.iv.data(), sizeof(int) * H.iv.size(), cudaMemcpyHostToDevice, st);
        if (!H.dv.empty())
            cudaMemcpyAsync(db, H.dv.data(), sizeof(double) * H.dv.size(),
                            cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(mut, 0, sizeof(double) * hm::karst_mut_len(H), st);
        hm::KDev d = hm::karst_view(H, ib, db, mut);
        hm::Axis ax{dK[0], dK[1], dK[2], hx, hy, hz};
        if (nk > 0) {
            cudaMemcpyAsync(stage, pc_old, sizeof(double) * mm, in, st);
            hm::k_ref_to_elem<<<hm::grid1(mm, 128), 128, 0, st>>>(d, H.mmax, stage, d.pc_old);
            HM_COUNT();
            if (mb > 0) {
                double *const fi[2] = {ucR, ucL};
                double *const fe[2] = {d.ucR, d.ucL};
                for (int a = 0; a < 2; a++) {
                    cudaMemcpyAsync(fstage, fi[a], sizeof(double) * mb, in, st);
                    hm::k_ref_to_frac<<<hm::grid1(mb, 128), 128, 0, st>>>(d, H.mbt, fstage, fe[a]);
                    HM_COUNT();
                }
            }
            const int cg = hm::grid1(nk, 64);
            hm::k_karst_keff<<<cg, 64, 0, st>>>(d, visc);
            HM_COUNT();
            hm::k_conduit<<<cg, 64, 0, st>>>(d, dp, ax, visc, rho);
            HM_COUNT();
            double *const outs[4] = {pc, kl, kr, kc};
            double *const src[4] = {d.pc, d.kl, d.kr, d.kc};
            for (int a = 0; a < 4; a++) {
                if (!outs[a]) continue;
                hm::k_elem_to_ref<<<hm::grid1(mm, 128), 128, 0, st>>>(d, H.mmax, src[a], stage);
                HM_COUNT();
                cudaMemcpyAsync(outs[a], stage, sizeof(double) * mm, outk, st);
                cudaStreamSynchronize(st);
            }
            if (mb > 0) {
                double *const fo[2] = {ucR, ucL};
                double *const fe[2] = {d.ucR, d.ucL};
                for (int a = 0; a < 2; a++) {
                    cudaMemcpyAsync(fstage, fo[a], sizeof(double) * mb, in, st);
                    hm::k_frac_to_ref<<<hm::grid1(mb, 128), 128, 0, st>>>(d, H.mbt, fe[a], fstage);
                    HM_COUNT();
                    cudaMemcpyAsync(fo[a], fstage, sizeof(double) * mb, outk, st);
                    cudaStreamSynchronize(st);
                }
            }
        }
        cudaError_t e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) {
            hm::set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
            rc = HMFEM_E_CUDA;
        }
    }
    if (buf) cudaFree(buf);
    if (ib) cudaFree(ib);
    cudaStreamDestroy(st);
    return rc;
}

}  // extern "C"
