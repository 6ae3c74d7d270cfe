// assemble.cu -- TPFA assembly, AoS stencil packing and flux reconstruction
// on the device.
//
// Every expression keeps the reference's operand order and rounding (no FMA
// contraction: __dmul_rn / __dadd_rn), so the matrix, right-hand side and
// fluxes are bit-identical to permeabilities.c / set_source_term.c /
// flux_reconstruction.c on the same inputs.
#include <string.h>

#include "hm.cuh"

namespace hm {

namespace {

struct Grid {
    int nx, ny, nz;
    double hx, hy, hz;
    double hx2v, hy2v, hz2v;  // h*h*visc as (h*h)*visc (permeabilities.c:222)
    double kdiv;              // visc*hx*hy*hz (permeabilities.c:486)
    double vve;               // visc*(hx*hy*hz) (set_source_term.c:209,213)
    int bc[6];                // l, r, u, d, t, b
    int allneu;               // all six faces Neumann
    int spec;                 // pindex(0, ny-1, nz/2) for the all-Neumann pin
};

Grid make_grid(int nx, int ny, int nz, double hx, double hy, double hz,
               double visc, const int bc[6])
{
    Grid g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.hx = hx; g.hy = hy; g.hz = hz;
    g.hx2v = hx * hx * visc;
    g.hy2v = hy * hy * visc;
    g.hz2v = hz * hz * visc;
    g.kdiv = visc * hx * hy * hz;
    double ve = hx * hy * hz;
    g.vve = visc * ve;
    int all = 1;
    for (int f = 0; f < 6; f++) { g.bc[f] = bc[f]; all &= (bc[f] == 1); }
    g.allneu = all;
    g.spec = 0 + (ny - 1) * nx + (nz / 2) * nx * ny;
    return g;
}

// hm(), permeabilities.c:188-193: 2*a*b/(a+b)
__device__ __forceinline__ double hmean(double a, double b)
{
    return dmul(dmul(2.0, a), b) / dadd(a, b);
}

// The six face coefficients of cell s exactly as permeabilidade_arestas
// leaves them in perm[s] (interior: harmonic mean; Dirichlet boundary:
// 2K/(h^2 mu); Neumann boundary: 0).
struct Faces { double u, d, l, r, t, b; };

__device__ __forceinline__ Faces cell_faces(const Grid &g, int i, int j, int k,
                                            long s, const double *KX,
                                            const double *KY, const double *KZ)
{
    const long nx = g.nx, nxy = (long)g.nx * g.ny;
    Faces F;
    double kx = KX[s], ky = KY[s], kz = KZ[s];
    F.u = (j < g.ny - 1) ? hmean(ky, KY[s + nx]) / g.hy2v
                         : (g.bc[2] == 0 ? dmul(2.0, ky) / g.hy2v : 0.0);
    F.d = (j > 0) ? hmean(ky, KY[s - nx]) / g.hy2v
                  : (g.bc[3] == 0 ? dmul(2.0, ky) / g.hy2v : 0.0);
    F.r = (i < g.nx - 1) ? hmean(kx, KX[s + 1]) / g.hx2v
                         : (g.bc[1] == 0 ? dmul(2.0, kx) / g.hx2v : 0.0);
    F.l = (i > 0) ? hmean(kx, KX[s - 1]) / g.hx2v
                  : (g.bc[0] == 0 ? dmul(2.0, kx) / g.hx2v : 0.0);
    if (g.allneu && s == g.spec) F.l = dmul(2.0, kx) / g.hx2v;
    F.t = (k < g.nz - 1) ? hmean(kz, KZ[s + nxy]) / g.hz2v
                         : (g.bc[4] == 0 ? dmul(2.0, kz) / g.hz2v : 0.0);
    F.b = (k > 0) ? hmean(kz, KZ[s - nxy]) / g.hz2v
                  : (g.bc[5] == 0 ? dmul(2.0, kz) / g.hz2v : 0.0);
    return F;
}

struct FacePtrs { const double *l, *r, *u, *d, *t, *b; };

__global__ void k_l0_rowcounts(int nx, int ny, int nz, int *cnt)
{
    long n = (long)nx * ny * nz;
    for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < n;
         s += (long)gridDim.x * blockDim.x) {
        int i = (int)(s % nx), j = (int)((s / nx) % ny), k = (int)(s / ((long)nx * ny));
        cnt[s] = 1 + (j > 0) + (i > 0) + (i < nx - 1) + (j < ny - 1) +
                 (k < nz - 1) + (k > 0);
    }
}

// Right-hand side of cell s (source_term, set_source_term.c:23-220; faces in
// the reference's interface order L,R,D,U,T,B, then the karst and well
// exchange terms of :206-220).
__device__ __forceinline__ double cell_rhs(const Grid &g, const FacePtrs &fv, int i,
                                           int j, int k, long s, const Faces &F,
                                           double ki, double wi, double pcs, double pws)
{
    double r = 0.0;
    if (i == 0) {
        double gv = fv.l[(long)k * g.ny + j];
        if (g.bc[0] == 0) r = dadd(r, dmul(F.l, gv));
        if (g.bc[0] == 1) r = dadd(r, gv / g.hx);
    }
    if (g.allneu && s == g.spec) r = dadd(r, dmul(F.l, 1.0));
    if (i == g.nx - 1) {
        double gv = fv.r[(long)k * g.ny + j];
        if (g.bc[1] == 0) r = dadd(r, dmul(F.r, gv));
        if (g.bc[1] == 1) r = dsub(r, gv / g.hx);
    }
    if (j == 0) {
        double gv = fv.d[(long)k * g.nx + i];
        if (g.bc[3] == 0) r = dadd(r, dmul(F.d, gv));
        if (g.bc[3] == 1) r = dadd(r, gv / g.hy);
    }
    if (j == g.ny - 1) {
        double gv = fv.u[(long)k * g.nx + i];
        if (g.bc[2] == 0) r = dadd(r, dmul(F.u, gv));
        if (g.bc[2] == 1) r = dsub(r, gv / g.hy);
    }
    if (k == g.nz - 1) {
        double gv = fv.t[(long)j * g.nx + i];
        if (g.bc[4] == 0) r = dadd(r, dmul(F.t, gv));
        if (g.bc[4] == 1) r = dsub(r, gv / g.hz);
    }
    if (k == 0) {
        double gv = fv.b[(long)j * g.nx + i];
        if (g.bc[5] == 0) r = dadd(r, dmul(F.b, gv));
        if (g.bc[5] == 1) r = dadd(r, gv / g.hz);
    }
    r = dadd(dadd(r, dmul(ki, pcs) / g.vve), dmul(wi, pws) / g.vve);
    return r;
}

// One thread per cell: faces, diagonal, CSR row (d,l,c,r,u,t,b as
// solve_linearsystem_AMG.c:103-139 packs it) and right-hand side.
__global__ void __launch_bounds__(256)
k_assemble(Grid g, const double *__restrict__ KX, const double *__restrict__ KY,
           const double *__restrict__ KZ, FacePtrs fv,
           const double *__restrict__ KI, const double *__restrict__ WI,
           const double *__restrict__ PC, const double *__restrict__ PW,
           const int *__restrict__ rowptr, int *__restrict__ col,
           double *__restrict__ val, double *__restrict__ b, int *bad)
{
    const long nx = g.nx, nxy = (long)g.nx * g.ny, n = nxy * g.nz;
    for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < n;
         s += (long)gridDim.x * blockDim.x) {
        int i = (int)(s % nx), j = (int)((s / nx) % g.ny), k = (int)(s / nxy);
        // a permeability that is NaN, infinite or negative makes every
        // coefficient that touches it meaningless (the reference does not
        // check): flag one such cell as 1 + its index
        if (bad) {
            const double kx = KX[s], ky = KY[s], kz = KZ[s];
            if (!(kx >= 0.0 && kx <= 1.7976931348623157e308) ||
                !(ky >= 0.0 && ky <= 1.7976931348623157e308) ||
                !(kz >= 0.0 && kz <= 1.7976931348623157e308))
                atomicExch(bad, (int)(s + 1));
        }
        Faces F = cell_faces(g, i, j, k, s, KX, KY, KZ);
        double ki = KI ? KI[s] : 0.0, wi = WI ? WI[s] : 0.0;
        // permeabilities.c:486: l + r + u + d + t + b + KI/(mu V) + WI/(mu V)
        double c = dadd(dadd(dadd(dadd(dadd(F.l, F.r), F.u), F.d), F.t), F.b);
        c = dadd(dadd(c, ki / g.kdiv), wi / g.kdiv);
        long q = rowptr[s];
        if (j > 0)          { col[q] = (int)(s - nx);  val[q] = -F.d; q++; }
        if (i > 0)          { col[q] = (int)(s - 1);   val[q] = -F.l; q++; }
        col[q] = (int)s; val[q] = c; q++;
        if (i < g.nx - 1)   { col[q] = (int)(s + 1);   val[q] = -F.r; q++; }
        if (j < g.ny - 1)   { col[q] = (int)(s + nx);  val[q] = -F.u; q++; }
        if (k < g.nz - 1)   { col[q] = (int)(s + nxy); val[q] = -F.t; q++; }
        if (k > 0)          { col[q] = (int)(s - nxy); val[q] = -F.b; q++; }
        b[s] = cell_rhs(g, fv, i, j, k, s, F, ki, wi, PC ? PC[s] : 0.0, PW ? PW[s] : 0.0);
    }
}

// The Picard loop's right-hand side patch (reservoir.c:19-52 /
// set_source_term.c:206-220): only the cells a conduit element exchanges
// with change between iterations.  Element e = own[t] owns reservoir cell
// ecell[e] (the last conduit element mapped to it, as pc_aux is filled) and
// brings its conduit pressure pc[e].
__global__ void k_exchange_rhs(Grid g, const double *__restrict__ KX,
                               const double *__restrict__ KY,
                               const double *__restrict__ KZ, FacePtrs fv, int m,
                               const int *__restrict__ own, const int *__restrict__ ecell,
                               const double *__restrict__ pc, const double *__restrict__ KI,
                               const double *__restrict__ WI, const double *__restrict__ PW,
                               double *__restrict__ b)
{
    const long nx = g.nx, nxy = (long)g.nx * g.ny;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
        int e = own[t];
        long s = ecell[e];
        int i = (int)(s % nx), j = (int)((s / nx) % g.ny), k = (int)(s / nxy);
        Faces F = cell_faces(g, i, j, k, s, KX, KY, KZ);
        b[s] = cell_rhs(g, fv, i, j, k, s, F, KI[s], WI ? WI[s] : 0.0, pc[e],
                        PW ? PW[s] : 0.0);
    }
}

// solve_linearsystem_AMG.c:58-139: count, then fill in d,l,c,r,u,t,b order.
// Pass 0 also validates the caller's indices: each is -1 (boundary) or a
// cell in [0, n), otherwise bad = 1 (the reference reads them unchecked).
__global__ void k_pack_stencil(int n, const hmfem_ele *__restrict__ perm,
                               const hmfem_ind *__restrict__ ind, int *cnt,
                               const int *__restrict__ rowptr, int *col,
                               double *val, int pass, int *bad)
{
    for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < n;
         s += (long)gridDim.x * blockDim.x) {
        hmfem_ind I = ind[s];
        if (pass == 0) {
            if (bad) {
                const int f[7] = {I.c, I.u, I.d, I.l, I.r, I.t, I.b};
                for (int q = 0; q < 7; q++)
                    if (f[q] < -1 || f[q] >= n) atomicExch(bad, 1);
            }
            cnt[s] = (I.d != -1) + (I.l != -1) + (I.c != -1) + (I.r != -1) +
                     (I.u != -1) + (I.t != -1) + (I.b != -1);
            continue;
        }
        hmfem_ele E = perm[s];
        long q = rowptr[s];
        if (I.d != -1) { col[q] = I.d; val[q] = -E.d; q++; }
        if (I.l != -1) { col[q] = I.l; val[q] = -E.l; q++; }
        if (I.c != -1) { col[q] = I.c; val[q] = E.c; q++; }
        if (I.r != -1) { col[q] = I.r; val[q] = -E.r; q++; }
        if (I.u != -1) { col[q] = I.u; val[q] = -E.u; q++; }
        if (I.t != -1) { col[q] = I.t; val[q] = -E.t; q++; }
        if (I.b != -1) { col[q] = I.b; val[q] = -E.b; q++; }
    }
}

// fluxos (flux_reconstruction.c:9-279) + divvel_pontual (:281-319).
// mm[0] / mm[1] collect min / max |div| as ordered bit patterns.
__global__ void __launch_bounds__(256)
k_flux(Grid g, const double *__restrict__ KX, const double *__restrict__ KY,
       const double *__restrict__ KZ, FacePtrs fv, const double *__restrict__ p,
       hmfem_ele *__restrict__ v, unsigned long long *mm)
{
    const long nx = g.nx, nxy = (long)g.nx * g.ny, n = nxy * g.nz;
    double lmin = 100.0, lmax = 0.0;  // divvel_pontual's initial values
    for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < n;
         s += (long)gridDim.x * blockDim.x) {
        int i = (int)(s % nx), j = (int)((s / nx) % g.ny), k = (int)(s / nxy);
        Faces F = cell_faces(g, i, j, k, s, KX, KY, KZ);
        double ps = p[s];
        double vu, vd, vl, vr, vt, vb;
        if (j < g.ny - 1) vu = dmul(dmul(g.hy, F.u), dsub(ps, p[s + nx]));
        else vu = g.bc[2] == 0 ? dmul(dmul(g.hy, F.u), dsub(ps, fv.u[(long)k * g.nx + i]))
                               : fv.u[(long)k * g.nx + i];
        if (i < g.nx - 1) vr = dmul(dmul(g.hx, F.r), dsub(ps, p[s + 1]));
        else vr = g.bc[1] == 0 ? dmul(dmul(g.hx, F.r), dsub(ps, fv.r[(long)k * g.ny + j]))
                               : fv.r[(long)k * g.ny + j];
        if (j > 0) vd = dmul(dmul(g.hy, F.d), dsub(ps, p[s - nx]));
        else vd = g.bc[3] == 0 ? dmul(dmul(g.hy, F.d), dsub(ps, fv.d[(long)k * g.nx + i]))
                               : -fv.d[(long)k * g.nx + i];
        if (i > 0) vl = dmul(dmul(g.hx, F.l), dsub(ps, p[s - 1]));
        else vl = g.bc[0] == 0 ? dmul(dmul(g.hx, F.l), dsub(ps, fv.l[(long)k * g.ny + j]))
                               : -fv.l[(long)k * g.ny + j];
        if (k < g.nz - 1) vt = dmul(dmul(g.hz, F.t), dsub(ps, p[s + nxy]));
        else vt = g.bc[4] == 0 ? dmul(dmul(g.hz, F.t), dsub(ps, fv.t[(long)j * g.nx + i]))
                               : fv.t[(long)j * g.nx + i];
        if (k > 0) vb = dmul(dmul(g.hz, F.b), dsub(ps, p[s - nxy]));
        else vb = g.bc[5] == 0 ? dmul(dmul(g.hz, F.b), dsub(ps, fv.b[(long)j * g.nx + i]))
                               : -fv.b[(long)j * g.nx + i];
        hmfem_ele *o = v + s;
        o->u = vu; o->d = vd; o->l = vl; o->r = vr; o->t = vt; o->b = vb;
        double dv = dadd(dadd(dadd(dadd(dadd(vr / g.hx, vl / g.hx), vd / g.hy),
                                   vu / g.hy), vb / g.hz), vt / g.hz);
        double a = fabs(dv);
        if (a > lmax) lmax = a;
        if (a < lmin) lmin = a;
    }
    // |div| >= 0, so the IEEE bit patterns order like the values
    for (int o = 16; o > 0; o >>= 1) {
        lmin = fmin(lmin, __shfl_xor_sync(0xffffffffu, lmin, o));
        lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(mm, (unsigned long long)__double_as_longlong(lmin));
        atomicMax(mm + 1, (unsigned long long)__double_as_longlong(lmax));
    }
}

int grid_for(long n, int threads)
{
    long b = ceil_div(n, threads);
    long cap = 148L * 16;
    return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

}  // namespace

int launch_l0_rowcounts(int nx, int ny, int nz, int *cnt, cudaStream_t st)
{
    long n = (long)nx * ny * nz;
    k_l0_rowcounts<<<grid_for(n, 256), 256, 0, st>>>(nx, ny, nz, cnt);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int launch_assemble(int nx, int ny, int nz, double hx, double hy, double hz,
                    double visc, const double *KX, const double *KY,
                    const double *KZ, const int bc[6], double *const face[6],
                    const double *KI, const double *WI, const double *pc,
                    const double *pw, const int *rowptr, int *col, double *val,
                    double *b, cudaStream_t st, int *bad)
{
    Grid g = make_grid(nx, ny, nz, hx, hy, hz, visc, bc);
    FacePtrs fv{face[0], face[1], face[2], face[3], face[4], face[5]};
    long n = (long)nx * ny * nz;
    k_assemble<<<grid_for(n, 256), 256, 0, st>>>(g, KX, KY, KZ, fv, KI, WI, pc,
                                                 pw, rowptr, col, val, b, bad);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int launch_exchange_rhs(int nx, int ny, int nz, double hx, double hy, double hz,
                        double visc, const double *KX, const double *KY,
                        const double *KZ, const int bc[6], double *const face[6],
                        int m, const int *own, const int *ecell, const double *pc,
                        const double *KI, const double *WI, const double *pw,
                        double *b, cudaStream_t st)
{
    if (m <= 0) return HMFEM_OK;
    Grid g = make_grid(nx, ny, nz, hx, hy, hz, visc, bc);
    FacePtrs fv{face[0], face[1], face[2], face[3], face[4], face[5]};
    k_exchange_rhs<<<grid_for(m, 128), 128, 0, st>>>(g, KX, KY, KZ, fv, m, own, ecell, pc,
                                                     KI, WI, pw, b);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int launch_pack_stencil(int n, const hmfem_ele *perm, const hmfem_ind *ind,
                        int *cnt, const int *rowptr, int *col, double *val,
                        int pass, cudaStream_t st, int *bad)
{
    k_pack_stencil<<<grid_for(n, 256), 256, 0, st>>>(n, perm, ind, cnt, rowptr,
                                                     col, val, pass, bad);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int launch_flux(int nx, int ny, int nz, double hx, double hy, double hz,
                double visc, const double *KX, const double *KY,
                const double *KZ, const int bc[6], double *const face[6],
                const double *p, hmfem_ele *v, double *mm, cudaStream_t st)
{
    Grid g = make_grid(nx, ny, nz, hx, hy, hz, visc, bc);
    FacePtrs fv{face[0], face[1], face[2], face[3], face[4], face[5]};
    long n = (long)nx * ny * nz;
    double d100 = 100.0;
    unsigned long long init[2] = {0ull, 0ull};
    memcpy(&init[0], &d100, sizeof(double));
    HM_CUDA(cudaMemcpyAsync(mm, init, sizeof(init), cudaMemcpyHostToDevice, st));
    k_flux<<<grid_for(n, 256), 256, 0, st>>>(g, KX, KY, KZ, fv, p, v,
                                             (unsigned long long *)mm);
    HM_LAUNCHED();
    return HMFEM_OK;
}

}  // namespace hm
