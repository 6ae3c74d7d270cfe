// noalloc.cu -- flux reconstruction for callers that cannot allocate device
// memory.
//
// hmfem_fluxes() works on a solver object whose boundary-value arrays and
// min/max accumulators live in memory the library allocated.  Some callers
// cannot let a library allocate: an application whose device memory is
// already fully reserved by its own (or a framework's) caching allocator, or
// code that runs where allocation is not permitted at all.  For them,
// hmfem_fluxes_noalloc() computes the same fluxes and divergence bounds with
// every piece of scratch in one file-scope __device__ array of fixed size:
// the six boundary-face value arrays (at most HMFEM_NOALLOC_MAX_FACE cells
// per face) and the two divergence accumulators.  Grids with a larger face
// are rejected with HMFEM_E_CAPACITY.
//
// The array exists once per device for as long as the library is loaded,
// and every call uses it: calls that overlap on the GPU (two streams, or two
// host threads) race on it.  Its device address is looked up the first time
// the entry point runs on a device (cudaGetSymbolAddress, with that device
// current, once per device even when several host threads make their first
// call at the same time); make that first call before any stream capture
// begins.  Every call reads the divergence bounds back to the host, so it
// returns only after its work on the stream has finished.
#include <string.h>

#include <mutex>

#include "hm.cuh"

namespace hm {
namespace {

constexpr long kFace = HMFEM_NOALLOC_MAX_FACE;
// six face arrays, then min / max |div| as ordered bit patterns
static __device__ __align__(256) double g_flux_scratch[6 * kFace + 32];

constexpr int kMaxDevices = 64;
double *g_scratch_addr[kMaxDevices];
cudaError_t g_scratch_err[kMaxDevices];
std::once_flag g_scratch_once[kMaxDevices];

struct NaGrid {
    int nx, ny, nz;
    double hx, hy, hz, hx2v, hy2v, hz2v;
    int bc[6];
    int allneu, spec;
};

__device__ __forceinline__ double na_hmean(double a, double b)
{
    return dmul(dmul(2.0, a), b) / dadd(a, b);
}

// The face coefficients of permeabilidade_arestas (permeabilities.c:214-477).
__device__ __forceinline__ void na_faces(const NaGrid &g, int i, int j, int k,
                                         long s, const double *KX,
                                         const double *KY, const double *KZ,
                                         double F[6])
{
    const long nx = g.nx, nxy = (long)g.nx * g.ny;
    const double kx = KX[s], ky = KY[s], kz = KZ[s];
    F[0] = (j < g.ny - 1) ? na_hmean(ky, KY[s + nx]) / g.hy2v
                          : (g.bc[2] == 0 ? dmul(2.0, ky) / g.hy2v : 0.0);  // u
    F[1] = (j > 0) ? na_hmean(ky, KY[s - nx]) / g.hy2v
                   : (g.bc[3] == 0 ? dmul(2.0, ky) / g.hy2v : 0.0);         // d
    F[2] = (i > 0) ? na_hmean(kx, KX[s - 1]) / g.hx2v
                   : (g.bc[0] == 0 ? dmul(2.0, kx) / g.hx2v : 0.0);         // l
    if (g.allneu && s == g.spec) F[2] = dmul(2.0, kx) / g.hx2v;
    F[3] = (i < g.nx - 1) ? na_hmean(kx, KX[s + 1]) / g.hx2v
                          : (g.bc[1] == 0 ? dmul(2.0, kx) / g.hx2v : 0.0);  // r
    F[4] = (k < g.nz - 1) ? na_hmean(kz, KZ[s + nxy]) / g.hz2v
                          : (g.bc[4] == 0 ? dmul(2.0, kz) / g.hz2v : 0.0);  // t
    F[5] = (k > 0) ? na_hmean(kz, KZ[s - nxy]) / g.hz2v
                   : (g.bc[5] == 0 ? dmul(2.0, kz) / g.hz2v : 0.0);         // b
}

// Boundary values (create_boundary, set_boundaries.c:8-125) into the
// scratch faces, and the divergence accumulators reset.
__global__ void k_na_prepare(double *scr, NaGrid g, double v0, double v1,
                             double v2, double v3, double v4, double v5)
{
    const double val[6] = {v0, v1, v2, v3, v4, v5};
    const long sz[6] = {(long)g.ny * g.nz, (long)g.ny * g.nz, (long)g.nx * g.nz,
                        (long)g.nx * g.nz, (long)g.nx * g.ny, (long)g.nx * g.ny};
    for (int f = 0; f < 6; f++)
        for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < sz[f];
             q += (long)gridDim.x * blockDim.x)
            scr[f * kFace + q] = val[f];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        unsigned long long *mm = (unsigned long long *)(scr + 6 * kFace);
        mm[0] = (unsigned long long)__double_as_longlong(100.0);  // divvel_pontual
        mm[1] = 0ull;
    }
}

// fluxos + divvel_pontual (flux_reconstruction.c:9-319) reading the
// boundary values from the scratch faces (l, r, u, d, t, b).
__global__ void __launch_bounds__(256)
k_na_flux(const double *scr, NaGrid g, const double *__restrict__ KX,
          const double *__restrict__ KY, const double *__restrict__ KZ,
          const double *__restrict__ p, hmfem_ele *__restrict__ v)
{
    const double *fl = scr, *fr = scr + kFace, *fu = scr + 2 * kFace,
                 *fd = scr + 3 * kFace, *ft = scr + 4 * kFace, *fb = scr + 5 * kFace;
    unsigned long long *mm = (unsigned long long *)(scr + 6 * kFace);
    const long nx = g.nx, nxy = (long)g.nx * g.ny, n = nxy * g.nz;
    double lmin = 100.0, lmax = 0.0;
    for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < n;
         s += (long)gridDim.x * blockDim.x) {
        const int i = (int)(s % nx), j = (int)((s / nx) % g.ny), k = (int)(s / nxy);
        double F[6];
        na_faces(g, i, j, k, s, KX, KY, KZ, F);
        const double ps = p[s];
        const long lxz = (long)k * g.nx + i, lyz = (long)k * g.ny + j,
                   lxy = (long)j * g.nx + i;
        double vu, vd, vl, vr, vt, vb;
        vu = j < g.ny - 1 ? dmul(dmul(g.hy, F[0]), dsub(ps, p[s + nx]))
             : g.bc[2] == 0 ? dmul(dmul(g.hy, F[0]), dsub(ps, fu[lxz])) : fu[lxz];
        vd = j > 0 ? dmul(dmul(g.hy, F[1]), dsub(ps, p[s - nx]))
             : g.bc[3] == 0 ? dmul(dmul(g.hy, F[1]), dsub(ps, fd[lxz])) : -fd[lxz];
        vl = i > 0 ? dmul(dmul(g.hx, F[2]), dsub(ps, p[s - 1]))
             : g.bc[0] == 0 ? dmul(dmul(g.hx, F[2]), dsub(ps, fl[lyz])) : -fl[lyz];
        vr = i < g.nx - 1 ? dmul(dmul(g.hx, F[3]), dsub(ps, p[s + 1]))
             : g.bc[1] == 0 ? dmul(dmul(g.hx, F[3]), dsub(ps, fr[lyz])) : fr[lyz];
        vt = k < g.nz - 1 ? dmul(dmul(g.hz, F[4]), dsub(ps, p[s + nxy]))
             : g.bc[4] == 0 ? dmul(dmul(g.hz, F[4]), dsub(ps, ft[lxy])) : ft[lxy];
        vb = k > 0 ? dmul(dmul(g.hz, F[5]), dsub(ps, p[s - nxy]))
             : g.bc[5] == 0 ? dmul(dmul(g.hz, F[5]), dsub(ps, fb[lxy])) : -fb[lxy];
        hmfem_ele *o = v + s;
        o->u = vu; o->d = vd; o->l = vl; o->r = vr; o->t = vt; o->b = vb;
        const double dv = dadd(dadd(dadd(dadd(dadd(vr / g.hx, vl / g.hx), vd / g.hy),
                                          vu / g.hy), vb / g.hz), vt / g.hz);
        const double a = fabs(dv);
        if (a > lmax) lmax = a;
        if (a < lmin) lmin = a;
    }
    for (int o = 16; o > 0; o >>= 1) {
        lmin = fmin(lmin, __shfl_xor_sync(0xffffffffu, lmin, o));
        lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(mm, (unsigned long long)__double_as_longlong(lmin));
        atomicMax(mm + 1, (unsigned long long)__double_as_longlong(lmax));
    }
}

}  // namespace
}  // namespace hm

extern "C" int hmfem_fluxes_noalloc(int nx, int ny, int nz, double hx, double hy,
                                    double hz, double visc, const double *KX,
                                    const double *KY, const double *KZ,
                                    const int bc_type[6], const double bc_value[6],
                                    const double *p, hmfem_ele *v, double *divmin,
                                    double *divmax, void *stream)
{
    using namespace hm;
    if (nx < 1 || ny < 1 || nz < 1 || !KX || !KY || !KZ || !bc_type || !bc_value ||
        !p || !v) {
        set_last_error("hmfem_fluxes_noalloc: invalid argument", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    for (int f = 0; f < 6; f++)
        if (bc_type[f] != 0 && bc_type[f] != 1) {
            set_last_error("hmfem_fluxes_noalloc: boundary types must be 0 or 1",
                           __FILE__, __LINE__);
            return HMFEM_E_ARG;
        }
    if ((long)nx * ny > kFace || (long)ny * nz > kFace || (long)nx * nz > kFace) {
        set_last_error("hmfem_fluxes_noalloc: a boundary face has more than "
                       "HMFEM_NOALLOC_MAX_FACE cells (the fixed scratch size)",
                       __FILE__, __LINE__);
        return HMFEM_E_CAPACITY;
    }
    int dev = 0;
    HM_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_last_error("hmfem_fluxes_noalloc: device ordinal out of range", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    // once per device, with that device current; concurrent first calls
    // wait here for the one that does the lookup
    std::call_once(g_scratch_once[dev], [dev] {
        void *addr = nullptr;
        g_scratch_err[dev] = cudaGetSymbolAddress(&addr, g_flux_scratch);
        g_scratch_addr[dev] = g_scratch_err[dev] == cudaSuccess ? (double *)addr : nullptr;
    });
    HM_CUDA(g_scratch_err[dev]);
    double *scr = g_scratch_addr[dev];
    cudaStream_t st = (cudaStream_t)stream;
    NaGrid g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.hx = hx; g.hy = hy; g.hz = hz;
    g.hx2v = hx * hx * visc;
    g.hy2v = hy * hy * visc;
    g.hz2v = hz * hz * visc;
    int all = 1;
    for (int f = 0; f < 6; f++) { g.bc[f] = bc_type[f]; all &= bc_type[f] == 1; }
    g.allneu = all;
    g.spec = (ny - 1) * nx + (nz / 2) * nx * ny;
    long face_max = (long)nx * ny;
    if ((long)ny * nz > face_max) face_max = (long)ny * nz;
    if ((long)nx * nz > face_max) face_max = (long)nx * nz;
    long pb = ceil_div(face_max, 256);
    k_na_prepare<<<(int)(pb < 1024 ? pb : 1024), 256, 0, st>>>(
        scr, g, bc_value[0], bc_value[1], bc_value[2], bc_value[3], bc_value[4],
        bc_value[5]);
    HM_LAUNCHED();
    const long n = (long)nx * ny * nz;
    long fb = ceil_div(n, 256);
    k_na_flux<<<(int)(fb < 148L * 16 ? fb : 148L * 16), 256, 0, st>>>(scr, g, KX, KY,
                                                                       KZ, p, v);
    HM_LAUNCHED();
    unsigned long long mm[2];
    HM_CUDA(cudaMemcpyAsync(mm, scr + 6 * kFace, sizeof(mm), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    double d[2];
    memcpy(d, mm, sizeof(d));
    if (divmin) *divmin = d[0];
    if (divmax) *divmax = d[1];
    return HMFEM_OK;
}
