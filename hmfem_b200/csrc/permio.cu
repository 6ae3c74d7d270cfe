// permio.cu -- heterogeneous-permeability inputs: the reference's readers of
// geological permeability files (read_set_perm_field, permeabilities.c:
// 494-668; read_layer_perm_field, :57-186; gaussian_permfield, :673-772)
// split into a host parse of the file and a device resample onto the
// simulation grid.
//
// The parse converts decimal text to doubles with strtod, as fscanf("%lf")
// does (both correctly rounded), and stores the geological cells in the
// reference's order and index ind(i, j, k) = i + nxg (j + nyg k)
// (solve_linearsystem_AMG.c:8-13).  The resample is one gather per
// simulation cell: the geological cell holding the cell centre,
// floor((i + 0.5) h / h_geo) per axis, evaluated with the reference's
// operations in double precision, so the fields are bit-identical.
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "solver.cuh"
#include "../../include/hmfem_permio.h"

namespace hm {
namespace {

// reads the whole file; numbers are whitespace-separated decimal text
int read_numbers(const char *path, long want, std::vector<double> &out)
{
    FILE *f = fopen(path, "rb");
    if (!f) {
        set_last_error("cannot open the permeability file", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    std::vector<char> text;
    char buf[1 << 16];
    size_t got;
    while ((got = fread(buf, 1, sizeof(buf), f)) > 0) text.insert(text.end(), buf, buf + got);
    fclose(f);
    text.push_back('\0');
    out.clear();
    out.reserve(want);
    const char *p = text.data();
    while ((long)out.size() < want) {
        char *end;
        errno = 0;
        const double v = strtod(p, &end);
        if (end == p) {
            set_last_error("permeability file: fewer values than the geological grid needs",
                           __FILE__, __LINE__);
            return HMFEM_E_ARG;
        }
        out.push_back(v);
        p = end;
    }
    return HMFEM_OK;
}

// floor(((i + 0.5) * h) / hg) as permeabilities.c:634-641 computes it,
// clamped into the geological grid (the reference's index never leaves it
// for a cell centre inside the domain)
__device__ __forceinline__ int geo_index(int i, double h, double hg, int ng)
{
    const double pos = __dmul_rn((double)i + 0.5, h);
    int g = (int)floor(__ddiv_rn(pos, hg));
    return g < 0 ? 0 : (g >= ng ? ng - 1 : g);
}

// variant 0: read_set_perm_field / gaussian_permfield (3-D);
// variant 1: read_layer_perm_field (one layer, plane k = 0 of the grid)
__global__ void k_resample(int variant, const double *__restrict__ GX,
                           const double *__restrict__ GY, const double *__restrict__ GZ,
                           int nxg, int nyg, int nzg, double hxg, double hyg, double hzg,
                           int nx, int ny, int nz, double hx, double hy, double hz,
                           double *KX, double *KY, double *KZ)
{
    const long nxy = (long)nx * ny;
    const long n = variant == 1 ? nxy : nxy * nz;
    for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < n;
         s += (long)gridDim.x * blockDim.x) {
        const int i = (int)(s % nx), j = (int)((s / nx) % ny), k = (int)(s / nxy);
        const int gi = geo_index(i, hx, hxg, nxg), gj = geo_index(j, hy, hyg, nyg);
        const int gk = variant == 1 ? 0 : geo_index(k, hz, hzg, nzg);
        const long g = gi + (long)nxg * (gj + (long)nyg * gk);
        KX[s] = GX[g];
        KY[s] = GY[g];
        KZ[s] = GZ[g];
    }
}

}  // namespace
}  // namespace hm

extern "C" {

int hmfem_read_spe(const char *path, int nxg, int nyg, int nzg, int layer, double *KXg,
                   double *KYg, double *KZg)
{
    if (!path || nxg < 1 || nyg < 1 || nzg < 1 || !KXg || !KYg || !KZg ||
        layer >= nzg)
        return HMFEM_E_ARG;
    const long ng = (long)nxg * nyg * nzg;
    std::vector<double> v;
    HM_CHECK(hm::read_numbers(path, 3 * ng, v));
    // permeabilities.c:541-611: three blocks (x, y, z), each k from the top
    // layer down, j, i ascending, stored at ind(nxg-1-i, nyg-1-j, k)
    double *dst[3] = {KXg, KYg, KZg};
    long q = 0;
    for (int c = 0; c < 3; c++)
        for (int k = nzg - 1; k >= 0; k--)
            for (int j = 0; j < nyg; j++)
                for (int i = 0; i < nxg; i++) {
                    const double bb = v[q++];
                    const long s2 = (nxg - i - 1) + (long)nxg * (nyg - j - 1);
                    if (layer < 0) dst[c][s2 + (long)nxg * nyg * k] = bb;
                    else if (k == layer) dst[c][s2] = c == 2 ? 1e-8 : bb;  // :150-163
                }
    return HMFEM_OK;
}

int hmfem_read_gaussian(const char *path, int nxg, int nyg, int nzg, double *Kg)
{
    if (!path || nxg < 1 || nyg < 1 || nzg < 1 || !Kg) return HMFEM_E_ARG;
    const long ng = (long)nxg * nyg * nzg;
    std::vector<double> v;
    HM_CHECK(hm::read_numbers(path, 3 * ng, v));
    // permeabilities.c:708-733: i, j, k loops, three columns, column 0 used
    long q = 0;
    for (int i = 0; i < nxg; i++)
        for (int j = 0; j < nyg; j++)
            for (int k = 0; k < nzg; k++) {
                Kg[i + (long)nxg * (j + (long)nyg * k)] = v[q];
                q += 3;
            }
    return HMFEM_OK;
}

int hmfem_resample_perm(int variant, const double *KXg, const double *KYg, const double *KZg,
                        int nxg, int nyg, int nzg, double Ix, double Iy, double Iz, int nx,
                        int ny, int nz, double *KX, double *KY, double *KZ, int mem)
{
    if (variant < 0 || variant > 2 || !KXg || !KYg || !KZg || !KX || !KY || !KZ ||
        nxg < 1 || nyg < 1 || nzg < 1 || nx < 1 || ny < 1 || nz < 1)
        return HMFEM_E_ARG;
    // the geological cell sizes of each reader: read_set_perm_field
    // (:538-540), read_layer_perm_field (:93-94, one layer), and
    // gaussian_permfield (:697-699, whose z size divides by the x count)
    const double hxg = Ix / (double)nxg, hyg = Iy / (double)nyg;
    const double hzg = variant == 2 ? Iz / (double)nxg : Iz / (double)nzg;
    const double hx = Ix / nx, hy = Iy / ny, hz = Iz / nz;   // main.c:163-165
    const long ng = (long)nxg * nyg * (variant == 1 ? 1 : nzg);
    const long n = (long)nx * ny * nz, nw = variant == 1 ? (long)nx * ny : n;
    cudaStream_t st;
    HM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    std::vector<void *> keep;
    const double *gx = KXg, *gy = KYg, *gz = KZg;
    double *ox = KX, *oy = KY, *oz = KZ;
    int rc = HMFEM_OK;
    auto dev = [&](size_t bytes) -> void * {
        void *p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
        keep.push_back(p);
        return p;
    };
    if (!mem) {
        double *g3[3];
        const double *h3[3] = {KXg, KYg, KZg};
        for (int a = 0; a < 3 && rc == HMFEM_OK; a++) {
            g3[a] = (double *)dev(sizeof(double) * ng);
            if (!g3[a]) { rc = HMFEM_E_CUDA; break; }
            cudaMemcpyAsync(g3[a], h3[a], sizeof(double) * ng, cudaMemcpyHostToDevice, st);
        }
        double *o3[3] = {nullptr, nullptr, nullptr};
        double *hout[3] = {KX, KY, KZ};
        for (int a = 0; a < 3 && rc == HMFEM_OK; a++) {
            o3[a] = (double *)dev(sizeof(double) * n);
            if (!o3[a]) { rc = HMFEM_E_CUDA; break; }
            // the layer reader writes plane 0 only: the rest keeps the
            // caller's values
            cudaMemcpyAsync(o3[a], hout[a], sizeof(double) * n, cudaMemcpyHostToDevice, st);
        }
        if (rc == HMFEM_OK) {
            gx = g3[0]; gy = g3[1]; gz = g3[2];
            ox = o3[0]; oy = o3[1]; oz = o3[2];
        }
    }
    if (rc == HMFEM_OK) {
        const long b = (nw + 255) / 256;
        hm::k_resample<<<(int)(b < 148L * 16 ? b : 148L * 16), 256, 0, st>>>(
            variant == 1 ? 1 : 0, gx, gy, gz, nxg, nyg, nzg, hxg, hyg, hzg, nx, ny, nz, hx,
            hy, hz, ox, oy, oz);
        HM_COUNT();
        if (!mem) {
            double *hout[3] = {KX, KY, KZ};
            const double *dsrc[3] = {ox, oy, oz};
            for (int a = 0; a < 3; a++)
                cudaMemcpyAsync(hout[a], dsrc[a], sizeof(double) * n, cudaMemcpyDeviceToHost, st);
        }
        cudaError_t e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) {
            hm::set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
            rc = HMFEM_E_CUDA;
        }
    } else {
        hm::set_last_error("out of device memory", __FILE__, __LINE__);
    }
    for (void *p : keep) cudaFree(p);
    cudaStreamDestroy(st);
    return rc;
}

}  // extern "C"
