// guess_ops.cu -- the data movement around the learned guess's convolutions,
// one pass over HBM each: input features, 2x2x2 average pooling, nearest
// upsampling fused with the skip concatenation, and the 1x1 head fused with
// the linear profile.  No counterpart in the reference.
//
// Activations are channel-blocked BF16 (C/8 slabs of the n cells, 8 channels
// per cell, 16 bytes): one thread moves one 16-byte cell of one slab.
#include <cuda_bf16.h>
#include <stdint.h>

#include "common.cuh"

namespace hm {

namespace {

constexpr int kOpsThreads = 256;

inline int ops_grid(long work)
{
    long g = (work + kOpsThreads - 1) / kOpsThreads;
    return (int)(g < 1 ? 1 : g);
}

// slab 0: (log10 K + 14) / 2, the conduit mask, the Dirichlet face mask
// (+1 at x = 0, -1 at x = nx-1), five zeros; slab 1: zeros
__global__ void k_features(const double *__restrict__ K, const unsigned char *__restrict__ mask,
                           int nx, long n, __nv_bfloat16 *__restrict__ out)
{
    const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int x = (int)(s % nx);
    __nv_bfloat16 v[8];
    v[0] = __float2bfloat16((float)((log10(K[s]) + 14.0) * 0.5));
    v[1] = __float2bfloat16(mask ? (float)mask[s] : 0.f);
    v[2] = __float2bfloat16((x == 0 ? 1.f : 0.f) - (x == nx - 1 ? 1.f : 0.f));
#pragma unroll
    for (int i = 3; i < 8; i++) v[i] = __float2bfloat16(0.f);
    ((uint4 *)out)[s] = *(uint4 *)v;
    ((uint4 *)out)[n + s] = make_uint4(0, 0, 0, 0);
}

// out[k][coarse cell] = mean of the 8 fine cells (FP32 sum, BF16 result)
__global__ void k_pool2(const __nv_bfloat16 *__restrict__ x, int S, int nx, int ny, int nz,
                        __nv_bfloat16 *__restrict__ out)
{
    const int cx = nx / 2, cy = ny / 2, cz = nz / 2;
    const long nc = (long)cx * cy * cz, nf = (long)nx * ny * nz;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)S * nc) return;
    const int k = (int)(i / nc);
    const long c = i - (long)k * nc;
    const int X = (int)(c % cx), Y = (int)((c / cx) % cy), Z = (int)(c / ((long)cx * cy));
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int d = 0; d < 8; d++) {
        const long f = (2 * X + (d & 1)) + (long)nx * ((2 * Y + ((d >> 1) & 1)) +
                                                       (long)ny * (2 * Z + (d >> 2)));
        const uint4 q = ((const uint4 *)x)[(long)k * nf + f];
        const __nv_bfloat16 *e = (const __nv_bfloat16 *)&q;
#pragma unroll
        for (int j = 0; j < 8; j++) acc[j] += __bfloat162float(e[j]);
    }
    __nv_bfloat16 o[8];
#pragma unroll
    for (int j = 0; j < 8; j++) o[j] = __float2bfloat16(acc[j] * 0.125f);
    ((uint4 *)out)[i] = *(uint4 *)o;
}

// out = [nearest-upsampled coarse (Sa slabs) | skip (Sb slabs)] on the fine grid
__global__ void k_up2_cat(const __nv_bfloat16 *__restrict__ coarse, int Sa,
                          const __nv_bfloat16 *__restrict__ skip, int Sb, int nx, int ny, int nz,
                          __nv_bfloat16 *__restrict__ out)
{
    const long nf = (long)nx * ny * nz;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)(Sa + Sb) * nf) return;
    const int k = (int)(i / nf);
    const long f = i - (long)k * nf;
    uint4 q;
    if (k < Sa) {
        const int cx = nx / 2, cy = ny / 2, cz = nz / 2;
        const int x = (int)(f % nx), y = (int)((f / nx) % ny), z = (int)(f / ((long)nx * ny));
        const long c = (x / 2) + (long)cx * ((y / 2) + (long)cy * (z / 2));
        q = ((const uint4 *)coarse)[(long)k * cx * cy * cz + c];
    } else {
        q = ((const uint4 *)skip)[(long)(k - Sa) * nf + f];
    }
    ((uint4 *)out)[i] = q;
}

// gradient of k_up2_cat's upsampled part: g_coarse[k][c] = sum of the 8 fine
// cells' gradients (FP32 sum, BF16 result)
__global__ void k_up2_grad(const __nv_bfloat16 *__restrict__ g, int Sa, int nx, int ny, int nz,
                           __nv_bfloat16 *__restrict__ out)
{
    const int cx = nx / 2, cy = ny / 2, cz = nz / 2;
    const long nc = (long)cx * cy * cz, nf = (long)nx * ny * nz;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)Sa * nc) return;
    const int k = (int)(i / nc);
    const long c = i - (long)k * nc;
    const int X = (int)(c % cx), Y = (int)((c / cx) % cy), Z = (int)(c / ((long)cx * cy));
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int d = 0; d < 8; d++) {
        const long f = (2 * X + (d & 1)) + (long)nx * ((2 * Y + ((d >> 1) & 1)) +
                                                       (long)ny * (2 * Z + (d >> 2)));
        const uint4 q = ((const uint4 *)g)[(long)k * nf + f];
        const __nv_bfloat16 *e = (const __nv_bfloat16 *)&q;
#pragma unroll
        for (int j = 0; j < 8; j++) acc[j] += __bfloat162float(e[j]);
    }
    __nv_bfloat16 o[8];
#pragma unroll
    for (int j = 0; j < 8; j++) o[j] = __float2bfloat16(acc[j]);
    ((uint4 *)out)[i] = *(uint4 *)o;
}

// p[s] = 1 - (x + 1/2)/nx + (sum_c x[c] w[c] + b): the 1x1 head (FP32) on the
// linear profile, FP64 out
__global__ void k_head_profile(const __nv_bfloat16 *__restrict__ x, int S,
                               const float *__restrict__ w, const float *__restrict__ b, int nx,
                               long n, double *__restrict__ p)
{
    const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float acc = b[0];
    for (int k = 0; k < S; k++) {
        const uint4 q = ((const uint4 *)x)[(long)k * n + s];
        const __nv_bfloat16 *e = (const __nv_bfloat16 *)&q;
#pragma unroll
        for (int j = 0; j < 8; j++) acc += __bfloat162float(e[j]) * __ldg(w + 8 * k + j);
    }
    const int xi = (int)(s % nx);
    p[s] = 1.0 - (xi + 0.5) / nx + (double)acc;
}

}  // namespace

}  // namespace hm

extern "C" {

int hmfem_guess_features(const double *K, const unsigned char *mask, int nx, int ny, int nz,
                         void *out, void *stream)
{
    if (!K || !out || nx < 1 || ny < 1 || nz < 1) return HMFEM_E_ARG;
    const long n = (long)nx * ny * nz;
    hm::k_features<<<hm::ops_grid(n), hm::kOpsThreads, 0, (cudaStream_t)stream>>>(
        K, mask, nx, n, (__nv_bfloat16 *)out);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int hmfem_guess_pool2(const void *x, int slabs, int nx, int ny, int nz, void *out, void *stream)
{
    if (!x || !out || slabs < 1 || nx < 2 || ny < 2 || nz < 2 || (nx | ny | nz) & 1) {
        hm::set_last_error("guess pool2: needs even grid dimensions", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    const long work = (long)slabs * (nx / 2) * (ny / 2) * (nz / 2);
    hm::k_pool2<<<hm::ops_grid(work), hm::kOpsThreads, 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16 *)x, slabs, nx, ny, nz, (__nv_bfloat16 *)out);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int hmfem_guess_up2_cat(const void *coarse, int slabs_a, const void *skip, int slabs_b, int nx,
                        int ny, int nz, void *out, void *stream)
{
    if (!coarse || !out || slabs_a < 1 || slabs_b < 0 || (slabs_b > 0 && !skip) || nx < 2 ||
        ny < 2 || nz < 2 || (nx | ny | nz) & 1) {
        hm::set_last_error("guess up2_cat: needs even fine-grid dimensions", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    const long work = (long)(slabs_a + slabs_b) * nx * ny * nz;
    hm::k_up2_cat<<<hm::ops_grid(work), hm::kOpsThreads, 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16 *)coarse, slabs_a, (const __nv_bfloat16 *)skip, slabs_b, nx, ny,
        nz, (__nv_bfloat16 *)out);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int hmfem_guess_up2_grad(const void *g, int slabs_a, int nx, int ny, int nz, void *out,
                         void *stream)
{
    if (!g || !out || slabs_a < 1 || nx < 2 || ny < 2 || nz < 2 || (nx | ny | nz) & 1) {
        hm::set_last_error("guess up2_grad: needs even fine-grid dimensions", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    const long work = (long)slabs_a * (nx / 2) * (ny / 2) * (nz / 2);
    hm::k_up2_grad<<<hm::ops_grid(work), hm::kOpsThreads, 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16 *)g, slabs_a, nx, ny, nz, (__nv_bfloat16 *)out);
    HM_LAUNCHED();
    return HMFEM_OK;
}

int hmfem_guess_head_profile(const void *x, int slabs, const float *w, const float *b, int nx,
                             int ny, int nz, double *p, void *stream)
{
    if (!x || !w || !b || !p || slabs < 1 || nx < 1 || ny < 1 || nz < 1) return HMFEM_E_ARG;
    const long n = (long)nx * ny * nz;
    hm::k_head_profile<<<hm::ops_grid(n), hm::kOpsThreads, 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16 *)x, slabs, w, b, nx, n, p);
    HM_LAUNCHED();
    return HMFEM_OK;
}

}  // extern "C"
