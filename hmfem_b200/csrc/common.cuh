// common.cuh -- shared device helpers for the hmfem B200 kernels (sm_100a).
#pragma once
#include <atomic>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/hmfem_gpu.h"

namespace hm {

constexpr int kSlice = 32;          // SELL slice height = warp width
constexpr int kRedBlocks = 148 * 6; // max blocks of a grid-stride reduction (6 resident per SM at 40 registers)

// Status plumbing: every host entry returns an hmfem status code.
#define HM_CUDA(call)                                                         \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) {                                              \
            hm::set_last_error(cudaGetErrorString(e_), __FILE__, __LINE__);   \
            return HMFEM_E_CUDA;                                              \
        }                                                                     \
    } while (0)
#define HM_CHECK(call)                                                        \
    do {                                                                      \
        int s_ = (call);                                                      \
        if (s_ != HMFEM_OK) return s_;                                        \
    } while (0)

void set_last_error(const char *msg, const char *file, int line);

// Number of this library's kernels launched (captured launches count once
// at capture; graph replays add the captured count).
// g_nlaunch counts every thread's launches; t_nlaunch the calling host
// thread's (what a graph capture on this thread recorded)
extern std::atomic<unsigned long long> g_nlaunch;
extern thread_local unsigned long long t_nlaunch;
#define HM_COUNT() (++hm::g_nlaunch, ++hm::t_nlaunch)
#define HM_LAUNCHED()                                                         \
    do {                                                                      \
        HM_COUNT();                                                           \
        HM_CUDA(cudaGetLastError());                                          \
    } while (0)

// Phase timing for diagnostics (HMFEM_VERBOSE=1 or options.verbose): syncs
// the stream and prints the host time since the previous mark to stderr.
extern int g_verbose;
void phase_mark(const char *label, cudaStream_t st);
#define HM_PHASE(label, st)                                                   \
    do {                                                                      \
        if (hm::g_verbose) hm::phase_mark(label, st);                         \
    } while (0)

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b)
{
    return (a + b - 1) / b;
}

// Non-contracted double arithmetic: keeps the reference's rounding where the
// setup results are required to match it bit for bit.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic grid reduction: every block leaves its partial in
// part[blockIdx.x]; the last block to arrive sums the partials in a fixed
// order and calls fin(total).  `ticket` must be zero on entry and is reset.
// blockDim.x must be a multiple of 32 and <= 1024.
template <typename Fin>
__device__ void grid_reduce_sum(double v, double *part, unsigned *ticket,
                                Fin fin)
{
    __shared__ double s_w[32];
    __shared__ bool s_last;
    __syncthreads();  // s_w may still be read by a previous reduction
    v = warp_sum(v);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) s_w[wid] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += s_w[w];
        part[blockIdx.x] = t;
        __threadfence();
        unsigned k = atomicAdd(ticket, 1u);
        s_last = (k == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double t = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
        t += ((volatile double *)part)[b];
    t = warp_sum(t);
    if (lane == 0) s_w[wid] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += s_w[w];
        *ticket = 0;
        fin(tot);
    }
}

// Bitonic sort of m (power of two) ints in shared memory by one warp.
__device__ inline void warp_bitonic_sort(int *a, int m)
{
    const int lane = threadIdx.x & 31;
    for (int k = 2; k <= m; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < m; i += 32) {
                int ixj = i ^ j;
                if (ixj > i) {
                    int x = a[i], y = a[ixj];
                    bool up = (i & k) == 0;
                    if ((x > y) == up) { a[i] = y; a[ixj] = x; }
                }
            }
            __syncwarp();
        }
    }
}

// Same, for a whole block (blockDim.x threads).
__device__ inline void block_bitonic_sort(int *a, int m)
{
    for (int k = 2; k <= m; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < m; i += blockDim.x) {
                int ixj = i ^ j;
                if (ixj > i) {
                    int x = a[i], y = a[ixj];
                    bool up = (i & k) == 0;
                    if ((x > y) == up) { a[i] = y; a[ixj] = x; }
                }
            }
            __syncthreads();
        }
    }
}

__host__ __device__ inline int next_pow2(int v)
{
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

}  // namespace hm
