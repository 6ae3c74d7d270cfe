// cycle.cuh -- arithmetic helpers shared by the V-cycle translation units.
#pragma once
#include "solver.cuh"

namespace hm {

template <class T> struct Ar;
template <> struct Ar<double> {
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return a / b; }
};
template <> struct Ar<float> {
    static __device__ __forceinline__ float mul(float a, float b) { return a * b; }
    static __device__ __forceinline__ float add(float a, float b) { return a + b; }
    static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
    static __device__ __forceinline__ float div(float a, float b) { return a / b; }
};

__device__ __forceinline__ double ld(const double *p, long long i) { return p[i]; }
__device__ __forceinline__ float ld(const float *p, long long i) { return __ldg(p + i); }
__device__ __forceinline__ float ld(const __nv_bfloat16 *p, long long i) { return __bfloat162float(p[i]); }

__device__ __forceinline__ bool finished(const Ctl *c) { return c && *(volatile const int *)&c->done; }

#define GRID_STRIDE(r, n)                                                     \
    for (long r = blockIdx.x * (long)blockDim.x + threadIdx.x; r < (n);       \
         r += (long)gridDim.x * blockDim.x)

// The first Jacobi iterate from zero, u = (w f) D^-1 (device_jacobi 3-arg,
// device_amg.h:35-42), written by the kernel that produces f (restriction,
// demotion, the CG residual update) so the pre-smoother reads u once
// instead of recomputing it from f and D^-1 at every neighbour.  u ==
// nullptr: the level is not Jacobi-smoothed.
template <class T> struct Seed {
    T *u;
    const T *d;
    T w;
    __device__ __forceinline__ void put(long i, T f) const
    {
        if (u) u[i] = Ar<T>::mul(Ar<T>::mul(w, f), d[i]);
    }
};

// sigma = (C r, r) once the preconditioner is applied (pcg.h:66-67, and
// 46-47 on the first application); run by the last block of the fused
// reduction.
__device__ __forceinline__ void sigma_finish(Ctl *ctl, double s, int first)
{
    if (s < 0.0) s = fabs(s);
    if (!(s == s) || isinf(s)) { ctl->status = HMFEM_E_BREAKDOWN; ctl->done = 1; }
    if (first) {
        ctl->sigma_first = s == 0.0 ? 1.0 : s;
        ctl->sigma_last = s;
        ctl->beta = 0.0;
    } else {
        ctl->beta = s / ctl->sigma_last;
    }
    ctl->sigma = s;
    if (ctl->stop_rule == 1 && s / ctl->sigma_first <= ctl->tol2) ctl->done = 1;
}

// alpha = sigma / (s, A s) after the CG's SpMV (pcg.h:59-63)
__device__ __forceinline__ void tau_finish(Ctl *ctl, double t)
{
    if (t < 0.0) t = fabs(t);
    ctl->tau = t;
    if (!(t > 0.0) || isinf(t)) { ctl->status = HMFEM_E_BREAKDOWN; ctl->done = 1; return; }
    ctl->alpha = ctl->sigma / t;
}

// (r, r) and (b, b) of a residual kernel; init: 1 = start of the solve,
// 0 = convergence check (residual replacement), 2 = report only
__device__ __forceinline__ void trr_finish(Ctl *ctl, double s, int init)
{
    ctl->trr = s;
    if (init == 2) return;
    ctl->rr = s;
    if (init == 1) {
        ctl->iters = 0;
        if (s <= ctl->tol2 * ctl->bb && ctl->stop_rule == 0) ctl->done = 1;
    } else {
        ctl->check = 0;
        if (s <= ctl->tol2 * ctl->bb) ctl->done = 1;
    }
}

}  // namespace hm
