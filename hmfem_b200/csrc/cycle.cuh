// cycle.cuh -- arithmetic helpers shared by the V-cycle translation units.
#pragma once
#include <utility>
#include <vector>

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

// Programmatic dependent launch: every solve-phase kernel is launched with
// launch_pdl, so the next kernel in the stream can be scheduled while this
// one drains; each such kernel calls pdl_wait() before touching memory its
// predecessors wrote (griddepcontrol.wait returns once they completed and
// their writes are visible; it returns at once for a plain launch), then
// pdl_trigger() to let its own successor be scheduled early.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;"); }
#define PDL_ENTRY()   \
    do {              \
        pdl_wait();   \
        pdl_trigger(); \
    } while (0)

extern int g_pdl;  // 0: plain stream order (HMFEM_PDL=0)
// set while capturing into a conditional node's body (plain stream order
// there: such bodies hold kernel nodes without programmatic edges)
extern thread_local int t_nopdl;

// Per-launch timing of the solve phase (hmfem_profile_iteration): while
// t_kprof is set on a host thread, launch_pdl brackets each of its launches
// with two events and records the kernel and t_klevel (the V-cycle level
// being worked on, -1 for the CG's level-0 vector work).
struct KRec {
    const void *fn;
    int level;
    cudaEvent_t e0, e1;
};
extern thread_local std::vector<KRec> *t_kprof;
extern thread_local int t_klevel;

template <class... KArgs, class... Args>
inline void launch_pdl(void (*kernel)(KArgs...), int grid, int block, cudaStream_t st,
                       Args &&...args)
{
    KRec rec{(const void *)kernel, t_klevel, nullptr, nullptr};
    if (t_kprof) {
        cudaEventCreate(&rec.e0);
        cudaEventCreate(&rec.e1);
        cudaEventRecord(rec.e0, st);
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = (g_pdl && !t_nopdl) ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);  // error: cudaGetLastError
    if (t_kprof) {
        cudaEventRecord(rec.e1, st);
        t_kprof->push_back(rec);
    }
}

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

// The FP32 cycle's right-hand side: the CG kernels that write r also write
// f = (float) r and its seed (f == nullptr: FP64 cycle, nothing to do).
struct Demote {
    float *f;
    Seed<float> sd;
    __device__ __forceinline__ void put(long i, double r) const
    {
        if (f) {
            const float fi = (float)r;
            f[i] = fi;
            sd.put(i, fi);
        }
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

// sigma = (z, r) of the CG's preconditioned residual z (and, flexible,
// rz = (z, A s_old)): breakdown test, beta, the reference stop rule; run by
// the last block of the reduction (k_finish_z, and the level-0
// prolongation that forms z when it does the dots itself).
__device__ __forceinline__ void zdots_finish(Ctl *ctl, double s, int first, int flexible)
{
    if (!(s == s) || isinf(s)) { ctl->status = HMFEM_E_BREAKDOWN; ctl->done = 1; }
    if (!flexible && s < 0.0) s = fabs(s);   // pcg.h:47, 68
    if (first) {
        ctl->sigma_first = s == 0.0 ? 1.0 : fabs(s);
        ctl->sigma_last = s;
        ctl->beta = 0.0;
    } else if (flexible) {
        ctl->beta = -ctl->rz_old / ctl->tau;
    } else {
        ctl->beta = s / ctl->sigma_last;
    }
    ctl->sigma = s;
    if (ctl->stop_rule == 1 && fabs(s) / ctl->sigma_first <= ctl->tol2) ctl->done = 1;
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
