// device_abi.cu -- the reference's device layer (toolbox/lib/toolbox.cu),
// same fifteen extern "C" entry points, same argument meaning, same launch
// stream (the legacy default stream), for toolbox host code that drives
// device_vector / device_amg_solver / device_conjugate_gradient.  Kernels
// are this project's: grid-stride loops sized to the B200's 148 SMs, no
// texture references (which CUDA 12 removed), and FP64 arithmetic without
// FMA contraction so results match the reference's CPU formulas.  Like the
// reference's, these return nothing; every launch is counted in
// hmfem_launch_count().
#include "hm.cuh"

namespace {

using hm::dadd;
using hm::dmul;
using hm::dsub;

constexpr int kL = 32;  // SELL slice height of the reference (toolbox.h:67)

inline int grid(unsigned long n)
{
    unsigned long b = (n + 255) / 256;
    if (b < 1) b = 1;
    return (int)(b < 148ul * 16 ? b : 148ul * 16);
}

#define STRIDE(i, n)                                                          \
    for (unsigned long i = blockIdx.x * (unsigned long)blockDim.x + threadIdx.x; \
         i < (n); i += (unsigned long)gridDim.x * blockDim.x)

__global__ void k_add_scale(double *x, const double *y, double s, unsigned m)
{ STRIDE(i, m) x[i] = dadd(x[i], dmul(y[i], s)); }
__global__ void k_sub_scale(double *x, const double *y, double s, unsigned m)
{ STRIDE(i, m) x[i] = dsub(x[i], dmul(y[i], s)); }
__global__ void k_scale_add(double *x, const double *y, double s, unsigned m)
{ STRIDE(i, m) x[i] = dadd(dmul(x[i], s), y[i]); }
__global__ void k_set_mul(double *x, const double *y, const double *z, double w, unsigned m)
{ STRIDE(i, m) x[i] = dmul(dmul(w, y[i]), z[i]); }
__global__ void k_add_mul(double *x, const double *y, const double *z, double w, unsigned m)
{ STRIDE(i, m) x[i] = dadd(x[i], dmul(dmul(w, y[i]), z[i])); }
__global__ void k_diag(double *x, const double *y, const double *z, unsigned m)
{ STRIDE(i, m) x[i] = dmul(y[i], z[i]); }
__global__ void k_sub(const double *x, double *y, unsigned m)
{ STRIDE(i, m) y[i] = dsub(y[i], x[i]); }
__global__ void k_add(const double *x, double *y, unsigned m)
{ STRIDE(i, m) y[i] = dadd(y[i], x[i]); }
__global__ void k_rsb(const double *x, double *y, unsigned m)
{ STRIDE(i, m) y[i] = dsub(x[i], y[i]); }
__global__ void k_com_snd(const double *x, double *svec, const int *rcom, unsigned n)
{ STRIDE(i, n) svec[i] = x[rcom[i]]; }
__global__ void k_com_rcv(double *x, const double *rvec, const int *rcom, unsigned n)
{ STRIDE(i, n) atomicAdd(x + rcom[i], rvec[i]); }

// Per-block partial dot products into w[0..m): the contract of
// device_binary_operator.h:29-49 (the host sums the m partials).
__global__ void k_vector_product(const double *u, const double *v, double *w,
                                 unsigned n)
{
    __shared__ double acc[32];
    double s = 0.0;
    for (unsigned j = blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += blockDim.x * gridDim.x)
        s += u[j] * v[j];
    s = hm::warp_sum(s);
    if ((threadIdx.x & 31) == 0) acc[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += acc[q];
        w[blockIdx.x] = t;
    }
}

// SELL-32 rows addressed by dsp[j] with stride L (device_amg.h:72-86).
__global__ void k_linear_operator(const int *cnt, const int *dsp, const int *col,
                                  const double *ele, int n, const double *u,
                                  double *v)
{
    STRIDE(j, (unsigned long)n) {
        long a = dsp[j], e = a + (long)kL * cnt[j];
        double s = 0.0;
        for (long i = a; i < e; i += kL) s = dadd(s, dmul(ele[i], u[col[i]]));
        v[j] = s;
    }
}

__global__ void k_jacobi(const int *cnt, const int *dsp, const int *col,
                         const double *ele, int n, const double *f,
                         const double *u, double *v)
{
    STRIDE(j, (unsigned long)n) {
        long a = dsp[j], e = a + (long)kL * cnt[j];
        double s = f[j];
        for (long i = a; i < e; i += kL) s = dsub(s, dmul(ele[i], u[col[i]]));
        v[j] = s;
    }
}

__global__ void k_matrix_conversion(const int *acnt, const int *adsp, int *acol,
                                    double *aele, const int *tdsp,
                                    const int *tcol, const double *tele, int n)
{
    STRIDE(j, (unsigned long)n) {
        long t = tdsp[j], k = adsp[j];
        for (int q = 0; q < acnt[j]; q++, k += kL) {
            acol[k] = tcol[t + q];
            aele[k] = tele[t + q];
        }
    }
}

}  // namespace

extern "C" {

void _device_add_scale(double *x, double *y, double s, unsigned int m)
{ if (m) { k_add_scale<<<grid(m), 256>>>(x, y, s, m); HM_COUNT(); } }
void _device_sub_scale(double *x, double *y, double s, unsigned int m)
{ if (m) { k_sub_scale<<<grid(m), 256>>>(x, y, s, m); HM_COUNT(); } }
void _device_scale_add(double *x, double *y, double s, unsigned int m)
{ if (m) { k_scale_add<<<grid(m), 256>>>(x, y, s, m); HM_COUNT(); } }
void _device_vector_product(double *x, double *y, double *z, unsigned int n,
                            unsigned int m)
{ if (m) { k_vector_product<<<m, 256>>>(x, y, z, n); HM_COUNT(); } }
void _device_linear_operator(int *cnt, int *dsp, int *col, double *ele, int l,
                             int m, int n, double *u, double *v)
{
    (void)l; (void)m;
    if (n > 0) { k_linear_operator<<<grid(n), 256>>>(cnt, dsp, col, ele, n, u, v); HM_COUNT(); }
}
void _device_jacobi(int *cnt, int *dsp, int *col, double *ele, int l, int n,
                    double *f, double *u, double *v)
{
    (void)l;
    if (n > 0) { k_jacobi<<<grid(n), 256>>>(cnt, dsp, col, ele, n, f, u, v); HM_COUNT(); }
}
void _device_set_mul(double *x, double *y, double *z, double omega, unsigned int m)
{ if (m) { k_set_mul<<<grid(m), 256>>>(x, y, z, omega, m); HM_COUNT(); } }
void _device_add_mul(double *x, double *y, double *z, double omega, unsigned int m)
{ if (m) { k_add_mul<<<grid(m), 256>>>(x, y, z, omega, m); HM_COUNT(); } }
void _device_diagonal_solver(double *x, double *y, double *z, unsigned int m)
{ if (m) { k_diag<<<grid(m), 256>>>(x, y, z, m); HM_COUNT(); } }
void _device_com_snd(double *x, double *svec, int *rcom, unsigned int n)
{ if (n) { k_com_snd<<<grid(n), 256>>>(x, svec, rcom, n); HM_COUNT(); } }
void _device_com_rcv(double *x, double *rvec, int *rcom, unsigned int n)
{ if (n) { k_com_rcv<<<grid(n), 256>>>(x, rvec, rcom, n); HM_COUNT(); } }
void _device_sub(double *x, double *y, unsigned int m)
{ if (m) { k_sub<<<grid(m), 256>>>(x, y, m); HM_COUNT(); } }
void _device_add(double *x, double *y, unsigned int m)
{ if (m) { k_add<<<grid(m), 256>>>(x, y, m); HM_COUNT(); } }
void _device_rsb(double *x, double *y, unsigned int m)
{ if (m) { k_rsb<<<grid(m), 256>>>(x, y, m); HM_COUNT(); } }
void _device_matrix_conversion(int *acnt, int *adsp, int *acol, double *aele,
                               int *tdsp, int *tcol, double *tele, int n)
{
    if (n > 0) { k_matrix_conversion<<<grid(n), 256>>>(acnt, adsp, acol, aele, tdsp, tcol, tele, n); HM_COUNT(); }
}

}  // extern "C"
