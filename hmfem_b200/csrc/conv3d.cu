// conv3d.cu -- 3x3x3 convolutions of the learned initial guess on the
// 5th-generation tensor cores (tcgen05, sm_100a): BF16 operands, FP32
// accumulation in tensor memory.  No counterpart in the reference.
//
// Activations are channels-last (cell s = x + nx (y + ny z), C contiguous
// BF16 values per cell); weights are [27 taps][Cout][Cin] with tap
// t = 9 (dz+1) + 3 (dy+1) + (dx+1); zero padding outside the grid.
//
// Forward (and, with flipped / transposed weights, the data gradient) is an
// implicit GEMM: D[m][n] = sum_tap sum_ci A_tap[m][ci] B_tap[n][ci] with m a
// run of 128 consecutive cells, n the output channel, A_tap the input at
// cell m shifted by the tap.  Per tap the 128 x Cin A tile and the Cout x
// Cin B tile are gathered by the CTA's threads into shared memory in the
// canonical K-major layout without swizzle (8-row x 16-byte core matrices:
// element (row r, k) at (k/8)*LBO + r*16 + (k%8)*2 bytes, LBO = rows*16,
// SBO = 128), then one thread issues Cin/16 tcgen05.mma (M=128, N=Cout,
// K=16) into a TMEM accumulator of Cout FP32 columns (TMEM lane = row m).
// Two buffers alternate between taps: the MMAs of tap t run while tap t+1
// is gathered; tcgen05.commit on a per-buffer mbarrier says when a buffer
// may be overwritten.  The epilogue reads TMEM with tcgen05.ld (each warp
// its 32 lanes), adds the bias, applies ReLU and stores BF16.
//
// Weight gradient: D[m = co][n = ci] = sum_cell dY[cell][co] X[cell+off][ci]
// per tap, the cells being the K dimension: a CTA takes one tap and a range
// of cells, stages dY^T (Cout rows, zero-padded to M = 128) and the shifted
// X^T (Cin rows) K-major in shared memory, accumulates in TMEM, and adds its
// partial [Cout][Cin] block into the FP32 gradient with atomics.
//
// Every mbarrier wait is bounded: on a timeout the kernel flags err, waits
// (bounded again) for its MMAs in flight, frees its TMEM and returns.
#include <cuda_bf16.h>
#include <stdint.h>

#include "common.cuh"

namespace hm {

namespace {

constexpr unsigned kWaitPolls = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, K-major without swizzle: start address,
// leading-dimension byte offset (between the two 8-element K halves of one
// MMA), stride byte offset (between 8-row groups), version 1 (sm_100).
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem, uint64_t da, uint64_t db,
                                          uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t *mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *m)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(m)));
}

__device__ __forceinline__ bool mbar_test(uint64_t *m, unsigned parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(m)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait for the phase with this parity to complete
__device__ __forceinline__ bool mbar_wait(uint64_t *m, unsigned parity)
{
    for (unsigned i = 0; i < kWaitPolls; i++) {
        if (mbar_test(m, parity)) return true;
        if (i > 64) __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void fence_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_before_sync()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_after_sync()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// TMEM allocation by warp 0 (whole warp), address left in *slot
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr),
                 "r"(ncols));
}

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
          "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
          "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__host__ __device__ constexpr int tmem_cols(int n)
{
    return n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : 256;
}

// ---- forward / data gradient ----------------------------------------------

// Taps gathered per stage (one barrier and one commit per stage) and
// whether all 27 taps of the weights stay resident in shared memory.
template <int CIN, int COUT>
struct FwdSmem {
    static constexpr int kStage = (24 * 1024) / (CIN * 256) < 1 ? 1
                                : (24 * 1024) / (CIN * 256) > 9 ? 9
                                : (24 * 1024) / (CIN * 256);
    static constexpr bool kWRes = 27 * COUT * CIN * 2 <= 56 * 1024;
    static constexpr int kATap = CIN * 256;       // 128 rows x CIN x 2 B
    static constexpr int kBTap = COUT * CIN * 2;  // COUT rows x CIN x 2 B
    static constexpr int kA = kStage * kATap;     // one A buffer
    static constexpr int kB = kWRes ? 27 * kBTap : kStage * kBTap;
    static constexpr int kBBufs = kWRes ? 1 : 2;
    static constexpr int kBytes = 2 * kA + kBBufs * kB + 64;
};

// B tile of one tap into shared memory (K-major: row n = output channel)
template <int CIN, int COUT>
__device__ __forceinline__ void stage_weights(const __nv_bfloat16 *__restrict__ w, int tap,
                                              unsigned char *dst, int tid)
{
    constexpr int ACH = CIN / 8;
    const uint4 *wt = (const uint4 *)(w + (long)tap * COUT * CIN);
    for (int i = tid; i < COUT * ACH; i += 128) {
        const int row = i / ACH, c = i % ACH;
        *(uint4 *)(dst + c * (COUT * 16) + row * 16) = wt[row * ACH + c];
    }
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(128)
k_conv3d(const __nv_bfloat16 *__restrict__ in, const __nv_bfloat16 *__restrict__ w,
         const float *__restrict__ bias, __nv_bfloat16 *__restrict__ out, int nx, int ny,
         int nz, int relu, int *err)
{
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 256, "channel counts");
    extern __shared__ __align__(128) unsigned char smem[];
    using S = FwdSmem<CIN, COUT>;
    constexpr int ST = S::kStage;
    unsigned char *abuf = smem, *bbuf = smem + 2 * S::kA;
    uint64_t *mbar = (uint64_t *)(smem + 2 * S::kA + S::kBBufs * S::kB);
    uint32_t *tslot = (uint32_t *)(mbar + 2);
    constexpr int NCOL = tmem_cols(COUT);
    constexpr uint32_t IDESC = idesc_bf16(128, COUT);
    constexpr int ACH = CIN / 8;  // 16-byte chunks per row

    const int tid = threadIdx.x, warp = tid >> 5;
    const long nxy = (long)nx * ny, n = nxy * nz;
    const long ntiles = (n + 127) / 128;
    if (tid == 0) {
        mbar_init(&mbar[0]);
        mbar_init(&mbar[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (S::kWRes)  // all taps' weights, once per CTA
        for (int t = 0; t < 27; t++) stage_weights<CIN, COUT>(w, t, bbuf + t * S::kBTap, tid);
    if (warp == 0) tmem_alloc(tslot, NCOL);
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tslot;
    unsigned parity[2] = {0u, 0u};
    int pending[2] = {0, 0};
    bool ok = true;

    for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const long m = tile * 128 + tid;
        const bool valid = m < n;
        const int x = valid ? (int)(m % nx) : 0, y = valid ? (int)((m / nx) % ny) : 0,
                  z = valid ? (int)(m / nxy) : 0;
        int stage = 0;
        for (int t0 = 0; t0 < 27 && ok; t0 += ST, stage++) {
            const int b = stage & 1;
            const int nt = 27 - t0 < ST ? 27 - t0 : ST;
            if (pending[b]) {  // the MMAs that read buffer b are done
                ok = mbar_wait(&mbar[b], parity[b]);
                parity[b] ^= 1u;
                pending[b] = 0;
                ok = __syncthreads_and(ok);
                if (!ok) break;
            }
            unsigned char *a = abuf + b * S::kA;
            for (int j = 0; j < nt; j++) {
                const int tap = t0 + j;
                const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
                const int xx = x + dx, yy = y + dy, zz = z + dz;
                const bool in_grid = valid && xx >= 0 && xx < nx && yy >= 0 && yy < ny &&
                                     zz >= 0 && zz < nz;
                const uint4 *src =
                    (const uint4 *)(in + (xx + (long)yy * nx + (long)zz * nxy) * CIN);
#pragma unroll
                for (int c = 0; c < ACH; c++) {
                    const uint4 v = in_grid ? src[c] : make_uint4(0, 0, 0, 0);
                    *(uint4 *)(a + j * S::kATap + c * 2048 + tid * 16) = v;
                }
                if (!S::kWRes)
                    stage_weights<CIN, COUT>(w, tap, bbuf + b * S::kB + j * S::kBTap, tid);
            }
            fence_async_smem();
            __syncthreads();
            if (tid == 0) {
                tc_after_sync();
                for (int j = 0; j < nt; j++) {
                    const int tap = t0 + j;
                    const uint32_t sa = smem_u32(a + j * S::kATap);
                    const uint32_t sb = smem_u32(S::kWRes ? bbuf + tap * S::kBTap
                                                          : bbuf + b * S::kB + j * S::kBTap);
#pragma unroll
                    for (int kk = 0; kk < CIN / 16; kk++) {
                        const uint64_t da = kmajor_desc(sa + kk * 2 * 2048, 2048, 128);
                        const uint64_t db =
                            kmajor_desc(sb + kk * 2 * (COUT * 16), COUT * 16, 128);
                        umma_bf16(tmem, da, db, IDESC, (tap | kk) != 0);
                    }
                }
                umma_commit(&mbar[b]);
            }
            pending[b] = 1;
        }
        if (!ok) break;
        // the last commit covers every MMA issued before it
        for (int b = 0; b < 2; b++) {
            if (pending[b]) {
                ok = ok && mbar_wait(&mbar[b], parity[b]);
                parity[b] ^= 1u;
                pending[b] = 0;
            }
        }
        ok = __syncthreads_and(ok);
        if (!ok) break;
        tc_after_sync();
        // epilogue: this warp's 32 TMEM lanes = rows 32 warp .. +31
#pragma unroll
        for (int c0 = 0; c0 < COUT; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + c0, v);
            if (valid) {
                __nv_bfloat16 o[16];
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    float t = v[i] + (bias ? bias[c0 + i] : 0.f);
                    if (relu) t = fmaxf(t, 0.f);
                    o[i] = __float2bfloat16(t);
                }
                uint4 *dst = (uint4 *)(out + m * COUT + c0);
                dst[0] = *(uint4 *)&o[0];
                dst[1] = *(uint4 *)&o[8];
            }
        }
        tc_before_sync();
        __syncthreads();
        tc_after_sync();
    }
    if (!ok) {
        if (tid == 0) atomicExch(err, 1);
        // MMAs possibly in flight: wait (bounded) before freeing their TMEM
        for (int b = 0; b < 2; b++)
            if (pending[b]) mbar_wait(&mbar[b], parity[b]);
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (warp == 0) tmem_free(tmem, NCOL);
}

// ---- weight gradient --------------------------------------------------------

constexpr int kWgCells = 64;  // cells (K) staged per round: 4 MMAs of K = 16

template <int CIN, int COUT>
struct WgSmem {
    // A: dY^T, 128 rows (COUT used, rest zero) x kWgCells; B: X^T, CIN rows
    static constexpr int kA = 128 * kWgCells * 2;
    static constexpr int kB = CIN * kWgCells * 2;
    static constexpr int kBytes = 2 * kA + 2 * kB + 64;
};

// grid (cell blocks, 27 taps); each CTA: tap blockIdx.y, cells
// [blockIdx.x * per_cta, +per_cta)
template <int CIN, int COUT>
__global__ void __launch_bounds__(128)
k_conv3d_wgrad(const __nv_bfloat16 *__restrict__ x, const __nv_bfloat16 *__restrict__ dy,
               float *__restrict__ dw, int nx, int ny, int nz, long per_cta, int *err)
{
    static_assert(CIN % 16 == 0 && CIN <= 256 && COUT <= 128 && COUT % 8 == 0, "channels");
    extern __shared__ __align__(128) unsigned char smem[];
    using S = WgSmem<CIN, COUT>;
    unsigned char *abuf = smem, *bbuf = smem + 2 * S::kA;
    uint64_t *mbar = (uint64_t *)(smem + 2 * S::kA + 2 * S::kB);
    uint32_t *tslot = (uint32_t *)(mbar + 2);
    constexpr int NCOL = tmem_cols(CIN);
    constexpr uint32_t IDESC = idesc_bf16(128, CIN);
    constexpr int KCH = kWgCells / 8;  // 16-byte K chunks per round

    const int tid = threadIdx.x, warp = tid >> 5;
    const int tap = blockIdx.y;
    const int dx = tap % 3 - 1, dyy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
    const long nxy = (long)nx * ny, n = nxy * nz;
    const long c_begin = (long)blockIdx.x * per_cta;
    const long c_end = c_begin + per_cta < n ? c_begin + per_cta : n;
    if (tid == 0) {
        mbar_init(&mbar[0]);
        mbar_init(&mbar[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // rows COUT..127 of both A buffers stay zero
    for (int i = tid; i < 2 * S::kA / 16; i += 128) ((uint4 *)abuf)[i] = make_uint4(0, 0, 0, 0);
    if (warp == 0) tmem_alloc(tslot, NCOL);
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tslot;
    unsigned parity[2] = {0u, 0u};
    int pending[2] = {0, 0};
    bool ok = true, any = false;
    int round = 0;
    for (long c0 = c_begin; c0 < c_end && ok; c0 += kWgCells, round++) {
        const int b = round & 1;
        if (pending[b]) {
            ok = mbar_wait(&mbar[b], parity[b]);
            parity[b] ^= 1u;
            pending[b] = 0;
            ok = __syncthreads_and(ok);
            if (!ok) break;
        }
        unsigned char *a = abuf + b * S::kA, *bb = bbuf + b * S::kB;
        // A[co][k] = dY[c0 + k][co]: thread k-pair stages the COUT values of
        // two cells (element (row co, k) at (k/8)*2048 + co*16 + (k%8)*2)
        for (int k = tid; k < kWgCells; k += 128) {
            const long cell = c0 + k;
            const bool v = cell < c_end;
            for (int co = 0; co < COUT; co += 8) {
                uint4 q = v ? *(const uint4 *)(dy + cell * COUT + co) : make_uint4(0, 0, 0, 0);
                const __nv_bfloat16 *e = (const __nv_bfloat16 *)&q;
#pragma unroll
                for (int j = 0; j < 8; j++)
                    *(__nv_bfloat16 *)(a + (k / 8) * 2048 + (co + j) * 16 + (k % 8) * 2) = e[j];
            }
        }
        // B[ci][k] = X[cell + off][ci] (zero outside the grid)
        for (int k = tid; k < kWgCells; k += 128) {
            const long cell = c0 + k;
            bool v = cell < c_end;
            long src = 0;
            if (v) {
                const int xx = (int)(cell % nx) + dx, yy = (int)((cell / nx) % ny) + dyy,
                          zz = (int)(cell / nxy) + dz;
                v = xx >= 0 && xx < nx && yy >= 0 && yy < ny && zz >= 0 && zz < nz;
                src = xx + (long)yy * nx + (long)zz * nxy;
            }
            for (int ci = 0; ci < CIN; ci += 8) {
                uint4 q = v ? *(const uint4 *)(x + src * CIN + ci) : make_uint4(0, 0, 0, 0);
                const __nv_bfloat16 *e = (const __nv_bfloat16 *)&q;
#pragma unroll
                for (int j = 0; j < 8; j++)
                    *(__nv_bfloat16 *)(bb + (k / 8) * (CIN * 16) + (ci + j) * 16 + (k % 8) * 2) =
                        e[j];
            }
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_after_sync();
            const uint32_t sa = smem_u32(a), sb = smem_u32(bb);
#pragma unroll
            for (int kk = 0; kk < KCH / 2; kk++) {
                const uint64_t da = kmajor_desc(sa + kk * 2 * 2048, 2048, 128);
                const uint64_t db = kmajor_desc(sb + kk * 2 * (CIN * 16), CIN * 16, 128);
                umma_bf16(tmem, da, db, IDESC, (round | kk) != 0);
            }
            umma_commit(&mbar[b]);
        }
        pending[b] = 1;
        any = true;
    }
    if (ok) {
        for (int b = 0; b < 2; b++) {
            if (pending[b]) {
                ok = ok && mbar_wait(&mbar[b], parity[b]);
                parity[b] ^= 1u;
                pending[b] = 0;
            }
        }
        ok = __syncthreads_and(ok);
    }
    if (ok && any) {
        tc_after_sync();
        // row co = 32 warp + lane of D, columns ci
        const int co = 32 * warp + (tid & 31);
#pragma unroll 1
        for (int c = 0; c < CIN; c += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + c, v);
            if (co < COUT)
#pragma unroll
                for (int i = 0; i < 16; i++)
                    atomicAdd(&dw[((long)tap * COUT + co) * CIN + c + i], v[i]);
        }
    }
    if (!ok) {
        if (tid == 0) atomicExch(err, 1);
        for (int b = 0; b < 2; b++)
            if (pending[b]) mbar_wait(&mbar[b], parity[b]);
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (warp == 0) tmem_free(tmem, NCOL);
}

template <int CIN, int COUT>
int launch_fwd(const void *in, const void *w, const float *bias, void *out, int nx, int ny,
               int nz, int relu, int *err, cudaStream_t st)
{
    using S = FwdSmem<CIN, COUT>;
    auto k = k_conv3d<CIN, COUT>;
    HM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, S::kBytes));
    HM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    const long n = (long)nx * ny * nz, ntiles = (n + 127) / 128;
    int per_sm = 0, dev = 0, nsm = 0, smem_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    // resident CTAs: shared memory (1 KB reserved per CTA), 16 per SM at most
    per_sm = smem_sm / (S::kBytes + 1024);
    if (per_sm > 16) per_sm = 16;
    // resident CTAs must also fit the SM's 512 TMEM columns
    const int tmem_fit = 512 / tmem_cols(COUT);
    if (per_sm > tmem_fit) per_sm = tmem_fit;
    long grid = (long)nsm * (per_sm > 0 ? per_sm : 1);
    if (grid > ntiles) grid = ntiles;
    k<<<(int)grid, 128, S::kBytes, st>>>((const __nv_bfloat16 *)in, (const __nv_bfloat16 *)w,
                                         bias, (__nv_bfloat16 *)out, nx, ny, nz, relu, err);
    HM_LAUNCHED();
    return HMFEM_OK;
}

template <int CIN, int COUT>
int launch_wgrad(const void *x, const void *dy, float *dw, int nx, int ny, int nz, int *err,
                 cudaStream_t st)
{
    using S = WgSmem<CIN, COUT>;
    auto k = k_conv3d_wgrad<CIN, COUT>;
    HM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, S::kBytes));
    HM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    const long n = (long)nx * ny * nz;
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // ~4 waves of CTAs over the 27 taps, whole rounds of kWgCells cells each
    long blocks_x = (4L * nsm + 26) / 27;
    long per = (n + blocks_x - 1) / blocks_x;
    per = (per + kWgCells - 1) / kWgCells * kWgCells;
    if (per < kWgCells) per = kWgCells;
    blocks_x = (n + per - 1) / per;
    k<<<dim3((unsigned)blocks_x, 27), 128, S::kBytes, st>>>((const __nv_bfloat16 *)x,
                                                           (const __nv_bfloat16 *)dy, dw, nx,
                                                           ny, nz, per, err);
    HM_LAUNCHED();
    return HMFEM_OK;
}

#define HM_CONV_SHAPES(X)                                                                \
    X(16, 16) X(16, 32) X(32, 16) X(32, 32) X(32, 64) X(64, 32) X(64, 64) X(96, 32)     \
    X(32, 96) X(48, 16) X(16, 48)

}  // namespace

}  // namespace hm

extern "C" {

int hmfem_conv3d_fwd(const void *in, const void *w, const float *bias, void *out, int nx,
                     int ny, int nz, int cin, int cout, int relu, int *err, void *stream)
{
    if (!in || !w || !out || !err || nx < 1 || ny < 1 || nz < 1) return HMFEM_E_ARG;
    cudaStream_t st = (cudaStream_t)stream;
#define X(a, b)                                                                               \
    if (cin == a && cout == b)                                                                \
        return hm::launch_fwd<a, b>(in, w, bias, out, nx, ny, nz, relu, err, st);
    HM_CONV_SHAPES(X)
#undef X
    hm::set_last_error("conv3d: unsupported channel counts", __FILE__, __LINE__);
    return HMFEM_E_ARG;
}

int hmfem_conv3d_wgrad(const void *x, const void *dy, float *dw, int nx, int ny, int nz,
                       int cin, int cout, int *err, void *stream)
{
    if (!x || !dy || !dw || !err || nx < 1 || ny < 1 || nz < 1) return HMFEM_E_ARG;
    cudaStream_t st = (cudaStream_t)stream;
#define X(a, b)                                                                               \
    if (cin == a && cout == b) return hm::launch_wgrad<a, b>(x, dy, dw, nx, ny, nz, err, st);
    HM_CONV_SHAPES(X)
#undef X
    hm::set_last_error("conv3d: unsupported channel counts", __FILE__, __LINE__);
    return HMFEM_E_ARG;
}

}  // extern "C"
