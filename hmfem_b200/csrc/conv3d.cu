// conv3d.cu -- 3x3x3 convolutions of the learned initial guess on the
// 5th-generation tensor cores (tcgen05, sm_100a): BF16 operands, FP32
// accumulation in tensor memory.  No counterpart in the reference.
//
// Activations are channel-blocked: C/8 slabs, each holding the grid's cells
// (s = x + nx (y + ny z)) with 8 consecutive BF16 channels per cell, i.e.
// channel c of cell s at (c/8) n + s) * 8 + c % 8; weights are
// [27 taps][Cout][Cin] with tap t = 9 (dz+1) + 3 (dy+1) + (dx+1); zero
// padding outside the grid.
//
// Forward (and, with flipped / transposed weights, the data gradient) is an
// implicit GEMM: D[m][n] = sum_tap sum_ci A_tap[m][ci] B_tap[n][ci] with m a
// run of 128 cells, n the output channel, A_tap the input at cell m shifted
// by the tap.  The input of a tile of cells, with its halo, is brought into
// shared memory once per 16 input channels by bulk copies and every tap's A operand
// is a shifted view of it (the layout and the roles are described at
// k_conv3d); tcgen05.mma (M = 128, N = Cout, K = 16) accumulates in tensor
// memory and the epilogue reads it with tcgen05.ld, adds the bias, applies
// ReLU and stores BF16.
//
// Weight gradient: D[m = co][n = ci] = sum_cell dY[cell][co] X[cell+off][ci]
// per tap, the cells being the K dimension: a CTA takes one tap and a range
// of cells, stages dY^T (Cout rows, zero-padded to M = 128) and the shifted
// X^T (Cin rows) K-major in shared memory, accumulates in TMEM, and adds its
// partial [Cout][Cin] block into the FP32 gradient with atomics.
//
// Every mbarrier wait is bounded: on a timeout the kernel flags err, waits
// (bounded again) for its MMAs in flight, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <mutex>

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

// 16 columns of this thread's TMEM lane into registers, without waiting:
// the registers are valid after tmem_wait_ld()
__device__ __forceinline__ void tmem_ld16_nw(uint32_t taddr, float v[16])
{
    uint32_t *r = reinterpret_cast<uint32_t *>(v);
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
          "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
          "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld()
{
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__host__ __device__ constexpr int tmem_cols(int n)
{
    return n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : 256;
}

// ---- forward / data gradient ----------------------------------------------
//
// A tile is bx x by x bz output cells.  Its input with a one-cell halo,
// (bx+2) x (by+2) x (bz+2) cells, is copied into shared memory once per
// 16-channel chunk of the input: halo cell q = xi + W (yi + H zi) (W = bx+2,
// H = by+2) at byte q*16 of each 8-channel slab, the chunk's two slabs SB
// bytes apart -- the K-major no-swizzle layout with rows 16 bytes apart, so
// any 128 consecutive halo cells form an MMA operand (LBO = SB, SBO = 128).
// An MMA run is 128 consecutive halo positions q0 .. q0+127; the operand of
// tap (dx, dy, dz) for the run is the same rows shifted by dx + W dy + W H dz,
// i.e. the run's descriptor with another start address: the 27 taps read the
// tile that was copied once.  Row mode (bx = 128): a run is one x row of the
// tile.  Plane mode (bx = nx, any width): the runs of a z plane cover its interior
// rows in steps of 128 positions; positions on halo columns or beyond the
// plane are computed and dropped by the epilogue.  The copy of a tile reads
// (bx+2)(by+2)(bz+2) / (bx by bz) times its cells from L2.
//
// Roles (one CTA per SM, persistent over the tiles): warp 4 loads each halo
// chunk into a ring of `ns` stages with one bulk copy per halo row and slab
// (a halo row of a slab is contiguous in the channel-blocked input); the
// cells and rows outside the grid (the convolution's zero padding) are
// stored by the warp itself and fenced for the tensor cores;
// lane 0 of warp 5 issues, per chunk, 27 taps x runs MMAs of M = 128,
// N = COUT, K = 16 into the tile's accumulator (runs x COUT FP32 columns of
// tensor memory, `nb` = 2 buffers when they fit) and commits the stage back
// to the producer; warps 0-3 read a finished accumulator (tcgen05.ld, warp w
// lanes 32w..32w+31), add the bias, apply ReLU, store BF16 and release the
// buffer -- loads, MMAs and the epilogue of different tiles overlap.  The
// weights of a chunk come as two TMA copies of box {8, COUT, 27} (the two
// 8-channel halves, each [tap][COUT][8]); all chunks stay resident when they
// fit in kWResMax bytes, otherwise each stage carries its chunk's weights.
// No multicast.
// Grouped x taps (XG, when 3 COUT <= 256 and the tile spans the whole x
// extent): an MMA's cost is set by its A operand (128 rows from shared
// memory) up to N ~ 90, so the three taps dx = -1, 0, +1 of a (dy, dz) pair
// share one A operand -- the run's rows shifted by W dy + W H dz only -- and
// one MMA with N = 3 COUT (B = the three taps' weights, consecutive rows of
// the weight tile) accumulates D_dx for all three: 9 MMAs per run and chunk
// instead of 27.  The output of row m is D_-1[m-1] + D_0[m] + D_+1[m+1]: the
// epilogue shifts by one TMEM lane (warp shuffles; shared memory across the
// warps' lane quarters and, in plane mode, between consecutive runs of a z
// plane).  Any other neighbour of a stored cell is a halo column, i.e. zero
// padding, because the tile covers the whole x extent.
struct ConvPlan {
    int bx, by, bz;          // tile (interior cells)
    int W, H;                // halo row pitch bx+2, halo rows per plane by+2
    int hc, hcp;             // halo cells; cells per slab with the run overrun (x8)
    int runs, rp;            // MMA runs per tile; runs per z plane
    int row_mode;            // 1: bx == 128, one run per x row
    int ntx, nty, ntz;       // tiles per axis
    int ns, nb;              // input stages, accumulator buffers
    int wres;                // weights of every chunk resident
    int xg;                  // x taps grouped: N = 3 COUT per MMA (see k_conv3d)
    int tmem_cols;
    unsigned stage_bytes, wbytes, smem_bytes;
};

constexpr int kConvThreads = 192;  // warps 0-3 epilogue, 4 TMA producer, 5 MMA
constexpr int kEpilogue = 128;
constexpr unsigned kWResMax = 64 * 1024;  // resident weights (all chunks) up to this size
constexpr unsigned kBarBytes = 128;       // mbarriers (ns, nb <= 4), TMEM slot, abort flag
constexpr int kMaxPlaneX = 1024;          // widest grid a plane-mode tile spans

// shared memory after the stages: barriers, then (grouped x taps) three
// exchange buffers of 4 + 4 + 1 boundary rows of COUT floats, then the bias
__host__ __device__ constexpr unsigned conv_tail_bytes(int cout, bool xg)
{
    return kBarBytes + (xg ? 3u * 9u * 4u * (unsigned)cout : 0u) + 4u * (unsigned)cout;
}

// The MMA warp runs its loop with all lanes (descriptor arithmetic stays
// warp-uniform); one elected lane issues.  Every MMA and commit of the
// kernel goes through the same election, so a commit tracks the MMAs it
// follows (both are per issuing thread).
__device__ __forceinline__ void umma_bf16_elect(uint32_t tmem, uint64_t da, uint64_t db,
                                                uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred e, p;\n\t"
        "elect.sync _|e, 0xffffffff;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "@e tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit_elect(uint64_t *mbar)
{
    asm volatile(
        "{\n\t.reg .pred e;\n\t"
        "elect.sync _|e, 0xffffffff;\n\t"
        "@e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n\t}\n"
        ::"r"(smem_u32(mbar))
        : "memory");
}

__device__ __forceinline__ void mbar_init_n(uint64_t *m, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t *m)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(m)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx_only(uint64_t *m, uint32_t bytes)
{
    asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes)
                 : "memory");
}

// bulk copy global -> this CTA's shared memory (16-byte aligned, multiple of 16)
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes,
                                          uint64_t *m)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(dst), "l"(src), "r"(bytes), "r"(smem_u32(m))
        : "memory");
}

// TMA tensor copies into this CTA's shared memory, completion on an mbarrier
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, int c0, int c1,
                                            int c2, uint64_t *m)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(m))
        : "memory");
}

// named barrier 1 among the epilogue warps; the reduction form returns the
// AND of every thread's predicate (all threads agree on leaving)
__device__ __forceinline__ void epi_sync()
{
    asm volatile("bar.sync 1, %0;" ::"n"(kEpilogue) : "memory");
}

__device__ __forceinline__ bool epi_all(bool v)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, 1, %2, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)v), "n"(kEpilogue)
        : "memory");
    return r != 0;
}

// bounded wait that also leaves when another role gave up (abort flag)
__device__ __forceinline__ bool role_wait(uint64_t *m, unsigned parity, volatile int *abort_flag,
                                          int *err)
{
    for (unsigned i = 0; i < kWaitPolls; i++) {
        if (mbar_test(m, parity)) return true;
        if (*abort_flag) return false;
        if (i > 64) __nanosleep(64);
    }
    *abort_flag = 1;
    atomicExch(err, 1);
    return false;
}

// first halo position of run r; its plane (0..bz-1) and, in row mode, row
__device__ __forceinline__ int run_start(const ConvPlan &p, int r, int &plane, int &row)
{
    if (p.row_mode) {
        plane = r / p.by;
        row = r - plane * p.by;
        return 1 + p.W * (row + 1) + p.W * p.H * (plane + 1);
    }
    plane = r / p.rp;
    row = -1;
    return 1 + p.W + p.W * p.H * (plane + 1) + 128 * (r - plane * p.rp);
}

template <int CIN, int COUT, bool XG>
__global__ void __launch_bounds__(kConvThreads, 1)
k_conv3d(const __nv_bfloat16 *__restrict__ in, const __grid_constant__ CUtensorMap tm_w,
         const float *__restrict__ bias, __nv_bfloat16 *__restrict__ out, int nx, int ny,
         int nz, int relu, const ConvPlan p, int *err)
{
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 256, "channel counts");
    static_assert(!XG || 3 * COUT <= 256, "grouped x taps: N = 3 COUT <= 256");
    constexpr int KC = CIN / 16;
    constexpr int NACC = XG ? 3 * COUT : COUT;  // accumulator columns per run
    constexpr uint32_t IDESC = idesc_bf16(128, NACC);
    constexpr int WTAP = COUT * 16;       // one tap's rows of one 8-channel half
    constexpr int WHALF = 27 * WTAP;      // the second half follows all 27 taps of the first
    extern __shared__ __align__(128) unsigned char smem[];
    const unsigned SB = (unsigned)p.hcp * 16u, SA = 2u * SB;
    unsigned char *wres = smem;                    // resident weights (p.wres)
    unsigned char *stages = smem + p.wbytes;
    uint64_t *bar = (uint64_t *)(stages + (size_t)p.ns * p.stage_bytes);
    uint64_t *full = bar, *empty = bar + p.ns, *tfull = bar + 2 * p.ns, *tempty = tfull + p.nb,
             *drain = tempty + p.nb;
    uint32_t *tslot = (uint32_t *)(drain + 1);
    volatile int *abort_flag = (volatile int *)(tslot + 1);
    // grouped x taps: boundary rows exchanged between warps / runs, three
    // buffers (by a running run count): lane 31's D_-1 of each warp, lane
    // 0's D_+1 of each warp, row 0's D_+1 of the next run
    float *xlo = (float *)(stages + (size_t)p.ns * p.stage_bytes + kBarBytes);
    float *xhi = xlo + 3 * 4 * COUT;
    float *xnx = xhi + 3 * 4 * COUT;
    float *sbias = (float *)(stages + (size_t)p.ns * p.stage_bytes + kBarBytes) +
                   (XG ? 27 * COUT : 0);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long ntiles = (long)p.ntx * p.nty * p.ntz;
    const int WH = p.W * p.H;
    if (tid == 0) {
        for (int s = 0; s < p.ns; s++) {
            mbar_init_n(&full[s], 1);
            mbar_init_n(&empty[s], 1);
        }
        for (int b = 0; b < p.nb; b++) {
            mbar_init_n(&tfull[b], 1);
            mbar_init_n(&tempty[b], kEpilogue);
        }
        mbar_init_n(drain, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 5) tmem_alloc(tslot, p.tmem_cols);
    for (int i = tid; i < COUT; i += kConvThreads) sbias[i] = bias ? bias[i] : 0.f;
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tslot;

    if (warp == 4) {
        // ---- producer (whole warp): bulk copies of the halo rows
        const long n = (long)nx * ny * nz;
        const int D = p.bz + 2, rows = p.H * D;
        unsigned wkc = 0xffffffffu;  // per stage (8 bits each): chunk of its weights
        long item = 0;
        bool ok = true;
        for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
            const int tx = (int)(tile % p.ntx), ty = (int)((tile / p.ntx) % p.nty),
                      tz = (int)(tile / ((long)p.ntx * p.nty));
            const int x0 = tx * p.bx - 1, y0 = ty * p.by - 1, z0 = tz * p.bz - 1;
            // the part [xa, xb) of every halo row inside the grid, and the
            // number of halo rows (of one slab) inside it
            const int xa = x0 < 0 ? 0 : x0, xb = x0 + p.W < nx ? x0 + p.W : nx;
            const int ya = y0 < 0 ? 0 : y0, yb = y0 + p.H < ny ? y0 + p.H : ny;
            const int za = z0 < 0 ? 0 : z0, zb = z0 + D < nz ? z0 + D : nz;
            const int rows_in = (yb - ya) * (zb - za);
            for (int kc = 0; kc < KC; kc++, item++) {
                const int s = (int)(item % p.ns);
                const unsigned use = (unsigned)(item / p.ns);
                if (!__all_sync(0xffffffffu,
                                role_wait(&empty[s], (use & 1u) ^ 1u, abort_flag, err))) {
                    ok = false;
                    break;
                }
                const uint32_t a = smem_u32(stages + (size_t)s * p.stage_bytes);
                const bool need_w = p.wres ? item == 0
                                           : ((wkc >> (8 * s)) & 0xffu) != (unsigned)kc;
                if (lane == 0)
                    mbar_expect_tx_only(&full[s], 32u * (unsigned)(rows_in * (xb - xa)) +
                                                      (need_w ? (p.wres ? KC : 1) * 2u * WHALF
                                                              : 0u));
                __syncwarp();
                const uint4 zero = make_uint4(0, 0, 0, 0);
                for (int i = lane; i < 2 * rows; i += 32) {
                    const int sl = i / rows, rr = i - sl * rows, zi = rr / p.H,
                              yi = rr - zi * p.H;
                    const int gy = y0 + yi, gz = z0 + zi;
                    unsigned char *drow_p = stages + (size_t)s * p.stage_bytes + (size_t)sl * SB +
                                            (size_t)(rr * p.W) * 16u;
                    if (gy < 0 || gy >= ny || gz < 0 || gz >= nz) {
                        for (int c = 0; c < p.W; c++) ((uint4 *)drow_p)[c] = zero;
                        continue;
                    }
                    const __nv_bfloat16 *src =
                        in + ((long)(2 * kc + sl) * n + xa + (long)nx * (gy + (long)ny * gz)) * 8;
                    bulk_load(smem_u32(drow_p) + (uint32_t)(xa - x0) * 16u, src,
                              (uint32_t)(xb - xa) * 16u, &full[s]);
                    for (int c = 0; c < xa - x0; c++) ((uint4 *)drow_p)[c] = zero;
                    for (int c = xb - x0; c < p.W; c++) ((uint4 *)drow_p)[c] = zero;
                }
                fence_async_smem();  // the zeros, written by this warp, for the MMAs
                if (need_w && lane == 0) {
                    for (int c = p.wres ? 0 : kc; c < (p.wres ? KC : kc + 1); c++) {
                        const uint32_t wb = p.wres ? smem_u32(wres) + (uint32_t)c * 2u * WHALF
                                                   : a + SA;
                        tma_load_3d(wb, &tm_w, 16 * c, 0, 0, &full[s]);
                        tma_load_3d(wb + WHALF, &tm_w, 16 * c + 8, 0, 0, &full[s]);
                    }
                }
                if (need_w) wkc = (wkc & ~(0xffu << (8 * s))) | ((unsigned)kc << (8 * s));
                __syncwarp();
                if (lane == 0) mbar_arrive(&full[s]);
            }
        }
        // copies still in flight land before the CTA leaves: wait for the
        // last use of every stage (already complete unless a role gave up)
        if (lane == 0)
            for (int j = 0; j < p.ns && j < item; j++) {
                const long it = item - 1 - j;
                if (!mbar_wait(&full[it % p.ns], (unsigned)(it / p.ns) & 1u)) atomicExch(err, 1);
            }
        __syncwarp();
    } else if (warp == 5) {
        // ---- MMA issue (the whole warp, one elected lane issuing).  Per run
        // the 27 taps are unrolled: the A descriptor is the run's base plus a
        // per-tap offset held in a register, the B descriptor the stage's
        // base plus an immediate.
        {
            constexpr int NT = XG ? 9 : 27;  // MMAs per run and chunk
            int offs[NT];
#pragma unroll
            for (int t = 0; t < NT; t++)
                offs[t] = XG ? p.W * (t % 3 - 1) + WH * (t / 3 - 1)
                             : (t % 3 - 1) + p.W * ((t / 3) % 3 - 1) + WH * (t / 9 - 1);
            long item = 0, jt = 0;
            bool ok = true;
            for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, jt++) {
                const int b = (int)(jt % p.nb);
                const unsigned u = (unsigned)(jt / p.nb);
                if (!__all_sync(0xffffffffu, role_wait(&tempty[b], (u & 1u) ^ 1u, abort_flag, err)))
                    break;
                tc_after_sync();
                const uint32_t acc0 = tmem + (uint32_t)(b * p.runs * NACC);
                for (int kc = 0; kc < KC; kc++, item++) {
                    const int s = (int)(item % p.ns);
                    const unsigned use = (unsigned)(item / p.ns);
                    if (!__all_sync(0xffffffffu, role_wait(&full[s], use & 1u, abort_flag, err))) {
                        ok = false;
                        break;
                    }
                    tc_after_sync();
                    const uint32_t a = smem_u32(stages + (size_t)s * p.stage_bytes);
                    const uint32_t wb =
                        p.wres ? smem_u32(wres) + (uint32_t)kc * 2u * WHALF : a + SA;
                    // descriptor start addresses count 16-byte units: a run's
                    // operand row q is one unit per position
                    const uint64_t da0 = kmajor_desc(a, SB, 128);
                    const uint64_t db0 = kmajor_desc(wb, WHALF, 128);
                    const uint32_t first = kc == 0 ? 0u : 1u;
                    // run starts without divisions (the order of run_start)
                    int plane = 0, j = 0;
                    for (int r = 0; r < p.runs; r++) {
                        const int q0 = p.row_mode
                                           ? 1 + p.W * (j + 1) + WH * (plane + 1)
                                           : 1 + p.W + WH * (plane + 1) + 128 * j;
                        if (++j == p.rp) {
                            j = 0;
                            plane++;
                        }
                        const uint64_t dar = da0 + (uint64_t)q0;
                        const uint32_t acc = acc0 + (uint32_t)(r * NACC);
                        // tap t (or group g: taps 3g .. 3g+2) starts at row t (3g) x COUT
                        // of the weight tile
#pragma unroll
                        for (int t = 0; t < NT; t++)
                            umma_bf16_elect(acc, dar + (uint64_t)offs[t],
                                            db0 + (uint64_t)(t * (XG ? 3 : 1) * (WTAP / 16)),
                                            IDESC, t == 0 ? first : 1u);
                    }
                    umma_commit_elect(&empty[s]);
                }
                if (ok) umma_commit_elect(&tfull[b]);
            }
        }
        __syncwarp();
    } else {
        // ---- epilogue: warp w reads TMEM lanes 32w .. 32w+31 (rows of a run)
        const int m = 32 * warp + lane;
        const long nc = (long)nx * ny * nz;
        long jt = 0, gr = 0;  // tiles, runs (running count: exchange buffers)
        for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, jt++) {
            const int b = (int)(jt % p.nb);
            const unsigned u = (unsigned)(jt / p.nb);
            bool okw = role_wait(&tfull[b], u & 1u, abort_flag, err);
            if (XG) okw = epi_all(okw);  // named barriers below: leave together
            if (!okw) break;
            tc_after_sync();
            const int tx = (int)(tile % p.ntx), ty = (int)((tile / p.ntx) % p.nty),
                      tz = (int)(tile / ((long)p.ntx * p.nty));
            const int X0 = tx * p.bx - 1, Y0 = ty * p.by - 1, Z0 = tz * p.bz - 1;
            for (int r = 0; r < p.runs; r++, gr++) {
                int plane, row;
                const int q = run_start(p, r, plane, row) + m;
                const int zi = q / WH, rem = q - zi * WH, yi = rem / p.W, xi = rem - yi * p.W;
                const int gx = X0 + xi, gy = Y0 + yi, gz = Z0 + zi;
                const bool v = zi == plane + 1 && yi >= 1 && yi <= p.by && xi >= 1 &&
                               xi <= p.bx && (row < 0 || yi == row + 1) && gx < nx && gy < ny &&
                               gz < nz;
                const uint32_t ta = tmem + ((uint32_t)(32 * warp) << 16) +
                                    (uint32_t)((b * p.runs + r) * NACC);
                const long cell = gx + (long)nx * (gy + (long)ny * gz);
                // runs r-1 and r+1 of the same z plane (plane mode only)
                const bool same_prev = !p.row_mode && r > 0 && r % p.rp != 0;
                const bool same_next = !p.row_mode && r + 1 < p.runs && (r + 1) % p.rp != 0;
                const int xb = (int)(gr % 3), xbp = (int)((gr + 2) % 3);
#pragma unroll
                for (int c0 = 0; c0 < COUT; c0 += 16) {
                    float f[16];
                    if (XG) {
                        float dm[16], dp[16], dn1[16];
                        tmem_ld16_nw(ta + c0, dm);              // D_-1
                        tmem_ld16_nw(ta + COUT + c0, f);        // D_0
                        tmem_ld16_nw(ta + 2 * COUT + c0, dp);   // D_+1
                        if (warp == 0 && same_next)
                            tmem_ld16_nw(ta + NACC + 2 * COUT + c0, dn1);  // next run's D_+1
                        tmem_wait_ld();
                        // publish the rows other warps (and the next run) need
                        float4 *lo = (float4 *)(xlo + (xb * 4 + warp) * COUT + c0);
                        float4 *hi = (float4 *)(xhi + (xb * 4 + warp) * COUT + c0);
                        if (lane == 31)
#pragma unroll
                            for (int i = 0; i < 4; i++)
                                lo[i] = make_float4(dm[4 * i], dm[4 * i + 1], dm[4 * i + 2],
                                                    dm[4 * i + 3]);
                        if (lane == 0) {
#pragma unroll
                            for (int i = 0; i < 4; i++)
                                hi[i] = make_float4(dp[4 * i], dp[4 * i + 1], dp[4 * i + 2],
                                                    dp[4 * i + 3]);
                            if (warp == 0 && same_next) {
                                float4 *nx4 = (float4 *)(xnx + xb * COUT + c0);
#pragma unroll
                                for (int i = 0; i < 4; i++)
                                    nx4[i] = make_float4(dn1[4 * i], dn1[4 * i + 1],
                                                         dn1[4 * i + 2], dn1[4 * i + 3]);
                            }
                        }
                        epi_sync();
                        // row m-1's D_-1 and row m+1's D_+1
                        float up[16], dn[16];
#pragma unroll
                        for (int i = 0; i < 16; i++) {
                            up[i] = __shfl_up_sync(0xffffffffu, dm[i], 1);
                            dn[i] = __shfl_down_sync(0xffffffffu, dp[i], 1);
                        }
                        if (lane == 0) {
                            const float *src = warp > 0 ? xlo + (xb * 4 + warp - 1) * COUT + c0
                                             : same_prev ? xlo + (xbp * 4 + 3) * COUT + c0
                                                         : nullptr;
#pragma unroll
                            for (int i = 0; i < 4; i++) {
                                const float4 t4 = src ? ((const float4 *)src)[i]
                                                      : make_float4(0.f, 0.f, 0.f, 0.f);
                                up[4 * i] = t4.x, up[4 * i + 1] = t4.y, up[4 * i + 2] = t4.z,
                                up[4 * i + 3] = t4.w;
                            }
                        }
                        if (lane == 31) {
                            const float *src = warp < 3 ? xhi + (xb * 4 + warp + 1) * COUT + c0
                                             : same_next ? xnx + xb * COUT + c0
                                                         : nullptr;
#pragma unroll
                            for (int i = 0; i < 4; i++) {
                                const float4 t4 = src ? ((const float4 *)src)[i]
                                                      : make_float4(0.f, 0.f, 0.f, 0.f);
                                dn[4 * i] = t4.x, dn[4 * i + 1] = t4.y, dn[4 * i + 2] = t4.z,
                                dn[4 * i + 3] = t4.w;
                            }
                        }
#pragma unroll
                        for (int i = 0; i < 16; i++) f[i] += up[i] + dn[i];
                    } else {
                        tmem_ld16_nw(ta + c0, f);
                        tmem_wait_ld();
                    }
                    if (v) {
                        __nv_bfloat16 o[16];
#pragma unroll
                        for (int i = 0; i < 16; i++) {
                            float t = f[i] + sbias[c0 + i];
                            if (relu) t = fmaxf(t, 0.f);
                            o[i] = __float2bfloat16(t);
                        }
                        *(uint4 *)(out + ((long)(c0 / 8) * nc + cell) * 8) = *(uint4 *)&o[0];
                        *(uint4 *)(out + ((long)(c0 / 8 + 1) * nc + cell) * 8) = *(uint4 *)&o[8];
                    }
                }
            }
            tc_before_sync();
            mbar_arrive(&tempty[b]);
        }
    }
    // teardown: every MMA this CTA issued has completed before TMEM is freed
    if (warp == 5) {
        umma_commit_elect(drain);
        if (lane == 0 && !mbar_wait(drain, 0)) atomicExch(err, 1);
        __syncwarp();
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (warp == 5) tmem_free(tmem, p.tmem_cols);
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
                uint4 q = v ? *(const uint4 *)(dy + ((long)(co / 8) * n + cell) * 8)
                            : make_uint4(0, 0, 0, 0);
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
                uint4 q = v ? *(const uint4 *)(x + ((long)(ci / 8) * n + src) * 8)
                            : make_uint4(0, 0, 0, 0);
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

// Tile choice for a forward launch: row mode (bx = 128) or plane mode (bx =
// nx, the whole x extent); the mode, the form (x taps grouped or not) and (by, bz)
// minimise an estimate of the makespan -- per tile the largest of the MMA
// issue (~42 cycles per MMA up to N = 84, N/2 above: the A operand read),
// the halo copy (a bulk copy per row and slab plus its bytes) and the
// epilogue (added instead with one accumulator buffer), times the tile
// waves over the SMs -- subject to the tensor-memory columns (runs x COUT,
// x3 grouped, doubled when two accumulators fit in 512) and the shared
// memory.  Grouping pays where the MMAs dominate: many input chunks and
// few output columns (48 -> 16 at 128^3: 255 -> 191 us).
ConvPlan plan_conv(int nx, int ny, int nz, int cin, int cout, int nsm, int smem_max)
{
    ConvPlan best{};
    double best_cost = 1e300;
    const int kc = cin / 16;
    const unsigned wchunk = 27u * (unsigned)cout * 32u;
    // row mode (bx = 128, x tiles) when nx >= 128; plane mode (bx = nx, the
    // whole x extent) for any width up to kMaxPlaneX
    for (int pm = 0; pm < 2; pm++)
    for (int xg = 0; xg < 2; xg++)
        for (int bz = 1; bz <= (nz < 16 ? nz : 16); bz++)
            for (int by = 1; by <= (ny < 64 ? ny : 64); by++) {
                const bool row_mode = pm == 0;
                if (row_mode ? nx < 128 : nx > kMaxPlaneX) continue;
                const int bx = row_mode ? 128 : nx;
                const int W = bx + 2;
                // grouped x taps need N = 3 COUT <= 256 and tiles spanning
                // the x extent (their x neighbours outside the tile are zero)
                if (xg && (3 * cout > 256 || (row_mode && nx != 128))) continue;
                ConvPlan p{};
                p.bx = bx;
                p.by = by;
                p.bz = bz;
                p.W = W;
                p.H = by + 2;
                p.hc = W * p.H * (bz + 2);
                p.hcp = (p.hc + 128 + 7) / 8 * 8;
                p.row_mode = row_mode;
                p.xg = xg;
                p.rp = row_mode ? by : (W * (by - 1) + bx + 127) / 128;
                p.runs = bz * p.rp;
                const int nacc = (xg ? 3 : 1) * cout;
                if (p.runs * nacc > 512) continue;
                p.nb = 2 * p.runs * nacc <= 512 ? 2 : 1;
                p.wres = (unsigned)kc * wchunk <= kWResMax;
                p.wbytes = p.wres ? (unsigned)kc * wchunk : 0;
                p.stage_bytes = 32u * (unsigned)p.hcp + (p.wres ? 0 : wchunk);
                const unsigned fixed = conv_tail_bytes(cout, xg);
                if ((unsigned)smem_max < fixed + p.wbytes + p.stage_bytes) continue;
                int ns = (int)(((unsigned)smem_max - fixed - p.wbytes) / p.stage_bytes);
                p.ns = ns > 4 ? 4 : ns;
                p.ntx = (nx + bx - 1) / bx;
                p.nty = (ny + by - 1) / by;
                p.ntz = (nz + bz - 1) / bz;
                const long tiles = (long)p.ntx * p.nty * p.ntz;
                const double mma_c = nacc / 2.0 > 42.0 ? nacc / 2.0 : 42.0;
                const double mma = (double)p.runs * (xg ? 9 : 27) * kc * mma_c;
                const double load = kc * (2.0 * p.H * (bz + 2) * 30.0 + 32.0 * p.hc / 48.0) +
                                    (p.wres ? 0.0 : 27.0 * cout * kc);
                // epilogue per run and 16 columns (measured): ~300 cycles, ~2000
                // grouped (three TMEM reads, the boundary exchange, a barrier)
                const double epi = (double)p.runs * (cout / 16) * (xg ? 2000.0 : 300.0);
                double tile_t = mma > load ? mma : load;
                if (p.ns < 2) tile_t = mma + load;
                tile_t = p.nb == 2 ? (tile_t > epi ? tile_t : epi) : tile_t + epi;
                const double cost = (double)((tiles + nsm - 1) / nsm) * (tile_t + 300.0);
                if (cost < best_cost) {
                    best_cost = cost;
                    best = p;
                }
            }
    const int nacc = (best.xg ? 3 : 1) * cout;
    best.tmem_cols = 32;
    while (best.tmem_cols < best.nb * best.runs * nacc) best.tmem_cols *= 2;
    best.smem_bytes = best.wbytes + (unsigned)best.ns * best.stage_bytes +
                      conv_tail_bytes(cout, best.xg);
    // one CTA per SM: its tensor-memory allocation may take all 512 columns
    if (best.smem_bytes < (unsigned)smem_max / 2 + 1024) best.smem_bytes = smem_max / 2 + 1024;
    return best;
}

// cuTensorMapEncodeTiled from the driver (no link against libcuda)
using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                 const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                 const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// A BF16 tensor map without swizzle: 16-byte aligned base and strides, boxes
// of box[] elements, zeros outside the tensor.
int encode_bf16_map(CUtensorMap *map, const void *base, int rank, const cuuint64_t *dims,
                    const cuuint64_t *strides, const cuuint32_t *box)
{
    static EncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiled)f;
    });
    if (!fn) {
        set_last_error("conv3d: cuTensorMapEncodeTiled unavailable", __FILE__, __LINE__);
        return HMFEM_E_CUDA;
    }
    if (((uintptr_t)base & 15u) != 0) {
        set_last_error("conv3d: tensors must be 16-byte aligned", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (cuuint32_t)rank,
                          const_cast<void *>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_last_error("conv3d: tensor map rejected", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    return HMFEM_OK;
}

template <int CIN, int COUT>
int launch_fwd(const void *in, const void *w, const float *bias, void *out, int nx, int ny,
               int nz, int relu, int *err, cudaStream_t st)
{
    int dev = 0, nsm = 0, smem_max = 0;
    HM_CUDA(cudaGetDevice(&dev));
    HM_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    HM_CUDA(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const ConvPlan p = plan_conv(nx, ny, nz, CIN, COUT, nsm, smem_max);
    auto k = k_conv3d<CIN, COUT, false>;
    if constexpr (3 * COUT <= 256)
        if (p.xg) k = k_conv3d<CIN, COUT, true>;
    if (p.ns < 1) {
        set_last_error("conv3d: no tile fits in shared memory", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    if (((uintptr_t)in & 15u) || ((uintptr_t)out & 15u)) {
        set_last_error("conv3d: tensors must be 16-byte aligned", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    CUtensorMap tm_w;
    {
        const cuuint64_t dims[3] = {(cuuint64_t)CIN, (cuuint64_t)COUT, 27};
        const cuuint64_t strides[2] = {(cuuint64_t)CIN * 2, (cuuint64_t)COUT * CIN * 2};
        const cuuint32_t box[3] = {8, (cuuint32_t)COUT, 27};
        const int rc = encode_bf16_map(&tm_w, w, 3, dims, strides, box);
        if (rc != HMFEM_OK) return rc;
    }
    HM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem_bytes));
    const long tiles = (long)p.ntx * p.nty * p.ntz;
    const int grid = (int)(tiles < nsm ? tiles : nsm);
    k<<<grid, kConvThreads, p.smem_bytes, st>>>((const __nv_bfloat16 *)in, tm_w, bias,
                                                (__nv_bfloat16 *)out, nx, ny, nz, relu, p, err);
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

int hmfem_conv3d_plan(int nx, int ny, int nz, int cin, int cout, int nsm, int smem_max,
                      int *plan)
{
    if (!plan || nx < 1 || ny < 1 || nz < 1 || cin < 16 || cin % 16 || cout < 16 ||
        cout % 16 || cout > 256 || nsm < 1 || smem_max < 1024)
        return HMFEM_E_ARG;
    const hm::ConvPlan p = hm::plan_conv(nx, ny, nz, cin, cout, nsm, smem_max);
    const int v[21] = {p.bx, p.by, p.bz, p.W, p.H, p.hc, p.hcp, p.runs, p.rp, p.row_mode,
                       p.ntx, p.nty, p.ntz, p.ns, p.nb, p.wres, p.tmem_cols,
                       (int)p.stage_bytes, (int)p.wbytes, (int)p.smem_bytes, p.xg};
    for (int i = 0; i < 21; i++) plan[i] = v[i];
    return p.ns >= 1 ? HMFEM_OK : HMFEM_E_ARG;
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
