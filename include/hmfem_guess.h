/* hmfem_guess.h -- kernels of the learned initial guess (a 3-level 3-D
 * U-Net mapping log K, the conduit mask and the Dirichlet mask to a pressure
 * guess).  No counterpart in the reference: the reference always starts its
 * CG from the previous pressure or zero.
 *
 * Tensors are device pointers, 16-byte aligned.  Activations are
 * channel-blocked BF16: C/8 slabs of the n = nx ny nz cells (s = x + nx (y +
 * ny z)), 8 consecutive channels per cell -- channel c of cell s at
 * ((c/8) n + s) * 8 + c % 8.  3x3x3 weights are BF16
 * [27][Cout][Cin] with tap t = 9 (dz+1) + 3 (dy+1) + (dx+1) (cross-
 * correlation, zero padding).  Supported (Cin, Cout): (16,16) (16,32)
 * (32,16) (32,32) (32,64) (64,32) (64,64) (96,32) (32,96) (48,16) (16,48).
 * `stream` is a cudaStream_t (NULL: legacy default stream); `err` a device
 * int the kernels set to 1 if a bounded tensor-core wait gave up. */
#ifndef HMFEM_GUESS_H
#define HMFEM_GUESS_H

#ifdef __cplusplus
extern "C" {
#endif

/* out = relu?(conv3x3x3(in, w) + bias) on the tcgen05 tensor cores (BF16
 * operands, FP32 accumulation in tensor memory); bias may be NULL.  With
 * weights flipped in the taps and transposed in the channels this is also
 * the data gradient of a convolution. */
int hmfem_conv3d_fwd(const void *in, const void *w, const float *bias, void *out, int nx,
                     int ny, int nz, int cin, int cout, int relu, int *err, void *stream);

/* The tiling hmfem_conv3d_fwd launches for this grid and channel counts on
 * a device with `nsm` SMs and `smem_max` bytes of opt-in shared memory per
 * block; host-only (no device call).  plan[21] = {bx, by, bz, W, H, hc, hcp,
 * runs, rp, row_mode, ntx, nty, ntz, ns, nb, wres, tmem_cols, stage_bytes,
 * wbytes, smem_bytes, xg}: the interior tile, the halo row pitch and rows
 * per plane, halo cells and cells per 8-channel slab, MMA runs per tile and
 * per z plane, row mode, tiles per axis, input stages, accumulator buffers,
 * resident weights, tensor-memory columns, shared-memory bytes and whether
 * the three x taps of each (dy, dz) share one MMA (N = 3 Cout). */
int hmfem_conv3d_plan(int nx, int ny, int nz, int cin, int cout, int nsm, int smem_max,
                      int *plan);

/* dw[27][cout][cin] += sum over cells of dy[cell][co] x[cell + tap][ci] (the
 * weight gradient), FP32, on the tensor cores. */
int hmfem_conv3d_wgrad(const void *x, const void *dy, float *dw, int nx, int ny, int nz,
                       int cin, int cout, int *err, void *stream);

/* The data movement around the convolutions (one HBM pass each; even grid
 * dimensions where a 2x level is involved).  Features: out[2][n][8] =
 * ((log10 K + 14)/2, conduit mask (NULL: 0), Dirichlet face mask +1 at x = 0
 * and -1 at x = nx-1, zeros) from device K (FP64) and mask (uint8). */
int hmfem_guess_features(const double *K, const unsigned char *mask, int nx, int ny, int nz,
                         void *out, void *stream);

/* 2x2x2 average pooling of `slabs` slabs of the fine grid nx x ny x nz. */
int hmfem_guess_pool2(const void *x, int slabs, int nx, int ny, int nz, void *out, void *stream);

/* out = [nearest-upsampled coarse (slabs_a slabs of the nx/2 x ny/2 x nz/2
 * grid) | skip (slabs_b slabs of the nx x ny x nz grid)]. */
int hmfem_guess_up2_cat(const void *coarse, int slabs_a, const void *skip, int slabs_b, int nx,
                        int ny, int nz, void *out, void *stream);

/* The gradient of the upsampling: out (slabs_a slabs of the coarse grid) =
 * the sum of the gradients of each coarse cell's 8 fine cells. */
int hmfem_guess_up2_grad(const void *g, int slabs_a, int nx, int ny, int nz, void *out,
                         void *stream);

/* p[s] = 1 - (x + 1/2)/nx + sum_c x[c] w[c] + b[0] (FP32 head, FP64 out):
 * the guess from the last activation (8 * slabs head weights). */
int hmfem_guess_head_profile(const void *x, int slabs, const float *w, const float *b, int nx,
                             int ny, int nz, double *p, void *stream);

#ifdef __cplusplus
}
#endif
#endif
