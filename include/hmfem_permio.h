/*
 * hmfem_permio.h -- heterogeneous permeability from geological files: the
 * reference's readers (permeabilities.c: read_set_perm_field :494-668,
 * read_layer_perm_field :57-186, gaussian_permfield :673-772) split into a
 * host parse and a device resample onto the simulation grid.
 *
 * Geological arrays are indexed like the reference's ind(i, j, k) =
 * i + nxg (j + nyg k) (solve_linearsystem_AMG.c:8-13); the reference fixes
 * the SPE10 model at nxg = 60, nyg = 220, nzg = 85 and the Gaussian field
 * at 60^3 (main.c:122-124), these take them as arguments.
 */
#ifndef HMFEM_PERMIO_H
#define HMFEM_PERMIO_H

#include "hmfem_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* SPE-format file: three blocks (K_x, K_y, K_z), each listing the layers
 * from k = nzg-1 down to 0, rows j and columns i ascending, into cell
 * ind(nxg-1-i, nyg-1-j, k) of KXg / KYg / KZg (host, nxg*nyg*nzg each).
 * layer < 0: every layer (read_set_perm_field); layer >= 0: only that layer
 * into the k = 0 plane, K_z set to 1e-8 (read_layer_perm_field; the arrays
 * then need nxg*nyg entries).  HMFEM_E_ARG on a missing file or too few
 * values. */
int hmfem_read_spe(const char *path, int nxg, int nyg, int nzg, int layer,
                   double *KXg, double *KYg, double *KZg);

/* gaussian_permfield's file: per cell (i, j, k loops, k fastest) three
 * columns, the first is the permeability (all directions). */
int hmfem_read_gaussian(const char *path, int nxg, int nyg, int nzg, double *Kg);

/* The resample onto an nx*ny*nz grid on a domain Ix*Iy*Iz: each cell takes
 * the geological cell holding its centre, floor((i + 0.5) h / h_geo) per
 * axis, with h = I/n and h_geo = I/n_geo as the reference computes them.
 * variant 0: read_set_perm_field; 1: read_layer_perm_field (the k = 0 plane
 * only, from the one-layer arrays; other planes keep their values);
 * 2: gaussian_permfield (its h_geo in z is Iz / nxg, as the reference
 * divides).  Host (mem 0) or device (mem 1) arrays. */
int hmfem_resample_perm(int variant, const double *KXg, const double *KYg,
                        const double *KZg, int nxg, int nyg, int nzg,
                        double Ix, double Iy, double Iz, int nx, int ny,
                        int nz, double *KX, double *KY, double *KZ, int mem);

#ifdef __cplusplus
}
#endif
#endif
