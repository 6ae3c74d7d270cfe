/*
 * hmfem_textio.h -- the reference's ASCII result files, formatted on the GPU.
 *
 * Each writer produces byte for byte the file the reference's writer
 * produces for the same arrays (every number converted as glibc's printf
 * converts it for the same format string: exact decimal digits of the
 * binary value, rounded half to even), with one GPU thread per line
 * instead of one fprintf per number.  Arrays are host (mem = 0) or device
 * (mem = 1) pointers; grid cell s = i + nx (j + ny k) as everywhere in this
 * library.  Lines holding a value outside the device's exact range (NaN,
 * infinity, or a magnitude beyond ~1e-77 .. 1e36 for %1.9e) are formatted
 * by the host C library with the same format string.  Return HMFEM_OK,
 * HMFEM_E_ARG (bad argument, file not writable) or HMFEM_E_CUDA.
 */
#ifndef HMFEM_TEXTIO_H
#define HMFEM_TEXTIO_H

#include "hmfem_gpu.h"
#include "hmfem_karst.h"

#ifdef __cplusplus
extern "C" {
#endif

/* posprocessing_output.c:200-234 (save_pressure): the file the reference
 * writes as <dirname>/pressure_reservoir.dat -- "%.6lf %.6lf %.6lf %1.9e\n"
 * per cell in i, j, k loop order, " \n" after every k column and after
 * every j-k plane. */
int hmfem_save_pressure(const char *path, int nx, int ny, int nz, double hx,
                        double hy, double hz, const double *p, int mem);

/* posprocessing_output.c:236-296 (save_flux): flux_reservoir.dat, cell
 * centre and 0.5 (r - l), 0.5 (u - d), 0.5 (t - b) of the face fluxes. */
int hmfem_save_flux(const char *path, int nx, int ny, int nz, double hx,
                    double hy, double hz, const hmfem_ele *v, int mem);

/* vtk.c:8-76 (vts_StructuredGrid_file): campos.vts with the velocity, the
 * pressure and the cell-centre points. */
int hmfem_save_vts(const char *path, int nx, int ny, int nz, double hx,
                   double hy, double hz, const hmfem_ele *v, const double *p,
                   int mem);

/* posprocessing_output.c:437-661 (save_pressure_1d, save_flux_1d): for
 * every conduit j, <dir>/pressure_karst_<j>.dat from pc and
 * <dir>/flux_karst_<j>.dat from 0.5 (ucr - ucl); pc / ucl / ucr in the
 * [i * number_karst + j] layout of hmfem_picard (nullable: that file is
 * skipped).  Position codes 1-7 as the writers know them (4-7: the
 * diagonal directions). */
int hmfem_save_karst(const char *dir, const hmfem_karst *k, double hx,
                     double hy, double hz, const double *pc, const double *ucl,
                     const double *ucr, int mem);

/* The conversion itself: "%.<prec>e\n" (conv 'e') or "%.<prec>f\n" (conv
 * 'f') for each of the n values, concatenated into out (cap bytes, host
 * memory); *used = bytes written (or needed: HMFEM_E_CAPACITY when they do
 * not fit in cap).  prec 0..17.  No reference counterpart:
 * the primitive the writers are built on, exposed for checks and callers
 * with their own file layouts. */
int hmfem_format_numbers(const double *x, long n, char conv, int prec,
                         char *out, long cap, long *used, int mem);

#ifdef __cplusplus
}
#endif
#endif
