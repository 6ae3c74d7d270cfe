/*
 * app_globals.h -- the global variables the reference application's main.c
 * defines (declared in its variables.h).  The reference's own C sources use
 * them, so every program that links those sources defines them exactly
 * once by including this file in one translation unit.  Test
 * infrastructure: used by the oracle harness (ref_harness.cpp) and by the
 * link test of the unmodified application (tests/link/app_main.cpp).
 */
#ifndef HMFEM_APP_GLOBALS_H
#define HMFEM_APP_GLOBALS_H
Dim N;
grid I, h;
Perm *P;
ELE *perm;
IND *indcol;
ELE *v;
Bound *B;
FACE boundary;
FACEK *BoundKarst;
IND *indcol1;
ELEK *uc;
Perm *KI;
DimK *M;
double *wi;
int *IDwi;
int Nwi;
int ix0, ixf, jy0, jyf;
double karst;
double viscosidade;
double **beta;
double rho;
int *n_brechas;
int **brechas;
double **pc_old;
double **ucL_old;
double **ucR_old;
double *hs;
double *Kc;
double **cont_karst;
int number_karst = 0;
int Mmax;
double **pc;
double **C;
double **C_contorno;
double nxg, nyg, nzg;
char fnam[1024];
const char *fn;
const char *fnwi;
const char *dirname = ".";
double time_total;
double time_amg;
int iter_amg;
int layer;
int lay;
#endif
