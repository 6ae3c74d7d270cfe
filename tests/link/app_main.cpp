/*
 * app_main.cpp -- link test of the drop-in boundary (test infrastructure).
 *
 * The reference application's own sources -- reservoir.c, permeabilities.c,
 * set_boundaries.c, set_source_term.c, solve_linearsystem_AMG.c,
 * create_variables.c -- are compiled unmodified from the hmfem tree
 * (tests/link/Makefile) and linked with this main() against
 * libhmfem_gpu.so instead of compute.cpp.  The call chain is the
 * application's: reservoir() (reservoir.c:8-57) -> permeabilidade_arestas
 * -> source_term -> solve_linsys (solve_linearsystem_AMG.c:37-157, the
 * application's own packing) -> compute(), which resolves to the GPU
 * library.  The library sets the application's iter_amg (defined here, in
 * the executable; the library's definition is weak).
 *
 *   app_link nx ny nz K.bin p.bin     (K: n float64, isotropic; p: output)
 *
 * Prints "iter_amg <n>".  Boundary conditions as main.c's run: Dirichlet
 * p = 1 on x = 0 and p = 0 on x = 1, no-flow elsewhere (val_bound and
 * boundary types of main.c:140-152, 347-359 with the y faces closed).
 */
#include <cstdio>
#include <cstdlib>

#include "structs.h"
#include "functions.h"
#include "app_globals.h"

int main(int argc, char **argv)
{
    if (argc != 6) {
        fprintf(stderr, "usage: app_link nx ny nz K.bin p.bin\n");
        return 2;
    }
    N.x = atoi(argv[1]); N.y = atoi(argv[2]); N.z = atoi(argv[3]);
    N.xy = N.x * N.y; N.t = N.xy * N.z;
    const int n = N.t;
    I.x = I.y = I.z = 1.0;
    h.x = 1.0 / N.x; h.y = 1.0 / N.y; h.z = 1.0 / N.z;
    viscosidade = 1.0;
    number_karst = 0;
    boundary.l = 0; boundary.r = 0;
    boundary.u = 1; boundary.d = 1; boundary.t = 1; boundary.b = 1;

    double *K = create_vector(n);
    FILE *f = fopen(argv[4], "rb");
    if (!f || fread(K, sizeof(double), n, f) != (size_t)n) {
        fprintf(stderr, "cannot read %s\n", argv[4]);
        return 2;
    }
    fclose(f);
    Perm Kp;
    Kp.X = K; Kp.Y = K; Kp.Z = K;

    B = (Bound *)malloc(sizeof(Bound));
    B->l = create_vector(n); B->r = create_vector(n); B->u = create_vector(n);
    B->d = create_vector(n); B->t = create_vector(n); B->b = create_vector(n);
    double val_bound[7] = {0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0};  /* L R U D T B */
    create_boundary(val_bound, B, N, boundary);

    perm = (ELE *)malloc(sizeof(ELE) * n);
    indcol = (IND *)malloc(sizeof(IND) * n);
    for (int s = 0; s < n; s++) {
        indcol[s].c = indcol[s].u = indcol[s].d = indcol[s].l = -1;
        indcol[s].r = indcol[s].t = indcol[s].b = -1;
    }
    double *WI = create_vector(n), *KIv = create_vector(n), *pw = create_vector(n);
    double *p = create_vector(n);
    iter_amg = -1;
    reservoir(N, &Kp, WI, KIv, nullptr, indcol, B, perm, h, boundary, viscosidade,
              pw, nullptr, p);
    f = fopen(argv[5], "wb");
    if (!f || fwrite(p, sizeof(double), n, f) != (size_t)n) {
        fprintf(stderr, "cannot write %s\n", argv[5]);
        return 2;
    }
    fclose(f);
    printf("iter_amg %d\n", iter_amg);
    return 0;
}
