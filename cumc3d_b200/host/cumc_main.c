/* cumc_main.c -- a plain C host program driving the engine through the C-ABI
 * (include/cumc3d_gpu.h), in the order of the reference's main program
 * (solver/mhd/main.f90:50-139):
 *
 *   GET_MODEL (here: the Brio-Wu shock tube of model/riemann/src/riemann1d.f90:229-250)
 *   -> cumc_create (BUILD_* + GETGRID + *_WEIGHT + POPULATE_DEVICE)
 *   -> cumc_set_state -> cumc_initial_update (INITIAL_UPDATE)
 *   -> DO WHILE (global_time < total_time)
 *        cumc_finddt ; IF (global_time + dt > total_time) dt = total_time - global_time
 *        cumc_rk3_step ; global_time = global_time + dt
 *   -> cumc_get_state -> cumc_destroy
 *
 * Usage: cumc_main NX OUTFILE
 * Writes prim (nz+6, ny+6, nx+6, 8) and epsilon (nz+6, ny+6, nx+6) as raw
 * little-endian doubles to OUTFILE and prints "steps <n> time <t>".
 * Build: gcc -std=c99 -I include cumc_main.c libcumc3d_gpu.so -o cumc_main
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "cumc3d_gpu.h"

static int check(cumc_handle *h, int rc, const char *what) {
    if (rc != CUMC_OK) fprintf(stderr, "%s failed (%d): %s\n", what, rc, cumc_last_error(h));
    return rc;
}

int main(int argc, char **argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: %s NX OUTFILE\n", argv[0]);
        return 2;
    }
    const int nx = atoi(argv[1]);
    if (nx < 8) return 2;
    const int NX = nx + 6, NY = 7, NZ = 7;
    const size_t n3 = (size_t)NX * NY * NZ;
    const double gamma = 2.0, total_time = 0.1;

    /* face coordinates -3..n+3 of [0,1] (getgrid.f90:26-34); y, z one cell */
    double *xF = malloc(sizeof(double) * (size_t)(nx + 7));
    double yF[8], zF[8];
    for (int j = -3; j <= nx + 3; ++j) xF[j + 3] = 0.0 + (double)j * ((1.0 - 0.0) / (double)nx);
    for (int j = -3; j <= 4; ++j) yF[j + 3] = zF[j + 3] = (double)j;

    /* GET_MODEL: Brio-Wu on cells 0..nx, split at x = 0.5; epsilon left
     * undefined (NaN) elsewhere, as the reference never sets it there */
    double *prim = calloc(8 * n3, sizeof(double));
    double *eps = malloc(sizeof(double) * n3);
    for (size_t i = 0; i < n3; ++i) eps[i] = NAN;
    for (int l = 0; l < NZ; ++l)
        for (int k = 0; k < NY; ++k)
            for (int j = 0; j <= nx; ++j) {
                const double xc = (xF[j + 3] + xF[j + 2]) / 2.0;  /* cell j spans faces j-1..j */
                const int left = xc <= 0.5;
                const size_t c = (size_t)(j + 2) + (size_t)NX * ((size_t)k + (size_t)NY * (size_t)l);
                double *p = prim + 8 * c;
                p[0] = left ? 1.0 : 0.125;  /* rho */
                p[4] = left ? 1.0 : 0.1;    /* p */
                p[6] = left ? 1.0 : -1.0;   /* By */
                p[5] = 0.75;                /* Bx */
                eps[c] = p[4] / p[0] / (gamma - 1.0);
            }

    cumc_config cfg = {0};
    cfg.nx = nx; cfg.ny = 1; cfg.nz = 1; cfg.n_dim = 1; cfg.coordinate_flag = 0;
    for (int i = 0; i < 6; ++i) cfg.boundary_flag[i] = 1; /* outflow */
    cfg.xF = xF; cfg.yF = yF; cfg.zF = zF;
    cfg.cfl = 0.8;
    cfg.recon = CUMC_RECON_PPM;
    cfg.riemann = CUMC_RS_HLLD;
    cfg.precision = CUMC_FP64;
    cfg.model.gamma = gamma;
    cfg.model.floor_kind = CUMC_FLOOR_EPS;

    cumc_handle *h = NULL;
    if (check(NULL, cumc_create(&cfg, &h), "cumc_create")) return 1;
    int rc = check(h, cumc_set_state(h, prim, eps), "cumc_set_state");
    if (!rc) rc = check(h, cumc_initial_update(h), "cumc_initial_update");
    double global_time = 0.0;
    int n_step = 0;
    while (!rc && global_time < total_time) {
        double dt = 0.0;
        rc = check(h, cumc_finddt(h, &dt), "cumc_finddt");
        if (rc) break;
        if (global_time + dt > total_time) dt = total_time - global_time;
        rc = check(h, cumc_rk3_step(h, dt), "cumc_rk3_step");
        n_step = n_step + 1;
        global_time = global_time + dt;
    }
    if (!rc) rc = check(h, cumc_get_state(h, prim, eps), "cumc_get_state");
    cumc_destroy(h);
    if (!rc) {
        FILE *f = fopen(argv[2], "wb");
        if (!f || fwrite(prim, sizeof(double), 8 * n3, f) != 8 * n3 || fwrite(eps, sizeof(double), n3, f) != n3) rc = 1;
        if (f) fclose(f);
        printf("steps %d time %.17g\n", n_step, global_time);
    }
    free(xF);
    free(prim);
    free(eps);
    return rc ? 1 : 0;
}
