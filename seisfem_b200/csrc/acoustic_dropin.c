/*
 * acoustic_dropin.c -- acoustic() and acoustic_pml() with the reference's
 * signatures and file behaviour (time_evolution/acoustic.c:1,
 * time_evolution/acoustic_pml.c:3), computed on the GPU through
 * sfg_acoustic_run.
 *
 * What each keeps from the reference:
 *   - the model of model_elastic_parameter/acoustic_model.c:17-42 (vp 2000
 *     where x >= 0 and y >= 0, else 3000; rho is not used by the solvers);
 *   - u.dat: the zero row, then u every 10 steps (acoustic.c:147-154,
 *     197-205) or every 20 steps (acoustic_pml.c:260-268, 448-455), "%f\t"
 *     per node; energy.dat: "%f\n" per step, entries 0 and 1 first;
 *   - acoustic_pml only: stif_p.dat / stif_j.dat / stif_x.dat, the canonical
 *     CSR of stiffness type 6 ("%d\n", "%d\n", "%f\n", acoustic_pml.c:252-258);
 *   - fatal conditions exit(1) with the reference's messages: an unknown
 *     solver (acoustic.c:176-182, acoustic_pml.c:387-393) and the PML energy
 *     bound (acoustic_pml.c:440-446; the rows of the steps before it are
 *     written first).
 * Solver "masslump" is the GPU path; "mgmres" (consistent-mass solves) is not
 * provided and exits like an unknown solver.  SFG_DEVICE picks the device.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/seisfem_acoustic.h"

static void acoustic_model_vp(int element_num, int order, const int *element_node, double **node_xy, double *vp)
{
    for (long long k = 0; k < (long long)element_num * order; k++) {
        const int p = element_node[k] - 1;
        const double x = node_xy[0][p], y = node_xy[1][p];
        vp[p] = (x >= 0 && y >= 0) ? 2000 : 3000;
    }
}

static void bad_solver(const char *who, const char *solver)
{
    fprintf(stderr, "\n");
    fprintf(stderr, "%s - Fatal error!\n", who);
    fprintf(stderr, "  Solver type is not set = \"%s\".\n", solver);
    exit(1);
}

static void write_outputs(int node_num, int step, int every, int last, const double *snap, const double *energy)
{
    FILE *fu = fopen("u.dat", "w"), *fe = fopen("energy.dat", "w");
    const size_t N = (size_t)node_num;
    int row = 0;
    if (fu) {
        for (size_t i = 0; i < N; i++) fprintf(fu, "%f\t", snap[i]);
        fprintf(fu, "\n");
    }
    row = 1;
    if (fe) {
        fprintf(fe, "%f\n", energy[0]);
        fprintf(fe, "%f\n", energy[1]);
    }
    for (int it = 2; it < step && it < last; it++) {
        if ((it + 1) % every == 0) {
            if (fu) {
                const double *r = snap + (size_t)row * N;
                for (size_t i = 0; i < N; i++) fprintf(fu, "%f\t", r[i]);
                fprintf(fu, "\n");
            }
            row++;
        }
        if (fe) fprintf(fe, "%f\n", energy[it]);
    }
    if (fu) fclose(fu);
    if (fe) fclose(fe);
}

static int run(const char *who, char *type, int node_num, int element_num, int element_order, int *element_node,
               double **node_xy, int step, double dt, double f0, double t0, double edge_size, double xmin,
               double xmax, double ymin, double ymax, int pml_nx, int pml_ny, int source_node, int pml)
{
    const size_t N = (size_t)node_num;
    double *vp = calloc(N ? N : 1, sizeof(double));
    acoustic_model_vp(element_num, element_order, element_node, node_xy, vp);
    const char *dev_s = getenv("SFG_DEVICE");
    sfg_ctx *ctx = sfg_create(dev_s ? atoi(dev_s) : 0);
    if (!ctx) {
        fprintf(stderr, "\n%s - Fatal error!\n  no usable sm_100 CUDA device.\n", who);
        exit(1);
    }
    sfg_mesh mesh = {type, node_num, element_num, element_order, element_node, node_xy[0], node_xy[1],
                     xmin, xmax, ymin, ymax, edge_size, pml_nx, pml_ny, 0};
    sfg_acoustic_desc desc = {pml, step, dt, f0, t0, source_node, NULL};
    const int rows = sfg_acoustic_snapshot_rows(step, pml);
    double *snap = calloc((size_t)rows * N, sizeof(double)), *energy = calloc((size_t)step, sizeof(double));
    sfg_acoustic_stats stats;
    int rc = sfg_acoustic_run(ctx, &mesh, vp, &desc, snap, energy, &stats);
    if (rc != SFG_OK && rc != SFG_ERR_BLOWUP) {
        fprintf(stderr, "\n%s - Fatal error!\n  %s: %s\n", who, sfg_error_string(rc), sfg_last_error(ctx));
        exit(1);
    }
    write_outputs(node_num, step, pml ? 20 : 10, rc == SFG_ERR_BLOWUP ? stats.blowup_step : step, snap, energy);
    free(snap);
    free(energy);
    free(vp);
    sfg_destroy(ctx);
    return rc;
}

void acoustic(char *type, int node_num, int element_num, int element_order, int *element_node, double **node_xy,
              int nnz, int csr_p_size, int step, double dt, double f0, double t0, int source_node, char *solver)
{
    (void)nnz;
    (void)csr_p_size;
    if (strcmp(solver, "masslump") != 0) bad_solver("ACOUSTIC", solver);
    run("ACOUSTIC", type, node_num, element_num, element_order, element_node, node_xy, step, dt, f0, t0, 0.0, 0.0,
        0.0, 0.0, 0.0, 0, 0, source_node, 0);
    printf("\n Acoutsic Normal End!\n");
}

void acoustic_pml(char *type, int node_num, int element_num, int element_order, int *element_node,
                  double **node_xy, int nnz, int csr_p_size, int step, double dt, double f0, double t0,
                  double edge_size, double xmin, double xmax, double ymin, double ymax, int pml_nx, int pml_ny,
                  int source_node, char *solver)
{
    if (strcmp(solver, "masslump") != 0) bad_solver("ACOUSTIC_PML", solver);
    /* stif_{p,j,x}.dat: the canonical CSR of stiffness type 6 (phi * dphidy) */
    int *si = malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1)), *sj = malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
    double *sx = malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
    int *bp = calloc((size_t)csr_p_size, sizeof(int)), *bj = calloc((size_t)(nnz > 0 ? nnz : 1), sizeof(int));
    double *bx = calloc((size_t)(nnz > 0 ? nnz : 1), sizeof(double));
    int csr_size = 0;
    int rc = sfg_stif_sparse_all(type, node_num, element_num, element_order, element_node, node_xy, si, sj, sx, 6);
    if (rc == SFG_OK) rc = sfg_coo2csr_canonical(&nnz, &csr_p_size, &csr_size, si, sj, sx, bp, bj, bx);
    if (rc != SFG_OK) {
        fprintf(stderr, "\nACOUSTIC_PML - Fatal error!\n  %s\n", sfg_error_string(rc));
        exit(1);
    }
    FILE *fp = fopen("stif_p.dat", "w"), *fj = fopen("stif_j.dat", "w"), *fx = fopen("stif_x.dat", "w");
    for (int i = 0; fp && i < csr_p_size; i++) fprintf(fp, "%d\n", bp[i]);
    for (int i = 0; fj && fx && i < csr_size; i++) {
        fprintf(fj, "%d\n", bj[i]);
        fprintf(fx, "%f\n", bx[i]);
    }
    if (fp) fclose(fp);
    if (fj) fclose(fj);
    if (fx) fclose(fx);
    free(si); free(sj); free(sx); free(bp); free(bj); free(bx);
    printf("\nTime iteration begin:\n");
    rc = run("ACOUSTIC_PML", type, node_num, element_num, element_order, element_node, node_xy, step, dt, f0, t0,
             edge_size, xmin, xmax, ymin, ymax, pml_nx, pml_ny, source_node, 1);
    if (rc == SFG_ERR_BLOWUP) {
        fprintf(stderr, "\n");
        fprintf(stderr, "ACOUSTIC_PML - Fatal error!\n");
        fprintf(stderr, "Energy exceeds maximum value!\n");
        exit(1);
    }
    printf("\nTime iteration end!\n");
    printf("\n Acoutsic Normal End!\n");
}
