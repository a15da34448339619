/*
 * elastic_wave_dropin.c -- elastic_wave() with the reference's signature and
 * file behaviour (time_evolution/elastic_wave.c:1-3), computed on the GPU
 * through the sfg_* C ABI.
 *
 * Link this library instead of compiling time_evolution/elastic_wave.c into
 * the driver (seisfem/seisfem.c:26, 277-278).  What it keeps from the
 * reference:
 *   - the model: ./mesh/velocity_and_density.txt is read when
 *     use_exterior_mesh == 1, otherwise the built-in homogeneous model
 *     (model_elastic_parameter.c:34-45) is used and written to that file
 *     (elastic_wave.c:198-220);
 *   - outputs: ./outputfile/seismogram_{u,w}_shot_<k>.txt, one row per step
 *     with "%f   " per receiver (:787-795), and wavefield_{u,w}_shot_<k>.txt,
 *     the zero initial row then every 200 steps with "%f\t" per node
 *     (:466-507, 797-806);
 *   - fatal conditions exit(1) with the reference's messages: an unknown
 *     solver (:747-753) and the energy bound (:779-785; the rows computed
 *     before the failing step are written first).
 * Solver "masslump" takes the lumped-mass GPU path; "pardiso" and "mgmres"
 * take the consistent-mass path (SFG_FP64_CONSISTENT: the 14 systems of each
 * step solved with M by preconditioned conjugate gradients on the GPU, FP64);
 * any other string exits(1) like the reference.
 * Environment: SFG_DEVICE (CUDA device, default 0), SFG_PRECISION for
 * "masslump" (fp32k = FP32 with Kahan-compensated displacement, the default;
 * fp32; fp64).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/seisfem_b200.h"

static void builtin_model(int node_num, int element_num, int order, const int *element_node,
                          double *rho, double *vp, double *vs, double **c)
{
    /* model_elastic_parameter.c:34-45: every node of every element */
    for (long long k = 0; k < (long long)element_num * order; k++) {
        int p = element_node[k] - 1;
        double RHO = 2200.0, VP = 2000.0, VS = 1154.7;
        double miu = VS * VS * RHO;
        double lamda = VP * VP * RHO - 2 * miu;
        rho[p] = RHO;
        vp[p] = VP;
        vs[p] = VS;
        c[0][p] = lamda + 2 * miu;
        c[1][p] = lamda;
        c[2][p] = lamda + 2 * miu;
        c[3][p] = miu;
    }
    (void)node_num;
}

static void die(const char *a, const char *b)
{
    fprintf(stderr, "\n");
    fprintf(stderr, "%s", a);
    if (b) fprintf(stderr, "%s", b);
    exit(1);
}

void elastic_wave(char *type, int node_num, int element_num, int element_order, int *element_node,
                  double **node_xy, int nnz, int csr_p_size, int step, double dt, double f0,
                  double t0, double edge_size, double xmin, double xmax, double ymin, double ymax,
                  int pml_nx, int pml_ny, int src_num, int *src_node, int rec_num, int *rec_node,
                  char *solver, int use_exterior_mesh, int free_surface_code)
{
    (void)nnz;
    (void)csr_p_size;
    const int consistent = strcmp(solver, "pardiso") == 0 || strcmp(solver, "mgmres") == 0;
    if (strcmp(solver, "masslump") != 0 && !consistent) {
        fprintf(stderr, "\nELASTIC_MPML- Fatal error!\n  Solver type is not set = \"%s\".\n", solver);
        exit(1);
    }
    size_t N = (size_t)node_num;
    double *rho = calloc(N, sizeof(double)), *vp = calloc(N, sizeof(double)),
           *vs = calloc(N, sizeof(double)), *cc = calloc(4 * N, sizeof(double));
    double *c[4] = {cc, cc + N, cc + 2 * N, cc + 3 * N};
    FILE *fp;
    if (use_exterior_mesh == 1) {
        if ((fp = fopen("./mesh/velocity_and_density.txt", "r")) == NULL) {
            printf("\n test velocity_and_density.txt file cannot open\n");
            exit(1);
        }
        for (size_t i = 0; i < N; i++)
            if (fscanf(fp, "%lf %lf  %lf  %lf  %lf  %lf  %lf\n", &rho[i], &vp[i], &vs[i], &c[0][i], &c[1][i],
                       &c[2][i], &c[3][i]) != 7)
                break;
        fclose(fp);
    } else {
        builtin_model(node_num, element_num, element_order, element_node, rho, vp, vs, c);
        if ((fp = fopen("./mesh/velocity_and_density.txt", "w")) == NULL)
            printf("\n velocity_and_density.txt file cannot open\n");
        else {
            for (size_t i = 0; i < N; i++)
                fprintf(fp, "%f\t%f\t%f\t%f\t%f\t%f\t%f\n", rho[i], vp[i], vs[i], c[0][i], c[1][i], c[2][i],
                        c[3][i]);
            fclose(fp);
        }
    }

    const char *dev_s = getenv("SFG_DEVICE");
    sfg_ctx *ctx = sfg_create(dev_s ? atoi(dev_s) : 0);
    if (!ctx) die("ELASTIC_WAVE - Fatal error!\n", "  no usable sm_100 CUDA device.\n");
    sfg_mesh mesh = {type, node_num, element_num, element_order, element_node, node_xy[0], node_xy[1],
                     xmin, xmax, ymin, ymax, edge_size, pml_nx, pml_ny, free_surface_code};
    sfg_model model = {rho, vp, vs, cc};
    int rc = sfg_setup(ctx, &mesh, &model);
    if (rc != SFG_OK) {
        fprintf(stderr, "\nELASTIC_WAVE - Fatal error!\n  %s: %s\n", sfg_error_string(rc), sfg_last_error(ctx));
        exit(1);
    }
    int precision = SFG_FP32_KAHAN;
    const char *ps = getenv("SFG_PRECISION");
    if (ps && strcmp(ps, "fp64") == 0) precision = SFG_FP64;
    else if (ps && strcmp(ps, "fp32") == 0) precision = SFG_FP32;
    if (consistent) precision = SFG_FP64_CONSISTENT;

    const int rows = step - 2, nsnap = sfg_snapshot_rows(step, 200);
    double *su = malloc(sizeof(double) * (size_t)src_num * rows * (rec_num > 0 ? rec_num : 1));
    double *sw = malloc(sizeof(double) * (size_t)src_num * rows * (rec_num > 0 ? rec_num : 1));
    double *pu = malloc(sizeof(double) * (size_t)src_num * nsnap * N);
    double *pw = malloc(sizeof(double) * (size_t)src_num * nsnap * N);
    sfg_run_desc run = {step, dt, f0, t0, src_num, src_node, rec_num, rec_node, precision, 200, 0};
    rc = sfg_run(ctx, &run, su, sw, pu, pw);
    sfg_stats stats;
    sfg_get_stats(ctx, &stats);
    if (rc != SFG_OK && rc != SFG_ERR_BLOWUP) {
        fprintf(stderr, "\nELASTIC_WAVE - Fatal error!\n  %s: %s\n", sfg_error_string(rc), sfg_last_error(ctx));
        exit(1);
    }
    int last_it = rc == SFG_ERR_BLOWUP ? stats.blowup_step : step;   /* rows it < last_it are valid */
    for (int shot = 0; shot < src_num; shot++) {
        char fu[128], fw[128];
        printf("\n ######## Shot num: %d ########\n", shot + 1);
        sprintf(fu, "./outputfile/wavefield_u_shot_%d.txt", shot + 1);
        sprintf(fw, "./outputfile/wavefield_w_shot_%d.txt", shot + 1);
        FILE *wu = fopen(fu, "w"), *ww = fopen(fw, "w");
        sprintf(fu, "./outputfile/seismogram_u_shot_%d.txt", shot + 1);
        sprintf(fw, "./outputfile/seismogram_w_shot_%d.txt", shot + 1);
        FILE *gu = fopen(fu, "w"), *gw = fopen(fw, "w");
        const double *psu = pu + (size_t)shot * nsnap * N, *psw = pw + (size_t)shot * nsnap * N;
        int srow = 0;
        if (wu && ww) {
            for (size_t i = 0; i < N; i++) { fprintf(wu, "%f\t", psu[i]); fprintf(ww, "%f\t", psw[i]); }
            fprintf(wu, "\n");
            fprintf(ww, "\n");
        }
        srow = 1;
        for (int it = 2; it < step && it < last_it; it++) {
            const double *ru = su + ((size_t)shot * rows + (it - 2)) * rec_num;
            const double *rw = sw + ((size_t)shot * rows + (it - 2)) * rec_num;
            if (gu && gw) {
                for (int r = 0; r < rec_num; r++) { fprintf(gu, "%f   ", ru[r]); fprintf(gw, "%f   ", rw[r]); }
                fprintf(gu, "\n");
                fprintf(gw, "\n");
            }
            if ((it + 1) % 200 == 0 && wu && ww) {
                const double *a = psu + (size_t)srow * N, *b = psw + (size_t)srow * N;
                for (size_t i = 0; i < N; i++) { fprintf(wu, "%f\t", a[i]); fprintf(ww, "%f\t", b[i]); }
                fprintf(wu, "\n");
                fprintf(ww, "\n");
                srow++;
            }
        }
        if (wu) fclose(wu);
        if (ww) fclose(ww);
        if (gu) fclose(gu);
        if (gw) fclose(gw);
        printf("\nTime iteration end!\n");
    }
    free(su); free(sw); free(pu); free(pw);
    free(rho); free(vp); free(vs); free(cc);
    sfg_destroy(ctx);
    if (rc == SFG_ERR_BLOWUP) die("ELASTIC_MPML - Fatal error!\n", "Energy exceeds maximum value!\n");
}
