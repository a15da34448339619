/*
 * ref_harness.c -- builds the REFERENCE's own C sources (compiled where they
 * lie, via -I<reference root>; nothing is copied) into oracle/_ref/libsfref.so
 * and exposes its functions through a small C API for the tests.
 *
 * TEST INFRASTRUCTURE ONLY (pins the oracle restatement; CPU baseline).
 *
 * The reference writes its results as "%f" text.  To compare in full FP64
 * precision, stdio calls made by the reference code are routed through the
 * sfr_* shims below (macros defined before the reference files are included):
 *   fopen/fprintf  record every double printed to seismogram_{u,w}_shot_k and
 *                  wavefield_{u,w}_shot_k into caller-provided arrays (the text
 *                  files are still written, so the timed I/O cost is kept);
 *   fclose         ignores the second close of the same FILE* (the reference
 *                  closes fp_wavefield_u twice, elastic_wave.c:812-813) and
 *                  files left open are closed after the run;
 *   malloc         zero-fills (Dirichlet_boundary_node_flag is never
 *                  initialised to 0, elastic_wave.c:136-155);
 *   exit           returns to the harness with status 1 (energy bound,
 *                  elastic_wave.c:779-785);
 *   printf         silenced unless SFR_VERBOSE is set.
 * PARDISO (a proprietary library, absent) is a stub that returns to the
 * harness with status 3; solver "mgmres" runs the reference's own
 * solver/mgmres/mgmres.c (the consistent-mass branch).
 */
#include <math.h>
#include <omp.h>
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

/* ----------------------------------------------------------------- shims */
enum { CAP_SU, CAP_SW, CAP_PU, CAP_PW, CAP_N };
typedef struct {
    double *buf[CAP_N];
    long per_shot[CAP_N];   /* values per shot */
    long count[CAP_N];      /* values recorded in the current file */
    FILE *fp[CAP_N];
    int shot[CAP_N];
} capture_t;
static capture_t g_cap;
static FILE *g_open[64];
static int g_nopen;
static jmp_buf g_jmp;
static int g_in_run;
/* exit() requested from inside an OpenMP parallel region (the energy bound,
 * elastic_wave.c:754-785): a worker thread cannot jump out, so the request
 * is recorded and served by the next shimmed call on the master thread */
static volatile int g_exit_code;

static void serve_exit(void)
{
    if (g_exit_code && g_in_run && !omp_in_parallel()) {
        int c = g_exit_code;
        g_exit_code = 0;
        longjmp(g_jmp, c);
    }
}
/* per-step timestamps: the reference ends every time step by writing "\n"
 * to seismogram_u_shot_k (elastic_wave.c:794) */
static double *g_step_t;
static long g_step_n, g_step_cap;

static double now_s(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static FILE *sfr_fopen(const char *path, const char *mode)
{
    serve_exit();
    FILE *f = fopen(path, mode);
    if (!f) return f;
    if (g_nopen < 64) g_open[g_nopen++] = f;
    static const char *tags[CAP_N] = {"seismogram_u_shot_", "seismogram_w_shot_",
                                      "wavefield_u_shot_", "wavefield_w_shot_"};
    for (int k = 0; k < CAP_N; k++) {
        const char *p = strstr(path, tags[k]);
        if (p) {
            g_cap.fp[k] = f;
            g_cap.shot[k] = atoi(p + strlen(tags[k])) - 1;
            g_cap.count[k] = 0;
        }
    }
    return f;
}

static int sfr_fclose(FILE *f)
{
    for (int i = 0; i < g_nopen; i++)
        if (g_open[i] == f) {
            g_open[i] = g_open[--g_nopen];
            for (int k = 0; k < CAP_N; k++) if (g_cap.fp[k] == f) g_cap.fp[k] = NULL;
            return fclose(f);
        }
    return 0;   /* already closed */
}

static int sfr_fprintf(FILE *f, const char *fmt, ...)
{
    serve_exit();
    va_list ap, ap2;
    va_start(ap, fmt);
    va_copy(ap2, ap);
    for (int k = 0; k < CAP_N; k++) {
        if (f && f == g_cap.fp[k] && fmt[0] == '%' && fmt[1] == 'f') {
            double v = va_arg(ap2, double);
            if (g_cap.buf[k] && g_cap.count[k] < g_cap.per_shot[k])
                g_cap.buf[k][(long)g_cap.shot[k] * g_cap.per_shot[k] + g_cap.count[k]] = v;
            g_cap.count[k]++;
            break;
        }
    }
    va_end(ap2);
    if (f && f == g_cap.fp[CAP_SU] && fmt[0] == '\n' && g_step_t && g_step_n < g_step_cap)
        g_step_t[g_step_n++] = now_s();
    int n = vfprintf(f, fmt, ap);
    va_end(ap);
    return n;
}

static int sfr_printf(const char *fmt, ...)
{
    serve_exit();
    if (!getenv("SFR_VERBOSE")) return 0;
    va_list ap;
    va_start(ap, fmt);
    int n = vprintf(fmt, ap);
    va_end(ap);
    return n;
}

static void *sfr_malloc(size_t n) { return calloc(1, n ? n : 1); }

static void sfr_exit(int code)
{
    if (g_in_run && omp_in_parallel()) {
        g_exit_code = code ? code : 1;
        return;
    }
    if (g_in_run) longjmp(g_jmp, code ? code : 1);
    exit(code);
}

void pardiso_unsym(int a, int b, int *c, int *d, double *e, double *f, double *g)
{
    (void)a; (void)b; (void)c; (void)d; (void)e; (void)f; (void)g;
    sfr_exit(3);
}

/* COO -> canonical CSR: the reference's Fortran module, restated in C
 * (oracle/coo2csr_f90abi.c) because no Fortran compiler is available */
void __coo2csr_lib_MOD_coo2csr_canonical(int *nnz, int *Bp_size, int *csr_size, int *Ai, int *Aj,
                                         double *Ax, int *Bp, int *Bj, double *Bx);

#define fopen sfr_fopen
#define fclose sfr_fclose
#define fprintf sfr_fprintf
#define printf sfr_printf
#define malloc sfr_malloc
#define exit sfr_exit

/* ---------------------------------------------- the reference's own code */
#include "mesh/element_type.c"
#include "mesh/mesh_element_order.c"
#include "mesh/mesh_node_num.c"
#include "mesh/mesh_element_num.c"
#include "mesh/mesh_element.c"
#include "mesh/mesh_xy.c"
#include "assemble/mass_sparse_all.c"
#include "assemble/stif_sparse_all.c"
#include "model_elastic_parameter/model_elastic_parameter.c"
#include "pml/abc_mpml.c"
#include "sparse_matrix/csr_matvec.c"
#include "source_receiver/node_location.c"
#include "source_receiver/set_receiver_node.c"
#include "source_receiver/set_source_node.c"
#include "source_receiver/seismic_source.c"
#include "source_receiver/set_rec_and_src.c"
#include "solver/solver_type.c"
#include "solver/mgmres/mgmres.c"
#include "time_evolution/elastic_wave.c"

#undef fopen
#undef fclose
#undef fprintf
#undef printf
#undef malloc
#undef exit

/* -------------------------------------------------------- exported API */

void sfr_mass_sparse_all(char *type, int node_num, int element_num, int order, int *element_node,
                         double *x, double *y, double *rho, int *mi, int *mj, double *mx,
                         int lumpflag)
{
    double *xy[2] = {x, y};
    mass_sparse_all(type, node_num, element_num, order, element_node, xy, rho, mi, mj, mx, lumpflag);
}

void sfr_stif_sparse_all(char *type, int node_num, int element_num, int order, int *element_node,
                         double *x, double *y, int *si, int *sj, double *sx, int stif_type)
{
    double *xy[2] = {x, y};
    stif_sparse_all(type, node_num, element_num, order, element_node, xy, si, sj, sx, stif_type);
}

void sfr_abc_mpml(int node_num, int element_num, int order, int *element_node, double *x, double *y,
                  int nx, int ny, double h, double xmin, double xmax, double ymin, double ymax,
                  double vp_max, int uxmin, int uxmax, int uymin, int uymax, double *out6)
{
    double *xy[2] = {x, y};
    size_t N = (size_t)node_num;
    for (size_t i = 0; i < 6 * N; i++) out6[i] = 0.0;
    abc_mpml(node_num, element_num, order, element_node, xy, nx, ny, h, xmin, xmax, ymin, ymax,
             vp_max, uxmin, uxmax, uymin, uymax, out6, out6 + N, out6 + 2 * N, out6 + 3 * N,
             out6 + 4 * N, out6 + 5 * N);
}

double sfr_seismic_source(double f0, double t0, double mag, double t)
{
    return seismic_source(f0, t0, mag, t);
}

int sfr_node_location(int node_num, double edge_size, double *x, double *y, double px, double py)
{
    double *xy[2] = {x, y};
    return node_location(node_num, edge_size, xy, px, py);
}

void sfr_csr_matvec(int p_size, int *Bp, int *Bj, double *Bx, double *x, double *y)
{
    csr_matvec(p_size, Bp, Bj, Bx, x, y);
}

void sfr_mesh(char *type, int nelemx, int nelemy, double xmin, double xmax, double ymin,
              double ymax, int *element_node, double *x, double *y)
{
    /* seisfem.c:216-232 internal mesh */
    int node_num = mesh_node_num(type, nelemx, nelemy);
    double *xy[2] = {x, y};
    mesh_element(type, nelemx, nelemy, element_node);
    mesh_xy(type, nelemx, nelemy, node_num, xmin, xmax, ymin, ymax, xy);
}

int sfr_mesh_sizes(char *type, int nelemx, int nelemy, int *node_num, int *element_num)
{
    *node_num = mesh_node_num(type, nelemx, nelemy);
    *element_num = mesh_element_num(type, nelemx, nelemy);
    return mesh_element_order(type);
}

/* Run the reference elastic_wave() in workdir (must hold mesh/ and
 * outputfile/; mesh/velocity_and_density.txt when use_exterior_mesh == 1).
 * Captured FP64 outputs: seis_u/seis_w [src_num][step-2][rec_num],
 * snap_u/snap_w [src_num][snap_rows][node_num] (any may be NULL).
 * Returns 0, 1 on the energy bound, 3 on a non-masslump solver; *seconds
 * gets the wall time of the elastic_wave() call; step_times (may be NULL)
 * gets the CLOCK_MONOTONIC time at the end of each time step of shot 1.
 * sfr_now() reads the same clock. */
double sfr_now(void) { return now_s(); }
int sfr_elastic_wave(const char *workdir, int nthreads, char *type, int node_num, int element_num,
                     int order, int *element_node, double *x, double *y, int step, double dt,
                     double f0, double t0, double edge_size, double xmin, double xmax, double ymin,
                     double ymax, int pml_nx, int pml_ny, int src_num, int *src_node, int rec_num,
                     int *rec_node, char *solver, int use_exterior_mesh, int free_surface,
                     double *seis_u, double *seis_w, double *snap_u, double *snap_w, int snap_rows,
                     double *seconds, double *step_times, int step_times_cap)
{
    char cwd[4096];
    if (!getcwd(cwd, sizeof cwd)) return 2;
    if (chdir(workdir) != 0) return 2;
    memset(&g_cap, 0, sizeof g_cap);
    g_cap.buf[CAP_SU] = seis_u; g_cap.per_shot[CAP_SU] = (long)(step - 2) * rec_num;
    g_cap.buf[CAP_SW] = seis_w; g_cap.per_shot[CAP_SW] = (long)(step - 2) * rec_num;
    g_cap.buf[CAP_PU] = snap_u; g_cap.per_shot[CAP_PU] = (long)snap_rows * node_num;
    g_cap.buf[CAP_PW] = snap_w; g_cap.per_shot[CAP_PW] = (long)snap_rows * node_num;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    g_step_t = step_times;
    g_step_n = 0;
    g_step_cap = step_times_cap;
    double *xy[2] = {x, y};
    struct timespec a, b;
    clock_gettime(CLOCK_MONOTONIC, &a);
    g_in_run = 1;
    g_exit_code = 0;
    int rc = setjmp(g_jmp);
    if (rc == 0)
        elastic_wave(type, node_num, element_num, order, element_node, xy,
                     element_num * order * order, node_num + 1, step, dt, f0, t0, edge_size,
                     xmin, xmax, ymin, ymax, pml_nx, pml_ny, src_num, src_node, rec_num, rec_node,
                     solver, use_exterior_mesh, free_surface);
    g_in_run = 0;
    g_step_t = NULL;
    clock_gettime(CLOCK_MONOTONIC, &b);
    while (g_nopen > 0) fclose(g_open[--g_nopen]);
    memset(&g_cap, 0, sizeof g_cap);
    if (seconds) *seconds = (double)(b.tv_sec - a.tv_sec) + 1e-9 * (double)(b.tv_nsec - a.tv_nsec);
    if (chdir(cwd) != 0) return 2;
    return rc;
}
