/*
 * ref_acoustic_harness.c -- builds the REFERENCE's scalar acoustic solvers
 * (time_evolution/acoustic.c and time_evolution/acoustic_pml.c, compiled
 * where they lie via -I<reference root>; nothing is copied) into
 * oracle/_ref/libsfacoustic.so.
 *
 * TEST INFRASTRUCTURE ONLY (pins the acoustic restatement in sfo.c).
 *
 * The two files are not wired into the reference's main() and were written
 * against older signatures of three helpers; the macros below bridge them
 * without touching the files:
 *   mass_sparse_all(10 arguments)  -> the current 11-argument function with
 *                                     rho = 1 everywhere (the older function
 *                                     had no density: M = integral phi_i phi_j;
 *                                     multiplying by 1.0 is exact, so the
 *                                     values are those of that function);
 *   absorbing_boundary_pml(...)    -> abc_pml (pml/abc_pml.c), the same list;
 *   acoustic_model(...)            -> fills vp from the caller's array (the
 *                                     reference's model file hard-codes two
 *                                     half-spaces; rho is not used by either
 *                                     solver).
 * stdio is shimmed as in ref_harness.c: every "%f" printed to u.dat is
 * recorded in FP64 (the snapshot rows), every "%f" printed to energy.dat is
 * recorded (the energy per step), exit() returns to the harness with status
 * 1 (the energy bound of acoustic_pml.c:440-446), printf and the messages to
 * stderr are silenced unless SFR_VERBOSE is set, and malloc zero-fills.
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

static FILE *g_fu, *g_fe, *g_open[16];
static int g_nopen;
static double *g_snap, *g_energy;
static long g_snap_cap, g_snap_n, g_energy_cap, g_energy_n;
static const double *g_vp;
static double *g_step_t;        /* CLOCK_MONOTONIC at each energy.dat value */
static long g_step_cap, g_step_n;
static double *g_ones;
static jmp_buf g_jmp;
static int g_in_run;

static FILE *sfa_fopen(const char *path, const char *mode)
{
    FILE *f = fopen(path, mode);
    if (!f) return f;
    if (g_nopen < 16) g_open[g_nopen++] = f;
    if (strcmp(path, "u.dat") == 0) g_fu = f;
    if (strcmp(path, "energy.dat") == 0) g_fe = f;
    return f;
}

static int sfa_fclose(FILE *f)
{
    for (int i = 0; i < g_nopen; i++)
        if (g_open[i] == f) {
            g_open[i] = g_open[--g_nopen];
            if (f == g_fu) g_fu = NULL;
            if (f == g_fe) g_fe = NULL;
            return fclose(f);
        }
    return 0;
}

static int sfa_fprintf(FILE *f, const char *fmt, ...)
{
    if (f == stderr && !getenv("SFR_VERBOSE")) return 0;
    va_list ap, ap2;
    va_start(ap, fmt);
    va_copy(ap2, ap);
    if (f && fmt[0] == '%' && fmt[1] == 'f') {
        const double v = va_arg(ap2, double);
        if (f == g_fu && g_snap && g_snap_n < g_snap_cap) g_snap[g_snap_n] = v;
        if (f == g_fu) g_snap_n++;
        if (f == g_fe && g_energy && g_energy_n < g_energy_cap) g_energy[g_energy_n] = v;
        if (f == g_fe) g_energy_n++;
        if (f == g_fe && g_step_t && g_step_n < g_step_cap) {
            struct timespec ts;
            clock_gettime(CLOCK_MONOTONIC, &ts);
            g_step_t[g_step_n++] = (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
        }
    }
    va_end(ap2);
    const int n = vfprintf(f, fmt, ap);
    va_end(ap);
    return n;
}

static int sfa_printf(const char *fmt, ...)
{
    if (!getenv("SFR_VERBOSE")) return 0;
    va_list ap;
    va_start(ap, fmt);
    const int n = vprintf(fmt, ap);
    va_end(ap);
    return n;
}

static void *sfa_malloc(size_t n) { return calloc(1, n ? n : 1); }

static void sfa_exit(int code)
{
    if (g_in_run) longjmp(g_jmp, code ? code : 1);
    exit(code);
}

/* COO -> canonical CSR: the reference's Fortran module restated in C
 * (oracle/coo2csr_f90abi.c, linked into this library) */
void __coo2csr_lib_MOD_coo2csr_canonical(int *nnz, int *Bp_size, int *csr_size, int *Ai, int *Aj,
                                         double *Ax, int *Bp, int *Bj, double *Bx);

static void sfa_model(int node_num, int element_num, int element_order, int *element_node,
                      double **node_xy, double *rho, double *vp)
{
    (void)element_num; (void)element_order; (void)element_node; (void)node_xy;
    for (int i = 0; i < node_num; i++) {
        rho[i] = 1.0;
        vp[i] = g_vp[i];
    }
}

#define fopen sfa_fopen
#define fclose sfa_fclose
#define fprintf sfa_fprintf
#define printf sfa_printf
#define malloc sfa_malloc
#define exit sfa_exit

/* ---------------------------------------------- the reference's own code */
#include "assemble/mass_sparse_all.c"
#include "assemble/stif_sparse_all.c"
#include "pml/abc_pml.c"
#include "sparse_matrix/csr_matvec.c"
#include "source_receiver/seismic_source.c"

#define mass_sparse_all(t, n, e, o, en, xy, mi, mj, mx, l) \
    mass_sparse_all(t, n, e, o, en, xy, g_ones, mi, mj, mx, l)
#define absorbing_boundary_pml abc_pml
#define acoustic_model sfa_model

#include "time_evolution/acoustic_pml.c" /* includes solver/mgmres/mgmres.c itself */
#include "time_evolution/acoustic.c"

#undef mass_sparse_all
#undef absorbing_boundary_pml
#undef acoustic_model
#undef fopen
#undef fclose
#undef fprintf
#undef printf
#undef malloc
#undef exit

/* -------------------------------------------------------- exported API */

/* Per-step timestamps of the next runs: the CLOCK_MONOTONIC time of every
 * value printed to energy.dat (two before the loop, then one at the end of
 * each time step, acoustic.c:206 / acoustic_pml.c:456); buf = NULL stops. */
void sfa_set_step_times(double *buf, long cap)
{
    g_step_t = buf;
    g_step_cap = cap;
    g_step_n = 0;
}

static int run_begin(const char *workdir, char *cwd, size_t ncwd, int nthreads, int node_num,
                     const double *vp, double *snap, long snap_cap, double *energy, long energy_cap)
{
    if (!getcwd(cwd, ncwd)) return 2;
    if (chdir(workdir) != 0) return 2;
    g_fu = g_fe = NULL;
    g_nopen = 0;
    g_snap = snap; g_snap_cap = snap_cap; g_snap_n = 0;
    g_energy = energy; g_energy_cap = energy_cap; g_energy_n = 0;
    g_vp = vp;
    g_ones = (double *)calloc((size_t)(node_num > 0 ? node_num : 1), sizeof(double));
    if (!g_ones) return 2;
    for (int i = 0; i < node_num; i++) g_ones[i] = 1.0;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    return 0;
}

static int run_end(const char *cwd, int rc, long *snap_values, long *energy_values)
{
    while (g_nopen > 0) fclose(g_open[--g_nopen]);
    g_fu = g_fe = NULL;
    free(g_ones);
    g_ones = NULL;
    if (snap_values) *snap_values = g_snap_n;
    if (energy_values) *energy_values = g_energy_n;
    g_snap = g_energy = NULL;
    if (chdir(cwd) != 0) return 2;
    return rc;
}

/* Run the reference acoustic() in workdir (u.dat and energy.dat are written
 * there).  snap [snap_cap] receives every value printed to u.dat: the zero
 * row, then u_now after every time step whose (it + 1) % 10 == 0
 * (acoustic.c:147-154,197-205); energy [energy_cap] receives energy[0..step-1]
 * (acoustic.c:156-158,206).  *snap_values / *energy_values get the counts.
 * Returns 0, 3 for a solver string other than masslump / mgmres (the
 * reference exits), 2 on a harness error or when step > node_num: acoustic.c
 * allocates energy[] with node_num entries (acoustic.c:84) and writes
 * energy[it] for it < step, past its end on such runs. */
int sfa_acoustic(const char *workdir, int nthreads, char *type, int node_num, int element_num,
                 int order, int *element_node, double *x, double *y, int step, double dt,
                 double f0, double t0, int source_node, char *solver, const double *vp,
                 double *snap, long snap_cap, double *energy, long energy_cap,
                 long *snap_values, long *energy_values, double *seconds)
{
    char cwd[4096];
    if (step > node_num) return 2;
    int rc = run_begin(workdir, cwd, sizeof cwd, nthreads, node_num, vp, snap, snap_cap, energy,
                       energy_cap);
    if (rc) return rc;
    double *xy[2] = {x, y};
    struct timespec a, b;
    clock_gettime(CLOCK_MONOTONIC, &a);
    g_in_run = 1;
    rc = setjmp(g_jmp);
    if (rc == 0)
        acoustic(type, node_num, element_num, order, element_node, xy, element_num * order * order,
                 node_num + 1, step, dt, f0, t0, source_node, solver);
    g_in_run = 0;
    clock_gettime(CLOCK_MONOTONIC, &b);
    if (seconds) *seconds = (double)(b.tv_sec - a.tv_sec) + 1e-9 * (double)(b.tv_nsec - a.tv_nsec);
    return run_end(cwd, rc == 1 ? 3 : rc, snap_values, energy_values);
}

/* Run the reference acoustic_pml() (classical split PML on all four sides,
 * acoustic_pml.c:93-96).  snap receives the zero row, then u_now after every
 * step whose (it + 1) % 20 == 0 (acoustic_pml.c:260-268,448-455); energy as
 * above.  Returns 0, 1 when the reference called exit(1) (the energy bound,
 * acoustic_pml.c:440-446, or an unknown solver string), 2 on a harness
 * error. */
int sfa_acoustic_pml(const char *workdir, int nthreads, char *type, int node_num, int element_num,
                     int order, int *element_node, double *x, double *y, int step, double dt,
                     double f0, double t0, double edge_size, double xmin, double xmax, double ymin,
                     double ymax, int pml_nx, int pml_ny, int source_node, char *solver,
                     const double *vp, double *snap, long snap_cap, double *energy,
                     long energy_cap, long *snap_values, long *energy_values, double *seconds)
{
    char cwd[4096];
    int rc = run_begin(workdir, cwd, sizeof cwd, nthreads, node_num, vp, snap, snap_cap, energy,
                       energy_cap);
    if (rc) return rc;
    double *xy[2] = {x, y};
    struct timespec a, b;
    clock_gettime(CLOCK_MONOTONIC, &a);
    g_in_run = 1;
    rc = setjmp(g_jmp);
    if (rc == 0)
        acoustic_pml(type, node_num, element_num, order, element_node, xy,
                     element_num * order * order, node_num + 1, step, dt, f0, t0, edge_size, xmin,
                     xmax, ymin, ymax, pml_nx, pml_ny, source_node, solver);
    g_in_run = 0;
    clock_gettime(CLOCK_MONOTONIC, &b);
    if (seconds) *seconds = (double)(b.tv_sec - a.tv_sec) + 1e-9 * (double)(b.tv_nsec - a.tv_nsec);
    return run_end(cwd, rc, snap_values, energy_values);
}
