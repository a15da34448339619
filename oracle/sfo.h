/*
 * sfo.h -- CPU oracle for the SeisFEM mass-lumped explicit time-stepping path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C, FP64 restatement of the
 * reference algorithm, used by tests/, bench.py's cpu_baseline leg and
 * __graft_entry__.smoke() as the checker.  The product (libseisfem_b200.so)
 * never links, loads or calls anything here.
 *
 * Each function follows the reference file:line given in its comment, with
 * the same floating-point operation order (build with -ffp-contract=off), so
 * that its results are bit-identical to the reference compiled from source.
 * Array conventions follow the reference: element_node is 1-based and
 * element-major ([element_num * order]); node coordinates are split into
 * x[node_num], y[node_num] (the reference's node_xy[0], node_xy[1]); CSR
 * output is 0-based.
 */
#ifndef SFO_H
#define SFO_H

#ifdef __cplusplus
extern "C" {
#endif

/* element types, same codes as mesh/element_type.c */
enum { SFO_T3 = 1, SFO_T6 = 2, SFO_T10 = 3, SFO_Q4 = 4, SFO_Q9 = 5, SFO_Q16 = 6 };

int sfo_type_code(const char *type);          /* "Q4" -> 4, unknown -> -1 */
int sfo_element_order(int type_code);         /* Q4 -> 4 ... */

/* shape functions at (r, s) on the reference element (shape/shape_*.c) */
void sfo_shape(int type_code, double r, double s, double *t, double *dtdr, double *dtds);

/* consistent mass COO (assemble/mass_sparse_*.c, lumpflag=0).  COO entry
 * index = e*p*p + iq*p + jq.  Returns 0, or -1-e on a zero-area element. */
int sfo_mass_coo(int type_code, int node_num, int element_num, const int *element_node,
                 const double *x, const double *y, const double *rho,
                 int *mi, int *mj, double *mx);

/* lumped mass (assemble/mass_sparse_*.c, lumpflag=1) */
int sfo_mass_lumped(int type_code, int node_num, int element_num, const int *element_node,
                    const double *x, const double *y, const double *rho, double *mass_lump);

/* stiffness COO of type 0..6 (assemble/stiffness_sparse_*.c) */
int sfo_stif_coo(int type_code, int stif_type, int node_num, int element_num,
                 const int *element_node, const double *x, const double *y,
                 int *si, int *sj, double *sx);

/* COO -> canonical CSR (sparse_matrix/coo2csr_lib.f90:6-41).  Ai/Aj are
 * read-only here (the reference's +1 mutation is replayed only by the
 * Fortran-ABI wrapper).  Bp has p_size entries, Bj/Bx room for nnz.
 * Returns the CSR size. */
int sfo_coo2csr_canonical(int nnz, int p_size, const int *Ai, const int *Aj, const double *Ax,
                          int *Bp, int *Bj, double *Bx);

/* iargsort_quicksort (coo2csr_lib.f90:191-246): map[k] = 0-based source
 * position of the k-th sorted element of vec[0..n) */
void sfo_iargsort(const int *vec, int n, int *map);

/* M-PML damping profiles (pml/abc_mpml.c:1-201) */
void sfo_abc_mpml(int node_num, int element_num, int order, const int *element_node,
                  const double *x, const double *y, int mpml_nx, int mpml_ny, double h,
                  double xmin, double xmax, double ymin, double ymax, double vp_max,
                  int use_xmin, int use_xmax, int use_ymin, int use_ymax,
                  double *dx, double *dy, double *dxx, double *dyy, double *dxx_pyx,
                  double *dyy_pxy);

/* Ricker wavelet (source_receiver/seismic_source.c:1-24) */
double sfo_ricker(double f0, double t0, double magnitude, double t);

/* nearest node, last match wins, -1 on a miss (source_receiver/node_location.c:1-28) */
int sfo_node_location(int node_num, double edge_size, const double *x, const double *y,
                      double px, double py);

/* Full elastic_wave() run (time_evolution/elastic_wave.c:1-941, masslump
 * solver) with outputs in memory instead of text files.
 *   c: 4*node_num, c11 | c13 | c33 | c44 (the reference's c[0..3])
 *   seis_u / seis_w: [src_num][step-2][rec_num]   (may be NULL)
 *   snap_u / snap_w: [src_num][nsnap][node_num]   (may be NULL); row 0 is
 *     the all-zero initial field, then every snap_every steps ((it+1) %
 *     snap_every == 0); nsnap = 1 + floor(step / snap_every) - (rows that
 *     fall before it=2).  snap_every = 200 reproduces the reference.
 *   energy_u / energy_w: [src_num][step] (may be NULL)
 * Returns 0; 1 when the reference would exit(1) on the energy bound (the
 * run stops there, outputs keep what was written so far); 2 on bad input;
 * 4 when a consistent-mass solve did not converge. */
typedef struct {
    int type_code, node_num, element_num, order;
    const int *element_node;
    const double *x, *y;
    const double *rho, *vp, *vs, *c;
    int step; double dt, f0, t0, edge_size;
    double xmin, xmax, ymin, ymax;
    int pml_nx, pml_ny;
    int src_num; const int *src_node;
    int rec_num; const int *rec_node;
    int free_surface;
    int snap_every;
    int nthreads;           /* OpenMP threads, <=0: library default */
    double *timing;         /* optional out: [0] set-up seconds, [1] time-loop seconds */
    int consistent;         /* 0: solver "masslump"; 1: the consistent-mass branch (solver
                               "pardiso" / "mgmres", elastic_wave.c:664-680, 730-746): the 14
                               right-hand sides solved with M (Jacobi-preconditioned CG to a
                               1e-12 relative residual, from the previous values) */
} sfo_problem;

int sfo_elastic_run(const sfo_problem *pb, double *seis_u, double *seis_w,
                    double *snap_u, double *snap_w, double *energy_u, double *energy_w);

/* number of snapshot rows sfo_elastic_run writes per shot */
int sfo_snapshot_rows(int step, int snap_every);

/* Plain SpMV (sparse_matrix/csr_matvec.c:1-18) */
void sfo_csr_matvec(int p_size, const int *Bp, const int *Bj, const double *Bx,
                    const double *x, double *y);

/* Scalar acoustic solvers (time_evolution/acoustic.c, acoustic_pml.c),
 * solver "masslump", geometric mass matrix (no density).
 *   snap:   [sfo_acoustic_snapshot_rows(step, pml)][node_num]: the zero row,
 *           then u after every step with (it + 1) % 10 == 0 (20 with PML)
 *   energy: [step] sum of u^2 per step (entries 0 and 1 are 0)
 * Returns 0; 1 when acoustic_pml's energy bound (1e7) ended the run (the
 * outputs keep what was written before that step); 2 on bad input; 3 on a
 * zero-area element. */
typedef struct {
    int type_code, node_num, element_num, order;
    const int *element_node;
    const double *x, *y;
    const double *vp;
    int step; double dt, f0, t0;
    int source_node;        /* 0-based; -1: no source */
    int pml;                /* 0: acoustic.c, 1: acoustic_pml.c (PML on four sides) */
    double edge_size, xmin, xmax, ymin, ymax;
    int pml_nx, pml_ny;
    int nthreads;
} sfo_acoustic_problem;

int sfo_acoustic_run(const sfo_acoustic_problem *pb, double *snap, double *energy);
int sfo_acoustic_snapshot_rows(int step, int pml);
void sfo_abc_pml(int node_num, int element_num, int order, const int *element_node,
                 const double *x, const double *y, int pml_nx, int pml_ny, double h,
                 double xmin, double xmax, double ymin, double ymax, double vp_max,
                 int use_xmin, int use_xmax, int use_ymin, int use_ymax,
                 double *pdx, double *pdy, double *pdxx, double *pdyy);

#ifdef __cplusplus
}
#endif
#endif
