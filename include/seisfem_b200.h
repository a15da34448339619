/*
 * seisfem_b200.h -- C ABI of libseisfem_b200.so, a B200 (sm_100a) drop-in for
 * SeisFEM's mass-lumped explicit time-stepping path.
 *
 * Three layers:
 *   1. elastic_wave()            the reference's own entry point, same
 *                                signature, same files, computed on the GPU;
 *   2. sfg_* seams               the inner reference functions elastic_wave()
 *                                calls (assembly, COO->CSR, M-PML, SpMV), same
 *                                argument meaning, computed on the GPU;
 *   3. sfg_ctx API               explicit context: assemble once, run many
 *                                shots (batched), read results, with int
 *                                status codes instead of exit(1).
 *
 * Conventions (as in the reference): element_node is 1-based and
 * element-major [element_num * element_order]; node coordinates are two
 * arrays x = node_xy[0], y = node_xy[1]; CSR output is 0-based; model c[] is
 * [4][node_num] = c11, c13, c33, c44.  All host pointers are borrowed for the
 * duration of a call only.  Every sfg_* call returns SFG_OK (0) or an
 * SFG_ERR_* code; sfg_last_error() gives the message.  One context is used
 * by one host thread at a time; contexts are independent.
 */
#ifndef SEISFEM_B200_H
#define SEISFEM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define SFG_OK 0
#define SFG_ERR_ARG 1         /* bad argument: NULL, size, type or solver string */
#define SFG_ERR_CUDA 2        /* CUDA runtime error (message in sfg_last_error) */
#define SFG_ERR_OOM 3         /* device allocation failed */
#define SFG_ERR_ZERO_AREA 4   /* an element of zero area (mass_sparse_q4.c:191-196) */
#define SFG_ERR_BADINDEX 5    /* element_node / source / receiver index out of range */
#define SFG_ERR_BLOWUP 6      /* energy above 1e7 or non-finite (elastic_wave.c:779-785) */
#define SFG_ERR_ROWLEN 7      /* a matrix row longer than the device canonicaliser handles */
#define SFG_ERR_STATE 8       /* call out of order (run before setup, ...) */
#define SFG_ERR_TIMEOUT 9     /* a bounded device-side wait gave up */
#define SFG_ERR_NODEVICE 10   /* no CUDA device / wrong architecture */
#define SFG_ERR_LIMIT 11      /* size above the fixed limit of a no-allocation entry point */
#define SFG_ERR_NOCONV 12     /* a consistent-mass solve did not converge in its iterations */

/* ------------------------------------------------------------- precision */
#define SFG_FP32_KAHAN 0      /* FP32 step, Kahan-compensated displacement (default) */
#define SFG_FP32 1            /* FP32 step, plain accumulation */
#define SFG_FP64 2            /* FP64 step, reference operation order, no FMA */
#define SFG_FP32_PLAIN_PATH 3 /* FP32, one SpMV launch per product + pointwise
                                 kernels, as elastic_wave.c structures the step
                                 (the unfused baseline) */
#define SFG_FP64_CONSISTENT 4 /* FP64 step with the consistent mass matrix: the 14 right-hand
                                 sides solved with M (solver "pardiso" / "mgmres",
                                 elastic_wave.c:664-680, 730-746) by Jacobi-preconditioned
                                 conjugate gradients to 1e-12 relative residual; one shot at
                                 a time, no Dirichlet zeroing (as the reference's branch) */

/* matrices: 0 = consistent mass M, 1..6 = stiffness types 1..6
 * (elastic_wave.c:6-17; stif type 0 is not on the path) */
#define SFG_MAT_MASS 0

typedef struct sfg_ctx sfg_ctx;

typedef struct {
    const char *type;          /* "T3","T6","T10","Q4","Q9","Q16" */
    int node_num;
    int element_num;
    int element_order;
    const int *element_node;   /* 1-based, [element_num * element_order] */
    const double *x;           /* node_xy[0] */
    const double *y;           /* node_xy[1] */
    double xmin, xmax, ymin, ymax;
    double edge_size;
    int pml_nx, pml_ny;        /* M-PML thickness in elements */
    int free_surface;          /* 1: x = xmax is a free surface */
} sfg_mesh;

typedef struct {
    const double *rho;         /* [node_num] */
    const double *vp;          /* [node_num] (vp_max sets the M-PML profile) */
    const double *vs;          /* [node_num] (carried, unused by the path) */
    const double *c;           /* [4][node_num] c11, c13, c33, c44 */
} sfg_model;

typedef struct {
    int step;                  /* the loop runs it = 2 .. step-1 (elastic_wave.c:519) */
    double dt, f0, t0;
    int src_num;  const int *src_node;   /* 0-based node per shot */
    int rec_num;  const int *rec_node;   /* 0-based node per receiver */
    int precision;             /* SFG_FP32_KAHAN, SFG_FP32, SFG_FP64, SFG_FP32_PLAIN_PATH,
                                  SFG_FP64_CONSISTENT */
    int snap_every;            /* 0: no snapshots; 200 reproduces the reference */
    int shots_per_batch;       /* shots advanced together; 0 = automatic */
} sfg_run_desc;

typedef struct {
    double setup_ms;           /* last sfg_setup: assembly + canonical CSR on the GPU */
    double loop_ms;            /* last sfg_run: time loop only (CUDA events) */
    double total_ms;           /* last sfg_run: including transfers */
    long long dof_steps;       /* 2 * node_num * shots * (step - 2) of the last run */
    long long union_nnz;       /* nonzeros of the union pattern the step kernel streams */
    long long csr_nnz[7];      /* nonzeros of M, K1..K6 after zero elimination */
    int kernel_launches;       /* kernels launched by the last run's time loop */
    int rows_per_block;        /* launch shapes the autotuner picked for the class-A and
                                  class-Z kernels: one shot: a * 16 + z (shape variants);
                                  batches: a * 256 + z, each spl * 16 + warps per block */
    int blowup_step;           /* first step whose energy bound failed, -1 if none */
    int interior_rows;         /* nodes advanced as totals only (outside the M-PML zone) */
    int pml_rows;              /* rows with a non-zero M-PML profile */
    int value_tuples;          /* distinct (M / rho, K1..K6) tuples the one-shot step kernels read
                                  from a dictionary; 0 when they stream full values per entry */
    int cm_iterations;         /* SFG_FP64_CONSISTENT: conjugate-gradient iterations of the last
                                  finished batch, all its steps together */
} sfg_stats;

/* ---------------------------------------------------------- context API */
sfg_ctx *sfg_create(int device);                  /* NULL when no usable device */
void sfg_destroy(sfg_ctx *ctx);
const char *sfg_error_string(int status);
const char *sfg_last_error(const sfg_ctx *ctx);

/* Assemble M, K1..K6 (FP64, bit-exact COO values), canonicalise them to CSR
 * (bit-exact with coo2csr_lib.f90), lumped mass, M-PML profiles, Dirichlet
 * flags, and build the device step data.  Replaces elastic_wave.c:136-313. */
int sfg_setup(sfg_ctx *ctx, const sfg_mesh *mesh, const sfg_model *model);

/* The canonical CSR of matrix 0..6 (M, K1..K6; coo2csr_lib.f90's output:
 * p [node_num+1], j and x [nnz], 0-based).  sfg_setup keeps the union of the
 * seven patterns with their values; the first sfg_csr_copy of a set-up forms
 * every matrix's CSR from it (its nonzero union entries in column order, the
 * same arrays) and keeps them on the device. */
int sfg_csr_nnz(sfg_ctx *ctx, int matrix, int *nnz);
int sfg_csr_copy(sfg_ctx *ctx, int matrix, int *p, int *j, double *x);
int sfg_lumped_mass_copy(sfg_ctx *ctx, double *mass_lump);         /* [node_num] */
/* the union sparsity pattern of M, K1..K6 that the step kernels stream
 * (p: [node_num+1], j: [*nnz]; either may be NULL to query the size) */
int sfg_union_copy(sfg_ctx *ctx, int *p, int *j, long long *nnz);
int sfg_mpml_copy(sfg_ctx *ctx, double *out6);                       /* [6][node_num] */
/* Replace the lumped mass used by the time loop (e.g. a caller's own
 * lumping).  The reference's normalisation mass_sum/diag_sum
 * (mass_sparse_q4.c:259-263) is a long sequential FP64 sum; sfg_setup forms
 * it with a fixed-shape parallel sum, equal to ~1e-14 relative. */
int sfg_lumped_mass_set(sfg_ctx *ctx, const double *mass_lump);     /* [node_num] */

/* Run every shot (elastic_wave.c:446-809).  Outputs (any may be NULL):
 *   seis_u, seis_w  [src_num][step-2][rec_num]  displacement at receivers
 *   snap_u, snap_w  [src_num][rows][node_num]   row 0 = initial zero field,
 *                   then each step with (it+1) % snap_every == 0
 * Returns SFG_ERR_BLOWUP (results up to the failing step are valid) when the
 * reference would have stopped on its energy bound. */
int sfg_run(sfg_ctx *ctx, const sfg_run_desc *run, double *seis_u, double *seis_w,
            double *snap_u, double *snap_w);
int sfg_snapshot_rows(int step, int snap_every);
int sfg_get_stats(const sfg_ctx *ctx, sfg_stats *stats);

/* Same run with the seismograms written to DEVICE pointers (FP64, layout as
 * sfg_run) and the work queued on `stream` (a cudaStream_t; NULL = the
 * context's stream).  Returns when the work is done. */
int sfg_run_device(sfg_ctx *ctx, const sfg_run_desc *run, void *d_seis_u, void *d_seis_w,
                   void *stream);

/* Prepared runs.  sfg_plan_create allocates one batch's device state, stages
 * every batch's sources on the device, picks the launch shape (autotuner) and
 * captures the whole time loop of a batch -- state reset, one fused kernel
 * per step, snapshot copies, receiver gathers -- into a CUDA graph.
 * sfg_plan_launch queues batch b (shots b*S .. b*S+S-1) on `stream`
 * asynchronously; sfg_plan_finish waits for it, copies its outputs to the
 * given host or device buffers (full [src_num]... layout as sfg_run; any may
 * be NULL) and applies the energy bound.  A plan is bound to its context and
 * to the context's current set-up. */
typedef struct sfg_plan sfg_plan;
int sfg_plan_create(sfg_ctx *ctx, const sfg_run_desc *run, sfg_plan **plan);
int sfg_plan_batches(const sfg_plan *plan);
int sfg_plan_launches(const sfg_plan *plan);   /* kernels one batch launches */
int sfg_plan_launch(sfg_plan *plan, int batch, void *stream);
int sfg_plan_finish(sfg_plan *plan, int batch, double *seis_u, double *seis_w, double *snap_u,
                    double *snap_w, void *stream);
void sfg_plan_destroy(sfg_plan *plan);

/* One model per shot (no counterpart in the reference, which runs one model
 * per call): shot s of the run uses models[s] -- the same mesh, its own rho,
 * vp and c[4] of node_num entries -- while the context's set-up model only
 * supplies the geometric matrices.  Shots of a batch advance together: the
 * consistent mass is applied as diag(rho) M_geo, each shot carries its own
 * constants, lumped mass (the reference's normalisation, per model) and
 * M-PML scale (d0 is proportional to vp_max).  Compensated FP32 only
 * (SFG_FP32_KAHAN), batches of 32 or 64 shots (shots_per_batch 0, 32 or 64). */
int sfg_plan_create_models(sfg_ctx *ctx, const sfg_run_desc *run, const sfg_model *models, sfg_plan **plan);
int sfg_run_models(sfg_ctx *ctx, const sfg_run_desc *run, const sfg_model *models, double *seis_u,
                   double *seis_w, double *snap_u, double *snap_w);

/* Plan groups: several single-batch plans -- independent problems on meshes
 * of any sizes, which the reference runs one after another
 * (time_evolution/elastic_wave.c:446-518 loops over shots; its callers over
 * meshes) -- advanced by one CUDA-graph launch.  The group's graph composes
 * the plans' own graphs side by side: every mesh advances on its own, with no
 * per-step join across meshes.  With SFG_GROUP_FUSED=1, when every plan is a
 * one-shot fused FP32 plan (SFG_FP32_KAHAN or SFG_FP32) with the same step
 * count and all or none of the meshes carry a value dictionary, the graph
 * instead issues one class-A and one class-Z kernel per time step for all
 * meshes together (each block finds its mesh in a block map; measured slower
 * on B200).
 * Results are read per plan with sfg_plan_finish(plan, 0, ...) after the
 * group's stream has finished.  A group uses its plans' buffers: do not
 * launch a member plan while the group runs; destroy the group before its
 * plans.  All plans must live on one device. */
typedef struct sfg_group sfg_group;
int sfg_group_create(sfg_plan *const *plans, int nplans, sfg_group **group);
int sfg_group_launch(sfg_group *group, void *stream);
int sfg_group_launches(const sfg_group *group);   /* kernels one launch runs */
/* 0: child graphs; else 1 + the multi-mesh kernels' launch shapes (class A * 16 + class Z) */
int sfg_group_fused(const sfg_group *group);
void sfg_group_destroy(sfg_group *group);
int sfg_sync(sfg_ctx *ctx);

/* ----------------------------------------------------------- the seams */
/* drop-in for time_evolution/elastic_wave.c:1-3 (solver "masslump"; any other
 * solver string exits like the reference, elastic_wave.c:747-753) */
void elastic_wave(char *type, int node_num, int element_num, int element_order, int *element_node,
                  double **node_xy, int nnz, int csr_p_size, int step, double dt, double f0,
                  double t0, double edge_size, double xmin, double xmax, double ymin, double ymax,
                  int pml_nx, int pml_ny, int src_num, int *src_node, int rec_num, int *rec_node,
                  char *solver, int use_exterior_mesh, int free_surface_code);

/* assemble/mass_sparse_all.c:13-68 (lumpflag 1: mass_coo_x[0..node_num) is the lumped mass) */
int sfg_mass_sparse_all(char *type, int node_num, int element_num, int element_order,
                        int *element_node, double **node_xy, double *rho, int *mass_coo_i,
                        int *mass_coo_j, double *mass_coo_x, int lumpflag);
/* assemble/stif_sparse_all.c:8-62 */
int sfg_stif_sparse_all(char *type, int node_num, int element_num, int element_order,
                        int *element_node, double **node_xy, int *stiffi, int *stiffj,
                        double *stiffness, int stif_type);
/* sparse_matrix/coo2csr_lib.f90:6-41 (Fortran ABI in elastic_wave.c:241): all
 * by pointer, Ai/Aj left incremented by one like the reference, 0-based output */
int sfg_coo2csr_canonical(int *nnz, int *Bp_size, int *csr_size, int *Ai, int *Aj, double *Ax,
                          int *Bp, int *Bj, double *Bx);
/* pml/abc_mpml.c:1-4 */
int sfg_abc_mpml(int node_num, int element_num, int element_order, int *element_node,
                 double **node_xy, int mpml_nx, int mpml_ny, double h, double xmin, double xmax,
                 double ymin, double ymax, double vp_max, int use_mpml_xmin, int use_mpml_xmax,
                 int use_mpml_ymin, int use_mpml_ymax, double *mpml_dx, double *mpml_dy,
                 double *mpml_dxx, double *mpml_dyy, double *mpml_dxx_pyx, double *mpml_dyy_pxy);
/* sparse_matrix/csr_matvec.c:1 (FP64, same per-row summation order) */
int sfg_csr_matvec(int Bp_size, int *Bp, int *Bj, double *Bx, double *x, double *y);
/* source_receiver/node_location.c:1-35 for npts points at once (host code):
 * out[k] = the LAST node index with |x - px[k]| <= edge_size / 2 and
 * |y - py[k]| <= edge_size / 2 (the reference's comparison), -1 when none;
 * a grid of edge_size cells replaces the O(node_num) scan per point.  The
 * reference's callers (set_source_node.c, set_receiver_node.c) print its
 * "-1" message themselves when they see -1. */
int sfg_node_location(int node_num, double edge_size, const double *x, const double *y, int npts,
                      const double *px, const double *py, int *out);

/* ------------------------------------------------ no-allocation entry point */
/* No counterpart in the reference.  The M-PML profiles of sfg_abc_mpml
 * (pml/abc_mpml.c:1-201, bit-identical results) for node arrays that are
 * already on the device, computed without allocating device memory: for
 * callers that must not call cudaMalloc/cudaFree while other work runs (both
 * synchronise the whole device), e.g. an inversion loop that recomputes the
 * profiles for each new velocity model next to streams that are stepping.
 *
 * d_element_node (1-based), d_x, d_y: device arrays; d_out6: device
 * [6][node_num] = dx, dy, dxx, dyy, dxx*pyx, dyy*pxy; nodes of no element keep
 * their values.  The work runs on `stream` (a cudaStream_t) and the call
 * returns after it has finished.  Use a stream created with
 * cudaStreamNonBlocking: NULL (the legacy default stream) is accepted, but it
 * waits for, and holds up, every blocking stream of the device, which defeats
 * running next to other work.
 *
 * Scratch: a fixed device array of SFG_NOALLOC_MAX_NODES + 256 bytes inside
 * the library (every device that loads the library holds it until exit); the
 * call clears what it uses itself, so nothing has to start at zero.
 * node_num above SFG_NOALLOC_MAX_NODES returns SFG_ERR_LIMIT.  Each call
 * looks up the scratch address in the current context (the first call on a
 * device loads it); make that first call before any stream capture.  The call
 * waits for its stream to read back an error word, so a stream that is being
 * captured is refused with SFG_ERR_ARG.  Calls that overlap in time on one
 * device (two host threads, or two streams) share the scratch and race:
 * serialise them.  Returns SFG_ERR_BADINDEX, with d_out6 untouched, when an
 * element_node entry is outside 1..node_num. */
#define SFG_NOALLOC_MAX_NODES (1 << 22)
int sfg_abc_mpml_device_noalloc(int node_num, int element_num, int element_order, const int *d_element_node,
                                const double *d_x, const double *d_y, int mpml_nx, int mpml_ny, double h,
                                double xmin, double xmax, double ymin, double ymax, double vp_max,
                                int use_mpml_xmin, int use_mpml_xmax, int use_mpml_ymin, int use_mpml_ymax,
                                double *d_out6, void *stream);

#ifdef __cplusplus
}
#endif
#endif
