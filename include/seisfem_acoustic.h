/*
 * seisfem_acoustic.h -- C ABI of the scalar acoustic solvers in
 * libseisfem_b200.so: SeisFEM's time_evolution/acoustic.c (no absorbing
 * boundary) and time_evolution/acoustic_pml.c (split-field classical PML on
 * four sides), solver "masslump", computed on the GPU.
 *
 * Both reference solvers advance
 *     M u_new = 2 M u_now - M u_old - vp^2 dt^2 K u_now + source   (acoustic.c:160-165)
 * (the PML solver in four split equations, acoustic_pml.c:277-353) and divide
 * by the lumped mass.  M is the geometric consistent mass (the reference
 * files call mass_sparse_all without a density), K the Laplacian stiffness
 * (stif_sparse_all type 0) or, with PML, the stiffness types 1, 5, 2, 6; all
 * assembled and canonicalised on the GPU with the same code as the elastic
 * path.  The step runs in FP64 in the reference's operation order (no FMA);
 * given the same lumped mass (sfg_acoustic_desc.mass_lump) the snapshots are
 * bit-identical to the reference's.
 */
#ifndef SEISFEM_ACOUSTIC_H
#define SEISFEM_ACOUSTIC_H

#include "seisfem_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int pml;                   /* 0: acoustic.c; 1: acoustic_pml.c (PML thickness pml_nx, pml_ny and
                                  edge_size of the mesh description, on all four sides) */
    int step;                  /* the loop runs it = 2 .. step-1 (acoustic.c:135) */
    double dt, f0, t0;         /* Ricker amplitude 1 (acoustic.c:137) */
    int source_node;           /* 0-based; -1: no source */
    const double *mass_lump;   /* [node_num] lumped mass to use, or NULL: assembled on the GPU (its
                                  normalisation sum is parallel, ~1e-14 relative to the reference's) */
} sfg_acoustic_desc;

typedef struct {
    double setup_ms;           /* assembly, canonical CSR, lumped mass, step data */
    double loop_ms;            /* time loop only (CUDA events around the graph launch) */
    long long union_nnz;       /* entries the step kernel streams per time step */
    long long csr_nnz[5];      /* canonical CSR sizes: M, then K0 (acoustic) or K1, K5, K2, K6 */
    int kernel_launches;       /* kernels in the time loop */
    int blowup_step;           /* first step whose energy passed 1e7 (PML only), -1 if none */
} sfg_acoustic_stats;

/* rows sfg_acoustic_run writes to snap: the zero row, then u after every
 * step with (it + 1) % 10 == 0 (acoustic.c:197), 20 with PML
 * (acoustic_pml.c:448) */
int sfg_acoustic_snapshot_rows(int step, int pml);

/* Assemble and run.  vp: [node_num].  Outputs (either may be NULL):
 *   snap    [sfg_acoustic_snapshot_rows(step, pml)][node_num]
 *   energy  [step]: sum of u^2 after each step (entries 0 and 1 are 0)
 * Returns SFG_ERR_BLOWUP when the PML solver's energy bound (1e7,
 * acoustic_pml.c:440-446) ended the run: snap and energy then hold what the
 * reference had written before that step.  stats may be NULL. */
int sfg_acoustic_run(sfg_ctx *ctx, const sfg_mesh *mesh, const double *vp, const sfg_acoustic_desc *desc,
                     double *snap, double *energy, sfg_acoustic_stats *stats);

/* Drop-in replacements with the reference's signatures
 * (time_evolution/acoustic.c:1, time_evolution/acoustic_pml.c:3): the model
 * of model_elastic_parameter/acoustic_model.c, u.dat and energy.dat (and, with
 * PML, stif_p.dat / stif_j.dat / stif_x.dat) written in the working
 * directory in the reference's formats.  Fatal conditions print the
 * reference's message and call exit(1). */
void acoustic(char *type, int node_num, int element_num, int element_order, int *element_node,
              double **node_xy, int nnz, int csr_p_size, int step, double dt, double f0, double t0,
              int source_node, char *solver);
void acoustic_pml(char *type, int node_num, int element_num, int element_order, int *element_node,
                  double **node_xy, int nnz, int csr_p_size, int step, double dt, double f0, double t0,
                  double edge_size, double xmin, double xmax, double ymin, double ymax, int pml_nx,
                  int pml_ny, int source_node, char *solver);

#ifdef __cplusplus
}
#endif
#endif
