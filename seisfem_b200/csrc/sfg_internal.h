// sfg_internal.h -- device data of one context and the launchers shared by
// the CUDA translation units (assembly, canonical CSR, step kernels, API).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/seisfem_b200.h"

namespace sfg {

// Error flags raised by device code (bitwise OR into one int).
enum DevFlag {
    FLAG_ZERO_AREA = 1,
    FLAG_ROWLEN = 2,
    FLAG_BADINDEX = 4,
    FLAG_SORT_STACK = 8,
};

// Device memory block with size, freed by the owner.
template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
};

// Canonical CSR (FP64) of one matrix on the device.
struct DevCsr {
    int *p = nullptr;
    int *j = nullptr;
    double *x = nullptr;
    long long nnz = 0;
};

// Assembled problem on the device (owned by the context).
struct DevProblem {
    int type_code = 0, order = 0, node_num = 0, element_num = 0;
    long long coo_nnz = 0;
    // union pattern of M, K1..K6 (all distinct columns of every row), FP64
    // values of the seven matrices at the union positions, [7][union_nnz]
    int *up = nullptr;
    int *uj = nullptr;
    double *ux = nullptr;
    long long union_nnz = 0;
    int max_row_len = 0;
    // the canonical CSR of each matrix, built from the union on first use
    // (csr_ensure); their nonzero counts from set-up
    DevCsr csr[7];
    long long csr_nnz[7] = {0, 0, 0, 0, 0, 0, 0};
    double *mass_lump = nullptr;     // [N]
    double *mpml = nullptr;          // [6][N]: dx, dy, dxx, dyy, dxx_pyx, dyy_pxy
    double *coef64 = nullptr;        // [4][N] c11, c13, c33, c44
    unsigned char *dirichlet = nullptr;  // [N]
    // FP32 fused step data, in the two-class numbering of sfg_step32.cuh:
    // row r' is mesh node perm[r'], node i is row inv[i]; rows [0, na) are
    // class A (interior), [na, N) class Z (split zone)
    float *coef32 = nullptr;         // [N][12], mesh order (unfused path)
    int *perm = nullptr, *inv = nullptr;
    std::vector<int> h_inv, h_perm;
    int na = 0;
    float *sellA = nullptr, *sellZ = nullptr;   // SELL-32 slots (6 / 8 planes of 32)
    int *sliceA = nullptr, *sliceZ = nullptr;
    long long slotsA = 0, slotsZ = 0;
    int *upp = nullptr;              // permuted union row pointers
    float *recp = nullptr;           // permuted row-major records [union_nnz][8]
    float *recA = nullptr;           // folded class-A records (batches with one model), built on first use
    // value dictionary of the one-shot kernels (sfg_dict.cu); dict_n = 0 without one
    int dict_n = 0;
    float4 *dict = nullptr;          // [2 dict_n]
    int2 *sellAd = nullptr, *sellZd = nullptr;   // SELL-32 slots (column, tuple id)
    float *rowrho = nullptr;         // [N] row density, permuted
    std::vector<float4> h_dict;      // host copy of dict
    // staged-gather tiles (sfg_step32.cuh: Step2::tile*); tileA_off == nullptr without them
    unsigned *sellAt = nullptr, *sellZt = nullptr;
    int *tileA_off = nullptr, *tileA_ext = nullptr, *tileZ_off = nullptr, *tileZ_ext = nullptr;
    int haloA_max = 0, haloZ_max = 0, slotsA_max = 0, slotsZ_max = 0;
    float4 *coefA = nullptr;         // [na]
    float *imA = nullptr;            // [na]
    float *coefZ = nullptr;          // [N - na][12]
    double *coefd = nullptr;         // [N][12] FP64 coefficients for the FP64 step
    // the set-up model's density and the Dirichlet flags, for runs with one
    // model per shot (geometric mass matrix, per-shot lumped masses)
    double *rho0 = nullptr;          // [N] device
    std::vector<double> h_rho0;
    std::vector<unsigned char> h_dir;
};

// ---- assembly (sfg_assemble.cu) ------------------------------------------
// All launchers queue work on `st` and return a cudaError_t.
cudaError_t launch_element_coo(int tc, int E, const int *d_en, const double *d_x, const double *d_y,
                               const double *d_rho, int nmat, const int *mats, int *d_ci, int *d_cj,
                               double *d_cx, int *d_flags, cudaStream_t st);
cudaError_t launch_lumped_mass(int tc, int N, int E, const int *d_en, const double *d_x,
                               const double *d_y, const double *d_rho, const int *d_row_start,
                               const int *d_bucket, const int *d_cj, double *d_mass,
                               double *d_scratch, int *d_flags, cudaStream_t st);
cudaError_t launch_mpml(int N, const double *d_x, const double *d_y, const int *d_row_start,
                        double d0x, double d0y, double tx, double ty, double x0, double x1,
                        double y0, double y1, int uxmin, int uxmax, int uymin, int uymax,
                        double *d_out6, cudaStream_t st);

// COO -> canonical CSR for nv value streams sharing one (i, j) pattern.
// Produces, per value stream, the CSR bit-exact with coo2csr_lib.f90, and
// optionally the union pattern with the nv values at each union entry.
struct CanonOut {
    DevCsr csr[8];
    int *up = nullptr, *uj = nullptr;
    double *ux = nullptr;   // [nv][union_nnz]
    long long union_nnz = 0;
    int max_row_len = 0;
    int *row_start = nullptr;   // COO bucket offsets [N+1] (kept for the lumped mass)
    int *bucket = nullptr;      // COO indices per row, ascending [nnz]
    long long nnz_v[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // nonzeros of each stream's CSR (also without want_csr)
};
// The canonical CSR of each of the nv streams from the union pattern and
// values (the union entries whose value is nonzero, in column order): the
// same arrays canonicalize's want_csr gives.
int csr_from_union(int N, int nv, const int *d_up, const int *d_uj, const double *d_ux, long long union_nnz,
                   DevCsr *out, cudaStream_t st, std::string &err);
// The lowest position of an element_node entry (1-based) outside [1, N] in
// d_en[0 .. cnt), or -1 in *first_bad.
cudaError_t check_element_nodes(const int *d_en, long long cnt, int N, long long *first_bad, cudaStream_t st);
int canonicalize(int N, long long nnz, const int *d_ci, const int *d_cj, const double *d_cx, int nv,
                 bool want_union, bool want_csr, CanonOut &out, int *d_flags, cudaStream_t st,
                 std::string &err);
void canon_free(CanonOut &o, bool keep_csr, cudaStream_t st = 0);

cudaError_t exclusive_scan_int(const int *d_in, int *d_out, int n, cudaStream_t st);
// the stream-ordered memory pool of a device, shared by the process (kept up
// to 8 GiB between uses), and a temporary allocation from it on `st`
cudaMemPool_t device_pool(int device);
inline cudaError_t tmp_alloc(void **p, size_t bytes, cudaStream_t st)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaMemPool_t pool = device_pool(dev);
    if (!pool) return cudaErrorMemoryAllocation;
    return cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, st);
}
// The long-lived arrays of a set-up (DevProblem) and of plans come from the
// same pool, which keeps released blocks mapped: allocating and releasing the
// ~1-2 GB of a large set-up then costs microseconds, where cudaMalloc and
// cudaFree map and unmap the pages of every block (up to ~300 ms per set-up
// and release of a 641,601-node Q9 problem).  Usable from any stream once
// `st` has reached the allocation; released in stream order on `st`.
template <typename T>
inline cudaError_t keep_alloc(T **p, size_t bytes, cudaStream_t st)
{
    return tmp_alloc((void **)p, bytes, st);
}
inline void keep_free(void *p, cudaStream_t st)
{
    if (p) cudaFreeAsync(p, st);
}

// ---- step data and kernels (sfg_step.cu) ---------------------------------
int build_step_data(DevProblem &P, const double *d_c, double dt_unused, std::string &err,
                    cudaStream_t st);

struct RunBuffers;
struct StepLaunch;

// ---- context access for units other than sfg_api.cu ----------------------
int ctx_device(const sfg_ctx *c);
cudaStream_t ctx_stream(const sfg_ctx *c);
int ctx_fail(sfg_ctx *c, int code, const std::string &msg);   // records msg, returns code
// Ricker wavelet, source_receiver/seismic_source.c:16-24
double ricker_amplitude(double f0, double t0, double mag, double t);

}  // namespace sfg

namespace sfg {
// mesh/mesh_element_order.c:2-57 (host side)
inline int elem_order_host(int tc)
{
    static const int order[7] = {-1, 3, 6, 10, 4, 9, 16};
    return (tc >= 1 && tc <= 6) ? order[tc] : -1;
}
}  // namespace sfg
