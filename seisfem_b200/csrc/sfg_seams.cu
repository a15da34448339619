// sfg_seams.cu -- GPU versions of the reference functions elastic_wave()
// calls, with the reference's signatures and argument meaning:
//   assemble/mass_sparse_all.c:13-68, assemble/stif_sparse_all.c:8-62,
//   sparse_matrix/coo2csr_lib.f90:6-41 (Fortran ABI of elastic_wave.c:241),
//   pml/abc_mpml.c:1-201, sparse_matrix/csr_matvec.c:1-18.
// Each call copies its host arrays in, computes on the device and copies the
// results back.  Compiled with -fmad=false (FP64 results bit-identical to
// the reference's scalar loops).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "sfg_internal.h"

using namespace sfg;

namespace {

int seam_device()
{
    const char *d = std::getenv("SFG_DEVICE");
    return d ? std::atoi(d) : 0;
}

int type_code(const char *t)
{
    static const char *names[] = {"T3", "T6", "T10", "Q4", "Q9", "Q16"};
    if (!t) return -1;
    for (int i = 0; i < 6; i++)
        if (std::strcmp(t, names[i]) == 0) return i + 1;
    return -1;
}

// RAII bundle of device buffers for one seam call
struct Scratch {
    std::vector<void *> ptrs;
    ~Scratch() { for (void *p : ptrs) cudaFree(p); }
    template <typename T>
    T *get(size_t n)
    {
        void *p = nullptr;
        if (cudaMalloc(&p, sizeof(T) * (n ? n : 1)) != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return (T *)p;
    }
    template <typename T>
    T *up(const T *h, size_t n)
    {
        T *d = get<T>(n);
        if (d && n) cudaMemcpy(d, h, sizeof(T) * n, cudaMemcpyHostToDevice);
        return d;
    }
};

int check(cudaError_t e) { return e == cudaSuccess ? SFG_OK : (e == cudaErrorMemoryAllocation ? SFG_ERR_OOM : SFG_ERR_CUDA); }

__global__ void csr_matvec64(int n, const int *__restrict__ p, const int *__restrict__ j,
                             const double *__restrict__ x, const double *__restrict__ v, double *__restrict__ y)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double t = 0.0;
    for (int k = p[i]; k <= p[i + 1] - 1; k++) t = t + x[k] * v[j[k]];
    y[i] = t;
}

int element_seam(char *type, int node_num, int element_num, int element_order, int *element_node,
                 double **node_xy, const double *rho, int mat, int *oi, int *oj, double *ox, int lumpflag)
{
    const int tc = type_code(type);
    if (tc < 0 || elem_order_host(tc) != element_order || node_num <= 0 || element_num <= 0) return SFG_ERR_ARG;
    if (cudaSetDevice(seam_device()) != cudaSuccess) return SFG_ERR_NODEVICE;
    const int p = element_order, N = node_num, E = element_num;
    const long long nnz = (long long)E * p * p;
    for (long long k = 0; k < (long long)E * p; k++)
        if (element_node[k] < 1 || element_node[k] > N) return SFG_ERR_BADINDEX;
    Scratch s;
    cudaStream_t st = 0;
    int *d_en = s.up(element_node, (size_t)E * p);
    double *d_x = s.up(node_xy[0], (size_t)N), *d_y = s.up(node_xy[1], (size_t)N);
    double *d_rho = rho ? s.up(rho, (size_t)N) : nullptr;
    int *d_flags = s.get<int>(1), *d_ci = s.get<int>(nnz), *d_cj = s.get<int>(nnz);
    double *d_cx = s.get<double>(nnz);
    if (!d_en || !d_x || !d_y || !d_flags || !d_ci || !d_cj || !d_cx) return SFG_ERR_OOM;
    cudaMemset(d_flags, 0, sizeof(int));
    int rc = check(launch_element_coo(tc, E, d_en, d_x, d_y, d_rho, 1, &mat, d_ci, d_cj, d_cx, d_flags, st));
    if (rc) return rc;
    int hflags = 0;
    cudaMemcpy(&hflags, d_flags, sizeof(int), cudaMemcpyDeviceToHost);
    if (hflags & FLAG_ZERO_AREA) return SFG_ERR_ZERO_AREA;
    if (lumpflag == 1) {
        CanonOut co;
        std::string err;
        rc = canonicalize(N, nnz, d_ci, d_cj, d_cx, 1, false, false, co, d_flags, st, err);
        if (rc) { canon_free(co, false); return rc; }
        double *d_m = s.get<double>(N), *d_scr = s.get<double>(2 * (size_t)E + 2);
        rc = check(launch_lumped_mass(tc, N, E, d_en, d_x, d_y, d_rho, co.row_start, co.bucket, d_cj, d_m, d_scr,
                                      d_flags, st));
        if (!rc) rc = check(cudaMemcpy(ox, d_m, sizeof(double) * N, cudaMemcpyDeviceToHost));
        canon_free(co, false);
        return rc;
    }
    rc = check(cudaMemcpy(oi, d_ci, sizeof(int) * nnz, cudaMemcpyDeviceToHost));
    if (!rc) rc = check(cudaMemcpy(oj, d_cj, sizeof(int) * nnz, cudaMemcpyDeviceToHost));
    if (!rc) rc = check(cudaMemcpy(ox, d_cx, sizeof(double) * nnz, cudaMemcpyDeviceToHost));
    return rc;
}

}  // namespace

extern "C" {

int sfg_mass_sparse_all(char *type, int node_num, int element_num, int element_order, int *element_node,
                        double **node_xy, double *rho, int *mass_coo_i, int *mass_coo_j, double *mass_coo_x,
                        int lumpflag)
{
    if (!rho || !node_xy || !element_node || !mass_coo_x) return SFG_ERR_ARG;
    return element_seam(type, node_num, element_num, element_order, element_node, node_xy, rho, -1, mass_coo_i,
                        mass_coo_j, mass_coo_x, lumpflag);
}

int sfg_stif_sparse_all(char *type, int node_num, int element_num, int element_order, int *element_node,
                        double **node_xy, int *stiffi, int *stiffj, double *stiffness, int stif_type)
{
    if (stif_type < 0 || stif_type > 6 || !node_xy || !element_node) return SFG_ERR_ARG;
    return element_seam(type, node_num, element_num, element_order, element_node, node_xy, nullptr, stif_type,
                        stiffi, stiffj, stiffness, 0);
}

int sfg_coo2csr_canonical(int *nnz_p, int *Bp_size, int *csr_size, int *Ai, int *Aj, double *Ax, int *Bp,
                          int *Bj, double *Bx)
{
    if (!nnz_p || !Bp_size || !csr_size || !Ai || !Aj || !Ax || !Bp || !Bj || !Bx) return SFG_ERR_ARG;
    const int nnz = *nnz_p, N = *Bp_size - 1;
    if (nnz < 0 || N < 0) return SFG_ERR_ARG;
    if (cudaSetDevice(seam_device()) != cudaSuccess) return SFG_ERR_NODEVICE;
    // coo2csr_lib.f90:24-26: the outputs are zeroed over their full extent
    for (int i = 0; i <= N; i++) Bp[i] = 0;
    for (int i = 0; i < nnz; i++) { Bj[i] = 0; Bx[i] = 0.0; }
    Scratch s;
    int *d_ci = s.up(Ai, (size_t)nnz), *d_cj = s.up(Aj, (size_t)nnz), *d_flags = s.get<int>(1);
    double *d_cx = s.up(Ax, (size_t)nnz);
    if (!d_ci || !d_cj || !d_cx || !d_flags) return SFG_ERR_OOM;
    cudaMemset(d_flags, 0, sizeof(int));
    CanonOut co;
    std::string err;
    int rc = canonicalize(N, nnz, d_ci, d_cj, d_cx, 1, false, true, co, d_flags, 0, err);
    if (rc == SFG_OK) {
        const DevCsr &c = co.csr[0];
        rc = check(cudaMemcpy(Bp, c.p, sizeof(int) * ((size_t)N + 1), cudaMemcpyDeviceToHost));
        if (!rc && c.nnz) rc = check(cudaMemcpy(Bj, c.j, sizeof(int) * c.nnz, cudaMemcpyDeviceToHost));
        if (!rc && c.nnz) rc = check(cudaMemcpy(Bx, c.x, sizeof(double) * c.nnz, cudaMemcpyDeviceToHost));
        *csr_size = (int)c.nnz;
    }
    canon_free(co, false);
    if (rc == SFG_OK)
        for (int i = 0; i < nnz; i++) { Ai[i] += 1; Aj[i] += 1; }   // coo2csr_lib.f90:27-28
    return rc;
}

int sfg_abc_mpml(int node_num, int element_num, int element_order, int *element_node, double **node_xy,
                 int mpml_nx, int mpml_ny, double h, double xmin, double xmax, double ymin, double ymax,
                 double vp_max, int use_mpml_xmin, int use_mpml_xmax, int use_mpml_ymin, int use_mpml_ymax,
                 double *mpml_dx, double *mpml_dy, double *mpml_dxx, double *mpml_dyy, double *mpml_dxx_pyx,
                 double *mpml_dyy_pxy)
{
    if (node_num <= 0 || element_num < 0 || !element_node || !node_xy) return SFG_ERR_ARG;
    if (cudaSetDevice(seam_device()) != cudaSuccess) return SFG_ERR_NODEVICE;
    const int N = node_num;
    std::vector<char> ref(N, 0);
    for (long long k = 0; k < (long long)element_num * element_order; k++) {
        int p = element_node[k] - 1;
        if (p < 0 || p >= N) return SFG_ERR_BADINDEX;
        ref[p] = 1;
    }
    const double Rcoef = 0.0001;
    const double tx = h * mpml_nx, ty = h * mpml_ny;
    const double d0x = 3.0 * vp_max * std::log10(1.0 / Rcoef) / (2.0 * tx);
    const double d0y = 3.0 * vp_max * std::log10(1.0 / Rcoef) / (2.0 * ty);
    Scratch s;
    double *d_x = s.up(node_xy[0], (size_t)N), *d_y = s.up(node_xy[1], (size_t)N), *d_o = s.get<double>(6 * (size_t)N);
    if (!d_x || !d_y || !d_o) return SFG_ERR_OOM;
    int rc = check(launch_mpml(N, d_x, d_y, nullptr, d0x, d0y, tx, ty, xmin + tx, xmax - tx, ymin + ty, ymax - ty,
                               use_mpml_xmin, use_mpml_xmax, use_mpml_ymin, use_mpml_ymax, d_o, 0));
    if (rc) return rc;
    std::vector<double> h6(6 * (size_t)N);
    rc = check(cudaMemcpy(h6.data(), d_o, sizeof(double) * h6.size(), cudaMemcpyDeviceToHost));
    if (rc) return rc;
    double *outs[6] = {mpml_dx, mpml_dy, mpml_dxx, mpml_dyy, mpml_dxx_pyx, mpml_dyy_pxy};
    for (int k = 0; k < 6; k++)
        for (int i = 0; i < N; i++)
            if (ref[i]) outs[k][i] = h6[(size_t)k * N + i];   // nodes of no element are left as they were
    return SFG_OK;
}

int sfg_csr_matvec(int Bp_size, int *Bp, int *Bj, double *Bx, double *x, double *y)
{
    const int n = Bp_size - 1;
    if (n < 0 || !Bp || !x || !y) return SFG_ERR_ARG;
    if (cudaSetDevice(seam_device()) != cudaSuccess) return SFG_ERR_NODEVICE;
    const int nz = n > 0 ? Bp[n] : 0;
    Scratch s;
    int *dp = s.up(Bp, (size_t)n + 1), *dj = s.up(Bj, (size_t)nz);
    double *dx = s.up(Bx, (size_t)nz), *dv = s.up(x, (size_t)n), *dy = s.get<double>(n);
    if (!dp || !dj || !dx || !dv || !dy) return SFG_ERR_OOM;
    if (n) csr_matvec64<<<(n + 255) / 256, 256>>>(n, dp, dj, dx, dv, dy);
    int rc = check(cudaGetLastError());
    if (!rc) rc = check(cudaMemcpy(y, dy, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return rc;
}

}  // extern "C"
