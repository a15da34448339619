// sfg_noalloc.cu -- M-PML damping profiles (pml/abc_mpml.c:1-201) of
// device-resident node arrays, computed without allocating device memory.
//
// The allocating seam (sfg_abc_mpml) copies host arrays in and marks the nodes
// that some element references on the host.  This entry point works on the
// caller's device buffers instead, and keeps its only scratch -- one
// "referenced" byte per node and an error word -- in a file-scope __device__
// array of fixed size, so it calls no cudaMalloc/cudaFree or allocating
// library routine.  Compiled with -fmad=false: the profiles are bit-identical
// to the reference's and to sfg_abc_mpml's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "../../include/seisfem_b200.h"
#include "sfg_mpml.cuh"

namespace {

constexpr int kErrOffset = 0;      // int: set to 1 when an element_node entry is out of range
constexpr int kFlagOffset = 256;   // node_num bytes: 1 = referenced by some element

__device__ __align__(256) unsigned char g_mpml_scratch[kFlagOffset + SFG_NOALLOC_MAX_NODES];

// Clears the error word and the first n flags (every call starts from zero;
// a previous call may have marked more nodes).
__global__ void noalloc_clear(unsigned char *scr, int n)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) *reinterpret_cast<int *>(scr + kErrOffset) = 0;
    uint4 *f = reinterpret_cast<uint4 *>(scr + kFlagOffset);
    const int n16 = (n + 15) / 16;
    for (int i = t; i < n16; i += gridDim.x * blockDim.x) f[i] = make_uint4(0u, 0u, 0u, 0u);
}

// Marks every node an element references (element_node is 1-based); entries
// outside 1..n are skipped and reported through the error word.
__global__ void noalloc_mark(const int *__restrict__ en, long long cnt, int n, unsigned char *scr)
{
    unsigned char *flag = scr + kFlagOffset;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < cnt;
         k += (long long)gridDim.x * blockDim.x) {
        const int v = en[k] - 1;
        if (v >= 0 && v < n) flag[v] = 1;
        else atomicOr(reinterpret_cast<int *>(scr + kErrOffset), 1);
    }
}

// Profiles of referenced nodes; nodes of no element keep their output values
// (as the reference, which assigns node by node inside its element loop).
__global__ void noalloc_mpml(int n, const double *__restrict__ xa, const double *__restrict__ ya,
                             const unsigned char *__restrict__ scr, double d0x, double d0y, double tx, double ty,
                             double x0, double x1, double y0, double y1, int uxmin, int uxmax, int uymin,
                             int uymax, double *__restrict__ out)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n || !scr[kFlagOffset + p]) return;
    const double pxy = 0.15, pyx = 0.15;
    double vdx, vdy, vdxx, vdyy;
    sfg::mpml_profile(xa[p], ya[p], d0x, d0y, tx, ty, x0, x1, y0, y1, uxmin, uxmax, uymin, uymax, vdx, vdy,
                      vdxx, vdyy);
    out[p] = vdx;
    out[(size_t)n + p] = vdy;
    out[2 * (size_t)n + p] = vdxx;
    out[3 * (size_t)n + p] = vdyy;
    out[4 * (size_t)n + p] = pyx * vdxx;
    out[5 * (size_t)n + p] = pxy * vdyy;
}

int status_of(cudaError_t e) { return e == cudaSuccess ? SFG_OK : SFG_ERR_CUDA; }

// Address of the scratch array in the current context, looked up on every
// call: a context that the caller reset and re-created reloads the module at
// another address, so a cached address could point at freed memory.  The
// lookup allocates nothing.
int scratch_address(unsigned char **out)
{
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_mpml_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return e == cudaErrorNoKernelImageForDevice || e == cudaErrorNoDevice ? SFG_ERR_NODEVICE : SFG_ERR_CUDA;
    }
    *out = static_cast<unsigned char *>(p);
    return SFG_OK;
}

// Reads the error word back (pageable host memory: the copy completes before
// the call returns) and waits for the stream.
int read_error_word(const unsigned char *scr, cudaStream_t st, int *bad)
{
    int rc = status_of(cudaMemcpyAsync(bad, scr + kErrOffset, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (rc) return rc;
    return status_of(cudaStreamSynchronize(st));
}

}  // namespace

extern "C" {

int sfg_abc_mpml_device_noalloc(int node_num, int element_num, int element_order, const int *d_element_node,
                                const double *d_x, const double *d_y, int mpml_nx, int mpml_ny, double h,
                                double xmin, double xmax, double ymin, double ymax, double vp_max,
                                int use_mpml_xmin, int use_mpml_xmax, int use_mpml_ymin, int use_mpml_ymax,
                                double *d_out6, void *stream)
{
    if (node_num <= 0 || element_num < 0 || element_order <= 0 || !d_element_node || !d_x || !d_y || !d_out6)
        return SFG_ERR_ARG;
    if (node_num > SFG_NOALLOC_MAX_NODES) return SFG_ERR_LIMIT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the call waits for its stream (it reads the error word back), which a
    // stream that is being captured does not allow: refuse rather than
    // invalidate the caller's capture
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) { cudaGetLastError(); return SFG_ERR_ARG; }
    if (cap != cudaStreamCaptureStatusNone) return SFG_ERR_ARG;
    unsigned char *scr = nullptr;
    int rc = scratch_address(&scr);
    if (rc) return rc;
    // abc_mpml.c:57-61 on the host (log10 of the host library)
    const double Rcoef = 0.0001;
    const double tx = h * mpml_nx, ty = h * mpml_ny;
    const double d0x = 3.0 * vp_max * std::log10(1.0 / Rcoef) / (2.0 * tx);
    const double d0y = 3.0 * vp_max * std::log10(1.0 / Rcoef) / (2.0 * ty);
    const long long cnt = (long long)element_num * element_order;
    const int nblk = (node_num + 255) / 256;
    noalloc_clear<<<(node_num + 16 * 256 - 1) / (16 * 256), 256, 0, st>>>(scr, node_num);
    if (cnt > 0) noalloc_mark<<<(unsigned)std::min<long long>((cnt + 255) / 256, 148 * 16), 256, 0, st>>>(
        d_element_node, cnt, node_num, scr);
    if ((rc = status_of(cudaGetLastError()))) return rc;
    // like sfg_abc_mpml, a bad element_node entry leaves d_out6 untouched
    int bad = 0;
    if ((rc = read_error_word(scr, st, &bad))) return rc;
    if (bad) return SFG_ERR_BADINDEX;
    noalloc_mpml<<<nblk, 256, 0, st>>>(node_num, d_x, d_y, scr, d0x, d0y, tx, ty, xmin + tx, xmax - tx, ymin + ty,
                                       ymax - ty, use_mpml_xmin, use_mpml_xmax, use_mpml_ymin, use_mpml_ymax,
                                       d_out6);
    if ((rc = status_of(cudaGetLastError()))) return rc;
    return status_of(cudaStreamSynchronize(st));
}

}  // extern "C"
