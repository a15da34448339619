// sfg_mpml.cuh -- M-PML damping profile of one node (pml/abc_mpml.c:73-199):
// the eight regions tested in the reference's order, quadratic profile,
// cross ratios pxy = pyx = 0.15.  Compile the including unit with
// -fmad=false so the FP64 values match the reference bit for bit.
#pragma once

namespace sfg {

// (X, Y): node coordinates; d0x/d0y: damping at the outer edge
// (abc_mpml.c:60-61, computed on the host); tx/ty: layer thickness;
// x0, x1, y0, y1: inner boundaries of the layer; u*: which sides are damped.
__device__ __forceinline__ void mpml_profile(double X, double Y, double d0x, double d0y, double tx, double ty,
                                             double x0, double x1, double y0, double y1, int uxmin, int uxmax,
                                             int uymin, int uymax, double &vdx, double &vdy, double &vdxx,
                                             double &vdyy)
{
    const double pxy = 0.15, pyx = 0.15;
    vdx = 0.0;
    vdy = 0.0;
    vdxx = 0.0;
    vdyy = 0.0;
    if (X <= x0 && Y >= y0 && Y <= y1 && uxmin == 1) {
        vdx = d0x * ((x0 - X) / tx) * ((x0 - X) / tx);
        vdy = pyx * vdx;
        vdxx = -d0x * 2 * (x0 - X) / (tx * tx);
        vdyy = 0.0;
    } else if (X >= x1 && Y >= y0 && Y <= y1 && uxmax == 1) {
        vdx = d0x * ((X - x1) / tx) * ((X - x1) / tx);
        vdy = pyx * vdx;
        vdxx = d0x * 2 * (X - x1) / (tx * tx);
        vdyy = 0.0;
    } else if (Y <= y0 && X >= x0 && X <= x1 && uymin == 1) {
        vdy = d0y * ((y0 - Y) / ty) * ((y0 - Y) / ty);
        vdx = pxy * vdy;
        vdxx = 0.0;
        vdyy = -d0y * 2 * (y0 - Y) / (ty * ty);
    } else if (Y >= y1 && X >= x0 && X <= x1 && uymax == 1) {
        vdy = d0y * ((Y - y1) / ty) * ((Y - y1) / ty);
        vdx = pxy * vdy;
        vdxx = 0.0;
        vdyy = d0y * 2 * (Y - y1) / (ty * ty);
    } else if (X <= x0 && Y <= y0 && (uxmin == 1 || uymin == 1)) {
        vdx = d0x * ((x0 - X) / tx) * ((x0 - X) / tx) + pxy * d0y * ((y0 - Y) / ty) * ((y0 - Y) / ty);
        vdy = d0y * ((y0 - Y) / ty) * ((y0 - Y) / ty) + pyx * d0x * ((x0 - X) / tx) * ((x0 - X) / tx);
        vdxx = -d0x * 2 * (x0 - X) / (tx * tx);
        vdyy = -d0y * 2 * (y0 - Y) / (ty * ty);
    } else if (X <= x0 && Y >= y1 && (uxmin == 1 || uymax == 1)) {
        vdx = d0x * ((x0 - X) / tx) * ((x0 - X) / tx) + pxy * d0y * ((Y - y1) / ty) * ((Y - y1) / ty);
        vdy = d0y * ((Y - y1) / ty) * ((Y - y1) / ty) + pyx * d0x * ((x0 - X) / tx) * ((x0 - X) / tx);
        vdyy = d0y * 2 * (Y - y1) / (ty * ty);
        vdxx = -d0x * 2 * (x0 - X) / (tx * tx);
    } else if (X >= x1 && Y <= y0 && (uxmax == 1 || uymin == 1)) {
        if (uymax == 1) {   // the reference tests ymax here (abc_mpml.c:147)
            vdx = d0x * ((X - x1) / tx) * ((X - x1) / tx) + pxy * d0y * ((y0 - Y) / ty) * ((y0 - Y) / ty);
            vdxx = d0x * 2 * (X - x1) / (tx * tx);
            vdy = d0y * ((y0 - Y) / ty) * ((y0 - Y) / ty) + pyx * d0x * ((X - x1) / tx) * ((X - x1) / tx);
        } else {
            vdx = pxy * d0y * ((y0 - Y) / ty) * ((y0 - Y) / ty);
            vdxx = 0.0;
            vdy = d0y * ((y0 - Y) / ty) * ((y0 - Y) / ty);
        }
        vdyy = -d0y * 2 * (y0 - Y) / (ty * ty);
    } else if (X >= x1 && Y >= y1 && (uxmax == 1 || uymax == 1)) {
        if (uymax == 1) {
            vdx = d0x * ((X - x1) / tx) * ((X - x1) / tx) + pxy * d0y * ((Y - y1) / ty) * ((Y - y1) / ty);
            vdy = d0y * ((Y - y1) / ty) * ((Y - y1) / ty) + pyx * d0x * ((X - x1) / tx) * ((X - x1) / tx);
            vdxx = d0x * 2 * (X - x1) / (tx * tx);
        } else {
            vdx = pxy * d0y * ((Y - y1) / ty) * ((Y - y1) / ty);
            vdy = d0y * ((Y - y1) / ty) * ((Y - y1) / ty);
            vdxx = 0.0;
        }
        vdyy = d0y * 2 * (Y - y1) / (ty * ty);
    }
}

}  // namespace sfg
