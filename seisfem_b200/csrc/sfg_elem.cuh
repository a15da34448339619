// sfg_elem.cuh -- reference elements, quadrature and shape functions for the
// FP64 assembly kernels.  The translation unit that includes this header is
// compiled with -fmad=false: every expression keeps the reference's
// left-to-right evaluation order, so element matrices are bit-identical to
// assemble/*_sparse_*.c.
#pragma once

#include <cuda_runtime.h>

namespace sfg {

enum ElemType { T3 = 1, T6 = 2, T10 = 3, Q4 = 4, Q9 = 5, Q16 = 6 };

__host__ __device__ constexpr int elem_order(int tc)
{
    // mesh/mesh_element_order.c:2-57
    switch (tc) {
    case T3: return 3;
    case T6: return 6;
    case T10: return 10;
    case Q4: return 4;
    case Q9: return 9;
    case Q16: return 16;
    default: return -1;
    }
}

__host__ __device__ constexpr bool elem_is_quad(int tc) { return tc == Q4 || tc == Q9 || tc == Q16; }

// Local positions of the nodes that define the element map
// (mass_sparse_q4.c:176-179; q16 corners 0,3,15,12: mass_sparse_q16.c:179-182;
// t10 uses positions 0,3,6: mass_sparse_t10.c:103-105).
__host__ __device__ inline void elem_geometry_nodes(int tc, int g[4])
{
    if (tc == Q16) { g[0] = 0; g[1] = 3; g[2] = 15; g[3] = 12; }
    else if (tc == T10) { g[0] = 0; g[1] = 3; g[2] = 6; g[3] = -1; }
    else if (tc == T3 || tc == T6) { g[0] = 0; g[1] = 1; g[2] = 2; g[3] = -1; }
    else { g[0] = 0; g[1] = 1; g[2] = 2; g[3] = 3; }
}

// 6x6 Gauss-Legendre rule on [0,1]^2 for quads, point q = 6*i + j at
// (g[i], g[j]); the weights are the reference's 15-digit literals
// (mass_sparse_q4.c:40-156).  12-point triangle rule (mass_sparse_t6.c:36-84).
__device__ __forceinline__ int quad_point(int tc, int q, double &r, double &s, double &w)
{
    const double g6[6] = {0.033765242898424, 0.169395306766868, 0.380690406958402,
                          0.619309593041599, 0.830604693233132, 0.966234757101576};
    const double w3[9] = {0.007338020422245, 0.015451823343096, 0.020041279329452,
                          0.015451823343096, 0.032537228147042, 0.042201341771897,
                          0.020041279329452, 0.042201341771897, 0.054735862541824};
    if (elem_is_quad(tc)) {
        int i = q / 6, j = q % 6;
        r = g6[i];
        s = g6[j];
        int a = i < 3 ? i : 5 - i, b = j < 3 ? j : 5 - j;
        w = w3[3 * a + b];
        return 36;
    }
    const double A = 0.87382197101699600, B = 0.06308901449150200, C = 0.50142650965817900,
                 D = 0.24928674517091000, E = 0.63650249912139900, F = 0.31035245103378500,
                 G = 0.05314504984481600;
    const double rr[12] = {A, B, B, C, D, D, E, E, F, F, G, G};
    const double ss[12] = {B, A, B, D, C, D, F, G, E, G, E, F};
    r = rr[q];
    s = ss[q];
    w = q < 3 ? 0.05084490637020700 : (q < 6 ? 0.11678627572637900 : 0.08285107561837400);
    return 12;
}

__host__ __device__ constexpr int quad_count(int tc) { return elem_is_quad(tc) ? 36 : 12; }

// Shape functions (shape/shape_*.c), products grouped left to right exactly as
// the reference writes them.
__device__ __forceinline__ void shape_eval(int tc, double r, double s, double *t, double *dr, double *ds)
{
    if (tc == Q4) {
        t[0] = (1.0 - r) * (1.0 - s);
        t[1] = r * (1.0 - s);
        t[2] = r * s;
        t[3] = (1.0 - r) * s;
        dr[0] = -1.0 + s; dr[1] = 1.0 - s; dr[2] = s; dr[3] = -s;
        ds[0] = -1.0 + r; ds[1] = -r; ds[2] = r; ds[3] = 1.0 - r;
    } else if (tc == Q9) {
        double rm1 = r - 1.0, rmh = r - 0.5, sm1 = s - 1.0, smh = s - 0.5;
        t[0] = 4.0 * rm1 * rmh * sm1 * smh;
        t[1] = 4.0 * r * rmh * sm1 * smh;
        t[2] = 4.0 * r * rmh * s * smh;
        t[3] = 4.0 * rm1 * rmh * s * smh;
        t[4] = -8.0 * r * rm1 * sm1 * smh;
        t[5] = -8.0 * r * rmh * s * sm1;
        t[6] = -8.0 * r * rm1 * s * smh;
        t[7] = -8.0 * rm1 * rmh * s * sm1;
        t[8] = 16.0 * r * rm1 * s * sm1;
        dr[0] = 4.0 * (2.0 * r - 1.5) * sm1 * smh;
        dr[1] = 4.0 * (2.0 * r - 0.5) * sm1 * smh;
        dr[2] = 4.0 * (2.0 * r - 0.5) * s * smh;
        dr[3] = 4.0 * (2.0 * r - 1.5) * s * smh;
        dr[4] = -8.0 * (2.0 * r - 1.0) * sm1 * smh;
        dr[5] = -8.0 * (2.0 * r - 0.5) * s * sm1;
        dr[6] = -8.0 * (2.0 * r - 1.0) * s * smh;
        dr[7] = -8.0 * (2.0 * r - 1.5) * s * sm1;
        dr[8] = 16.0 * (2.0 * r - 1.0) * s * sm1;
        ds[0] = 4.0 * rm1 * rmh * (2.0 * s - 1.5);
        ds[1] = 4.0 * r * rmh * (2.0 * s - 1.5);
        ds[2] = 4.0 * r * rmh * (2.0 * s - 0.5);
        ds[3] = 4.0 * rm1 * rmh * (2.0 * s - 0.5);
        ds[4] = -8.0 * r * rm1 * (2.0 * s - 1.5);
        ds[5] = -8.0 * r * rmh * (2.0 * s - 1.0);
        ds[6] = -8.0 * r * rm1 * (2.0 * s - 0.5);
        ds[7] = -8.0 * rm1 * rmh * (2.0 * s - 1.0);
        ds[8] = 16.0 * r * rm1 * (2.0 * s - 1.0);
    } else if (tc == T3) {
        t[0] = 1.0 - r - s; t[1] = r; t[2] = s;
        dr[0] = -1.0; dr[1] = 1.0; dr[2] = 0.0;
        ds[0] = -1.0; ds[1] = 0.0; ds[2] = 1.0;
    } else if (tc == T6) {
        t[0] = 2.0 * (1.0 - r - s) * (0.5 - r - s);
        t[1] = 2.0 * r * (r - 0.5);
        t[2] = 2.0 * s * (s - 0.5);
        t[3] = 4.0 * r * (1.0 - r - s);
        t[4] = 4.0 * r * s;
        t[5] = 4.0 * s * (1.0 - r - s);
        dr[0] = -3.0 + 4.0 * r + 4.0 * s;
        dr[1] = -1.0 + 4.0 * r;
        dr[2] = 0.0;
        dr[3] = 4.0 - 8.0 * r - 4.0 * s;
        dr[4] = 4.0 * s;
        dr[5] = -4.0 * s;
        ds[0] = -3.0 + 4.0 * r + 4.0 * s;
        ds[1] = 0.0;
        ds[2] = -1.0 + 4.0 * s;
        ds[3] = -4.0 * r;
        ds[4] = 4.0 * r;
        ds[5] = 4.0 - 4.0 * r - 8.0 * s;
    } else if (tc == T10) {
        const double a = 1.0 / 3.0, b = 2.0 / 3.0, c = 1.0;
        t[0] = 4.5 * (a - r - s) * (b - r - s) * (c - r - s);
        t[1] = 13.5 * r * (b - r - s) * (c - r - s);
        t[2] = -13.5 * r * (a - r) * (c - r - s);
        t[3] = 4.5 * r * (a - r) * (b - r);
        t[4] = 13.5 * s * (b - r - s) * (c - r - s);
        t[5] = 27.0 * r * s * (c - r - s);
        t[6] = 13.5 * r * s * (r - a);
        t[7] = 13.5 * s * (s - a) * (c - r - s);
        t[8] = 13.5 * r * s * (s - a);
        t[9] = 4.5 * s * (a - s) * (b - s);
        dr[0] = 4.5 * ((a - s) * (2.0 * r - c - b + 2.0 * s) - (s - b) * (s - c)
                       - 2.0 * (2.0 * s - b - c) * r - 3.0 * r * r);
        dr[1] = 13.5 * ((s - b) * (s - c) + 2.0 * (2.0 * s - b - c) * r + 3.0 * r * r);
        dr[2] = -13.5 * (a * (c - s) + 2.0 * (s - a - c) * r + 3.0 * r * r);
        dr[3] = 4.5 * (a * b - 2.0 * (a + b) * r + 3.0 * r * r);
        dr[4] = 13.5 * s * (2.0 * s - b - c + 2.0 * r);
        dr[5] = 27.0 * s * (c - s - 2.0 * r);
        dr[6] = 13.5 * s * (2.0 * r - a);
        dr[7] = -13.5 * s * (s - a);
        dr[8] = 13.5 * s * (s - a);
        dr[9] = 0.0;
        ds[0] = 4.5 * ((a - r) * (2.0 * s - c - b + 2.0 * r) - (r - b) * (r - c)
                       - 2.0 * (2.0 * r - b - c) * s - 3.0 * s * s);
        ds[1] = 13.5 * r * (2.0 * s + 2.0 * r - b - c);
        ds[2] = 13.5 * r * (a - r);
        ds[3] = 0.0;
        ds[4] = 13.5 * ((r - b) * (r - c) + 2.0 * (2.0 * r - b - c) * s + 3.0 * s * s);
        ds[5] = 27.0 * r * (c - r - 2.0 * s);
        ds[6] = 13.5 * r * (r - a);
        ds[7] = -13.5 * (a * (c - r) + 2.0 * (r - c - a) * s + 3.0 * s * s);
        ds[8] = 13.5 * r * (2.0 * s - a);
        ds[9] = 4.5 * (a * b - 2.0 * (a + b) * s + 3.0 * s * s);
    } else {  // Q16: tensor-product cubic, node k = 4*j + i
        const double R[4] = {r - 0.0, r - 1.0 / 3.0, r - 2.0 / 3.0, r - 1.0};
        const double S[4] = {s - 0.0, s - 1.0 / 3.0, s - 2.0 / 3.0, s - 1.0};
        const double c1 = 81.0 / 4.0, c3 = 243.0 / 4.0, c9 = 729.0 / 4.0;
        const double coef[16] = {c1, -c3, c3, -c1, -c3, c9, -c9, c3,
                                 c3, -c9, c9, -c3, -c1, c3, -c3, c1};
        double dR[4], dS[4];
        dR[0] = 3.0 * r * r - 4.0 * r + 11.0 / 9.0;
        dR[1] = 3.0 * r * r - 10.0 * r / 3.0 + 2.0 / 3.0;
        dR[2] = 3.0 * r * r - 8.0 * r / 3.0 + 1.0 / 3.0;
        dR[3] = 3.0 * r * r - 2.0 * r + 2.0 / 9.0;
        dS[0] = 3.0 * s * s - 4.0 * s + 11.0 / 9.0;
        dS[1] = 3.0 * s * s - 10.0 * s / 3.0 + 2.0 / 3.0;
        dS[2] = 3.0 * s * s - 8.0 * s / 3.0 + 1.0 / 3.0;
        dS[3] = 3.0 * s * s - 2.0 * s + 2.0 / 9.0;
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int i = 0; i < 4; i++) {
                int k = 4 * j + i;
                double v = coef[k], d = coef[k] * dR[i];
#pragma unroll
                for (int m = 0; m < 4; m++) if (m != i) v = v * R[m];
                double e = v;
#pragma unroll
                for (int m = 0; m < 4; m++) if (m != j) { v = v * S[m]; d = d * S[m]; }
                t[k] = v;
                dr[k] = d;
                ds[k] = e * dS[j];
            }
    }
}

// Element geometry: corner coordinates, area, and (triangles) the constant
// inverse map.  Quads take the Jacobian per quadrature point in map_point().
struct ElemGeom {
    double x1, x2, x3, x4, y1, y2, y3, y4;
    double area;
    double drdx, drdy, dsdx, dsdy;
};

__device__ __forceinline__ void elem_geom(int tc, const int *en, const double *x, const double *y, ElemGeom &g)
{
    int gn[4];
    elem_geometry_nodes(tc, gn);
    int p1 = en[gn[0]] - 1, p2 = en[gn[1]] - 1, p3 = en[gn[2]] - 1;
    g.x1 = x[p1]; g.y1 = y[p1];
    g.x2 = x[p2]; g.y2 = y[p2];
    g.x3 = x[p3]; g.y3 = y[p3];
    if (elem_is_quad(tc)) {
        int p4 = en[gn[3]] - 1;
        g.x4 = x[p4]; g.y4 = y[p4];
        // two-triangle area (mass_sparse_q4.c:189)
        g.area = 0.5 * fabs(g.x1 * (g.y2 - g.y3) + g.x2 * (g.y3 - g.y1) + g.x3 * (g.y1 - g.y2))
               + 0.5 * fabs(g.x1 * (g.y4 - g.y3) + g.x4 * (g.y3 - g.y1) + g.x3 * (g.y1 - g.y4));
        g.drdx = g.drdy = g.dsdx = g.dsdy = 0.0;
    } else {
        g.x4 = g.y4 = 0.0;
        g.area = 0.5 * fabs(g.x1 * (g.y2 - g.y3) + g.x2 * (g.y3 - g.y1) + g.x3 * (g.y1 - g.y2));
        double det = (g.x2 - g.x1) * (g.y3 - g.y1) - (g.x3 - g.x1) * (g.y2 - g.y1);
        g.drdx = (g.y3 - g.y1) / det;
        g.drdy = (g.x1 - g.x3) / det;
        g.dsdx = (g.y1 - g.y2) / det;
        g.dsdy = (g.x2 - g.x1) / det;
    }
}

// Inverse-map terms at (r, s): bilinear Jacobian from the four geometry
// nodes for quads (mass_sparse_q4.c:204-213), constant for triangles.
__device__ __forceinline__ void map_point(int tc, const ElemGeom &g, double r, double s,
                                          double &drdx, double &drdy, double &dsdx, double &dsdy)
{
    if (elem_is_quad(tc)) {
        double dxdr = -(1 - s) * g.x1 + (1 - s) * g.x2 + s * g.x3 - s * g.x4;
        double dxds = -(1 - r) * g.x1 - r * g.x2 + r * g.x3 + (1 - r) * g.x4;
        double dydr = -(1 - s) * g.y1 + (1 - s) * g.y2 + s * g.y3 - s * g.y4;
        double dyds = -(1 - r) * g.y1 - r * g.y2 + r * g.y3 + (1 - r) * g.y4;
        double det = dxdr * dyds - dxds * dydr;
        drdx = dyds / det;
        drdy = -dxds / det;
        dsdx = -dydr / det;
        dsdy = dxdr / det;
    } else {
        drdx = g.drdx; drdy = g.drdy; dsdx = g.dsdx; dsdy = g.dsdy;
    }
}

}  // namespace sfg
