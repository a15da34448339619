/*
 * sfo.c -- CPU oracle (FP64) for the SeisFEM mass-lumped explicit path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product, never part of
 * it.  Build: gcc -O2 -fopenmp -ffp-contract=off -fPIC -shared (oracle/Makefile).
 *
 * Floating-point expressions keep the reference's evaluation order (C
 * left-to-right, no contraction) so results are bit-identical to the
 * reference compiled from its own sources; the quadrature literals are the
 * reference's own 15-digit values for the same reason (a more precise table
 * would change the last bits).
 */
#include "sfo.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static double wall_s(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

/* ------------------------------------------------------------------ types */

int sfo_type_code(const char *type)
{
    /* mesh/element_type.c:2-64 */
    static const char *names[] = {"T3", "T6", "T10", "Q4", "Q9", "Q16"};
    for (int i = 0; i < 6; i++)
        if (strcmp(type, names[i]) == 0) return i + 1;
    return -1;
}

int sfo_element_order(int tc)
{
    /* mesh/mesh_element_order.c:2-57 */
    static const int order[7] = {0, 3, 6, 10, 4, 9, 16};
    return (tc >= 1 && tc <= 6) ? order[tc] : -1;
}

static int is_quad(int tc) { return tc == SFO_Q4 || tc == SFO_Q9 || tc == SFO_Q16; }

/* Nodes that define the element geometry: the assembly routines take the
 * bilinear (quads) or affine (triangles) map from these local positions
 * (mass_sparse_q4.c:176-179, mass_sparse_q16.c:179-182, mass_sparse_t10.c:103-105). */
static void geometry_nodes(int tc, int g[4])
{
    switch (tc) {
    case SFO_Q16: g[0] = 0; g[1] = 3; g[2] = 15; g[3] = 12; break;
    case SFO_T10: g[0] = 0; g[1] = 3; g[2] = 6; g[3] = -1; break;
    case SFO_T3: case SFO_T6: g[0] = 0; g[1] = 1; g[2] = 2; g[3] = -1; break;
    default: g[0] = 0; g[1] = 1; g[2] = 2; g[3] = 3; break;
    }
}

/* -------------------------------------------------------------- quadrature */

/* 6x6 Gauss rule on [0,1]^2, points indexed quad = 6*i + j with r = g[i],
 * s = g[j] (mass_sparse_q4.c:40-156).  Weight literals are the reference's
 * rounded products; the table is symmetric under i -> 5-i, j -> 5-j. */
static const double QG[6] = {0.033765242898424, 0.169395306766868, 0.380690406958402,
                             0.619309593041599, 0.830604693233132, 0.966234757101576};
static const double QW3[3][3] = {{0.007338020422245, 0.015451823343096, 0.020041279329452},
                                 {0.015451823343096, 0.032537228147042, 0.042201341771897},
                                 {0.020041279329452, 0.042201341771897, 0.054735862541824}};

/* 12-point triangle rule (mass_sparse_t6.c:36-84) */
static const double TA = 0.87382197101699600, TB = 0.06308901449150200,
                    TC = 0.50142650965817900, TD = 0.24928674517091000,
                    TE = 0.63650249912139900, TF = 0.31035245103378500,
                    TG = 0.05314504984481600, TU = 0.05084490637020700,
                    TV = 0.11678627572637900, TWW = 0.08285107561837400;

static int quad_rule(int tc, double *r, double *s, double *w)
{
    if (is_quad(tc)) {
        for (int i = 0; i < 6; i++)
            for (int j = 0; j < 6; j++) {
                int q = 6 * i + j;
                r[q] = QG[i];
                s[q] = QG[j];
                int a = i < 3 ? i : 5 - i, b = j < 3 ? j : 5 - j;
                w[q] = QW3[a][b];
            }
        return 36;
    }
    const double rr[12] = {TA, TB, TB, TC, TD, TD, TE, TE, TF, TF, TG, TG};
    const double ss[12] = {TB, TA, TB, TD, TC, TD, TF, TG, TE, TG, TE, TF};
    const double ww[12] = {TU, TU, TU, TV, TV, TV, TWW, TWW, TWW, TWW, TWW, TWW};
    for (int q = 0; q < 12; q++) { r[q] = rr[q]; s[q] = ss[q]; w[q] = ww[q]; }
    return 12;
}

/* --------------------------------------------------------- shape functions */

static void shape_q4(double r, double s, double *t, double *dr, double *ds)
{
    /* shape/shape_q4.c:24-37 */
    t[0] = (1.0 - r) * (1.0 - s);
    t[1] = r * (1.0 - s);
    t[2] = r * s;
    t[3] = (1.0 - r) * s;
    dr[0] = -1.0 + s; dr[1] = 1.0 - s; dr[2] = s; dr[3] = -s;
    ds[0] = -1.0 + r; ds[1] = -r; ds[2] = r; ds[3] = 1.0 - r;
}

static void shape_q9(double r, double s, double *t, double *dr, double *ds)
{
    /* shape/shape_q9.c:63-91; products grouped left to right as written there */
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
}

static void shape_t3(double r, double s, double *t, double *dr, double *ds)
{
    /* shape/shape_t3.c:161-171 */
    t[0] = 1.0 - r - s; t[1] = r; t[2] = s;
    dr[0] = -1.0; dr[1] = 1.0; dr[2] = 0.0;
    ds[0] = -1.0; ds[1] = 0.0; ds[2] = 1.0;
}

static void shape_t6(double r, double s, double *t, double *dr, double *ds)
{
    /* shape/shape_t6.c:117-136 */
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
}

static void shape_t10(double r, double s, double *t, double *dr, double *ds)
{
    /* shape/shape_t10.c (cubic triangle, a=1/3, b=2/3, c=1) */
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
}

static void shape_q16(double r, double s, double *t, double *dr, double *ds)
{
    /* shape/shape_q16.c: tensor-product cubic Lagrange, node k = 4*j + i.
     * Each value is coef * (three r-factors) * (three s-factors), multiplied
     * left to right in the order the reference writes them. */
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
    for (int j = 0; j < 4; j++)
        for (int i = 0; i < 4; i++) {
            int k = 4 * j + i;
            double v = coef[k], d = coef[k] * dR[i];
            for (int m = 0; m < 4; m++) if (m != i) v = v * R[m];
            double e = v;           /* coef * r-factors, before the s-factors */
            for (int m = 0; m < 4; m++) if (m != j) { v = v * S[m]; d = d * S[m]; }
            t[k] = v;
            dr[k] = d;
            ds[k] = e * dS[j];
        }
}

void sfo_shape(int tc, double r, double s, double *t, double *dr, double *ds)
{
    switch (tc) {
    case SFO_T3: shape_t3(r, s, t, dr, ds); break;
    case SFO_T6: shape_t6(r, s, t, dr, ds); break;
    case SFO_T10: shape_t10(r, s, t, dr, ds); break;
    case SFO_Q4: shape_q4(r, s, t, dr, ds); break;
    case SFO_Q9: shape_q9(r, s, t, dr, ds); break;
    case SFO_Q16: shape_q16(r, s, t, dr, ds); break;
    default: break;
    }
}

/* ---------------------------------------------------- element integration */

typedef struct {
    double area;
    double phi[16], dphidx[16], dphidy[16];
} quad_point;

/* Element area and inverse-map terms.  Quads: two-triangle area
 * (mass_sparse_q4.c:189), Jacobian per quadrature point (:204-213).
 * Triangles: area and constant inverse map (mass_sparse_t6.c:113-126). */
typedef struct {
    double x1, x2, x3, x4, y1, y2, y3, y4;
    double area;
    double drdx, drdy, dsdx, dsdy;   /* triangles only */
} elem_geom;

static void element_geom(int tc, const int *en, const double *x, const double *y, elem_geom *g)
{
    int gn[4];
    geometry_nodes(tc, gn);
    int p1 = en[gn[0]] - 1, p2 = en[gn[1]] - 1, p3 = en[gn[2]] - 1;
    g->x1 = x[p1]; g->y1 = y[p1];
    g->x2 = x[p2]; g->y2 = y[p2];
    g->x3 = x[p3]; g->y3 = y[p3];
    if (is_quad(tc)) {
        int p4 = en[gn[3]] - 1;
        g->x4 = x[p4]; g->y4 = y[p4];
        g->area = 0.5 * fabs(g->x1 * (g->y2 - g->y3) + g->x2 * (g->y3 - g->y1) + g->x3 * (g->y1 - g->y2))
                + 0.5 * fabs(g->x1 * (g->y4 - g->y3) + g->x4 * (g->y3 - g->y1) + g->x3 * (g->y1 - g->y4));
    } else {
        g->area = 0.5 * fabs(g->x1 * (g->y2 - g->y3) + g->x2 * (g->y3 - g->y1) + g->x3 * (g->y1 - g->y2));
        double det = (g->x2 - g->x1) * (g->y3 - g->y1) - (g->x3 - g->x1) * (g->y2 - g->y1);
        g->drdx = (g->y3 - g->y1) / det;
        g->drdy = (g->x1 - g->x3) / det;
        g->dsdx = (g->y1 - g->y2) / det;
        g->dsdy = (g->x2 - g->x1) / det;
    }
}

static void eval_point(int tc, int p, const elem_geom *g, double r, double s, quad_point *qp)
{
    double w[16], dwdr[16], dwds[16];
    double drdx, drdy, dsdx, dsdy;
    if (is_quad(tc)) {
        double dxdr = -(1 - s) * g->x1 + (1 - s) * g->x2 + s * g->x3 - s * g->x4;
        double dxds = -(1 - r) * g->x1 - r * g->x2 + r * g->x3 + (1 - r) * g->x4;
        double dydr = -(1 - s) * g->y1 + (1 - s) * g->y2 + s * g->y3 - s * g->y4;
        double dyds = -(1 - r) * g->y1 - r * g->y2 + r * g->y3 + (1 - r) * g->y4;
        double det = dxdr * dyds - dxds * dydr;
        drdx = dyds / det;
        drdy = -dxds / det;
        dsdx = -dydr / det;
        dsdy = dxdr / det;
    } else {
        drdx = g->drdx; drdy = g->drdy; dsdx = g->dsdx; dsdy = g->dsdy;
    }
    sfo_shape(tc, r, s, w, dwdr, dwds);
    qp->area = g->area;
    for (int k = 0; k < p; k++) {
        qp->phi[k] = w[k];
        qp->dphidx[k] = dwdr[k] * drdx + dwds[k] * dsdx;
        qp->dphidy[k] = dwdr[k] * drdy + dwds[k] * dsdy;
    }
}

/* one stiffness integrand (stiffness_sparse_q4.c:246-259) */
static double stif_term(int type, const quad_point *qp, double aw, int iq, int jq)
{
    switch (type) {
    case 0: return aw * (qp->dphidx[iq] * qp->dphidx[jq] + qp->dphidy[iq] * qp->dphidy[jq]);
    case 1: return aw * (qp->dphidx[iq] * qp->dphidx[jq]);
    case 2: return aw * (qp->dphidy[iq] * qp->dphidy[jq]);
    case 3: return aw * (qp->dphidx[iq] * qp->dphidy[jq]);
    case 4: return aw * (qp->dphidy[iq] * qp->dphidx[jq]);
    case 5: return aw * (qp->phi[iq] * qp->dphidx[jq]);
    default: return aw * (qp->phi[iq] * qp->dphidy[jq]);
    }
}

int sfo_mass_coo(int tc, int node_num, int element_num, const int *element_node,
                 const double *x, const double *y, const double *rho,
                 int *mi, int *mj, double *mx)
{
    /* assemble/mass_sparse_q4.c:158-257 (lumpflag == 0), same for every type */
    (void)node_num;
    int p = sfo_element_order(tc);
    double rq[36], sq[36], wq[36];
    int nq = quad_rule(tc, rq, sq, wq);
    long long total = (long long)element_num * p * p;
    for (long long i = 0; i < total; i++) { mi[i] = 0; mj[i] = 0; mx[i] = 0.0; }
    int bad = 0;
    #pragma omp parallel for schedule(static)
    for (int e = 0; e < element_num; e++) {
        const int *en = element_node + (long long)e * p;
        elem_geom g;
        element_geom(tc, en, x, y, &g);
        if (g.area == 0.0) { bad = -1 - e; continue; }
        double *out = mx + (long long)e * p * p;
        for (int q = 0; q < nq; q++) {
            quad_point qp;
            eval_point(tc, p, &g, rq[q], sq[q], &qp);
            for (int iq = 0; iq < p; iq++) {
                int ip = en[iq] - 1;
                for (int jq = 0; jq < p; jq++) {
                    out[iq * p + jq] = out[iq * p + jq]
                        + g.area * wq[q] * rho[ip] * qp.phi[iq] * qp.phi[jq];
                }
            }
        }
        for (int iq = 0; iq < p; iq++)
            for (int jq = 0; jq < p; jq++) {
                mi[(long long)e * p * p + iq * p + jq] = en[iq] - 1;
                mj[(long long)e * p * p + iq * p + jq] = en[jq] - 1;
            }
    }
    return bad;
}

int sfo_mass_lumped(int tc, int node_num, int element_num, const int *element_node,
                    const double *x, const double *y, const double *rho, double *mass)
{
    /* assemble/mass_sparse_q4.c:159-163, 238-246, 259-263 (lumpflag == 1):
     * a single sequential pass; mass_sum and diag_sum run over every term in
     * (element, quad, iq, jq) order. */
    int p = sfo_element_order(tc);
    double rq[36], sq[36], wq[36];
    int nq = quad_rule(tc, rq, sq, wq);
    double mass_sum = 0.0, diag_sum = 0.0;
    for (int i = 0; i < node_num; i++) mass[i] = 0.0;
    for (int e = 0; e < element_num; e++) {
        const int *en = element_node + (long long)e * p;
        elem_geom g;
        element_geom(tc, en, x, y, &g);
        if (g.area == 0.0) return -1 - e;
        for (int q = 0; q < nq; q++) {
            quad_point qp;
            eval_point(tc, p, &g, rq[q], sq[q], &qp);
            for (int iq = 0; iq < p; iq++) {
                int ip = en[iq] - 1;
                for (int jq = 0; jq < p; jq++) {
                    int jp = en[jq] - 1;
                    double term = g.area * wq[q] * rho[ip] * qp.phi[iq] * qp.phi[jq];
                    mass_sum = mass_sum + term;
                    if (ip == jp) {
                        diag_sum = diag_sum + term;
                        mass[ip] = mass[ip] + term;
                    }
                }
            }
        }
    }
    for (int i = 0; i < node_num; i++) mass[i] = mass[i] * mass_sum / diag_sum;
    return 0;
}

int sfo_stif_coo(int tc, int type, int node_num, int element_num, const int *element_node,
                 const double *x, const double *y, int *si, int *sj, double *sx)
{
    /* assemble/stiffness_sparse_q4.c:168-273 */
    (void)node_num;
    int p = sfo_element_order(tc);
    double rq[36], sq[36], wq[36];
    int nq = quad_rule(tc, rq, sq, wq);
    long long total = (long long)element_num * p * p;
    for (long long i = 0; i < total; i++) { si[i] = 0; sj[i] = 0; sx[i] = 0.0; }
    int bad = 0;
    #pragma omp parallel for schedule(static)
    for (int e = 0; e < element_num; e++) {
        const int *en = element_node + (long long)e * p;
        elem_geom g;
        element_geom(tc, en, x, y, &g);
        if (g.area == 0.0) { bad = -1 - e; continue; }
        double *out = sx + (long long)e * p * p;
        for (int q = 0; q < nq; q++) {
            quad_point qp;
            eval_point(tc, p, &g, rq[q], sq[q], &qp);
            double aw = g.area * wq[q];
            for (int iq = 0; iq < p; iq++)
                for (int jq = 0; jq < p; jq++)
                    out[iq * p + jq] = out[iq * p + jq] + stif_term(type, &qp, aw, iq, jq);
        }
        for (int iq = 0; iq < p; iq++)
            for (int jq = 0; jq < p; jq++) {
                si[(long long)e * p * p + iq * p + jq] = en[iq] - 1;
                sj[(long long)e * p * p + iq * p + jq] = en[jq] - 1;
            }
    }
    return bad;
}

/* ------------------------------------------------------- COO -> CSR (F90) */

/* interchange_sort_map_int (coo2csr_lib.f90:256-267): selection sort that
 * swaps in the FIRST minimum of the tail (Fortran minloc semantics) */
static void interchange_sort(int *v, int *m, int n)
{
    for (int i = 0; i < n - 1; i++) {
        int best = i;
        for (int k = i + 1; k < n; k++)
            if (v[k] < v[best]) best = k;
        if (best != i) {
            int t = v[i]; v[i] = v[best]; v[best] = t;
            t = m[i]; m[i] = m[best]; m[best] = t;
        }
    }
}

void sfo_iargsort(const int *vec_in, int n, int *map)
{
    /* iargsort_quicksort (coo2csr_lib.f90:191-246).  Values are compared as
     * given; the pivot is the truncated mean of the two ends. */
    enum { LEVELS = 300, SMALL = 20 };
    int lb[LEVELS + 1], ub[LEVELS + 1];
    int *vec = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    for (int i = 0; i < n; i++) { vec[i] = vec_in[i]; map[i] = i; }
    if (n <= 0) { free(vec); return; }
    int sp = 0;
    lb[0] = 0; ub[0] = n - 1;
    while (sp >= 0) {
        int left = lb[sp], right = ub[sp];
        if (right - left < SMALL) {
            if (left < right) interchange_sort(vec + left, map + left, right - left + 1);
            sp--;
            continue;
        }
        int pivot = (vec[left] + vec[right]) / 2;
        left--; right++;
        for (;;) {
            do { left++; } while (vec[left] < pivot);
            do { right--; } while (vec[right] > pivot);
            if (left < right) {
                int t = vec[left]; vec[left] = vec[right]; vec[right] = t;
                t = map[left]; map[left] = map[right]; map[right] = t;
            } else if (left == right) {
                if (left == lb[sp]) left++; else right--;
                break;
            } else {
                break;
            }
        }
        ub[sp + 1] = ub[sp];
        lb[sp + 1] = left;
        ub[sp] = right;
        sp++;
    }
    free(vec);
}

int sfo_coo2csr_canonical(int nnz, int p_size, const int *Ai, const int *Aj, const double *Ax,
                          int *Bp, int *Bj, double *Bx)
{
    int nrow = p_size - 1;
    /* coo2csr (coo2csr_lib.f90:43-78): stable bucketing by row, COO order kept */
    int *start = (int *)calloc((size_t)nrow + 1, sizeof(int));
    int *tj = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    double *tx = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
    for (int n = 0; n < nnz; n++) start[Ai[n] + 1]++;
    for (int i = 0; i < nrow; i++) start[i + 1] += start[i];
    int *fill = (int *)malloc(sizeof(int) * ((size_t)nrow + 1));
    memcpy(fill, start, sizeof(int) * ((size_t)nrow + 1));
    for (int n = 0; n < nnz; n++) {
        int d = fill[Ai[n]]++;
        tj[d] = Aj[n];
        tx[d] = Ax[n];
    }
    free(fill);
    /* csr_sort_indices (:80-97) with 1-based values as the Fortran sees them,
     * then csr_sum_duplicates (:99-134), csr_eliminate_zeros (:136-161) */
    int maxlen = 0;
    for (int i = 0; i < nrow; i++)
        if (start[i + 1] - start[i] > maxlen) maxlen = start[i + 1] - start[i];
    int *v1 = (int *)malloc(sizeof(int) * (maxlen > 0 ? maxlen : 1));
    int *map = (int *)malloc(sizeof(int) * (maxlen > 0 ? maxlen : 1));
    int out = 0;
    Bp[0] = 0;
    for (int i = 0; i < nrow; i++) {
        int r1 = start[i], l = start[i + 1] - start[i];
        for (int k = 0; k < l; k++) v1[k] = tj[r1 + k] + 1;
        sfo_iargsort(v1, l, map);
        int k = 0;
        while (k < l) {
            int j = tj[r1 + map[k]];
            double xs = tx[r1 + map[k]];
            k++;
            while (k < l && tj[r1 + map[k]] == j) {
                xs = xs + tx[r1 + map[k]];
                k++;
            }
            if (xs != 0.0) {
                Bj[out] = j;
                Bx[out] = xs;
                out++;
            }
        }
        Bp[i + 1] = out;
    }
    free(v1); free(map); free(start); free(tj); free(tx);
    return out;
}

/* ------------------------------------------------------------------ M-PML */

void sfo_abc_mpml(int node_num, int element_num, int order, const int *element_node,
                  const double *x, const double *y, int mpml_nx, int mpml_ny, double h,
                  double xmin, double xmax, double ymin, double ymax, double vp_max,
                  int use_xmin, int use_xmax, int use_ymin, int use_ymax,
                  double *mdx, double *mdy, double *mdxx, double *mdyy, double *mdxx_pyx,
                  double *mdyy_pxy)
{
    /* pml/abc_mpml.c:41-201.  Region tests in the reference's order; every
     * node of every element is (re)written with the same value. */
    const double pxy = 0.15, pyx = 0.15, Rcoef = 0.0001;
    double tx = h * mpml_nx, ty = h * mpml_ny;
    double x0 = xmin + tx, x1 = xmax - tx, y0 = ymin + ty, y1 = ymax - ty;
    double d0x = 3.0 * vp_max * log10(1.0 / Rcoef) / (2.0 * tx);
    double d0y = 3.0 * vp_max * log10(1.0 / Rcoef) / (2.0 * ty);
    for (int i = 0; i < node_num; i++)
        mdx[i] = mdy[i] = mdxx[i] = mdyy[i] = mdxx_pyx[i] = mdyy_pxy[i] = 0.0;
    for (long long k = 0; k < (long long)element_num * order; k++) {
        int p = element_node[k] - 1;
        double X = x[p], Y = y[p];
        double vdx, vdy, vdxx, vdyy;
        if (X <= x0 && Y >= y0 && Y <= y1 && use_xmin == 1) {                    /* area 1 */
            vdx = d0x * ((x0 - X) / tx) * ((x0 - X) / tx);
            vdy = pyx * vdx;
            vdxx = -d0x * 2 * (x0 - X) / (tx * tx);
            vdyy = 0.0;
        } else if (X >= x1 && Y >= y0 && Y <= y1 && use_xmax == 1) {             /* area 3 */
            vdx = d0x * ((X - x1) / tx) * ((X - x1) / tx);
            vdy = pyx * vdx;
            vdxx = d0x * 2 * (X - x1) / (tx * tx);
            vdyy = 0.0;
        } else if (Y <= y0 && X >= x0 && X <= x1 && use_ymin == 1) {             /* area 2 */
            vdy = d0y * ((y0 - Y) / ty) * ((y0 - Y) / ty);
            vdx = pxy * vdy;
            vdxx = 0.0;
            vdyy = -d0y * 2 * (y0 - Y) / (ty * ty);
        } else if (Y >= y1 && X >= x0 && X <= x1 && use_ymax == 1) {             /* area 4 */
            vdy = d0y * ((Y - y1) / ty) * ((Y - y1) / ty);
            vdx = pxy * vdy;
            vdxx = 0.0;
            vdyy = d0y * 2 * (Y - y1) / (ty * ty);
        } else if (X <= x0 && Y <= y0 && (use_xmin == 1 || use_ymin == 1)) {     /* area 12 */
            vdx = d0x * ((x0 - X) / tx) * ((x0 - X) / tx) + pxy * d0y * ((y0 - Y) / ty) * ((y0 - Y) / ty);
            vdy = d0y * ((y0 - Y) / ty) * ((y0 - Y) / ty) + pyx * d0x * ((x0 - X) / tx) * ((x0 - X) / tx);
            vdxx = -d0x * 2 * (x0 - X) / (tx * tx);
            vdyy = -d0y * 2 * (y0 - Y) / (ty * ty);
        } else if (X <= x0 && Y >= y1 && (use_xmin == 1 || use_ymax == 1)) {     /* area 14 */
            vdx = d0x * ((x0 - X) / tx) * ((x0 - X) / tx) + pxy * d0y * ((Y - y1) / ty) * ((Y - y1) / ty);
            vdy = d0y * ((Y - y1) / ty) * ((Y - y1) / ty) + pyx * d0x * ((x0 - X) / tx) * ((x0 - X) / tx);
            vdyy = d0y * 2 * (Y - y1) / (ty * ty);
            vdxx = -d0x * 2 * (x0 - X) / (tx * tx);
        } else if (X >= x1 && Y <= y0 && (use_xmax == 1 || use_ymin == 1)) {     /* area 23 */
            if (use_ymax == 1) {   /* the reference tests ymax here (abc_mpml.c:147) */
                vdx = d0x * ((X - x1) / tx) * ((X - x1) / tx) + pxy * d0y * ((y0 - Y) / ty) * ((y0 - Y) / ty);
                vdxx = d0x * 2 * (X - x1) / (tx * tx);
                vdy = d0y * ((y0 - Y) / ty) * ((y0 - Y) / ty) + pyx * d0x * ((X - x1) / tx) * ((X - x1) / tx);
            } else {
                vdx = pxy * d0y * ((y0 - Y) / ty) * ((y0 - Y) / ty);
                vdxx = 0.0;
                vdy = d0y * ((y0 - Y) / ty) * ((y0 - Y) / ty);
            }
            vdyy = -d0y * 2 * (y0 - Y) / (ty * ty);
        } else if (X >= x1 && Y >= y1 && (use_xmax == 1 || use_ymax == 1)) {     /* area 34 */
            if (use_ymax == 1) {
                vdx = d0x * ((X - x1) / tx) * ((X - x1) / tx) + pxy * d0y * ((Y - y1) / ty) * ((Y - y1) / ty);
                vdy = d0y * ((Y - y1) / ty) * ((Y - y1) / ty) + pyx * d0x * ((X - x1) / tx) * ((X - x1) / tx);
                vdxx = d0x * 2 * (X - x1) / (tx * tx);
            } else {
                vdx = pxy * d0y * ((Y - y1) / ty) * ((Y - y1) / ty);
                vdy = d0y * ((Y - y1) / ty) * ((Y - y1) / ty);
                vdxx = 0.0;
            }
            vdyy = d0y * 2 * (Y - y1) / (ty * ty);
        } else {
            vdx = vdy = vdxx = vdyy = 0.0;
        }
        mdx[p] = vdx; mdy[p] = vdy; mdxx[p] = vdxx; mdyy[p] = vdyy;
        mdxx_pyx[p] = pyx * vdxx;
        mdyy_pxy[p] = pxy * vdyy;
    }
}

/* ---------------------------------------------------- sources / receivers */

double sfo_ricker(double f0, double t0, double magnitude, double t)
{
    /* source_receiver/seismic_source.c:16-24 */
    const double pi = 3.141592653589793238462643;
    double a = (pi * f0 * (t - t0)) * (pi * f0 * (t - t0));
    return magnitude * (1 - 2 * a) * exp(-a);
}

int sfo_node_location(int node_num, double edge_size, const double *x, const double *y,
                      double px, double py)
{
    /* source_receiver/node_location.c:13-27: the last matching index wins */
    int node = -1;
    for (int i = 0; i < node_num; i++)
        if (fabs(x[i] - px) <= edge_size / 2.0 && fabs(y[i] - py) <= edge_size / 2.0) node = i;
    return node;
}

/* -------------------------------------------------------------- time loop */

void sfo_csr_matvec(int p_size, const int *Bp, const int *Bj, const double *Bx,
                    const double *x, double *y)
{
    /* sparse_matrix/csr_matvec.c:1-18: per-row sequential sum from 0.0 */
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < p_size - 1; i++) {
        double t = 0.0;
        for (int k = Bp[i]; k <= Bp[i + 1] - 1; k++) t = t + Bx[k] * x[Bj[k]];
        y[i] = t;
    }
}

int sfo_snapshot_rows(int step, int snap_every)
{
    int n = 1;
    for (int it = 2; it < step; it++)
        if ((it + 1) % snap_every == 0) n++;
    return n;
}

typedef struct { int *p, *j; double *x; int nnz; } csr_t;

static int build_csr(int nnz, int p_size, const int *ci, const int *cj, const double *cx, csr_t *m)
{
    m->p = (int *)malloc(sizeof(int) * p_size);
    m->j = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    m->x = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
    m->nnz = sfo_coo2csr_canonical(nnz, p_size, ci, cj, cx, m->p, m->j, m->x);
    return m->nnz;
}

/* M x = b by conjugate gradients with the Jacobi preconditioner (M is
 * symmetric positive definite), x holding the first guess; stops when
 * |r| <= 1e-12 |b| (or |r|^2 <= 1e-200).  work: 4 * n doubles.  Returns 0,
 * or 1 after 1000 iterations without convergence.  It stands in for the
 * reference's PARDISO (direct) and restarted GMRES + ILU (tolerance 1e-8)
 * solves of the same systems. */
static int cg_mass(const csr_t *M, const double *dinv, const double *b, double *x, double *work, int n)
{
    double *r = work, *z = work + n, *p = work + 2 * (size_t)n, *q = work + 3 * (size_t)n;
    sfo_csr_matvec(n + 1, M->p, M->j, M->x, x, q);
    double bb = 0.0, rz = 0.0, rr = 0.0;
    for (int i = 0; i < n; i++) {
        r[i] = b[i] - q[i];
        z[i] = r[i] * dinv[i];
        p[i] = z[i];
        bb += b[i] * b[i];
        rz += r[i] * z[i];
        rr += r[i] * r[i];
    }
    for (int it = 0; it < 1000; it++) {
        if (rr <= 1e-24 * bb || rr <= 1e-200) return 0;
        sfo_csr_matvec(n + 1, M->p, M->j, M->x, p, q);
        double pq = 0.0;
        for (int i = 0; i < n; i++) pq += p[i] * q[i];
        const double alpha = rz / pq;
        double rz1 = 0.0;
        rr = 0.0;
        for (int i = 0; i < n; i++) {
            x[i] += alpha * p[i];
            r[i] -= alpha * q[i];
            z[i] = r[i] * dinv[i];
            rz1 += r[i] * z[i];
            rr += r[i] * r[i];
        }
        const double beta = rz1 / rz;
        rz = rz1;
        for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
    }
    return 1;
}

int sfo_elastic_run(const sfo_problem *pb, double *seis_u, double *seis_w,
                    double *snap_u, double *snap_w, double *energy_u, double *energy_w)
{
    /* time_evolution/elastic_wave.c:1-941 with solver "masslump" */
    const int N = pb->node_num, E = pb->element_num, P = pb->order, tc = pb->type_code;
    if (N <= 0 || E <= 0 || sfo_element_order(tc) != P || pb->step < 3) return 2;
    for (int s = 0; s < pb->src_num; s++) if (pb->src_node[s] < 0 || pb->src_node[s] >= N) return 2;
    for (int r = 0; r < pb->rec_num; r++) if (pb->rec_node[r] < 0 || pb->rec_node[r] >= N) return 2;
#ifdef _OPENMP
    int saved_threads = omp_get_max_threads();
    if (pb->nthreads > 0) omp_set_num_threads(pb->nthreads);
#endif
    const int snap_every = pb->snap_every > 0 ? pb->snap_every : 200;
    const double t_start = wall_s();
    const double dt = pb->dt, es = pb->edge_size;
    const double *x = pb->x, *y = pb->y;
    const double *c0 = pb->c, *c1 = pb->c + N, *c2 = pb->c + 2 * (size_t)N, *c3 = pb->c + 3 * (size_t)N;
    const double Angle_force = 90.0, pi_src = 3.1415926535898;   /* elastic_wave.c:66-67 */
    const double delta = 1.5, alpha = 1.0;                          /* :97 */

    /* Dirichlet flags (:136-155); zero-initialised here (the reference
     * relies on fresh malloc memory being zero) */
    char *dir = (char *)calloc(N, 1);
    for (int i = 0; i < N; i++) {
        if (pb->free_surface == 0) {
            if (x[i] <= pb->xmin + es / 4.0 || x[i] >= pb->xmax - es / 4.0 ||
                y[i] <= pb->ymin + es / 4.0 || y[i] >= pb->ymax - es / 4.0) dir[i] = 1;
        } else {
            if (x[i] <= pb->xmin + es / 4.0 || y[i] <= pb->ymin + es / 4.0 ||
                y[i] >= pb->ymax - es / 4.0) dir[i] = 1;
        }
    }
    int use_xmax = 1 - pb->free_surface;                              /* :157 */

    double vp_max = pb->vp[0];                                        /* :221-226 */
    for (int i = 0; i < N; i++) if (pb->vp[i] > vp_max) vp_max = pb->vp[i];
    double *mp = (double *)malloc(sizeof(double) * 6 * (size_t)N);
    double *dx = mp, *dy = mp + N, *dxx = mp + 2 * (size_t)N, *dyy = mp + 3 * (size_t)N,
           *dxx_pyx = mp + 4 * (size_t)N, *dyy_pxy = mp + 5 * (size_t)N;
    sfo_abc_mpml(N, E, P, pb->element_node, x, y, pb->pml_nx, pb->pml_ny, es, pb->xmin, pb->xmax,
                 pb->ymin, pb->ymax, vp_max, 1, use_xmax, 1, 1, dx, dy, dxx, dyy, dxx_pyx, dyy_pxy);

    /* assembly (:235-313) */
    long long nnz = (long long)E * P * P;
    int *ci = (int *)malloc(sizeof(int) * nnz), *cj = (int *)malloc(sizeof(int) * nnz);
    double *cx = (double *)malloc(sizeof(double) * nnz);
    double *mass_lump = (double *)malloc(sizeof(double) * N);
    int rc = sfo_mass_lumped(tc, N, E, pb->element_node, x, y, pb->rho, mass_lump);
    csr_t M, K[7];
    sfo_mass_coo(tc, N, E, pb->element_node, x, y, pb->rho, ci, cj, cx);
    build_csr((int)nnz, N + 1, ci, cj, cx, &M);
    for (int k = 1; k <= 6; k++) {
        sfo_stif_coo(tc, k, N, E, pb->element_node, x, y, ci, cj, cx);
        build_csr((int)nnz, N + 1, ci, cj, cx, &K[k]);
    }
    free(ci); free(cj); free(cx);
    (void)rc;

    /* state (:371-444) */
    enum { U1, U2, U3, W1, W2, W3, U1t, U2t, U3t, W1t, W2t, W3t, U1tt, U2tt, U3tt, W1tt, W2tt, W3tt,
           U1n, U2n, U3n, W1n, W2n, W3n, Lx1, Lx2, Lx3, Lx4, Ly1, Ly2, Ly3, Ly4, Un, Wn,
           NSTATE };
    enum { NEQ = 22, NRHS = 14 };
    double *st = (double *)malloc(sizeof(double) * NSTATE * (size_t)N);
    double *eq = (double *)malloc(sizeof(double) * NEQ * (size_t)N);
    double *rh = (double *)malloc(sizeof(double) * NRHS * (size_t)N);
#define S_(k) (st + (size_t)(k) * N)
#define E_(k) (eq + (size_t)(k) * N)
#define R_(k) (rh + (size_t)(k) * N)
    const int nsnap = sfo_snapshot_rows(pb->step, snap_every);
    const int nrow = pb->step - 2;
    int status = 0;
    double *cm_dinv = NULL, *cm_work = NULL;
    if (pb->consistent) {
        cm_dinv = (double *)calloc(N, sizeof(double));
        cm_work = (double *)malloc(sizeof(double) * 4 * (size_t)N);
        for (int i = 0; i < N; i++)
            for (int k = M.p[i]; k < M.p[i + 1]; k++)
                if (M.j[k] == i) cm_dinv[i] = M.x[k] != 0.0 ? 1.0 / M.x[k] : 0.0;
    }
    const double t_loop = wall_s();
    for (int shot = 0; shot < pb->src_num && status == 0; shot++) {
        const int src = pb->src_node[shot];
        for (size_t i = 0; i < (size_t)NSTATE * N; i++) st[i] = 0.0;   /* :466-501 */
        double *su = seis_u ? seis_u + (size_t)shot * nrow * pb->rec_num : NULL;
        double *sw = seis_w ? seis_w + (size_t)shot * nrow * pb->rec_num : NULL;
        double *pu = snap_u ? snap_u + (size_t)shot * nsnap * N : NULL;
        double *pw = snap_w ? snap_w + (size_t)shot * nsnap * N : NULL;
        double *eu = energy_u ? energy_u + (size_t)shot * pb->step : NULL;
        double *ew = energy_w ? energy_w + (size_t)shot * pb->step : NULL;
        int srow = 0;
        if (pu) { for (int i = 0; i < N; i++) { pu[i] = 0.0; pw[i] = 0.0; } srow = 1; }
        if (eu) { eu[0] = eu[1] = 0.0; ew[0] = ew[1] = 0.0; }
        for (int it = 2; it < pb->step; it++) {
            double time = (it + 1) * dt;
            double point_source = sfo_ricker(pb->f0, pb->t0, 1.0e10, time);
            double *Un_ = S_(Un), *Wn_ = S_(Wn);
            /* u half (:533-580), then the rhs (:582-592) */
            sfo_csr_matvec(N + 1, K[1].p, K[1].j, K[1].x, Un_, E_(0));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(U1t), E_(1));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(U1), E_(2));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(Lx1), E_(3));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(Lx2), E_(4));
            sfo_csr_matvec(N + 1, K[3].p, K[3].j, K[3].x, S_(Wn), E_(5));
            sfo_csr_matvec(N + 1, K[4].p, K[4].j, K[4].x, S_(Wn), E_(6));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(U2t), E_(7));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(U2), E_(8));
            sfo_csr_matvec(N + 1, K[2].p, K[2].j, K[2].x, Un_, E_(9));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(U3t), E_(10));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(U3), E_(11));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(Lx3), E_(12));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(Lx4), E_(13));
            sfo_csr_matvec(N + 1, K[5].p, K[5].j, K[5].x, Un_, E_(14));
            sfo_csr_matvec(N + 1, K[5].p, K[5].j, K[5].x, Wn_, E_(15));
            sfo_csr_matvec(N + 1, K[6].p, K[6].j, K[6].x, Wn_, E_(16));
            sfo_csr_matvec(N + 1, K[6].p, K[6].j, K[6].x, Un_, E_(17));
            {
                const double *e11 = E_(0), *e12 = E_(1), *e13 = E_(2), *e14 = E_(3), *e15 = E_(4),
                             *e21 = E_(5), *e22 = E_(6), *e23 = E_(7), *e24 = E_(8), *e31 = E_(9),
                             *e32 = E_(10), *e33 = E_(11), *e34 = E_(12), *e35 = E_(13),
                             *e41 = E_(14), *e51 = E_(15), *e61 = E_(16), *e71 = E_(17);
                double sf = sin(Angle_force * pi_src / 180.0);
                #pragma omp parallel for schedule(static)
                for (int i = 0; i < N; i++) {
                    double src_term = (i == src) * point_source * sf;
                    R_(0)[i] = -c0[i] * e11[i] - 2.0 * dx[i] * e12[i] - dx[i] * dx[i] * e13[i] + e14[i] + e15[i] + src_term;
                    R_(1)[i] = -c1[i] * e21[i] - c3[i] * e22[i] - dx[i] * e23[i] - dy[i] * e23[i] - dx[i] * dy[i] * e24[i];
                    R_(2)[i] = -c3[i] * e31[i] - 2.0 * dy[i] * e32[i] - dy[i] * dy[i] * e33[i] + e34[i] + e35[i];
                    /* equ4_2 == equ1_4, equ5_2 == equ1_5, equ6_2 == equ3_4, equ7_2 == equ3_5 */
                    R_(3)[i] = -dt * c0[i] * dxx[i] * e41[i] - dt * dx[i] * e14[i] + e14[i];
                    R_(4)[i] = -dt * c3[i] * dyy_pxy[i] * e51[i] - dt * dy[i] * e15[i] + e15[i];
                    R_(5)[i] = -dt * c1[i] * dxx_pyx[i] * e61[i] - dt * dx[i] * e34[i] + e34[i];
                    R_(6)[i] = -dt * c3[i] * dyy[i] * e71[i] - dt * dy[i] * e35[i] + e35[i];
                }
            }
            /* w half (:599-646), then the rhs (:648-658) */
            sfo_csr_matvec(N + 1, K[1].p, K[1].j, K[1].x, Wn_, E_(0));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(W1t), E_(1));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(W1), E_(2));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(Ly1), E_(3));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(Ly2), E_(4));
            sfo_csr_matvec(N + 1, K[3].p, K[3].j, K[3].x, Un_, E_(5));
            sfo_csr_matvec(N + 1, K[4].p, K[4].j, K[4].x, Un_, E_(6));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(W2t), E_(7));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(W2), E_(8));
            sfo_csr_matvec(N + 1, K[2].p, K[2].j, K[2].x, Wn_, E_(9));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(W3t), E_(10));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(W3), E_(11));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(Ly3), E_(12));
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, S_(Ly4), E_(13));
            sfo_csr_matvec(N + 1, K[5].p, K[5].j, K[5].x, Wn_, E_(14));
            sfo_csr_matvec(N + 1, K[5].p, K[5].j, K[5].x, Un_, E_(15));
            sfo_csr_matvec(N + 1, K[6].p, K[6].j, K[6].x, Un_, E_(16));
            sfo_csr_matvec(N + 1, K[6].p, K[6].j, K[6].x, Wn_, E_(17));
            {
                const double *e11 = E_(0), *e12 = E_(1), *e13 = E_(2), *e14 = E_(3), *e15 = E_(4),
                             *e21 = E_(5), *e22 = E_(6), *e23 = E_(7), *e24 = E_(8), *e31 = E_(9),
                             *e32 = E_(10), *e33 = E_(11), *e34 = E_(12), *e35 = E_(13),
                             *e41 = E_(14), *e51 = E_(15), *e61 = E_(16), *e71 = E_(17);
                double cf = cos(Angle_force * pi_src / 180.0);
                #pragma omp parallel for schedule(static)
                for (int i = 0; i < N; i++) {
                    double src_term = (i == src) * point_source * cf;
                    R_(7)[i] = -c3[i] * e11[i] - 2.0 * dx[i] * e12[i] - dx[i] * dx[i] * e13[i] + e14[i] + e15[i] + src_term;
                    R_(8)[i] = -c3[i] * e21[i] - c1[i] * e22[i] - dx[i] * e23[i] - dy[i] * e23[i] - dx[i] * dy[i] * e24[i];
                    R_(9)[i] = -c2[i] * e31[i] - 2.0 * dy[i] * e32[i] - dy[i] * dy[i] * e33[i] + e34[i] + e35[i];
                    R_(10)[i] = -dt * c3[i] * dxx[i] * e41[i] - dt * dx[i] * e14[i] + e14[i];
                    R_(11)[i] = -dt * c1[i] * dyy_pxy[i] * e51[i] - dt * dy[i] * e15[i] + e15[i];
                    R_(12)[i] = -dt * c3[i] * dxx_pyx[i] * e61[i] - dt * dx[i] * e34[i] + e34[i];
                    R_(13)[i] = -dt * c2[i] * dyy[i] * e71[i] - dt * dy[i] * e35[i] + e35[i];
                }
            }
            /* consistent-mass solves (:664-680, 730-746): M x = rhs per field,
             * from the previous values, without the Dirichlet zeroing */
            if (pb->consistent) {
                static const int dst[NRHS] = {U1n, U2n, U3n, Lx1, Lx2, Lx3, Lx4,
                                              W1n, W2n, W3n, Ly1, Ly2, Ly3, Ly4};
                for (int k = 0; k < NRHS && status == 0; k++)
                    if (cg_mass(&M, cm_dinv, R_(k), S_(dst[k]), cm_work, N) != 0) status = 4;
                if (status) break;
            } else
            /* mass-lumped solve (:681-729): Dirichlet nodes -> 0; a zero lumped
             * mass leaves the previous values in place */
            {
                static const int dst[NRHS] = {U1n, U2n, U3n, Lx1, Lx2, Lx3, Lx4,
                                              W1n, W2n, W3n, Ly1, Ly2, Ly3, Ly4};
                #pragma omp parallel for schedule(static)
                for (int i = 0; i < N; i++) {
                    if (mass_lump[i] != 0.0) {
                        for (int k = 0; k < NRHS; k++)
                            S_(dst[k])[i] = dir[i] == 1 ? 0.0 : R_(k)[i] / (1.0 * mass_lump[i]);
                    }
                }
            }
            /* Newmark update (:754-786) */
            {
                #pragma omp parallel for schedule(static)
                for (int i = 0; i < N; i++) {
                    for (int k = 0; k < 6; k++) {
                        double *Uk = S_(U1 + k), *Ukt = S_(U1t + k), *Ukt2 = S_(U1tt + k), *Ukn = S_(U1n + k);
                        Uk[i] = Uk[i] + Ukt[i] * dt + ((0.5 - alpha) * Ukt2[i] + alpha * Ukn[i]) * dt * dt;
                        Ukt[i] = Ukt[i] + ((1 - delta) * Ukt2[i] + delta * Ukn[i]) * dt;
                        Ukt2[i] = Ukn[i];
                    }
                    S_(Un)[i] = S_(U1)[i] + S_(U2)[i] + S_(U3)[i];
                    S_(Wn)[i] = S_(W1)[i] + S_(W2)[i] + S_(W3)[i];
                }
                /* energy bound (:777-785), summed in node order */
                double e_u = 0.0, e_w = 0.0;
                int blow = 0;
                for (int i = 0; i < N; i++) {
                    e_u += S_(Un)[i] * S_(Un)[i];
                    e_w += S_(Wn)[i] * S_(Wn)[i];
                    if (e_u > 10e6 || e_w > 10e6) blow = 1;
                }
                if (eu) { eu[it] = e_u; ew[it] = e_w; }
                if (blow) { status = 1; break; }
            }
            /* receivers (:787-795) and snapshots (:797-806) */
            for (int r = 0; r < pb->rec_num; r++) {
                if (su) su[(size_t)(it - 2) * pb->rec_num + r] = S_(Un)[pb->rec_node[r]];
                if (sw) sw[(size_t)(it - 2) * pb->rec_num + r] = S_(Wn)[pb->rec_node[r]];
            }
            if ((it + 1) % snap_every == 0 && pu) {
                memcpy(pu + (size_t)srow * N, S_(Un), sizeof(double) * N);
                memcpy(pw + (size_t)srow * N, S_(Wn), sizeof(double) * N);
                srow++;
            }
        }
    }
#undef S_
#undef E_
#undef R_
    if (pb->timing) { pb->timing[0] = t_loop - t_start; pb->timing[1] = wall_s() - t_loop; }
    free(st); free(eq); free(rh); free(mp); free(dir); free(mass_lump); free(cm_dinv); free(cm_work);
    free(M.p); free(M.j); free(M.x);
    for (int k = 1; k <= 6; k++) { free(K[k].p); free(K[k].j); free(K[k].x); }
#ifdef _OPENMP
    omp_set_num_threads(saved_threads);
#endif
    return status;
}

/* ------------------------------------------------------ scalar acoustics */

void sfo_abc_pml(int node_num, int element_num, int order, const int *element_node,
                 const double *x, const double *y, int pml_nx, int pml_ny, double h,
                 double xmin, double xmax, double ymin, double ymax, double vp_max,
                 int use_xmin, int use_xmax, int use_ymin, int use_ymax,
                 double *pdx, double *pdy, double *pdxx, double *pdyy)
{
    /* pml/abc_pml.c:41-103: classical quadratic profile per axis, written for
     * every node of every element (nodes of no element are zeroed here) */
    const double Rcoef = 0.0001;
    const double tx = h * pml_nx, ty = h * pml_ny;
    const double x0 = xmin + tx, x1 = xmax - tx, y0 = ymin + ty, y1 = ymax - ty;
    const double d0x = 3.0 * vp_max * log10(1.0 / Rcoef) / (2.0 * tx);
    const double d0y = 3.0 * vp_max * log10(1.0 / Rcoef) / (2.0 * ty);
    for (int i = 0; i < node_num; i++) pdx[i] = pdy[i] = pdxx[i] = pdyy[i] = 0.0;
    for (long long k = 0; k < (long long)element_num * order; k++) {
        const int p = element_node[k] - 1;
        const double X = x[p], Y = y[p];
        if (X <= x0 && use_xmin == 1) {
            pdx[p] = d0x * ((x0 - X) / tx) * ((x0 - X) / tx);
            pdxx[p] = -d0x * 2 * (x0 - X) / (tx * tx);
        } else if (X >= x1 && use_xmax == 1) {
            pdx[p] = d0x * ((X - x1) / tx) * ((X - x1) / tx);
            pdxx[p] = d0x * 2 * (X - x1) / (tx * tx);
        } else {
            pdx[p] = 0.0;
            pdxx[p] = 0.0;
        }
        if (Y <= y0 && use_ymin == 1) {
            pdy[p] = d0y * ((y0 - Y) / ty) * ((y0 - Y) / ty);
            pdyy[p] = -d0y * 2 * (y0 - Y) / (ty * ty);
        } else if (Y >= y1 && use_ymax == 1) {
            pdy[p] = d0y * ((Y - y1) / ty) * ((Y - y1) / ty);
            pdyy[p] = d0y * 2 * (Y - y1) / (ty * ty);
        } else {
            pdy[p] = 0.0;
            pdyy[p] = 0.0;
        }
    }
}

int sfo_acoustic_snapshot_rows(int step, int pml)
{
    /* acoustic.c:147-154,197-205 (every 10 steps) and acoustic_pml.c:260-268,
     * 448-455 (every 20), after the zero row */
    return sfo_snapshot_rows(step, pml ? 20 : 10);
}

int sfo_acoustic_run(const sfo_acoustic_problem *pb, double *snap, double *energy)
{
    /* time_evolution/acoustic.c:1-223 (pml == 0) and
     * time_evolution/acoustic_pml.c:3-485 (pml == 1), solver "masslump".
     * The mass matrices carry no density (the files call mass_sparse_all
     * without rho): M = integral phi_i phi_j, lumped as in mass_sparse_q4.c. */
    const int N = pb->node_num, E = pb->element_num, P = pb->order, tc = pb->type_code;
    if (N <= 0 || E <= 0 || sfo_element_order(tc) != P || pb->step < 3) return 2;
    if (pb->source_node < -1 || pb->source_node >= N) return 2;
#ifdef _OPENMP
    int saved_threads = omp_get_max_threads();
    if (pb->nthreads > 0) omp_set_num_threads(pb->nthreads);
#endif
    const long long nnz = (long long)E * P * P;
    const double dt = pb->dt;
    const double *vp = pb->vp;
    double *ones = (double *)malloc(sizeof(double) * N);
    for (int i = 0; i < N; i++) ones[i] = 1.0;
    double *mass_lump = (double *)malloc(sizeof(double) * N);
    int *ci = (int *)malloc(sizeof(int) * nnz), *cj = (int *)malloc(sizeof(int) * nnz);
    double *cx = (double *)malloc(sizeof(double) * nnz);
    int bad = sfo_mass_lumped(tc, N, E, pb->element_node, pb->x, pb->y, ones, mass_lump);
    csr_t M = {0}, K[4] = {{0}};
    /* acoustic.c:95-98: K0; acoustic_pml.c:183-187: K1, K5, K2, K6 */
    const int types_pml[4] = {1, 5, 2, 6};
    const int nk = pb->pml ? 4 : 1;
    if (!bad) bad = sfo_mass_coo(tc, N, E, pb->element_node, pb->x, pb->y, ones, ci, cj, cx);
    if (!bad) build_csr((int)nnz, N + 1, ci, cj, cx, &M);
    for (int k = 0; k < nk && !bad; k++) {
        bad = sfo_stif_coo(tc, pb->pml ? types_pml[k] : 0, N, E, pb->element_node, pb->x, pb->y, ci, cj, cx);
        if (!bad) build_csr((int)nnz, N + 1, ci, cj, cx, &K[k]);
    }
    free(ci); free(cj); free(cx); free(ones);
    int status = bad ? 3 : 0;
    double *pdx = NULL, *pdy = NULL, *pdxx = NULL, *pdyy = NULL;
    double *buf = NULL;
    int srow = 0;
    if (!bad && !pb->pml) {
        /* acoustic.c:124-207 */
        buf = (double *)calloc((size_t)6 * N, sizeof(double));
        double *u_old = buf, *u_now = buf + N, *y1 = buf + 2 * (size_t)N, *y2 = buf + 3 * (size_t)N,
               *y3 = buf + 4 * (size_t)N, *rhs = buf + 5 * (size_t)N;
        if (snap) memcpy(snap + (size_t)srow++ * N, u_old, sizeof(double) * N);
        if (energy) energy[0] = energy[1] = 0.0;
        for (int it = 2; it < pb->step; it++) {
            const double time = (it + 1) * dt;
            const double ps = sfo_ricker(pb->f0, pb->t0, 1.0, time);
            sfo_csr_matvec(N + 1, K[0].p, K[0].j, K[0].x, u_now, y1);
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, u_now, y2);
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, u_old, y3);
            for (int i = 0; i < N; i++) {
                rhs[i] = (i == pb->source_node) * ps - vp[i] * vp[i] * dt * dt * y1[i] + 2.0 * y2[i] - y3[i];
                u_old[i] = u_now[i];
            }
            for (int i = 0; i < N; i++)
                if (mass_lump[i] != 0.0) u_now[i] = rhs[i] / (1.0 * mass_lump[i]);
            double e = 0.0;
            for (int i = 0; i < N; i++) e += u_now[i] * u_now[i];
            if (energy) energy[it] = e;
            if ((it + 1) % 10 == 0 && snap) memcpy(snap + (size_t)srow++ * N, u_now, sizeof(double) * N);
        }
    } else if (!bad) {
        /* acoustic_pml.c:170-178 (vp_max), 178-179 (profiles), 270-456 */
        double vp_max = vp[0];
        for (int i = 0; i < N; i++) if (vp[i] > vp_max) vp_max = vp[i];
        pdx = (double *)malloc(sizeof(double) * N); pdy = (double *)malloc(sizeof(double) * N);
        pdxx = (double *)malloc(sizeof(double) * N); pdyy = (double *)malloc(sizeof(double) * N);
        sfo_abc_pml(N, E, P, pb->element_node, pb->x, pb->y, pb->pml_nx, pb->pml_ny, pb->edge_size,
                    pb->xmin, pb->xmax, pb->ymin, pb->ymax, vp_max, 1, 1, 1, 1, pdx, pdy, pdxx, pdyy);
        buf = (double *)calloc((size_t)15 * N, sizeof(double));
        double *u_now = buf, *u1_old = buf + N, *u1_now = buf + 2 * (size_t)N, *u2_old = buf + 3 * (size_t)N,
               *u2_now = buf + 4 * (size_t)N, *p1_now = buf + 5 * (size_t)N, *p2_now = buf + 6 * (size_t)N,
               *y1 = buf + 7 * (size_t)N, *y2 = buf + 8 * (size_t)N, *y3 = buf + 9 * (size_t)N,
               *y4 = buf + 10 * (size_t)N, *rhs1 = buf + 11 * (size_t)N, *rhs2 = buf + 12 * (size_t)N,
               *rhs3 = buf + 13 * (size_t)N, *rhs4 = buf + 14 * (size_t)N;
        const csr_t *K1 = &K[0], *K5 = &K[1], *K2 = &K[2], *K6 = &K[3];
        if (snap) memcpy(snap + (size_t)srow++ * N, u_now, sizeof(double) * N);
        if (energy) energy[0] = energy[1] = 0.0;
        for (int it = 2; it < pb->step; it++) {
            const double time = (it + 1) * dt;
            const double ps = sfo_ricker(pb->f0, pb->t0, 1.0, time);
            /* equation 1 (:289-306) */
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, u1_now, y1);
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, u1_old, y2);
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, p1_now, y3);
            sfo_csr_matvec(N + 1, K1->p, K1->j, K1->x, u_now, y4);
            for (int i = 0; i < N; i++)
                rhs1[i] = 2.0 * y1[i] - y2[i] - 2.0 * dt * pdx[i] * y1[i] + 2 * dt * pdx[i] * y2[i]
                        - dt * dt * pdx[i] * pdx[i] * y1[i] + vp[i] * vp[i] * dt * dt * y4[i]
                        + vp[i] * vp[i] * dt * dt * y3[i] + (i == pb->source_node) * ps;
            /* equation 2 (:308-320) */
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, p1_now, y1);
            sfo_csr_matvec(N + 1, K5->p, K5->j, K5->x, u_now, y2);
            for (int i = 0; i < N; i++) rhs2[i] = y1[i] - dt * pdx[i] * y1[i] - dt * pdxx[i] * y2[i];
            /* equation 3 (:322-339) */
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, u2_now, y1);
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, u2_old, y2);
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, p2_now, y3);
            sfo_csr_matvec(N + 1, K2->p, K2->j, K2->x, u_now, y4);
            for (int i = 0; i < N; i++)
                rhs3[i] = 2.0 * y1[i] - y2[i] - 2.0 * dt * pdy[i] * y1[i] + 2 * dt * pdy[i] * y2[i]
                        - dt * dt * pdy[i] * pdy[i] * y1[i] + vp[i] * vp[i] * dt * dt * y4[i]
                        + vp[i] * vp[i] * dt * dt * y3[i];
            /* equation 4 (:341-353) */
            sfo_csr_matvec(N + 1, M.p, M.j, M.x, p2_now, y1);
            sfo_csr_matvec(N + 1, K6->p, K6->j, K6->x, u_now, y2);
            for (int i = 0; i < N; i++) rhs4[i] = y1[i] - dt * pdy[i] * y1[i] - dt * pdyy[i] * y2[i];
            /* :355-375 */
            for (int i = 0; i < N; i++) { u1_old[i] = u1_now[i]; u2_old[i] = u2_now[i]; }
            for (int i = 0; i < N; i++)
                if (mass_lump[i] != 0.0) {
                    u1_now[i] = rhs1[i] / (1.0 * mass_lump[i]);
                    p1_now[i] = rhs2[i] / (1.0 * mass_lump[i]);
                    u2_now[i] = rhs3[i] / (1.0 * mass_lump[i]);
                    p2_now[i] = rhs4[i] / (1.0 * mass_lump[i]);
                }
            /* :432-447: the run ends as soon as the running sum passes 1e7 */
            double e = 0.0;
            int blow = 0;
            for (int i = 0; i < N; i++) {
                u_now[i] = u1_now[i] + u2_now[i];
                e += u_now[i] * u_now[i];
                if (e > 10e6) { blow = 1; break; }
            }
            if (blow) { status = 1; break; }
            if (energy) energy[it] = e;
            if ((it + 1) % 20 == 0 && snap) memcpy(snap + (size_t)srow++ * N, u_now, sizeof(double) * N);
        }
    }
    free(buf); free(pdx); free(pdy); free(pdxx); free(pdyy); free(mass_lump);
    free(M.p); free(M.j); free(M.x);
    for (int k = 0; k < 4; k++) { free(K[k].p); free(K[k].j); free(K[k].x); }
#ifdef _OPENMP
    omp_set_num_threads(saved_threads);
#endif
    return status;
}
