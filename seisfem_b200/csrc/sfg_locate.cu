// sfg_locate.cu -- node location for sources and receivers (host code).
//
// source_receiver/node_location.c:13-27 scans every node for each point and
// keeps the LAST index whose coordinates lie within edge_size / 2 of the
// point in both axes (-1 when none does): O(N) per point.  This replacement
// buckets the nodes once into a uniform grid of cells edge_size wide and, per
// point, tests only the nodes of the cells its box can touch (one cell more
// on each side, so rounding in the cell arithmetic can never drop a
// candidate), with the reference's own comparison
//   fabs(x[i] - px) <= edge_size / 2.0 && fabs(y[i] - py) <= edge_size / 2.0
// and the largest matching index kept.  The answers are therefore those of
// the linear scan, bit for bit.
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/seisfem_b200.h"

namespace {

int scan(int n, double edge, const double *x, const double *y, double px, double py)
{
    int node = -1;
    for (int i = 0; i < n; i++)
        if (std::fabs(x[i] - px) <= edge / 2.0 && std::fabs(y[i] - py) <= edge / 2.0) node = i;
    return node;
}

}  // namespace

extern "C" int sfg_node_location(int node_num, double edge_size, const double *x, const double *y, int npts,
                                 const double *px, const double *py, int *out)
{
    if (node_num < 0 || npts < 0 || (npts > 0 && (!px || !py || !out)) || (node_num > 0 && (!x || !y)))
        return SFG_ERR_ARG;
    if (npts == 0) return SFG_OK;
    double x0 = INFINITY, x1 = -INFINITY, y0 = INFINITY, y1 = -INFINITY;
    bool finite = true;
    for (int i = 0; i < node_num; i++) {
        finite = finite && std::isfinite(x[i]) && std::isfinite(y[i]);
        x0 = std::min(x0, x[i]); x1 = std::max(x1, x[i]);
        y0 = std::min(y0, y[i]); y1 = std::max(y1, y[i]);
    }
    // the linear scan where a grid does not apply (no nodes, a non-positive
    // or non-finite edge, non-finite coordinates)
    if (node_num == 0 || !(edge_size > 0.0) || !std::isfinite(edge_size) || !finite) {
        for (int k = 0; k < npts; k++) out[k] = scan(node_num, edge_size, x, y, px[k], py[k]);
        return SFG_OK;
    }
    // cells edge_size wide, coarsened if that would give more than ~4 cells per node
    double c = edge_size;
    const double w = x1 - x0, h = y1 - y0;
    while ((w / c + 1.0) * (h / c + 1.0) > 4.0 * node_num + 64.0) c *= 2.0;
    const long long nx = (long long)(w / c) + 1, ny = (long long)(h / c) + 1;
    // cell of a coordinate, clamped to one cell beyond the grid before the
    // conversion (points far outside stay representable)
    auto cell_x = [&](double v) { return (long long)std::min(std::max(std::floor((v - x0) / c), -2.0), (double)nx + 1.0); };
    auto cell_y = [&](double v) { return (long long)std::min(std::max(std::floor((v - y0) / c), -2.0), (double)ny + 1.0); };
    std::vector<int> start((size_t)(nx * ny) + 1, 0), items((size_t)node_num);
    std::vector<long long> cell((size_t)node_num);
    for (int i = 0; i < node_num; i++) {
        const long long cx = std::min(std::max(cell_x(x[i]), 0LL), nx - 1);
        const long long cy = std::min(std::max(cell_y(y[i]), 0LL), ny - 1);
        cell[i] = cy * nx + cx;
        start[(size_t)cell[i] + 1]++;
    }
    for (size_t k = 1; k < start.size(); k++) start[k] += start[k - 1];
    {
        std::vector<int> fill(start.begin(), start.end() - 1);
        for (int i = 0; i < node_num; i++) items[(size_t)fill[(size_t)cell[i]]++] = i;   // ascending per cell
    }
    const double half = edge_size / 2.0;
    for (int k = 0; k < npts; k++) {
        const double qx = px[k], qy = py[k];
        if (!std::isfinite(qx) || !std::isfinite(qy)) {
            out[k] = scan(node_num, edge_size, x, y, qx, qy);
            continue;
        }
        const long long ax = std::max(cell_x(qx - half) - 1, 0LL), bx = std::min(cell_x(qx + half) + 1, nx - 1);
        const long long ay = std::max(cell_y(qy - half) - 1, 0LL), by = std::min(cell_y(qy + half) + 1, ny - 1);
        int node = -1;
        for (long long cy = ay; cy <= by; cy++)
            for (long long cx = ax; cx <= bx; cx++) {
                const long long id = cy * nx + cx;
                for (int t = start[(size_t)id]; t < start[(size_t)id + 1]; t++) {
                    const int i = items[(size_t)t];
                    if (i > node && std::fabs(x[i] - qx) <= edge_size / 2.0 && std::fabs(y[i] - qy) <= edge_size / 2.0)
                        node = i;
                }
            }
        out[k] = node;
    }
    return SFG_OK;
}
