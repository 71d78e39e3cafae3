// sw2d_mapper.cu — the porosity mapper's geometry on the GPU (sw2dPorosityMapper, footprint
// input): for every cell the fraction of its area outside the building footprints, for every
// edge the fraction of its length outside them, at each elevation of a level list (a building
// counts at level h when it is taller than h; with one level and heights ignored for SP and
// DIP).  swPorosityMapperPipeline::cellPorosity / edgePorosity
// (src/sw2dPorosityMapper/swPorosityMapperPipeline.cpp:31-90, 256-388) over the polygon
// routines of swGeometry (src/common/swGeometry.cpp:9-483), restated per thread:
//   - sort_vertices: by the angle about the vertex mean (atan2, in [0, 2 pi)), selection sort;
//   - intersection_area: the vertices of each polygon inside the other (ray casting), the
//     pairwise side intersections not yet listed, sorted, then the cross-product sum / 2;
//   - length_in_polygon: the segment cut at the polygon's sides, points sorted along x (y for
//     a vertical segment), alternating inside / outside from the first portion's test.
// One thread per (cell or edge, level) loops over the buildings in file order, so every sum
// adds the same terms in the same order as the reference; a building whose bounding box is
// disjoint from the element's adds exactly zero there and is skipped.  Polygons are limited in
// size (kMaxCellVerts, kMaxBldVerts, kMaxPoly intersection points): a larger one sets the
// status word and the call fails.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/sw2d_b200.h"

namespace {

constexpr int kMaxCellVerts = 8;
constexpr int kMaxBldVerts = 64;
constexpr int kMaxPoly = 96;
constexpr double kTwoPi = 6.283185307179586;  // 2 M_PI

__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }  // std::max

// swGeometry::sortVertices (:417-466)
__device__ void sort_vertices(double* x, double* y, int n)
{
    double xc = 0, yc = 0;
    for (int k = 0; k < n; k++) {
        xc += x[k];
        yc += y[k];
    }
    xc /= n;
    yc /= n;
    double ang[kMaxPoly];
    for (int k = 0; k < n; k++) {
        double a = atan2(y[k] - yc, x[k] - xc);
        if (a < 0) a += kTwoPi;
        ang[k] = a;
    }
    for (int i = 0; i < n; i++) {
        int jm = i;
        for (int j = i; j < n; j++)
            if (ang[j] < ang[jm]) jm = j;
        double t = x[i];
        x[i] = x[jm];
        x[jm] = t;
        t = y[i];
        y[i] = y[jm];
        y[jm] = t;
        t = ang[i];
        ang[i] = ang[jm];
        ang[jm] = t;
    }
}

// swGeometry::isInsidePolygon with small = 0 (:111-142); the polygon is already sorted, which
// sorting again leaves as it is
__device__ bool inside_polygon(double x, double y, const double* px, const double* py, int n)
{
    int cnt = 0;
    for (int k = 0; k < n; k++) {
        const double x1 = px[k], y1 = py[k], x2 = px[(k + 1) % n], y2 = py[(k + 1) % n];
        if (fabs(y1 - y2) < 0.0) continue;
        const double xi = (x2 - x1) * (y - y1) / (y2 - y1) + x1;
        if ((xi > x) && (((y1 < y) && y2 >= y) || (y2 < y && y1 >= y))) cnt++;
    }
    return (cnt % 2) == 1;
}

// swGeometry::isOnSegment (:170-193)
__device__ bool on_segment(double x, double y, double sx0, double sy0, double sx1, double sy1)
{
    if (sy1 == sy0) return (y == sy0) && (x >= dmin(sx0, sx1)) && (x <= dmax(sx0, sx1));
    return (x == (y - sy0) * (sx1 - sx0) / (sy1 - sy0) + sx0) && (y >= dmin(sy0, sy1)) && (y <= dmax(sy0, sy1));
}

// swGeometry::isOnPolygonContour (:144-168), polygon sorted
__device__ bool on_contour(double x, double y, const double* px, const double* py, int n)
{
    for (int k = 0; k < n; k++)
        if (on_segment(x, y, px[k], py[k], px[(k + 1) % n], py[(k + 1) % n])) return true;
    return false;
}

// swGeometry::segmentsIntersection (:195-264)
__device__ bool seg_intersection(double ax0, double ay0, double ax1, double ay1, double bx0, double by0, double bx1,
                                 double by1, double& xo, double& yo)
{
    double xi, yi;
    if ((ax0 != ax1) && (bx0 != bx1)) {
        const double a1 = (ay1 - ay0) / (ax1 - ax0);
        const double b1 = ay0 - a1 * ax0;
        const double a2 = (by1 - by0) / (bx1 - bx0);
        const double b2 = by0 - a2 * bx0;
        if (a1 == a2) return false;
        xi = -(b2 - b1) / (a2 - a1);
        yi = a1 * xi + b1;
    } else if ((ax0 == ax1) && (bx0 != bx1)) {
        const double a2 = (by1 - by0) / (bx1 - bx0);
        const double b2 = by0 - a2 * bx0;
        xi = ax0;
        yi = a2 * xi + b2;
    } else if ((ax0 != ax1) && (bx0 == bx1)) {
        const double a1 = (ay1 - ay0) / (ax1 - ax0);
        const double b1 = ay0 - a1 * ax0;
        xi = bx0;
        yi = a1 * xi + b1;
    } else {
        return false;
    }
    if (((dmin(ax0, ax1) <= xi) && (xi <= dmax(ax0, ax1))) && ((dmin(bx0, bx1) <= xi) && (xi <= dmax(bx0, bx1))) &&
        ((dmin(ay0, ay1) <= yi) && (yi <= dmax(ay0, ay1))) && ((dmin(by0, by1) <= yi) && (yi <= dmax(by0, by1)))) {
        xo = xi;
        yo = yi;
        return true;
    }
    return false;
}

__device__ bool is_vertex(const double* px, const double* py, int n, double x, double y)
{
    for (int k = 0; k < n; k++)
        if (px[k] == x && py[k] == y) return true;
    return false;
}

// swGeometry::computeIntersectionArea (:32-96); both polygons sorted on entry
__device__ double intersection_area(const double* x1, const double* y1, int n1, const double* x2, const double* y2,
                                    int n2, bool& overflow)
{
    double x3[kMaxPoly], y3[kMaxPoly];
    int n3 = 0;
    auto push = [&](double x, double y) {
        if (n3 < kMaxPoly) {
            x3[n3] = x;
            y3[n3] = y;
            n3++;
        } else {
            overflow = true;
        }
    };
    for (int k = 0; k < n1; k++)
        if (inside_polygon(x1[k], y1[k], x2, y2, n2)) push(x1[k], y1[k]);
    for (int k = 0; k < n2; k++)
        if (inside_polygon(x2[k], y2[k], x1, y1, n1)) push(x2[k], y2[k]);
    for (int a = 0; a < n1; a++)
        for (int b = 0; b < n2; b++) {
            double xi = 0, yi = 0;
            if (seg_intersection(x1[a], y1[a], x1[(a + 1) % n1], y1[(a + 1) % n1], x2[b], y2[b], x2[(b + 1) % n2],
                                 y2[(b + 1) % n2], xi, yi) &&
                !is_vertex(x3, y3, n3, xi, yi))
                push(xi, yi);
        }
    // swGeometry::computeArea (:9-30)
    sort_vertices(x3, y3, n3);
    double area = 0;
    for (int k = 0; k < n3; k++) area += x3[k] * y3[(k + 1) % n3] - x3[(k + 1) % n3] * y3[k];
    area /= 2;
    return area;
}

// swGeometry::lenghtSegmentInPolygon (:286-387); the polygon sorted on entry
__device__ double length_in_polygon(const double* px, const double* py, int n, double sx0, double sy0, double sx1,
                                    double sy1, bool& overflow)
{
    double xs[kMaxBldVerts + 2], ys[kMaxBldVerts + 2];
    int m = 2;
    xs[0] = sx0;
    ys[0] = sy0;
    xs[1] = sx1;
    ys[1] = sy1;
    for (int k = 0; k < n; k++) {
        double xi = 0, yi = 0;
        if (seg_intersection(px[k], py[k], px[(k + 1) % n], py[(k + 1) % n], sx0, sy0, sx1, sy1, xi, yi) &&
            !is_vertex(xs, ys, m, xi, yi)) {
            if (m < kMaxBldVerts + 2) {
                xs[m] = xi;
                ys[m] = yi;
                m++;
            } else {
                overflow = true;
            }
        }
    }
    const bool by_x = xs[0] != xs[1];
    for (int i = 0; i < m; i++) {
        int jm = i;
        for (int j = i; j < m; j++)
            if ((by_x ? xs[j] < xs[jm] : ys[j] < ys[jm])) jm = j;
        double t = xs[i];
        xs[i] = xs[jm];
        xs[jm] = t;
        t = ys[i];
        ys[i] = ys[jm];
        ys[jm] = t;
    }
    bool inside;
    if (on_contour(xs[0], ys[0], px, py, n)) {
        const double xm = (xs[0] + xs[1]) / 2, ym = (ys[0] + ys[1]) / 2;
        inside = inside_polygon(xm, ym, px, py, n) || on_contour(xm, ym, px, py, n);
    } else {
        inside = inside_polygon(xs[0], ys[0], px, py, n);
    }
    double len = 0;
    for (int k = 0; k < m - 1; k++) {
        if (inside) {
            const double dx = xs[k + 1] - xs[k], dy = ys[k + 1] - ys[k];
            len += sqrt(dx * dx + dy * dy);
        }
        inside = !inside;
    }
    return len;
}

struct Blds {
    int n;
    const int* off;     // [n + 1]
    const double* x;    // flat
    const double* y;
    const double* h;    // heights (null: every building counts at every level)
    const double4* bb;  // {xmin, ymin, xmax, ymax}
};

__device__ __forceinline__ bool counts(const Blds& b, int k, double level) { return !b.h || b.h[k] > level; }

__device__ __forceinline__ bool disjoint(double4 a, double4 b)
{
    return a.z < b.x || b.z < a.x || a.w < b.y || b.w < a.y;
}

// load a building's footprint, sorted (the reference sorts the copy it receives)
__device__ int load_building(const Blds& b, int k, double* x, double* y, bool& overflow)
{
    const int o = b.off[k], n = b.off[k + 1] - o;
    if (n > kMaxBldVerts || n < 1) {
        overflow = true;
        return 0;
    }
    for (int i = 0; i < n; i++) {
        x[i] = b.x[o + i];
        y[i] = b.y[o + i];
    }
    sort_vertices(x, y, n);
    return n;
}

// cellPorosity (:31-90): 1 - sum_k area(cell, building k) / cell area
__global__ void k_cell_porosity(int nc, const int* __restrict__ coff, const int* __restrict__ cnodes,
                                const double* __restrict__ nx, const double* __restrict__ ny,
                                const double* __restrict__ area, Blds b, const double* __restrict__ levels, int nl,
                                double* out, unsigned* status)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)nc * nl) return;
    const int c = (int)(i / nl), l = (int)(i % nl);
    const double level = levels[l];
    const int o = coff[c], n = coff[c + 1] - o;
    bool overflow = n > kMaxCellVerts || n < 3;
    double cx[kMaxCellVerts], cy[kMaxCellVerts];
    double4 cb = make_double4(1e300, 1e300, -1e300, -1e300);
    for (int k = 0; k < n && k < kMaxCellVerts; k++) {
        cx[k] = nx[cnodes[o + k]];
        cy[k] = ny[cnodes[o + k]];
        cb = make_double4(fmin(cb.x, cx[k]), fmin(cb.y, cy[k]), fmax(cb.z, cx[k]), fmax(cb.w, cy[k]));
    }
    double built = 0;
    if (!overflow) {
        sort_vertices(cx, cy, n);
        double bx[kMaxBldVerts], by[kMaxBldVerts];
        for (int k = 0; k < b.n && !overflow; k++) {
            if (!counts(b, k, level) || disjoint(cb, b.bb[k])) continue;
            const int m = load_building(b, k, bx, by, overflow);
            if (!overflow) built += intersection_area(cx, cy, n, bx, by, m, overflow);
        }
    }
    if (overflow) atomicOr(status, 1u);
    out[(size_t)c * nl + l] = 1 - built / area[c];
}

// edgePorosity (:256-388): 1 - sum_k length of the edge in building k / edge length
__global__ void k_edge_porosity(int ne, const int2* __restrict__ enodes, const double* __restrict__ nx,
                                const double* __restrict__ ny, const double* __restrict__ len, Blds b,
                                const double* __restrict__ levels, int nl, double* out, unsigned* status)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)ne * nl) return;
    const int e = (int)(i / nl), l = (int)(i % nl);
    const double level = levels[l];
    const int2 en = enodes[e];
    const double x0 = nx[en.x], y0 = ny[en.x], x1 = nx[en.y], y1 = ny[en.y];
    const double4 eb = make_double4(fmin(x0, x1), fmin(y0, y1), fmax(x0, x1), fmax(y0, y1));
    bool overflow = false;
    double built = 0;
    double bx[kMaxBldVerts], by[kMaxBldVerts];
    for (int k = 0; k < b.n && !overflow; k++) {
        if (!counts(b, k, level) || disjoint(eb, b.bb[k])) continue;
        const int m = load_building(b, k, bx, by, overflow);
        if (!overflow) built += length_in_polygon(bx, by, m, x0, y0, x1, y1, overflow);
    }
    if (overflow) atomicOr(status, 1u);
    out[(size_t)e * nl + l] = 1 - built / len[e];
}

// ---- raster input (swRasterBuildings, src/sw2dPorosityMapper/swRasterBuildings.cpp): a grid of
// building heights, pixel centres xc [nx] and yc [ny] ascending, heights b [ny x nx]
struct Raster {
    int nx, ny;
    const double* xc;
    const double* yc;
    const double* b;
    double dx, dy;
};

// getIndexX / getIndexY (:268-331): the pixel holding x (y); the y test of the first pixel uses
// yc[1], as the reference does.  Outside the raster (the reference stops) sets `bad`.
__device__ int index_x(const Raster& r, double x, bool& bad)
{
    if (x < r.xc[0] - r.dx / 2 || x > r.xc[r.nx - 1] + r.dx / 2) bad = true;
    if (x < r.xc[0] + r.dx / 2) return 0;
    int i = 0;
    while ((i < r.nx - 1) && (x > r.xc[i + 1] - r.dx / 2)) i++;
    return i;
}
__device__ int index_y(const Raster& r, double y, bool& bad)
{
    if (y < r.yc[0] - r.dy / 2 || y > r.yc[r.ny - 1] + r.dy / 2) bad = true;
    if (y < r.yc[1] + r.dy / 2) return 0;
    int i = 0;
    while ((i < r.ny - 1) && (y > r.yc[i + 1] - r.dy / 2)) i++;
    return i;
}

// the pixel (i, j) as the reference builds it (corners in the order x-, x+, x-, x+ / y-, y-,
// y+, y+), sorted
__device__ void pixel(const Raster& r, int i, int j, double* x, double* y)
{
    x[0] = r.xc[i] - r.dx / 2;
    x[1] = r.xc[i] + r.dx / 2;
    x[2] = r.xc[i] - r.dx / 2;
    x[3] = r.xc[i] + r.dx / 2;
    y[0] = r.yc[j] - r.dy / 2;
    y[1] = r.yc[j] - r.dy / 2;
    y[2] = r.yc[j] + r.dy / 2;
    y[3] = r.yc[j] + r.dy / 2;
    sort_vertices(x, y, 4);
}

// cellPorosity, raster branch (:64-87): the pixels of the cell's bounding box taller than h
__global__ void k_cell_porosity_raster(int nc, const int* __restrict__ coff, const int* __restrict__ cnodes,
                                       const double* __restrict__ nx, const double* __restrict__ ny,
                                       const double* __restrict__ area, Raster r, const double* __restrict__ levels,
                                       int nl, double* out, unsigned* status)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nc * nl) return;
    const int c = (int)(t / nl), l = (int)(t % nl);
    const double level = levels[l];
    const int o = coff[c], n = coff[c + 1] - o;
    bool overflow = n > kMaxCellVerts || n < 3;
    double cx[kMaxCellVerts], cy[kMaxCellVerts];
    double built = 0;
    if (!overflow) {
        double x0 = nx[cnodes[o]], y0 = ny[cnodes[o]], x1 = x0, y1 = y0;  // getBoundingBox (:147-181)
        for (int k = 0; k < n; k++) {
            cx[k] = nx[cnodes[o + k]];
            cy[k] = ny[cnodes[o + k]];
            if (cx[k] < x0) x0 = cx[k];
            if (cy[k] < y0) y0 = cy[k];
            if (cx[k] > x1) x1 = cx[k];
            if (cy[k] > y1) y1 = cy[k];
        }
        int i0 = index_x(r, x0, overflow), j0 = index_y(r, y0, overflow);
        int i1 = index_x(r, x1, overflow) + 1, j1 = index_y(r, y1, overflow) + 1;
        if (i1 > r.nx - 1) i1 -= 1;
        if (j1 > r.ny - 1) j1 -= 1;
        sort_vertices(cx, cy, n);
        double px[4], py[4];
        for (int i = i0; i <= i1 && !overflow; i++)
            for (int j = j0; j <= j1 && !overflow; j++) {
                if (!(r.b[(size_t)j * r.nx + i] > level)) continue;
                pixel(r, i, j, px, py);
                built += intersection_area(cx, cy, n, px, py, 4, overflow);
            }
    }
    if (overflow) atomicOr(status, 1u);
    out[(size_t)c * nl + l] = 1 - built / area[c];
}

// edgePorosity, raster branch (:283-318): a pixel side shared by two built pixels along the
// edge counts half in each
__global__ void k_edge_porosity_raster(int ne, const int2* __restrict__ enodes, const double* __restrict__ nx,
                                       const double* __restrict__ ny, const double* __restrict__ len, Raster r,
                                       const double* __restrict__ levels, int nl, double* out, unsigned* status)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ne * nl) return;
    const int e = (int)(t / nl), l = (int)(t % nl);
    const double level = levels[l];
    const int2 en = enodes[e];
    const double x0 = nx[en.x], y0 = ny[en.x], x1 = nx[en.y], y1 = ny[en.y];
    bool overflow = false;
    // getBoundingBox of an edge (:183-240)
    const double mnx = dmin(x0, x1), mny = dmin(y0, y1), mxx = dmax(x0, x1), mxy = dmax(y0, y1);
    const int i0 = index_x(r, mnx, overflow), j0 = index_y(r, mny, overflow);
    int i1 = index_x(r, mxx, overflow) + 1, j1 = index_y(r, mxy, overflow) + 1;
    if (mxx == r.xc[0] - r.dx / 2) i1 -= 1;
    if (mxy == r.yc[0] - r.dy / 2) j1 -= 1;
    if (i1 > r.nx - 1) i1 -= 1;
    if (j1 > r.ny - 1) j1 -= 1;
    const bool horizontal = (y0 == y1) && (y0 == r.yc[j1] - r.dy / 2) && j0 != j1;
    const bool vertical = (x0 == x1) && (x0 == r.xc[i1] - r.dx / 2) && i0 != i1;
    double built = 0;
    double px[4], py[4];
    for (int i = i0; i <= i1 && !overflow; i++)
        for (int j = j0; j <= j1 && !overflow; j++) {
            if (!(r.b[(size_t)j * r.nx + i] > level)) continue;
            pixel(r, i, j, px, py);
            double li = length_in_polygon(px, py, 4, x0, y0, x1, y1, overflow);
            if ((horizontal && (r.b[(size_t)j0 * r.nx + i] > level) && (r.b[(size_t)j1 * r.nx + i] > level)) ||
                (vertical && (r.b[(size_t)j * r.nx + i0] > level) && (r.b[(size_t)j * r.nx + i1] > level)))
                li /= 2;
            built += li;
        }
    if (overflow) atomicOr(status, 1u);
    out[(size_t)e * nl + l] = 1 - built / len[e];
}

struct DevBuf {
    std::vector<void*> p;
    ~DevBuf()
    {
        for (void* q : p) cudaFree(q);
    }
    // a device copy of src[0, n), or n zeroed elements when src is null
    template <class T>
    cudaError_t up(const T* src, size_t n, T** dst)
    {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
        if (e != cudaSuccess) return e;
        p.push_back(q);
        *dst = static_cast<T*>(q);
        if (!n) return cudaSuccess;
        return src ? cudaMemcpy(q, src, n * sizeof(T), cudaMemcpyHostToDevice) : cudaMemset(q, 0, n * sizeof(T));
    }
};

std::string g_map_error;

int map_fail(int code, const std::string& msg)
{
    g_map_error = msg;
    return code;
}

// The mesh on the device and the outputs, shared by both inputs.
struct MeshDev {
    DevBuf d;
    int nc = 0, nl = 0, ni = 0, nb = 0;
    int *coff = nullptr, *cn = nullptr;
    int2 *ei = nullptr, *eb = nullptr;
    double *nx = nullptr, *ny = nullptr, *area = nullptr, *il = nullptr, *bl = nullptr, *lev = nullptr;
    double *cell = nullptr, *eint = nullptr, *ebnd = nullptr;
    unsigned* status = nullptr;
};

int mesh_setup(int device, const sw2d_map_mesh* mesh, const double* levels, int n_levels, bool want_int,
               bool want_bnd, MeshDev& md)
{
    if (!mesh || !levels || n_levels < 1) return map_fail(SW2D_E_ARG, "invalid arguments");
    if (mesh->cell_nb <= 0 || mesh->node_nb <= 0 || mesh->cell_nb >= (1LL << 30) || mesh->node_nb >= (1LL << 31) ||
        mesh->edge_int_nb < 0 || mesh->edge_bnd_nb < 0 || mesh->edge_int_nb >= (1LL << 30) ||
        mesh->edge_bnd_nb >= (1LL << 30))
        return map_fail(SW2D_E_ARG, "mesh sizes");
    if (!mesh->node_x || !mesh->node_y || !mesh->cell_node_offsets || !mesh->cell_nodes || !mesh->cell_area)
        return map_fail(SW2D_E_ARG, "mesh arrays missing");
    if ((want_int && (!mesh->edge_int_nodes || !mesh->edge_int_length)) ||
        (want_bnd && (!mesh->edge_bnd_nodes || !mesh->edge_bnd_length)))
        return map_fail(SW2D_E_ARG, "edge arrays missing");
    const int64_t nc = mesh->cell_nb, nn = mesh->node_nb;
    // host-side checks and conversions: offsets and node indices in range
    std::vector<int> coff(nc + 1), cn((size_t)std::max<int64_t>(0, mesh->cell_node_offsets[nc]));
    for (int64_t c = 0; c <= nc; c++) {
        const int64_t v = mesh->cell_node_offsets[c];
        if (v < 0 || (c > 0 && v < mesh->cell_node_offsets[c - 1])) return map_fail(SW2D_E_ARG, "cell node offsets");
        coff[c] = (int)v;
    }
    for (size_t k = 0; k < cn.size(); k++) {
        const int64_t v = mesh->cell_nodes[k];
        if (v < 0 || v >= nn) return map_fail(SW2D_E_ARG, "cell node index out of range");
        cn[k] = (int)v;
    }
    auto edges = [&](int64_t ne, const int64_t* en, std::vector<int2>& out) {
        out.resize(ne);
        for (int64_t e = 0; e < ne; e++) {
            if (en[2 * e] < 0 || en[2 * e] >= nn || en[2 * e + 1] < 0 || en[2 * e + 1] >= nn) return false;
            out[e] = make_int2((int)en[2 * e], (int)en[2 * e + 1]);
        }
        return true;
    };
    std::vector<int2> ei, eb;
    if (want_int && !edges(mesh->edge_int_nb, mesh->edge_int_nodes, ei))
        return map_fail(SW2D_E_ARG, "internal edge node index out of range");
    if (want_bnd && !edges(mesh->edge_bnd_nb, mesh->edge_bnd_nodes, eb))
        return map_fail(SW2D_E_ARG, "boundary edge node index out of range");
    if (cudaSetDevice(device) != cudaSuccess) return map_fail(SW2D_E_NO_DEVICE, "cudaSetDevice failed");
    md.nc = (int)nc;
    md.nl = n_levels;
    md.ni = want_int ? (int)mesh->edge_int_nb : 0;
    md.nb = want_bnd ? (int)mesh->edge_bnd_nb : 0;
    DevBuf& d = md.d;
    cudaError_t e = d.up(coff.data(), coff.size(), &md.coff);
    if (e == cudaSuccess) e = d.up(cn.data(), cn.size(), &md.cn);
    if (e == cudaSuccess) e = d.up(mesh->node_x, (size_t)nn, &md.nx);
    if (e == cudaSuccess) e = d.up(mesh->node_y, (size_t)nn, &md.ny);
    if (e == cudaSuccess) e = d.up(mesh->cell_area, (size_t)nc, &md.area);
    if (e == cudaSuccess) e = d.up(levels, (size_t)n_levels, &md.lev);
    if (e == cudaSuccess) e = d.up((const double*)nullptr, (size_t)nc * n_levels, &md.cell);
    if (e == cudaSuccess) e = d.up((const unsigned*)nullptr, 1, &md.status);
    if (e == cudaSuccess && want_int) {
        e = d.up(ei.data(), ei.size(), &md.ei);
        if (e == cudaSuccess) e = d.up(mesh->edge_int_length, (size_t)mesh->edge_int_nb, &md.il);
        if (e == cudaSuccess) e = d.up((const double*)nullptr, (size_t)mesh->edge_int_nb * n_levels, &md.eint);
    }
    if (e == cudaSuccess && want_bnd) {
        e = d.up(eb.data(), eb.size(), &md.eb);
        if (e == cudaSuccess) e = d.up(mesh->edge_bnd_length, (size_t)mesh->edge_bnd_nb, &md.bl);
        if (e == cudaSuccess) e = d.up((const double*)nullptr, (size_t)mesh->edge_bnd_nb * n_levels, &md.ebnd);
    }
    if (e != cudaSuccess) return map_fail(SW2D_E_CUDA, std::string("mapper buffers: ") + cudaGetErrorString(e));
    return SW2D_OK;
}

int mesh_finish(MeshDev& md, double* cell_phi, double* edge_int_phi, double* edge_bnd_phi, const char* limits)
{
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    unsigned st = 0;
    const size_t nl = (size_t)md.nl;
    if (e == cudaSuccess) e = cudaMemcpy(&st, md.status, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(cell_phi, md.cell, (size_t)md.nc * nl * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && md.eint && md.ni > 0)
        e = cudaMemcpy(edge_int_phi, md.eint, (size_t)md.ni * nl * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && md.ebnd && md.nb > 0)
        e = cudaMemcpy(edge_bnd_phi, md.ebnd, (size_t)md.nb * nl * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return map_fail(SW2D_E_CUDA, std::string("mapper kernels: ") + cudaGetErrorString(e));
    if (st) return map_fail(SW2D_E_ARG, limits);
    return SW2D_OK;
}

constexpr int kMapBlock = 128;
unsigned map_blocks(int64_t n) { return (unsigned)((n + kMapBlock - 1) / kMapBlock); }

}  // namespace

extern "C" {

const char* sw2d_map_last_error(void) { return g_map_error.c_str(); }

int sw2d_map_porosity(int device, const sw2d_map_mesh* mesh, const sw2d_buildings* blds, const double* levels,
                      int n_levels, double* cell_phi, double* edge_int_phi, double* edge_bnd_phi)
{
    g_map_error.clear();
    if (!blds || !cell_phi) return map_fail(SW2D_E_ARG, "invalid arguments");
    if (blds->n < 0 || (blds->n > 0 && (!blds->offsets || !blds->x || !blds->y)))
        return map_fail(SW2D_E_ARG, "building arrays missing");
    const int64_t nb = blds->n;
    std::vector<int> boff(nb + 1);
    std::vector<double4> bbox(nb);
    for (int64_t k = 0; k <= nb; k++) boff[k] = nb ? (int)blds->offsets[k] : 0;
    for (int64_t k = 0; k < nb; k++) {
        const int64_t o = blds->offsets[k], e = blds->offsets[k + 1];
        if (e - o < 1 || e - o > kMaxBldVerts) return map_fail(SW2D_E_ARG, "a building has 0 or more than 64 vertices");
        double4 b = make_double4(1e300, 1e300, -1e300, -1e300);
        for (int64_t i = o; i < e; i++)
            b = make_double4(std::min(b.x, blds->x[i]), std::min(b.y, blds->y[i]), std::max(b.z, blds->x[i]),
                             std::max(b.w, blds->y[i]));
        bbox[k] = b;
    }
    MeshDev md;
    int rc = mesh_setup(device, mesh, levels, n_levels, edge_int_phi != nullptr, edge_bnd_phi != nullptr, md);
    if (rc) return rc;
    int* d_boff = nullptr;
    double *d_bx = nullptr, *d_by = nullptr, *d_bh = nullptr;
    double4* d_bb = nullptr;
    const size_t nbv = nb ? (size_t)blds->offsets[nb] : 0;
    cudaError_t e = md.d.up(boff.data(), boff.size(), &d_boff);
    if (e == cudaSuccess) e = md.d.up(blds->x, nbv, &d_bx);
    if (e == cudaSuccess) e = md.d.up(blds->y, nbv, &d_by);
    if (e == cudaSuccess && blds->height) e = md.d.up(blds->height, (size_t)nb, &d_bh);
    if (e == cudaSuccess) e = md.d.up(bbox.data(), bbox.size(), &d_bb);
    if (e != cudaSuccess) return map_fail(SW2D_E_CUDA, std::string("mapper buffers: ") + cudaGetErrorString(e));
    Blds b{(int)nb, d_boff, d_bx, d_by, d_bh, d_bb};
    k_cell_porosity<<<map_blocks((int64_t)md.nc * md.nl), kMapBlock>>>(md.nc, md.coff, md.cn, md.nx, md.ny, md.area, b,
                                                                      md.lev, md.nl, md.cell, md.status);
    if (md.ni > 0)
        k_edge_porosity<<<map_blocks((int64_t)md.ni * md.nl), kMapBlock>>>(md.ni, md.ei, md.nx, md.ny, md.il, b, md.lev,
                                                                          md.nl, md.eint, md.status);
    if (md.nb > 0)
        k_edge_porosity<<<map_blocks((int64_t)md.nb * md.nl), kMapBlock>>>(md.nb, md.eb, md.nx, md.ny, md.bl, b, md.lev,
                                                                          md.nl, md.ebnd, md.status);
    return mesh_finish(md, cell_phi, edge_int_phi, edge_bnd_phi,
                       "a cell with more than 8 nodes or an intersection of more than 96 points");
}

int sw2d_map_porosity_raster(int device, const sw2d_map_mesh* mesh, const sw2d_raster* raster, const double* levels,
                             int n_levels, double* cell_phi, double* edge_int_phi, double* edge_bnd_phi)
{
    g_map_error.clear();
    if (!raster || !cell_phi || !raster->x || !raster->y || !raster->height)
        return map_fail(SW2D_E_ARG, "invalid arguments");
    if (raster->nx < 2 || raster->ny < 2 || raster->nx * raster->ny >= (1LL << 31))
        return map_fail(SW2D_E_ARG, "the raster needs at least 2 x 2 pixels");
    MeshDev md;
    int rc = mesh_setup(device, mesh, levels, n_levels, edge_int_phi != nullptr, edge_bnd_phi != nullptr, md);
    if (rc) return rc;
    double *d_x = nullptr, *d_y = nullptr, *d_b = nullptr;
    cudaError_t e = md.d.up(raster->x, (size_t)raster->nx, &d_x);
    if (e == cudaSuccess) e = md.d.up(raster->y, (size_t)raster->ny, &d_y);
    if (e == cudaSuccess) e = md.d.up(raster->height, (size_t)(raster->nx * raster->ny), &d_b);
    if (e != cudaSuccess) return map_fail(SW2D_E_CUDA, std::string("mapper buffers: ") + cudaGetErrorString(e));
    // swRasterBuildings::build (:124-125): the pixel sizes from the first two centres
    Raster r{(int)raster->nx, (int)raster->ny, d_x, d_y, d_b, raster->x[1] - raster->x[0], raster->y[1] - raster->y[0]};
    k_cell_porosity_raster<<<map_blocks((int64_t)md.nc * md.nl), kMapBlock>>>(md.nc, md.coff, md.cn, md.nx, md.ny,
                                                                             md.area, r, md.lev, md.nl, md.cell,
                                                                             md.status);
    if (md.ni > 0)
        k_edge_porosity_raster<<<map_blocks((int64_t)md.ni * md.nl), kMapBlock>>>(md.ni, md.ei, md.nx, md.ny, md.il, r,
                                                                                 md.lev, md.nl, md.eint, md.status);
    if (md.nb > 0)
        k_edge_porosity_raster<<<map_blocks((int64_t)md.nb * md.nl), kMapBlock>>>(md.nb, md.eb, md.nx, md.ny, md.bl, r,
                                                                                 md.lev, md.nl, md.ebnd, md.status);
    return mesh_finish(md, cell_phi, edge_int_phi, edge_bnd_phi,
                       "a cell with more than 8 nodes, or a cell or an edge outside the raster");
}

}  // extern "C"
