// sw2d_sp.cu — SW2D single-porosity explicit step on the B200 (sm_100a), FP64, and the C ABI of
// include/sw2d_b200.h.
//
// One time step (the body of swSp::execute's loop, src/sw2dSolver/models/sp/swSp.cpp:522-589)
// is four kernels, all predicated on device state so that a CUDA graph of many steps runs
// without the host:
//
//   k_slopes   per cell   limited free-surface slopes (MUSCL-EVR only)      swSpHypMusclEvr.cpp:11-115
//   k_edges    per edge   Riemann states, max wave speed, HLLC / boundary    swSpHypGodunov.cpp, swSpHypMusclEvr.cpp:119-277,
//                         fluxes                                            swSpHyp.cpp:13-135,276-402,664-998
//   k_cfl      per cell   swept length, CFL dt, warp -> block -> grid min,   swSpHyp.cpp:430-512
//                         dt_map snap and t_max clip on the device
//   k_update   per cell   flux balance (CSR gather in the reference's per-   swSpHyp.cpp:214-273,184-209,
//                         cell order), round-off flush, negative-depth clamp, swSpSourceFriction.cpp:11-219,
//                         friction, singular head loss, velocity cap, t += dt swSp.cpp:447-479
//
// Cells are renumbered along a Hilbert curve and internal edges by their first cell, for
// locality; every per-cell sum still runs in the reference's order (boundary edges, then
// internal edges, by increasing ORIGINAL index), so the renumbering changes no bit.  No
// floating-point atomics are used anywhere.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/sw2d_b200.h"
#include "sp_math.cuh"

using namespace sw2d;

namespace {

constexpr int kBlock = 256;

// Device-resident loop control.  t and t_max decide whether a step runs; `go` and `dt` are
// written by the CFL kernel's last block and read by the update kernel.
struct Ctrl {
    double t;
    double dt;
    double t_max;
    long long steps;
    unsigned int status;
    unsigned int blocks_done;
    int go;
    int pad;
};

struct DevMesh {
    int nc, ni, nb;
    // cells
    double *h, *q, *r;
    const double *zb, *area, *cx, *cy, *phi, *bous;
    const double *fk1, *fk2, *fcos, *fsin;               // friction (may be null)
    const double *hs, *hk1, *hk2, *hcos, *hsin;          // singular head loss (may be null)
    const int *cb_off, *cb_idx;                          // boundary edges of each cell
    const int *ci_off, *ci_ent, *ci_nbr;                 // internal edges (edge*2 + side) and neighbour
    double *sx, *sy;                                      // MUSCL slopes
    // internal edges
    const int2* lr;
    const double *len, *nx, *ny, *mx, *my, *coefL, *coefR;
    double *F1, *F2, *F3, *S2L, *S2R, *lmax;
    // boundary edges
    const int* bcell;
    const int* bbc;
    const double *blen, *bnx, *bny, *bcoef;
    double *F1b, *F2b, *F3b, *lmaxb;
    // boundary series
    const int* bctype;
    const long long* bcoff;
    const double *bctimes, *bcvals;
    // parameters
    double h_min, phi_min, cfl_max, dt_max, dt_map, v_max, fr_max;
    int scheme, topo, friction, head_loss, neg_detect;
    // dt reduction scratch
    double* part;
    Ctrl* ctrl;
};

__device__ __forceinline__ bool step_active(const Ctrl* c) { return c->t < c->t_max; }

// ------------------------------------------------------------------------------------------
// k_slopes: swSp::computeMusclSlopes (swSpHypMusclEvr.cpp:11-115) per cell.  Step 1 sums the
// neighbour contributions in increasing internal-edge order; step 2 applies, edge after edge
// in the same order, the under/overshoot rescaling of this cell's slope (that rescaling only
// reads this cell's slope, so the reference's global edge loop decomposes exactly per cell).
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_slopes(DevMesh m)
{
    if (!step_active(m.ctrl)) return;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const double zc = m.h[c] + m.zb[c];
    const double xc = m.cx[c], yc = m.cy[c];
    const int k0 = m.ci_off[c], k1 = m.ci_off[c + 1];
    double sx = 0.0, sy = 0.0, wsum = 0.0;
    if (k1 - k0 > 1) {
        for (int k = k0; k < k1; k++) {
            int j = m.ci_nbr[k];
            double dx = m.cx[j] - xc;
            double dy = m.cy[j] - yc;
            double dist = sqrt(dx * dx + dy * dy);
            double w = 1.0 / dist;
            double zj = m.h[j] + m.zb[j];
            sx += (zj - zc) * dx / dist / dist * w;
            sy += (zj - zc) * dy / dist / dist * w;
            wsum += w;
        }
        sx /= wsum;
        sy /= wsum;
    }
    for (int k = k0; k < k1; k++) {
        int ent = m.ci_ent[k];
        int e = ent >> 1;
        int j = m.ci_nbr[k];
        double zj = m.h[j] + m.zb[j];
        double zL = (ent & 1) ? zj : zc;
        double zR = (ent & 1) ? zc : zj;
        double fmx = smax(zL, zR);
        double fmn = smin(zL, zR);
        double rec = zc + (m.mx[e] - xc) * sx + (m.my[e] - yc) * sy;
        if (rec < fmn) {
            double fac = (fmn - zc) / (rec - zc);
            sx *= fac;
            sy *= fac;
        }
        if (rec > fmx) {
            double fac = (fmx - zc) / (rec - zc);
            sx *= fac;
            sy *= fac;
        }
    }
    m.sx[c] = sx;
    m.sy[c] = sy;
}

// ------------------------------------------------------------------------------------------
// k_edges: one thread per internal edge, then one per boundary edge.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_edges(DevMesh m)
{
    if (!step_active(m.ctrl)) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned bad = 0;
    if (i < m.ni) {
        const int e = i;
        const int2 lr = m.lr[e];
        const int a = lr.x, b = lr.y;
        const double nx = m.nx[e], ny = m.ny[e];
        const double zbL = m.zb[a], zbR = m.zb[b];
        const double bL = m.bous[a], bR = m.bous[b];
        SideState SL, SR;
        if (m.scheme == SW2D_SCHEME_GODUNOV) {
            SL = godunov_side(m.h[a], m.q[a], m.r[a], zbL, bL, nx, ny);
            SR = godunov_side(m.h[b], m.q[b], m.r[b], zbR, bR, nx, ny);
        } else {
            const double dtp = m.ctrl->dt;
            const double mx = m.mx[e], my = m.my[e];
            const double ha = m.h[a], hb = m.h[b];
            SL = evr_side(true, ha, m.q[a], m.r[a], zbL, bL, ha + zbL, m.sx[a], m.sy[a], m.cx[a], m.cy[a], mx, my, nx,
                          ny, dtp);
            SR = evr_side(false, hb, m.q[b], m.r[b], zbR, bR, hb + zbR, m.sx[b], m.sy[b], m.cx[b], m.cy[b], mx, my, nx,
                          ny, dtp);
        }
        m.lmax[e] = max4(fabs(SL.lm), fabs(SL.lp), fabs(SR.lm), fabs(SR.lp));
        const double hL = SL.z - zbL, hR = SR.z - zbR;
        if ((hL > m.h_min) || (hR > m.h_min)) {
            EdgeFlux f = hllc(m.topo == SW2D_TOPO_BLENDING, bL, bR, m.phi[a], m.phi[b], zbL, zbR, SL, SR, m.h_min,
                              m.phi_min, &bad);
            if (isnan(f.f1)) bad |= kStatusNanFlux;
            m.F1[e] = f.f1;
            m.F2[e] = f.f2;
            m.F3[e] = f.f3;
            m.S2L[e] = f.sl;
            m.S2R[e] = f.sr;
        }
    } else if (i < m.ni + m.nb) {
        const int e = i - m.ni;
        const int c = m.bcell[e];
        const double zbc = m.zb[c];
        SideState S = godunov_side(m.h[c], m.q[c], m.r[c], zbc, m.bous[c], m.bnx[e], m.bny[e]);
        m.lmaxb[e] = (m.scheme == SW2D_SCHEME_GODUNOV) ? smax(fabs(S.lp), fabs(S.lm)) : smax(fabs(S.lm), fabs(S.lp));
        const int k = m.bbc[e];
        const long long o0 = m.bcoff[k], o1 = m.bcoff[k + 1];
        const double v = bc_value(m.bctimes + o0, m.bcvals + o0, o1 - o0, m.ctrl->t);
        double f1, f2, f3;
        boundary_flux(m.bous[c], m.phi[c], zbc, S, m.bctype[k], v, m.h_min, &f1, &f2, &f3, &bad);
        m.F1b[e] = f1;
        m.F2b[e] = f2;
        m.F3b[e] = f3;
    }
    if (bad) atomicOr(&m.ctrl->status, bad);
}

// ------------------------------------------------------------------------------------------
// k_cfl: swSp::hypComputeTimeStep (swSpHyp.cpp:430-512).  swept[c] gathers, in the reference's
// order, lambda_max * length over the boundary edges (cell wet) and internal edges; on an
// internal edge the R cell also counts when only L is wet, because the reference carries the
// variable `lambda` over from the L test to the R side (:456-476).  dt = min over cells of
// cfl * area / max(swept, 1e-16), reduced warp -> block -> grid (last block done), then the
// dt_map snap (:496-504) and the t_max clip, all on the device.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ double min_keep(double a, double b) { return (b < a) ? b : a; }

__global__ void __launch_bounds__(kBlock) k_cfl(DevMesh m)
{
    Ctrl* ctrl = m.ctrl;
    if (!step_active(ctrl)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) ctrl->go = 0;
        return;
    }
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    double best = m.dt_max;
    if (c < m.nc) {
        const double hc = m.h[c];
        const bool wet = hc > m.h_min;
        double sw = 0.0;
        if (wet) {
            for (int k = m.cb_off[c]; k < m.cb_off[c + 1]; k++) {
                int e = m.cb_idx[k];
                sw += m.lmaxb[e] * m.blen[e];
            }
        }
        for (int k = m.ci_off[c]; k < m.ci_off[c + 1]; k++) {
            int ent = m.ci_ent[k];
            int e = ent >> 1;
            bool count = wet;
            if ((ent & 1) && !wet) count = m.h[m.ci_nbr[k]] > m.h_min;
            if (count) sw += m.lmax[e] * m.len[e];
        }
        double x = m.cfl_max * (m.area[c] / smax(sw, kSmallReal));
        if (x < best) best = x;
    }
    // warp then block minimum (NaN candidates never win: comparisons with NaN are false)
    for (int off = 16; off > 0; off >>= 1) best = min_keep(best, __shfl_down_sync(0xffffffffu, best, off));
    __shared__ double wmin[kBlock / 32];
    __shared__ bool last;
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) wmin[wid] = best;
    __syncthreads();
    if (wid == 0) {
        best = (lane < kBlock / 32) ? wmin[lane] : m.dt_max;
        for (int off = 16; off > 0; off >>= 1) best = min_keep(best, __shfl_down_sync(0xffffffffu, best, off));
        if (lane == 0) {
            m.part[blockIdx.x] = best;
            __threadfence();
            unsigned done = atomicAdd(&ctrl->blocks_done, 1u);
            last = (done == gridDim.x - 1);
        }
    }
    __syncthreads();
    if (!last) return;
    // last block: reduce the per-block minima
    __threadfence();
    double b2 = m.dt_max;
    for (int i = threadIdx.x; i < gridDim.x; i += blockDim.x) b2 = min_keep(b2, ((volatile double*)m.part)[i]);
    for (int off = 16; off > 0; off >>= 1) b2 = min_keep(b2, __shfl_down_sync(0xffffffffu, b2, off));
    if (lane == 0) wmin[wid] = b2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double dt = m.dt_max;
        for (int w = 0; w < kBlock / 32; w++)
            if (wmin[w] < dt) dt = wmin[w];
        const double t = ctrl->t;
        if (m.dt_map > kSmallReal) {
            int now = (int)(t / m.dt_map);
            int later = (int)((t + dt) / m.dt_map);
            if (later > now) dt = later * m.dt_map - t;
        }
        if ((t + dt) > ctrl->t_max) dt = ctrl->t_max - t;
        ctrl->dt = dt;
        ctrl->go = 1;
        ctrl->blocks_done = 0;
    }
}

// ------------------------------------------------------------------------------------------
// k_update: balance + sources for one cell, then t += dt (block 0).
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_update(DevMesh m)
{
    Ctrl* ctrl = m.ctrl;
    if (!ctrl->go) return;
    const double dt = ctrl->dt;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0) {
        ctrl->t = ctrl->t + dt;  // swSp.cpp:592; no other thread of this kernel reads t
        ctrl->steps += 1;
    }
    if (c >= m.nc) return;
    double hh = m.h[c], qq = m.q[c], rr = m.r[c];
    // hypComputeBalance (swSpHyp.cpp:214-273): boundary edges, then internal edges, each in
    // increasing original index; factors of swSp::computeEdgeFactors (swSp.cpp:338-444)
    for (int k = m.cb_off[c]; k < m.cb_off[c + 1]; k++) {
        const int e = m.cb_idx[k];
        const double cf = m.bcoef[e], nx = m.bnx[e], ny = m.bny[e];
        const double f1 = +cf, f2F2 = +cf * nx, f2F3 = -cf * ny, f2S2 = +cf * nx;
        const double f3F2 = +cf * ny, f3F3 = +cf * nx, f3S2 = +cf * ny;
        const double s2 = 0.0;  // boundary geometric source: never set by hypBoundaryFlux
        hh += f1 * m.F1b[e] * dt;
        qq += (f2F2 * m.F2b[e] + f2S2 * s2 + f2F3 * m.F3b[e]) * dt;
        rr += (f3F2 * m.F2b[e] + f3S2 * s2 + f3F3 * m.F3b[e]) * dt;
    }
    for (int k = m.ci_off[c]; k < m.ci_off[c + 1]; k++) {
        const int ent = m.ci_ent[k];
        const int e = ent >> 1;
        const double nx = m.nx[e], ny = m.ny[e];
        const double F1 = m.F1[e], F2 = m.F2[e], F3 = m.F3[e];
        if (ent & 1) {  // this cell is R
            const double cf = m.coefR[e];
            const double s2 = m.S2R[e];
            const double f1 = +cf, f2F2 = +cf * nx, f2F3 = -cf * ny, f2S2 = +cf * nx;
            const double f3F2 = +cf * ny, f3F3 = +cf * nx, f3S2 = +cf * ny;
            hh += f1 * F1 * dt;
            qq += (f2F2 * F2 + f2S2 * s2 + f2F3 * F3) * dt;
            rr += (f3F2 * F2 + f3S2 * s2 + f3F3 * F3) * dt;
        } else {        // this cell is L
            const double cf = m.coefL[e];
            const double s2 = m.S2L[e];
            const double f1 = -cf, f2F2 = -cf * nx, f2F3 = +cf * ny, f2S2 = +cf * nx;
            const double f3F2 = -cf * ny, f3F3 = -cf * nx, f3S2 = +cf * ny;
            hh += f1 * F1 * dt;
            qq += (f2F2 * F2 + f2S2 * s2 + f2F3 * F3) * dt;
            rr += (f3F2 * F2 + f3S2 * s2 + f3F3 * F3) * dt;
        }
    }
    if (fabs(hh) < kSmallReal) hh = 0.;
    if (fabs(qq) < kSmallReal) qq = 0.;
    if (fabs(rr) < kSmallReal) rr = 0.;
    // negative depth (swSpHyp.cpp:182-210)
    if (m.neg_detect) {
        if (hh < 0) atomicOr(&ctrl->status, kStatusNegDepth);
    } else if (hh < 0.) {
        hh = 0.;
        qq = 0.;
        rr = 0.;
    }
    const double hthr = smax(m.h_min, kSmallReal);
    // friction (swSpSourceFriction.cpp:39-171)
    if (m.friction != SW2D_FRICTION_NONE) {
        if (hh > hthr) {
            double u = qq / hh;
            double v = rr / hh;
            double ca = m.fcos[c], sa = m.fsin[c];
            double ul = u * ca + v * sa;
            double vl = -u * sa + v * ca;
            double un = sqrt(u * u + v * v);
            double f1 = friction_factor(m.friction, m.fk1[c], hh, un, dt);
            double f2 = friction_factor(m.friction, m.fk2[c], hh, un, dt);
            ul *= f1;
            vl *= f2;
            qq = (ul * ca - vl * sa) * hh;
            rr = (ul * sa + vl * ca) * hh;
        } else {
            qq = 0.;
            rr = 0.;
        }
    }
    // singular head loss (swSpSourceFriction.cpp:174-219)
    if (m.head_loss) {
        double ca = m.hcos[c], sa = m.hsin[c];
        double qx = qq * ca + rr * sa;
        double qy = -qq * sa + rr * ca;
        if (hh > hthr) {
            double ax = 0, ay = 0;
            if (hh > m.hs[c]) {
                ax = sqrt(qx * qx + qy * qy) * m.hk1[c] / hh;
                ay = sqrt(qx * qx + qy * qy) * m.hk2[c] / hh;
            }
            qx = qx * exp(-ax * dt);
            qy = qy * exp(-ay * dt);
        } else {
            qx = 0.;
            qy = 0.;
        }
        qq = qx * ca - qy * sa;
        rr = qx * sa + qy * ca;
    }
    // swSp::correctVelocity (swSp.cpp:447-479)
    if (hh > m.h_min) {
        double qn = sqrt(qq * qq + rr * rr);
        double cc = sqrt(kGravity * hh);
        double Fr = qn / cc / hh;
        double fact = smax(qn / (hh * m.v_max), Fr / m.fr_max);
        if (fact > 1.0) {
            qq = qq / fact;
            rr = rr / fact;
        }
    }
    m.h[c] = hh;
    m.q[c] = qq;
    m.r[c] = rr;
}

// swSp::computeEdgeFactors coefficient w / area / phi (swSp.cpp:364-368, 397-405)
__global__ void k_edge_coefficients(DevMesh m, double* coefL, double* coefR, double* bcoef)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m.ni) {
        int2 lr = m.lr[i];
        double w = m.len[i];
        coefL[i] = (m.phi[lr.x] > m.phi_min) ? w / m.area[lr.x] / m.phi[lr.x] : 0.0;
        coefR[i] = (m.phi[lr.y] > m.phi_min) ? w / m.area[lr.y] / m.phi[lr.y] : 0.0;
    } else if (i < m.ni + m.nb) {
        int e = i - m.ni;
        int c = m.bcell[e];
        bcoef[e] = (m.phi[c] > m.phi_min) ? m.blen[e] / m.area[c] / m.phi[c] : 0.0;
    }
}

// caller numbering <-> internal numbering
__global__ void k_gather3(const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c,
                          const int* __restrict__ perm, double* oa, double* ob, double* oc, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        int p = perm[i];
        oa[i] = a[p];
        ob[i] = b[p];
        oc[i] = c[p];
    }
}

__global__ void k_scatter3(const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c,
                           const int* __restrict__ perm, double* oa, double* ob, double* oc, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        int p = perm[i];
        oa[p] = a[i];
        ob[p] = b[i];
        oc[p] = c[i];
    }
}

__global__ void k_scatter1(const double* __restrict__ a, const int* __restrict__ perm, double* oa, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) oa[perm[i]] = a[i];
}

inline unsigned grid_for(long long n) { return (unsigned)((n + kBlock - 1) / kBlock); }

// Hilbert index of (x, y) on a 2^16 x 2^16 grid (the classic rotate-and-flip walk).
uint64_t hilbert_d(uint32_t x, uint32_t y)
{
    uint64_t d = 0;
    for (uint32_t s = 1u << 15; s > 0; s >>= 1) {
        uint32_t rx = (x & s) ? 1u : 0u;
        uint32_t ry = (y & s) ? 1u : 0u;
        d += (uint64_t)s * s * ((3u * rx) ^ ry);
        if (ry == 0) {
            if (rx == 1) {
                x = s - 1 - x;
                y = s - 1 - y;
            }
            std::swap(x, y);
        }
    }
    return d;
}

}  // namespace

// ------------------------------------------------------------------------------------------
// handle
// ------------------------------------------------------------------------------------------
struct sw2d_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    int64_t nc = 0, ni = 0, nb = 0;
    sw2d_params p{};
    std::vector<int> cell_perm, int_perm, bnd_perm;  // [new] = caller index
    std::vector<void*> allocs;
    DevMesh m{};
    Ctrl* ctrl = nullptr;
    Ctrl* ctrl_host = nullptr;  // pinned
    int* d_cell_perm = nullptr;
    int* d_int_perm = nullptr;
    int* d_bnd_perm = nullptr;
    double* stage = nullptr;    // 3 * nc doubles
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    std::string err;
};

namespace {

std::string g_create_error;

int fail(sw2d_handle* h, int code, const std::string& msg)
{
    if (h) h->err = msg;
    else g_create_error = msg;
    return code;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return fail(h, SW2D_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

template <class T>
int dev_upload(sw2d_handle* h, const std::vector<T>& v, T** out)
{
    size_t bytes = std::max<size_t>(1, v.size()) * sizeof(T);
    void* p = nullptr;
    CK(cudaMalloc(&p, bytes));
    h->allocs.push_back(p);
    if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, h->stream));
    *out = static_cast<T*>(p);
    return SW2D_OK;
}

template <class T>
int dev_alloc(sw2d_handle* h, size_t n, T** out)
{
    void* p = nullptr;
    CK(cudaMalloc(&p, std::max<size_t>(1, n) * sizeof(T)));
    h->allocs.push_back(p);
    CK(cudaMemsetAsync(p, 0, std::max<size_t>(1, n) * sizeof(T), h->stream));
    *out = static_cast<T*>(p);
    return SW2D_OK;
}

int status_to_code(sw2d_handle* h, unsigned st)
{
    if (st & kStatusNanFlux) return fail(h, SW2D_E_NAN_FLUX, "SP - mass flux is not a number on an internal interface");
    if (st & kStatusHllcConfig) return fail(h, SW2D_E_HLLC_CONFIG, "impossible flow configuration in the HLLC solver");
    if (st & kStatusNegDepth) return fail(h, SW2D_E_NEG_DEPTH, "SP - negative water depth");
    if (st & kStatusBcType) return fail(h, SW2D_E_BC_TYPE, "boundary condition type not handled");
    if (st & kStatusBcFr) return fail(h, SW2D_E_BC_FR, "incorrect value for 'fr'-type boundary condition");
    return SW2D_OK;
}

int launch_step(sw2d_handle* h)
{
    DevMesh& m = h->m;
    if (h->p.scheme == SW2D_SCHEME_MUSCL_EVR) k_slopes<<<grid_for(m.nc), kBlock, 0, h->stream>>>(m);
    k_edges<<<grid_for((long long)m.ni + m.nb), kBlock, 0, h->stream>>>(m);
    k_cfl<<<grid_for(m.nc), kBlock, 0, h->stream>>>(m);
    k_update<<<grid_for(m.nc), kBlock, 0, h->stream>>>(m);
    return SW2D_OK;
}

int ensure_graph(sw2d_handle* h, int steps)
{
    if (h->graph && h->graph_steps == steps) return SW2D_OK;
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < steps; i++) launch_step(h);
    CK(cudaStreamEndCapture(h->stream, &g));
    CK(cudaGraphInstantiate(&h->graph, g, 0));
    cudaGraphDestroy(g);
    h->graph_steps = steps;
    return SW2D_OK;
}

int check_mesh(const sw2d_mesh* m)
{
    if (!m || m->cell_nb <= 0 || m->edge_int_nb < 0 || m->edge_bnd_nb < 0) return SW2D_E_ARG;
    if (m->cell_nb >= (1LL << 30) || m->edge_int_nb >= (1LL << 29) || m->edge_bnd_nb >= (1LL << 30)) return SW2D_E_ARG;
    if (!m->cell_area || !m->cell_x || !m->cell_y || !m->cell_z_b) return SW2D_E_ARG;
    if (m->edge_int_nb && (!m->edge_int_cells || !m->edge_int_length || !m->edge_int_nx || !m->edge_int_ny ||
                           !m->edge_int_mx || !m->edge_int_my))
        return SW2D_E_ARG;
    if (m->edge_bnd_nb && (!m->edge_bnd_cell || !m->edge_bnd_length || !m->edge_bnd_nx || !m->edge_bnd_ny ||
                           !m->edge_bnd_bc))
        return SW2D_E_ARG;
    for (int64_t e = 0; e < 2 * m->edge_int_nb; e++)
        if (m->edge_int_cells[e] < 0 || m->edge_int_cells[e] >= m->cell_nb) return SW2D_E_ARG;
    for (int64_t e = 0; e < m->edge_int_nb; e++)
        if (m->edge_int_cells[2 * e] == m->edge_int_cells[2 * e + 1]) return SW2D_E_ARG;
    for (int64_t e = 0; e < m->edge_bnd_nb; e++)
        if (m->edge_bnd_cell[e] < 0 || m->edge_bnd_cell[e] >= m->cell_nb) return SW2D_E_ARG;
    return SW2D_OK;
}

}  // namespace

// ------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------
extern "C" {

int sw2d_abi_version(void) { return SW2D_ABI_VERSION; }

int sw2d_create(const sw2d_mesh* mesh, const sw2d_params* params, const sw2d_cell_fields* fields,
                const sw2d_bc_table* bc, const double* h0, const double* q0, const double* r0, int device,
                sw2d_handle** out)
{
    sw2d_handle* h = nullptr;
    if (!out) return fail(h, SW2D_E_ARG, "out is NULL");
    *out = nullptr;
    if (check_mesh(mesh) != SW2D_OK) return fail(h, SW2D_E_ARG, "invalid mesh tables");
    if (!params || !fields || !fields->phi || !fields->boussinesq || !bc || !h0 || !q0 || !r0)
        return fail(h, SW2D_E_ARG, "missing parameters, porosity, Boussinesq map, boundary table or state");
    if (params->variant != SW2D_VARIANT_NATIVE)
        return fail(h, SW2D_E_UNSUPPORTED, "only the native SP variant is implemented");
    if (params->scheme != SW2D_SCHEME_GODUNOV && params->scheme != SW2D_SCHEME_MUSCL_EVR)
        return fail(h, SW2D_E_ARG, "numerical scheme not implemented");
    if (params->topo != SW2D_TOPO_DISCONTINUOUS && params->topo != SW2D_TOPO_BLENDING)
        return fail(h, SW2D_E_ARG, "'topo_discretization' value not recognised");
    if (params->friction < 0 || params->friction > 3) return fail(h, SW2D_E_ARG, "friction model unknown");
    if (params->friction != SW2D_FRICTION_NONE && (!fields->friction_1 || !fields->friction_2 || !fields->friction_alpha))
        return fail(h, SW2D_E_ARG, "friction map missing");
    if (params->singular_head_loss &&
        (!fields->hl_h_sing || !fields->hl_coeff_1 || !fields->hl_coeff_2 || !fields->hl_alpha))
        return fail(h, SW2D_E_ARG, "singular head loss map missing");
    if (bc->bc_nb < 0 || (mesh->edge_bnd_nb > 0 && bc->bc_nb == 0)) return fail(h, SW2D_E_ARG, "boundary table empty");
    for (int k = 0; k < bc->bc_nb; k++) {
        if (bc->offset[k + 1] - bc->offset[k] < 1) return fail(h, SW2D_E_ARG, "boundary series without records");
    }
    for (int64_t e = 0; e < mesh->edge_bnd_nb; e++)
        if (mesh->edge_bnd_bc[e] < 0 || mesh->edge_bnd_bc[e] >= bc->bc_nb)
            return fail(h, SW2D_E_ARG, "boundary edge refers to a missing boundary series");
    // swSp::checkParameterConsistency (swSp.cpp:33-335), the checks on this path
    for (int64_t c = 0; c < mesh->cell_nb; c++) {
        if (!(fields->boussinesq[c] >= 1.0)) return fail(h, SW2D_E_ARG, "boussinesq coeff. should be >= 1");
        if ((fields->phi[c] < 0.0) || (fields->phi[c] > 1.0)) return fail(h, SW2D_E_ARG, "porosity should belong to [0,1]");
    }

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0)
        return fail(h, SW2D_E_NO_DEVICE, "no usable CUDA device");

    h = new sw2d_handle();
    h->device = device;
    h->p = *params;
    h->nc = mesh->cell_nb;
    h->ni = mesh->edge_int_nb;
    h->nb = mesh->edge_bnd_nb;
    const int64_t nc = h->nc, ni = h->ni, nb = h->nb;
    auto bail = [&](int code) {
        g_create_error = h->err;
        sw2d_destroy(h);
        return code;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bail(fail(h, SW2D_E_NO_DEVICE, "cudaSetDevice failed"));
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(h, SW2D_E_CUDA, "cudaStreamCreate failed"));

    // ---- cell renumbering along a Hilbert curve of the centroids
    double xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300;
    for (int64_t c = 0; c < nc; c++) {
        xmin = std::min(xmin, mesh->cell_x[c]);
        xmax = std::max(xmax, mesh->cell_x[c]);
        ymin = std::min(ymin, mesh->cell_y[c]);
        ymax = std::max(ymax, mesh->cell_y[c]);
    }
    double span = std::max(xmax - xmin, ymax - ymin);
    if (!(span > 0)) span = 1.0;
    std::vector<uint64_t> key(nc);
    for (int64_t c = 0; c < nc; c++) {
        uint32_t ix = (uint32_t)std::min(65535.0, std::max(0.0, (mesh->cell_x[c] - xmin) / span * 65535.0));
        uint32_t iy = (uint32_t)std::min(65535.0, std::max(0.0, (mesh->cell_y[c] - ymin) / span * 65535.0));
        key[c] = hilbert_d(ix, iy);
    }
    h->cell_perm.resize(nc);
    std::iota(h->cell_perm.begin(), h->cell_perm.end(), 0);
    std::stable_sort(h->cell_perm.begin(), h->cell_perm.end(), [&](int a, int b) { return key[a] < key[b]; });
    std::vector<int> inv(nc);
    for (int64_t i = 0; i < nc; i++) inv[h->cell_perm[i]] = (int)i;

    // ---- internal edges ordered by their lower new cell, boundary edges by their new cell
    h->int_perm.resize(ni);
    std::iota(h->int_perm.begin(), h->int_perm.end(), 0);
    std::vector<uint64_t> ekey(ni);
    for (int64_t e = 0; e < ni; e++) {
        uint64_t a = inv[mesh->edge_int_cells[2 * e]], b = inv[mesh->edge_int_cells[2 * e + 1]];
        ekey[e] = (std::min(a, b) << 32) | std::max(a, b);
    }
    std::stable_sort(h->int_perm.begin(), h->int_perm.end(), [&](int a, int b) { return ekey[a] < ekey[b]; });
    std::vector<int> inv_int(ni);
    for (int64_t i = 0; i < ni; i++) inv_int[h->int_perm[i]] = (int)i;
    h->bnd_perm.resize(nb);
    std::iota(h->bnd_perm.begin(), h->bnd_perm.end(), 0);
    std::stable_sort(h->bnd_perm.begin(), h->bnd_perm.end(),
                     [&](int a, int b) { return inv[mesh->edge_bnd_cell[a]] < inv[mesh->edge_bnd_cell[b]]; });
    std::vector<int> inv_bnd(nb);
    for (int64_t i = 0; i < nb; i++) inv_bnd[h->bnd_perm[i]] = (int)i;

    // ---- per-cell lists in the reference's order (swParent::setMeshTables, swParent.cpp:469-486):
    // walking edges by increasing original index appends them in that order.
    std::vector<int> cb_off(nc + 1, 0), ci_off(nc + 1, 0);
    for (int64_t e = 0; e < nb; e++) cb_off[inv[mesh->edge_bnd_cell[e]] + 1]++;
    for (int64_t e = 0; e < ni; e++) {
        ci_off[inv[mesh->edge_int_cells[2 * e]] + 1]++;
        ci_off[inv[mesh->edge_int_cells[2 * e + 1]] + 1]++;
    }
    for (int64_t c = 0; c < nc; c++) {
        cb_off[c + 1] += cb_off[c];
        ci_off[c + 1] += ci_off[c];
    }
    std::vector<int> cb_idx(nb), ci_ent(2 * ni), ci_nbr(2 * ni);
    {
        std::vector<int> fb(cb_off.begin(), cb_off.end() - 1), fi(ci_off.begin(), ci_off.end() - 1);
        for (int64_t e = 0; e < nb; e++) cb_idx[fb[inv[mesh->edge_bnd_cell[e]]]++] = inv_bnd[e];
        for (int64_t e = 0; e < ni; e++) {
            int a = inv[mesh->edge_int_cells[2 * e]], b = inv[mesh->edge_int_cells[2 * e + 1]];
            int ne = inv_int[e];
            ci_ent[fi[a]] = ne * 2 + 0;
            ci_nbr[fi[a]++] = b;
            ci_ent[fi[b]] = ne * 2 + 1;
            ci_nbr[fi[b]++] = a;
        }
    }

    // ---- gather host tables into the new numbering
    auto cellv = [&](const double* src, double fill) {
        std::vector<double> v(nc);
        for (int64_t i = 0; i < nc; i++) v[i] = src ? src[h->cell_perm[i]] : fill;
        return v;
    };
    auto intv = [&](const double* src) {
        std::vector<double> v(ni);
        for (int64_t i = 0; i < ni; i++) v[i] = src[h->int_perm[i]];
        return v;
    };
    auto bndv = [&](const double* src) {
        std::vector<double> v(nb);
        for (int64_t i = 0; i < nb; i++) v[i] = src[h->bnd_perm[i]];
        return v;
    };
    std::vector<int2> lr(ni);
    for (int64_t i = 0; i < ni; i++) {
        int oe = h->int_perm[i];
        lr[i] = make_int2(inv[mesh->edge_int_cells[2 * oe]], inv[mesh->edge_int_cells[2 * oe + 1]]);
    }
    std::vector<int> bcell(nb), bbc(nb);
    for (int64_t i = 0; i < nb; i++) {
        bcell[i] = inv[mesh->edge_bnd_cell[h->bnd_perm[i]]];
        bbc[i] = mesh->edge_bnd_bc[h->bnd_perm[i]];
    }
    // friction and head-loss angles: degrees -> radians and cos/sin on the host, with the
    // expressions of swSp::setFrictionParameters (swSp.cpp:1063-1068) and
    // sourceSingularHeadLoss (swSpSourceFriction.cpp:185-187)
    std::vector<double> fcos, fsin, hcos, hsin;
    if (params->friction != SW2D_FRICTION_NONE) {
        fcos.resize(nc);
        fsin.resize(nc);
        for (int64_t i = 0; i < nc; i++) {
            double a = fields->friction_alpha[h->cell_perm[i]] * atan(1.0) / 45.0;
            fcos[i] = cos(a);
            fsin[i] = sin(a);
        }
    }
    if (params->singular_head_loss) {
        hcos.resize(nc);
        hsin.resize(nc);
        for (int64_t i = 0; i < nc; i++) {
            double a = fields->hl_alpha[h->cell_perm[i]] * atan(1.0) / 45.0;
            hcos[i] = cos(a);
            hsin[i] = sin(a);
        }
    }

    DevMesh& m = h->m;
    m.nc = (int)nc;
    m.ni = (int)ni;
    m.nb = (int)nb;
    double* tmp = nullptr;
    int st = SW2D_OK;
#define UP(vec, dst)                                        \
    do {                                                    \
        st = dev_upload(h, vec, &tmp);                      \
        if (st) return bail(st);                            \
        dst = tmp;                                          \
    } while (0)
    double *dh, *dq, *dr;
    UP(cellv(h0, 0), dh);
    UP(cellv(q0, 0), dq);
    UP(cellv(r0, 0), dr);
    m.h = dh;
    m.q = dq;
    m.r = dr;
    UP(cellv(mesh->cell_z_b, 0), m.zb);
    UP(cellv(mesh->cell_area, 0), m.area);
    UP(cellv(mesh->cell_x, 0), m.cx);
    UP(cellv(mesh->cell_y, 0), m.cy);
    UP(cellv(fields->phi, 1), m.phi);
    UP(cellv(fields->boussinesq, 1), m.bous);
    if (params->friction != SW2D_FRICTION_NONE) {
        UP(cellv(fields->friction_1, 0), m.fk1);
        UP(cellv(fields->friction_2, 0), m.fk2);
        UP(fcos, m.fcos);
        UP(fsin, m.fsin);
    }
    if (params->singular_head_loss) {
        UP(cellv(fields->hl_h_sing, 0), m.hs);
        UP(cellv(fields->hl_coeff_1, 0), m.hk1);
        UP(cellv(fields->hl_coeff_2, 0), m.hk2);
        UP(hcos, m.hcos);
        UP(hsin, m.hsin);
    }
    UP(intv(mesh->edge_int_length), m.len);
    UP(intv(mesh->edge_int_nx), m.nx);
    UP(intv(mesh->edge_int_ny), m.ny);
    UP(intv(mesh->edge_int_mx), m.mx);
    UP(intv(mesh->edge_int_my), m.my);
    UP(bndv(mesh->edge_bnd_length), m.blen);
    UP(bndv(mesh->edge_bnd_nx), m.bnx);
    UP(bndv(mesh->edge_bnd_ny), m.bny);
#undef UP
    {
        int* ip = nullptr;
        int2* lp = nullptr;
        if ((st = dev_upload(h, lr, &lp))) return bail(st);
        m.lr = lp;
        if ((st = dev_upload(h, bcell, &ip))) return bail(st);
        m.bcell = ip;
        if ((st = dev_upload(h, bbc, &ip))) return bail(st);
        m.bbc = ip;
        if ((st = dev_upload(h, cb_off, &ip))) return bail(st);
        m.cb_off = ip;
        if ((st = dev_upload(h, cb_idx, &ip))) return bail(st);
        m.cb_idx = ip;
        if ((st = dev_upload(h, ci_off, &ip))) return bail(st);
        m.ci_off = ip;
        if ((st = dev_upload(h, ci_ent, &ip))) return bail(st);
        m.ci_ent = ip;
        if ((st = dev_upload(h, ci_nbr, &ip))) return bail(st);
        m.ci_nbr = ip;
        if ((st = dev_upload(h, h->cell_perm, &h->d_cell_perm))) return bail(st);
        if ((st = dev_upload(h, h->int_perm, &h->d_int_perm))) return bail(st);
        if ((st = dev_upload(h, h->bnd_perm, &h->d_bnd_perm))) return bail(st);
        std::vector<int> bct(bc->type, bc->type + bc->bc_nb);
        std::vector<long long> bco(bc->offset, bc->offset + bc->bc_nb + 1);
        int64_t nrec = bc->offset[bc->bc_nb];
        std::vector<double> bt(bc->times, bc->times + nrec), bv(bc->values, bc->values + nrec);
        if ((st = dev_upload(h, bct, &ip))) return bail(st);
        m.bctype = ip;
        long long* lp2 = nullptr;
        if ((st = dev_upload(h, bco, &lp2))) return bail(st);
        m.bcoff = lp2;
        if ((st = dev_upload(h, bt, &tmp))) return bail(st);
        m.bctimes = tmp;
        if ((st = dev_upload(h, bv, &tmp))) return bail(st);
        m.bcvals = tmp;
    }
    double *cl, *cr, *cbf;
    if ((st = dev_alloc(h, ni, &cl)) || (st = dev_alloc(h, ni, &cr)) || (st = dev_alloc(h, nb, &cbf))) return bail(st);
    m.coefL = cl;
    m.coefR = cr;
    m.bcoef = cbf;
    // persistent flux arrays start at zero, like the reference's resized member vectors
    if ((st = dev_alloc(h, ni, &m.F1)) || (st = dev_alloc(h, ni, &m.F2)) || (st = dev_alloc(h, ni, &m.F3)) ||
        (st = dev_alloc(h, ni, &m.S2L)) || (st = dev_alloc(h, ni, &m.S2R)) || (st = dev_alloc(h, ni, &m.lmax)) ||
        (st = dev_alloc(h, nb, &m.F1b)) || (st = dev_alloc(h, nb, &m.F2b)) || (st = dev_alloc(h, nb, &m.F3b)) ||
        (st = dev_alloc(h, nb, &m.lmaxb)) || (st = dev_alloc(h, nc, &m.sx)) || (st = dev_alloc(h, nc, &m.sy)) ||
        (st = dev_alloc(h, grid_for(nc) + 1, &m.part)) || (st = dev_alloc(h, 3 * nc, &h->stage)))
        return bail(st);
    m.h_min = params->h_min;
    m.phi_min = params->phi_min;
    m.cfl_max = params->cfl_max;
    m.dt_max = params->dt_max;
    m.dt_map = params->dt_map;
    m.v_max = params->v_max;
    m.fr_max = params->fr_max;
    m.scheme = params->scheme;
    m.topo = params->topo;
    m.friction = params->friction;
    m.head_loss = params->singular_head_loss ? 1 : 0;
    m.neg_detect = params->negative_depth_detection ? 1 : 0;
    if (cudaMalloc(&h->ctrl, sizeof(Ctrl)) != cudaSuccess) return bail(fail(h, SW2D_E_CUDA, "cudaMalloc ctrl"));
    h->allocs.push_back(h->ctrl);
    if (cudaMallocHost(&h->ctrl_host, sizeof(Ctrl)) != cudaSuccess) return bail(fail(h, SW2D_E_CUDA, "cudaMallocHost"));
    m.ctrl = h->ctrl;
    Ctrl c0{};
    c0.t = params->t_0;
    c0.dt = 0.0;  // swSp.h:155
    c0.t_max = params->t_max;
    *h->ctrl_host = c0;
    if (cudaMemcpyAsync(h->ctrl, h->ctrl_host, sizeof(Ctrl), cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
        return bail(fail(h, SW2D_E_CUDA, "ctrl upload"));
    k_edge_coefficients<<<grid_for(ni + nb), kBlock, 0, h->stream>>>(m, cl, cr, cbf);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess)
        return bail(fail(h, SW2D_E_CUDA, "initialisation kernels failed"));
    *out = h;
    return SW2D_OK;
}

int sw2d_step_n(sw2d_handle* h, int64_t n_steps, int64_t* steps_done)
{
    if (!h || n_steps < 0) return fail(h, SW2D_E_ARG, "invalid arguments");
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const long long before = h->ctrl_host->steps;
    const int chunk = 32;
    int64_t full = n_steps / chunk, rem = n_steps % chunk;
    if (full > 0) {
        int st = ensure_graph(h, chunk);
        if (st) return st;
        for (int64_t i = 0; i < full; i++) CK(cudaGraphLaunch(h->graph, h->stream));
    }
    for (int64_t i = 0; i < rem; i++) launch_step(h);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (steps_done) *steps_done = h->ctrl_host->steps - before;
    return status_to_code(h, h->ctrl_host->status);
}

int sw2d_execute(sw2d_handle* h, int64_t* steps_done)
{
    if (!h) return fail(h, SW2D_E_ARG, "invalid handle");
    int64_t total = 0;
    for (;;) {
        int64_t k = 0;
        int st = sw2d_step_n(h, 1024, &k);
        total += k;
        if (st) {
            if (steps_done) *steps_done = total;
            return st;
        }
        if (k < 1024) break;
    }
    if (steps_done) *steps_done = total;
    return SW2D_OK;
}

int sw2d_phase_times(sw2d_handle* h, int64_t n_steps, double* ms, int capacity)
{
    if (!h || !ms || n_steps <= 0) return fail(h, SW2D_E_ARG, "invalid arguments");
    const int nph = 4;
    if (capacity < nph) return fail(h, SW2D_E_ARG, "capacity < 4");
    CK(cudaSetDevice(h->device));
    cudaEvent_t ev[nph + 1];
    for (int i = 0; i <= nph; i++) CK(cudaEventCreate(&ev[i]));
    double acc[nph] = {0, 0, 0, 0};
    DevMesh& m = h->m;
    for (int64_t s = 0; s < n_steps; s++) {
        cudaEventRecord(ev[0], h->stream);
        if (h->p.scheme == SW2D_SCHEME_MUSCL_EVR) k_slopes<<<grid_for(m.nc), kBlock, 0, h->stream>>>(m);
        cudaEventRecord(ev[1], h->stream);
        k_edges<<<grid_for((long long)m.ni + m.nb), kBlock, 0, h->stream>>>(m);
        cudaEventRecord(ev[2], h->stream);
        k_cfl<<<grid_for(m.nc), kBlock, 0, h->stream>>>(m);
        cudaEventRecord(ev[3], h->stream);
        k_update<<<grid_for(m.nc), kBlock, 0, h->stream>>>(m);
        cudaEventRecord(ev[4], h->stream);
        CK(cudaEventSynchronize(ev[4]));
        for (int i = 0; i < nph; i++) {
            float t = 0.f;
            cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
            acc[i] += t;
        }
    }
    for (int i = 0; i <= nph; i++) cudaEventDestroy(ev[i]);
    CK(cudaGetLastError());
    for (int i = 0; i < nph; i++) ms[i] = acc[i] / (double)n_steps;
    CK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    int st = status_to_code(h, h->ctrl_host->status);
    return st ? st : nph;
}

const char* sw2d_phase_name(int i)
{
    static const char* names[] = {"k_slopes", "k_edges", "k_cfl", "k_update"};
    return (i >= 0 && i < 4) ? names[i] : "";
}

int sw2d_get_state_device(sw2d_handle* h, double* dh, double* dq, double* dr)
{
    if (!h || !dh || !dq || !dr) return fail(h, SW2D_E_ARG, "invalid arguments");
    CK(cudaSetDevice(h->device));
    k_scatter3<<<grid_for(h->nc), kBlock, 0, h->stream>>>(h->m.h, h->m.q, h->m.r, h->d_cell_perm, dh, dq, dr, (int)h->nc);
    CK(cudaGetLastError());
    return SW2D_OK;
}

int sw2d_set_state_device(sw2d_handle* h, const double* dh, const double* dq, const double* dr)
{
    if (!h || !dh || !dq || !dr) return fail(h, SW2D_E_ARG, "invalid arguments");
    CK(cudaSetDevice(h->device));
    k_gather3<<<grid_for(h->nc), kBlock, 0, h->stream>>>(dh, dq, dr, h->d_cell_perm, h->m.h, h->m.q, h->m.r, (int)h->nc);
    CK(cudaGetLastError());
    return SW2D_OK;
}

int sw2d_get_state(sw2d_handle* h, double* wd, double* qx, double* qy)
{
    if (!h || !wd || !qx || !qy) return fail(h, SW2D_E_ARG, "invalid arguments");
    int st = sw2d_get_state_device(h, h->stage, h->stage + h->nc, h->stage + 2 * h->nc);
    if (st) return st;
    size_t bytes = h->nc * sizeof(double);
    CK(cudaMemcpyAsync(wd, h->stage, bytes, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(qx, h->stage + h->nc, bytes, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(qy, h->stage + 2 * h->nc, bytes, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return SW2D_OK;
}

int sw2d_set_state(sw2d_handle* h, const double* wd, const double* qx, const double* qy)
{
    if (!h || !wd || !qx || !qy) return fail(h, SW2D_E_ARG, "invalid arguments");
    CK(cudaSetDevice(h->device));
    size_t bytes = h->nc * sizeof(double);
    CK(cudaMemcpyAsync(h->stage, wd, bytes, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->stage + h->nc, qx, bytes, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->stage + 2 * h->nc, qy, bytes, cudaMemcpyHostToDevice, h->stream));
    int st = sw2d_set_state_device(h, h->stage, h->stage + h->nc, h->stage + 2 * h->nc);
    if (st) return st;
    CK(cudaStreamSynchronize(h->stream));
    return SW2D_OK;
}

int sw2d_get_time(sw2d_handle* h, double* t, double* dt)
{
    if (!h) return fail(h, SW2D_E_ARG, "invalid handle");
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (t) *t = h->ctrl_host->t;
    if (dt) *dt = h->ctrl_host->dt;
    return SW2D_OK;
}

int sw2d_set_time(sw2d_handle* h, double t, double dt)
{
    if (!h) return fail(h, SW2D_E_ARG, "invalid handle");
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->ctrl_host->t = t;
    h->ctrl_host->dt = dt;
    CK(cudaMemcpyAsync(h->ctrl, h->ctrl_host, sizeof(Ctrl), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return SW2D_OK;
}

int64_t sw2d_get_array(sw2d_handle* h, const char* name, double* out, int64_t capacity)
{
    if (!h || !name || !out) return fail(h, SW2D_E_ARG, "invalid arguments");
    struct Entry {
        const char* n;
        const double* p;
        int64_t len;
        const int* perm;
    } tab[] = {
        {"F1_int", h->m.F1, h->ni, h->d_int_perm},        {"F2_int", h->m.F2, h->ni, h->d_int_perm},
        {"F3_int", h->m.F3, h->ni, h->d_int_perm},        {"s2L_int", h->m.S2L, h->ni, h->d_int_perm},
        {"s2R_int", h->m.S2R, h->ni, h->d_int_perm},      {"lambda_max_int", h->m.lmax, h->ni, h->d_int_perm},
        {"F1_bnd", h->m.F1b, h->nb, h->d_bnd_perm},       {"F2_bnd", h->m.F2b, h->nb, h->d_bnd_perm},
        {"F3_bnd", h->m.F3b, h->nb, h->d_bnd_perm},       {"lambda_max_bnd", h->m.lmaxb, h->nb, h->d_bnd_perm},
        {"slope_x", h->m.sx, h->nc, h->d_cell_perm},      {"slope_y", h->m.sy, h->nc, h->d_cell_perm},
    };
    for (const Entry& e : tab) {
        if (std::strcmp(e.n, name) != 0) continue;
        if (capacity < e.len) return fail(h, SW2D_E_ARG, "output buffer too small");
        CK(cudaSetDevice(h->device));
        double* tmp = nullptr;
        CK(cudaMalloc(&tmp, std::max<int64_t>(1, e.len) * sizeof(double)));
        k_scatter1<<<grid_for(e.len), kBlock, 0, h->stream>>>(e.p, e.perm, tmp, (int)e.len);
        cudaError_t ce = cudaMemcpyAsync(out, tmp, e.len * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
        cudaStreamSynchronize(h->stream);
        cudaFree(tmp);
        if (ce != cudaSuccess) return fail(h, SW2D_E_CUDA, cudaGetErrorString(ce));
        return e.len;
    }
    if (std::strcmp(name, "s2R_bnd") == 0) {
        if (capacity < h->nb) return fail(h, SW2D_E_ARG, "output buffer too small");
        for (int64_t i = 0; i < h->nb; i++) out[i] = 0.0;
        return h->nb;
    }
    return fail(h, SW2D_E_ARG, std::string("unknown array ") + name);
}

int sw2d_get_cell_permutation(sw2d_handle* h, int64_t* perm)
{
    if (!h || !perm) return fail(h, SW2D_E_ARG, "invalid arguments");
    for (int64_t i = 0; i < h->nc; i++) perm[i] = h->cell_perm[i];
    return SW2D_OK;
}

void* sw2d_get_stream(sw2d_handle* h) { return h ? (void*)h->stream : nullptr; }

int sw2d_kernels_per_step(sw2d_handle* h)
{
    if (!h) return 0;
    return h->p.scheme == SW2D_SCHEME_MUSCL_EVR ? 4 : 3;
}

int sw2d_destroy(sw2d_handle* h)
{
    if (!h) return SW2D_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    for (void* p : h->allocs) cudaFree(p);
    if (h->ctrl_host) cudaFreeHost(h->ctrl_host);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return SW2D_OK;
}

const char* sw2d_last_error(sw2d_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

}  // extern "C"
