// sw2d_sp.cu — SW2D single-porosity explicit step on the B200 (sm_100a), FP64, and the C ABI of
// include/sw2d_b200.h.
//
// One time step (the body of swSp::execute's loop, src/sw2dSolver/models/sp/swSp.cpp:522-589)
// is four kernels, all predicated on device state so that a CUDA graph of many steps runs
// without the host:
//
//   k_slopes   per cell   limited free-surface slopes (MUSCL-EVR only)      swSpHypMusclEvr.cpp:11-115
//   k_edges    per edge   Riemann states, max wave speed, HLLC / boundary    swSpHypGodunov.cpp, swSpHypMusclEvr.cpp:119-277,
//                         fluxes, per-side CFL contributions                 swSpHyp.cpp:13-135,276-402,664-998
//   k_cfl      per cell   swept length, CFL dt, warp -> block -> grid min,   swSpHyp.cpp:430-512
//                         dt_map snap and t_max clip on the device
//   k_update   per cell   flux balance (CSR gather in the reference's per-   swSpHyp.cpp:214-273,184-209,
//                         cell order), round-off flush, negative-depth clamp, swSpSourceFriction.cpp:11-219,
//                         friction, singular head loss, velocity cap, t += dt swSp.cpp:447-479
//
// Data layout (all in HBM, internal numbering): the state of a cell is one 32-byte record
// {h, q, r, z = h + z_b} so that a neighbour gather touches one sector; cell statics
// {z_b, boussinesq, phi, area}, centroids {x, y} and slopes {sx, sy} are 32/16-byte records;
// edges keep {L, R}, normals {nx, ny}, midpoints {mx, my} and the edge-factor coefficients
// {w/(A_L phi_L), w/(A_R phi_R)}.
//
// Balance slots.  The reference adds each edge's contribution to a cell as
//   h += (factor * F1) * dt,  q += (f2F2*F2 + f2S2*S2 + f2F3*F3) * dt,  r += (...) * dt
// (swSpHyp.cpp:221-263): the products before "* dt" do not depend on dt.  k_edges therefore
// writes, for every (cell, edge) pair, the three dt-free terms {a, b, c} into a per-cell slot
// range laid out in the reference's summation order (boundary edges, then internal edges, by
// increasing original index), plus the edge's CFL contribution.  k_cfl and k_update then read
// their cell's slots contiguously, without any gather.  The slots persist between steps: the
// reference keeps the previous fluxes of an edge whose two sides are dry (swSpHyp.cpp:339), and
// since the factors are static, keeping the previous {a, b, c} is the same thing.
//
// Cells are renumbered along a Hilbert curve and internal edges by their first cell, for
// locality; every per-cell sum still runs in the reference's order (boundary edges, then
// internal edges, by increasing ORIGINAL index), so the renumbering changes no bit.  No
// floating-point atomics are used anywhere.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <mutex>
#include <string>
#include <vector>

#include "sp_phases.cuh"
#include "sw2d_internal.cuh"

using namespace sw2d;

namespace {


// k_slopes: the limited slopes of one cell per thread (slopes_cell, sp_phases.cuh)
template <int kB, int kMinB>
__global__ void __launch_bounds__(kB, kMinB) k_slopes(DevMesh m)
{
    if (!step_active(m.ctrl)) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    slopes_cell<LdNc>(m, c);
}

// k_edges: one thread per internal edge, then one per boundary edge (edge_internal and
// edge_boundary, sp_phases.cuh)
template <int kScheme, bool kBlending, int kModel, int kB, int kMinB>
__global__ void __launch_bounds__(kB, kMinB) k_edges(DevMesh m)
{
    if (!step_active(m.ctrl)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned bad = 0;
    if (i < m.ni) bad = edge_internal<kScheme, kBlending, kModel, LdNc>(m, i);
    else if (i < m.ni + m.nb) bad = edge_boundary<kScheme, kModel, LdNc>(m, i - m.ni);
    if (bad) atomicOr(&m.ctrl->status, bad);
}

// ------------------------------------------------------------------------------------------
// k_cfl: swSp::hypComputeTimeStep (swSpHyp.cpp:430-512).  swept[c] sums the cell's slot
// contributions in the reference's order; dt = min over cells of cfl * area / max(swept,
// 1e-16), reduced warp -> block -> grid (last block done), then the dt_map snap (:496-504)
// and the t_max clip, all on the device.  A skipped contribution is stored as 0, and adding
// +0 to the (non-negative) sum changes no bit, so the sum is the reference's.
// ------------------------------------------------------------------------------------------

// k_cfl's grid: 8 blocks of kBlock threads per SM (a full SM), at most one block per kBlock cells
unsigned cfl_grid(sw2d_handle* h, int nc)
{
    if (!h->sms) {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device) != cudaSuccess || sms <= 0) sms = 148;
        h->sms = sms;
    }
    return std::min<unsigned>(grid_for(nc), (unsigned)(8 * h->sms));
}

// kDdpSnap: the DDP model's form of the snap, which truncates t and t + dt to integers before
// dividing by dt_map (swDdpHyp.cpp:588-600: `(int)t / dt_map`).
template <bool kDdpSnap>
__global__ void __launch_bounds__(kBlock) k_cfl(DevMesh m)
{
    Ctrl* ctrl = m.ctrl;
    if (!step_active(ctrl)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) ctrl->go = 0;
        return;
    }
    // grid-stride over the cells (the grid is a few blocks per SM, see cfl_grid), several cells
    // per thread in flight; the minimum does not depend on the order it is taken in
    double best = m.dt_max;
    const int stride = gridDim.x * blockDim.x;
#pragma unroll 4
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < m.nc; c += stride) {
        const double x = cfl_cell<LdNc>(m, c);
        if (x < best) best = x;
    }
    // warp then block minimum (NaN candidates never win: comparisons with NaN are false)
    for (int off = 16; off > 0; off >>= 1) best = min_keep(best, __shfl_down_sync(0xffffffffu, best, off));
    __shared__ double wmin[kBlock / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
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
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) b2 = min_keep(b2, ((volatile double*)m.part)[i]);
    for (int off = 16; off > 0; off >>= 1) b2 = min_keep(b2, __shfl_down_sync(0xffffffffu, b2, off));
    if (lane == 0) wmin[wid] = b2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double dt = m.dt_max;
        for (int w = 0; w < kBlock / 32; w++)
            if (wmin[w] < dt) dt = wmin[w];
        dt_finalize<kDdpSnap>(m, ctrl, dt);
        ctrl->blocks_done = 0;
    }
}

// ------------------------------------------------------------------------------------------
// k_update: balance + sources for one cell, then t += dt (thread 0).
// ------------------------------------------------------------------------------------------
template <int kFriction, bool kHeadLoss, bool kStoreB, bool kDissip>
__global__ void __launch_bounds__(kBlock, 4) k_update(DevMesh m)
{
    Ctrl* ctrl = m.ctrl;
    if (!ctrl->go) return;
    const double dt = ctrl->dt;
    // with rev_update the blocks take the cells from the end: the flux kernel finishes on the last
    // tiles, whose slots and states are then still in L2
    const int blk = m.rev_update ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
    const int c = blk * blockDim.x + threadIdx.x;
    if (c == 0) {
        ctrl->t = ctrl->t + dt;  // swSp.cpp:592; no other thread of this kernel reads t
        ctrl->steps += 1;
    }
    if (c >= m.nc) return;
    update_cell<kFriction, kHeadLoss, kStoreB, kDissip, LdNc>(m, c, dt);
}

// swSp::computeEdgeFactors coefficient w / area / phi (swSp.cpp:364-368, 397-405)
__global__ void k_edge_coefficients(DevMesh m, double2* coef, double4* bgeo)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m.ni) {
        const int2 lr = m.lr[i];
        const double w = m.len[i];
        const double4 a = m.cst[lr.x], b = m.cst[lr.y];
        coef[i] = make_double2((a.z > m.phi_min) ? w / a.w / a.z : 0.0, (b.z > m.phi_min) ? w / b.w / b.z : 0.0);
    } else if (i < m.ni + m.nb) {
        const int e = i - m.ni;
        const double4 c = m.cst[m.bcell[e]];
        double4 g = bgeo[e];
        g.w = (c.z > m.phi_min) ? g.z / c.w / c.z : 0.0;
        bgeo[e] = g;
    }
}

// caller numbering <-> internal numbering
__global__ void k_gather_state(const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c,
                               const int* __restrict__ perm, const double4* __restrict__ cst, double4* st, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int p = perm[i];
        const double h = a[p];
        st[i] = make_double4(h, b[p], c[p], h + cst[i].x);
    }
}

__global__ void k_scatter_state(const double4* __restrict__ st, const int* __restrict__ perm, double* oa, double* ob,
                                double* oc, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int p = perm[i];
        const double4 s = st[i];
        oa[p] = s.x;
        ob[p] = s.y;
        oc[p] = s.z;
    }
}

// per-edge/per-cell arrays back to the caller's numbering: out[perm[i]] = src[i*stride + offset]
__global__ void k_scatter_strided(const double* __restrict__ src, int stride, int offset, const int* __restrict__ perm,
                                  double* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[perm[i]] = src[(size_t)i * stride + offset];
}

__global__ void k_eval_math(int fn, const double* __restrict__ x, double* y, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = x[i];
    y[i] = fn == 0 ? sw2d_exp(v) : fn == 1 ? sw2d_log(v) : fn == 2 ? exp(v) : fn == 3 ? log(v)
         : fn == 4 ? sw2d_cbrt(v) : cbrt(v);
}

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


namespace {

std::string g_create_error;

}  // namespace

namespace sw2d {

int fail(sw2d_handle* h, int code, const std::string& msg)
{
    if (h) h->err = msg;
    else g_create_error = msg;
    return code;
}

int status_to_code(sw2d_handle* h, unsigned st)
{
    if (st & kStatusNanFlux) return fail(h, SW2D_E_NAN_FLUX, "SP - mass flux is not a number on an internal interface");
    if (st & kStatusHllcConfig) return fail(h, SW2D_E_HLLC_CONFIG, "impossible flow configuration in the HLLC solver");
    if (st & kStatusNegDepth)
        return fail(h, SW2D_E_NEG_DEPTH, h->model == kModelDdp ? "DDP - negative theta" : "SP - negative water depth");
    if (st & kStatusBcType) return fail(h, SW2D_E_BC_TYPE, "boundary condition type not handled");
    if (st & kStatusBcFr) return fail(h, SW2D_E_BC_FR, "incorrect value for 'fr'-type boundary condition");
    if (st & kStatusPhiG) return fail(h, SW2D_E_PHIG, "specificForce : phiG is < small");
    if (st & kStatusTable)
        return fail(h, SW2D_E_DDP_TABLE, "DDP - NaN elevation or volume in a porosity-table lookup");
    if (st & kStatusUnsupported)
        return fail(h, SW2D_E_UNSUPPORTED, "cell with more neighbours than the adjoint's slope reverse handles");
    return SW2D_OK;
}

}  // namespace sw2d

namespace {

constexpr int kDefaultTileCells = 384;  // cells per tile of the fused step

// Launch variants {threads per block, minimum resident blocks per SM (register cap)} of the
// two heaviest kernels; sw2d_autotune times them on the live state and keeps the fastest.
struct Variant {
    int block, minb;
};
constexpr Variant kVariants[] = {{256, 3}, {256, 2}, {256, 4}, {128, 4}, {128, 8}, {512, 1}};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

template <int kScheme, bool kBlending, int kModel, int V>
void launch_edges_v(sw2d_handle* h, const DevMesh& m, unsigned n)
{
    constexpr int B = kVariants[V].block, M = kVariants[V].minb;
    k_edges<kScheme, kBlending, kModel, B, M><<<(n + B - 1) / B, B, 0, h->stream>>>(m);
}

template <int kScheme, bool kBlending, int kModel>
void launch_edges_s(sw2d_handle* h, const DevMesh& m, unsigned n, int v)
{
    switch (v) {
        case 1: launch_edges_v<kScheme, kBlending, kModel, 1>(h, m, n); break;
        case 2: launch_edges_v<kScheme, kBlending, kModel, 2>(h, m, n); break;
        case 3: launch_edges_v<kScheme, kBlending, kModel, 3>(h, m, n); break;
        case 4: launch_edges_v<kScheme, kBlending, kModel, 4>(h, m, n); break;
        case 5: launch_edges_v<kScheme, kBlending, kModel, 5>(h, m, n); break;
        default: launch_edges_v<kScheme, kBlending, kModel, 0>(h, m, n); break;
    }
}

template <int kModel>
void launch_edges_m(sw2d_handle* h, const DevMesh& m, int v)
{
    const unsigned n = (unsigned)(m.ni + m.nb);
    const bool bl = h->p.topo == SW2D_TOPO_BLENDING;
    if (h->p.scheme == SW2D_SCHEME_GODUNOV) {
        if (bl) launch_edges_s<SW2D_SCHEME_GODUNOV, true, kModel>(h, m, n, v);
        else launch_edges_s<SW2D_SCHEME_GODUNOV, false, kModel>(h, m, n, v);
    } else {
        if (bl) launch_edges_s<SW2D_SCHEME_MUSCL_EVR, true, kModel>(h, m, n, v);
        else launch_edges_s<SW2D_SCHEME_MUSCL_EVR, false, kModel>(h, m, n, v);
    }
}

void launch_edges(sw2d_handle* h, const DevMesh& m, int v)
{
    if (h->model == kModelDdp) launch_ddp_edges(h, m, v);
    else if (h->model == kModelDip) launch_edges_m<kModelDip>(h, m, v);
    else launch_edges_m<kModelSp>(h, m, v);
}

void launch_edges(sw2d_handle* h, int v) { launch_edges(h, h->m, v); }

template <int V>
void launch_slopes_v(sw2d_handle* h, const DevMesh& m)
{
    constexpr int B = kVariants[V].block, M = kVariants[V].minb;
    k_slopes<B, M><<<((unsigned)m.nc + B - 1) / B, B, 0, h->stream>>>(m);
}

void launch_slopes(sw2d_handle* h, const DevMesh& m, int v)
{
    switch (v) {
        case 1: launch_slopes_v<1>(h, m); break;
        case 2: launch_slopes_v<2>(h, m); break;
        case 3: launch_slopes_v<3>(h, m); break;
        case 4: launch_slopes_v<4>(h, m); break;
        case 5: launch_slopes_v<5>(h, m); break;
        default: launch_slopes_v<0>(h, m); break;
    }
}

void launch_slopes(sw2d_handle* h, int v) { launch_slopes(h, h->m, v); }

template <int kF, bool kStoreB, bool kDissip>
void launch_update_f(sw2d_handle* h, const DevMesh& m, unsigned g)
{
    if (h->p.singular_head_loss) k_update<kF, true, kStoreB, kDissip><<<g, kBlock, 0, h->stream>>>(m);
    else k_update<kF, false, kStoreB, kDissip><<<g, kBlock, 0, h->stream>>>(m);
}

template <bool kStoreB, bool kDissip>
void launch_update_d(sw2d_handle* h, const DevMesh& m)
{
    const unsigned g = grid_for(m.nc);
    switch (h->p.friction) {
        case SW2D_FRICTION_CHEZY: launch_update_f<SW2D_FRICTION_CHEZY, kStoreB, kDissip>(h, m, g); break;
        case SW2D_FRICTION_MANNING: launch_update_f<SW2D_FRICTION_MANNING, kStoreB, kDissip>(h, m, g); break;
        case SW2D_FRICTION_STRICKLER: launch_update_f<SW2D_FRICTION_STRICKLER, kStoreB, kDissip>(h, m, g); break;
        default: launch_update_f<SW2D_FRICTION_NONE, kStoreB, kDissip>(h, m, g); break;
    }
}

// the recorded post-balance state serves the adjoint, which covers the SP model only
template <bool kStoreB>
void launch_update_s(sw2d_handle* h, const DevMesh& m)
{
    // with a learned closure attached the update runs the network at the closure site (and the
    // plain closure where the features leave the training hull)
    if (!kStoreB && h->closure) closure_update(h, m);
    else if (!kStoreB && h->dissipation) launch_update_d<false, true>(h, m);
    else launch_update_d<kStoreB, false>(h, m);
}

// kernels of one step: the fused step's k_flux and k_update (with k_slopes first when the
// MUSCL-EVR slopes are not computed inside k_flux), or the four-kernel step
bool slopes_first(const sw2d_handle* h) { return h->p.scheme == SW2D_SCHEME_MUSCL_EVR && !h->tiles.slopes_in; }
int n_phases(const sw2d_handle* h) { return h->fused ? (slopes_first(h) ? 3 : 2) : 4; }

// phase i of one step on the handle's stream: fused step 0 flux, 1 update; four-kernel step (and
// DDP) 0 slopes, 1 edges, 2 cfl, 3 update
void launch_phase(sw2d_handle* h, int i)
{
    if (h->model == kModelDdp) {
        launch_ddp_phase(h, i);
        return;
    }
    DevMesh& m = h->m;
    if (h->fused) {
        if (slopes_first(h)) {
            if (i == 0) launch_slopes(h, h->slope_variant);
            else if (i == 1) launch_flux(h, m, h->flux_variant, false);
            else launch_update_s<false>(h, m);
            return;
        }
        if (i == 0) launch_flux(h, m, h->flux_variant, false);
        else launch_update_s<false>(h, m);
        return;
    }
    switch (i) {
        case 0:
            if (h->p.scheme == SW2D_SCHEME_MUSCL_EVR) launch_slopes(h, h->slope_variant);
            break;
        case 1: launch_edges(h, h->edge_variant); break;
        case 2: k_cfl<false><<<cfl_grid(h, m.nc), kBlock, 0, h->stream>>>(m); break;
        default: launch_update_s<false>(h, m); break;
    }
}

void launch_step(sw2d_handle* h)
{
    for (int i = 0; i < n_phases(h); i++) launch_phase(h, i);
    if (h->result) result_after_step(h);
}

// host-side set-up a step's launches need before they are captured in a graph
int prepare_step(sw2d_handle* h)
{
    if (h->fused) {
        const cudaError_t e = launch_flux(h, h->m, h->flux_variant, true);
        if (e != cudaSuccess) return fail(h, SW2D_E_CUDA, std::string("k_flux attributes: ") + cudaGetErrorString(e));
    }
    return SW2D_OK;
}

}  // namespace

namespace sw2d {

void launch_slopes_on(sw2d_handle* h, const DevMesh& m)
{
    if (h->p.scheme == SW2D_SCHEME_MUSCL_EVR) launch_slopes(h, m, h->slope_variant);
}

void launch_edges_on(sw2d_handle* h, const DevMesh& m) { launch_edges(h, m, h->edge_variant); }

void launch_cfl_on(sw2d_handle* h, const DevMesh& m) { k_cfl<false><<<cfl_grid(h, m.nc), kBlock, 0, h->stream>>>(m); }

void launch_cfl_ddp_on(sw2d_handle* h, const DevMesh& m) { k_cfl<true><<<cfl_grid(h, m.nc), kBlock, 0, h->stream>>>(m); }

void launch_step_on(sw2d_handle* h) { launch_step(h); }

void launch_update_on(sw2d_handle* h, const DevMesh& m, bool store_balance)
{
    if (store_balance) launch_update_s<true>(h, m);
    else launch_update_s<false>(h, m);
}

}  // namespace sw2d

namespace {

// steps per launch of the captured step graph (sw2d_step_n without a result file)
constexpr int kGraphSteps = 32;

int ensure_graph(sw2d_handle* h, int steps)
{
    if (h->graph && h->graph_steps == steps) return SW2D_OK;
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    const int rc = prepare_step(h);
    if (rc) return rc;
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

int create_model(const sw2d_mesh* mesh, const sw2d_params* params, const sw2d_cell_fields* fields,
                 const sw2d_dip_fields* dip, const sw2d_ddp_fields* ddp, const sw2d_bc_table* bc, const double* h0,
                 const double* q0, const double* r0, int device, sw2d_handle** out);

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
    return create_model(mesh, params, fields, nullptr, nullptr, bc, h0, q0, r0, device, out);
}

int sw2d_create_dip(const sw2d_mesh* mesh, const sw2d_params* params, const sw2d_cell_fields* fields,
                    const sw2d_dip_fields* dip, const sw2d_bc_table* bc, const double* h0, const double* q0,
                    const double* r0, int device, sw2d_handle** out)
{
    if (!dip) return fail(nullptr, SW2D_E_ARG, "DIP fields missing");
    return create_model(mesh, params, fields, dip, nullptr, bc, h0, q0, r0, device, out);
}

int sw2d_create_ddp(const sw2d_mesh* mesh, const sw2d_params* params, const sw2d_cell_fields* fields,
                    const sw2d_ddp_fields* ddp, const sw2d_bc_table* bc, const double* ic_level, const double* ic_x,
                    const double* ic_y, int device, sw2d_handle** out)
{
    if (!ddp) return fail(nullptr, SW2D_E_ARG, "DDP fields missing");
    return create_model(mesh, params, fields, nullptr, ddp, bc, ic_level, ic_x, ic_y, device, out);
}

int64_t sw2d_ddp_get_table(sw2d_handle* h, int which, int64_t record, double* z, double* phi, double* theta,
                           int64_t capacity)
{
    if (!h || capacity < 0) return fail(h, SW2D_E_ARG, "invalid arguments");
    return ddp_get_table(h, which, record, z, phi, theta, capacity);
}

}  // extern "C"

namespace {

// sw2d_create / sw2d_create_dip / sw2d_create_ddp: `dip` selects the DIP model, `ddp` the DDP
// model (h0, q0, r0 then hold its initial-condition columns)
int create_model(const sw2d_mesh* mesh, const sw2d_params* params, const sw2d_cell_fields* fields,
                 const sw2d_dip_fields* dip, const sw2d_ddp_fields* ddp, const sw2d_bc_table* bc, const double* h0,
                 const double* q0, const double* r0, int device, sw2d_handle** out)
{
    sw2d_handle* h = nullptr;
    if (!out) return fail(h, SW2D_E_ARG, "out is NULL");
    *out = nullptr;
    if (check_mesh(mesh) != SW2D_OK) return fail(h, SW2D_E_ARG, "invalid mesh tables");
    if (!params || !fields || (!ddp && !fields->phi) || !fields->boussinesq || !bc || !h0 || !q0 || !r0)
        return fail(h, SW2D_E_ARG, "missing parameters, porosity, Boussinesq map, boundary table or state");
    if (ddp) {
        // swDdp::hypComputeLRStates and hypComputeFluxes (swDdpHyp.cpp:434-458,496-516): Godunov
        // and the discontinuous topography only
        if (params->scheme != SW2D_SCHEME_GODUNOV)
            return fail(h, SW2D_E_UNSUPPORTED, "the DDP model runs the Godunov scheme only (swDdpHyp.cpp:506-510)");
        if (params->topo != SW2D_TOPO_DISCONTINUOUS)
            return fail(h, SW2D_E_UNSUPPORTED, "the DDP model runs the discontinuous topography only (swDdpHyp.cpp:454-458)");
        std::string why;
        int rc0 = ddp_check(mesh, ddp, why);
        if (rc0) return fail(h, rc0, why);
    }
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
        if (!ddp && ((fields->phi[c] < 0.0) || (fields->phi[c] > 1.0)))
            return fail(h, SW2D_E_ARG, "porosity should belong to [0,1]");
    }
    // swDip::checkParameterConsistency (dip/swDip.cpp:121-240): phiG in [0,1], not above phiW
    if (dip) {
        if ((mesh->edge_int_nb && !dip->phi_g_int) || (mesh->edge_bnd_nb && !dip->phi_g_bnd))
            return fail(h, SW2D_E_ARG, "DIP edge porosity map missing");
        if (dip->momentum_dissipation && (!dip->mu_1 || !dip->mu_2 || !dip->mu_alpha))
            return fail(h, SW2D_E_ARG, "momentum dissipation map missing");
        for (int64_t e = 0; e < mesh->edge_bnd_nb; e++) {
            const double g = dip->phi_g_bnd[e];
            if (g < 0.0 || g > 1.0 || g > fields->phi[mesh->edge_bnd_cell[e]])
                return fail(h, SW2D_E_ARG, "boundary edge porosity outside [0, cell porosity]");
        }
        for (int64_t e = 0; e < mesh->edge_int_nb; e++) {
            const double g = dip->phi_g_int[e];
            if (g < 0.0 || g > 1.0 || g > fields->phi[mesh->edge_int_cells[2 * e]] ||
                g > fields->phi[mesh->edge_int_cells[2 * e + 1]])
                return fail(h, SW2D_E_ARG, "internal edge porosity outside [0, cell porosity]");
        }
    }

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0)
        return fail(h, SW2D_E_NO_DEVICE, "no usable CUDA device");

    h = new sw2d_handle();
    h->device = device;
    h->p = *params;
    h->model = dip ? kModelDip : ddp ? kModelDdp : kModelSp;
    h->dissipation = ((dip && dip->momentum_dissipation) || (ddp && ddp->momentum_dissipation)) ? 1 : 0;
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
    // walking edges by increasing original index appends them in that order.  Balance slots of
    // a cell: its boundary edges, then its internal edges (hypComputeBalance, swSpHyp.cpp:221-263).
    std::vector<int> cb_cnt(nc + 1, 0), ci_cnt(nc + 1, 0);
    for (int64_t e = 0; e < nb; e++) cb_cnt[inv[mesh->edge_bnd_cell[e]] + 1]++;
    for (int64_t e = 0; e < ni; e++) {
        ci_cnt[inv[mesh->edge_int_cells[2 * e]] + 1]++;
        ci_cnt[inv[mesh->edge_int_cells[2 * e + 1]] + 1]++;
    }
    std::vector<int2> coff(nc + 1);
    {
        int ci = 0, sl = 0;
        for (int64_t c = 0; c < nc; c++) {
            coff[c] = make_int2(ci, sl);
            ci += ci_cnt[c + 1];
            sl += cb_cnt[c + 1] + ci_cnt[c + 1];
        }
        coff[nc] = make_int2(ci, sl);
    }
    std::vector<int2> cint(2 * ni), eslot(ni);
    std::vector<int> bslot(nb);
    {
        std::vector<int> fi(nc), fs(nc);
        for (int64_t c = 0; c < nc; c++) {
            fi[c] = coff[c].x;
            fs[c] = coff[c].y;
        }
        for (int64_t e = 0; e < nb; e++) bslot[inv_bnd[e]] = fs[inv[mesh->edge_bnd_cell[e]]]++;
        for (int64_t e = 0; e < ni; e++) {
            int a = inv[mesh->edge_int_cells[2 * e]], b = inv[mesh->edge_int_cells[2 * e + 1]];
            int ne = inv_int[e];
            cint[fi[a]++] = make_int2(ne * 2 + 0, b);
            cint[fi[b]++] = make_int2(ne * 2 + 1, a);
            eslot[ne] = make_int2(fs[a]++, fs[b]++);
        }
    }
    const int64_t nslot = (int64_t)coff[nc].y;

    // ---- tables in the new numbering
    std::vector<double4> st(nc), cst(nc);
    std::vector<double2> cxy(nc);
    std::vector<double> zbv(nc), area(nc);
    for (int64_t i = 0; i < nc; i++) {
        const int o = h->cell_perm[i];
        const double zb = mesh->cell_z_b[o];
        st[i] = make_double4(h0[o], q0[o], r0[o], h0[o] + zb);
        // DDP: the SP coefficient w / area / phi with phi = 1 is the DDP factor w / area
        // (swDdp.cpp:430-466); the DDP set-up then stores the lowest table level in .z
        cst[i] = make_double4(zb, fields->boussinesq[o], ddp ? 1.0 : fields->phi[o], mesh->cell_area[o]);
        cxy[i] = make_double2(mesh->cell_x[o], mesh->cell_y[o]);
        zbv[i] = zb;
        area[i] = mesh->cell_area[o];
    }
    std::vector<int2> lr(ni);
    std::vector<double2> nxy(ni), mxy(ni);
    std::vector<double> len(ni);
    for (int64_t i = 0; i < ni; i++) {
        const int oe = h->int_perm[i];
        lr[i] = make_int2(inv[mesh->edge_int_cells[2 * oe]], inv[mesh->edge_int_cells[2 * oe + 1]]);
        nxy[i] = make_double2(mesh->edge_int_nx[oe], mesh->edge_int_ny[oe]);
        mxy[i] = make_double2(mesh->edge_int_mx[oe], mesh->edge_int_my[oe]);
        len[i] = mesh->edge_int_length[oe];
    }
    // per internal edge, midpoint - centroid of L and R: the first difference of the MUSCL-EVR
    // reconstruction (swSpHypMusclEvr.cpp:197-207), a static of the mesh computed once
    std::vector<double4> emc(ni);
    for (int64_t i = 0; i < ni; i++) {
        const double2 a = cxy[lr[i].x], b = cxy[lr[i].y], mp = mxy[i];
        emc[i] = make_double4(mp.x - a.x, mp.y - a.y, mp.x - b.x, mp.y - b.y);
    }
    std::vector<int> bcell(nb), bbc(nb);
    std::vector<double4> bgeo(nb);
    for (int64_t i = 0; i < nb; i++) {
        const int oe = h->bnd_perm[i];
        bcell[i] = inv[mesh->edge_bnd_cell[oe]];
        bbc[i] = mesh->edge_bnd_bc[oe];
        bgeo[i] = make_double4(mesh->edge_bnd_nx[oe], mesh->edge_bnd_ny[oe], mesh->edge_bnd_length[oe], 0.0);
    }
    // friction and head-loss angles: degrees -> radians and cos/sin on the host, with the
    // expressions of swSp::setFrictionParameters (swSp.cpp:1063-1068) and
    // sourceSingularHeadLoss (swSpSourceFriction.cpp:185-187)
    std::vector<double4> fric, hla;
    std::vector<double2> hlb;
    if (params->friction != SW2D_FRICTION_NONE) {
        fric.resize(nc);
        for (int64_t i = 0; i < nc; i++) {
            const int o = h->cell_perm[i];
            double a = fields->friction_alpha[o] * atan(1.0) / 45.0;
            fric[i] = make_double4(fields->friction_1[o], fields->friction_2[o], cos(a), sin(a));
        }
    }
    if (params->singular_head_loss) {
        hla.resize(nc);
        hlb.resize(nc);
        for (int64_t i = 0; i < nc; i++) {
            const int o = h->cell_perm[i];
            double a = fields->hl_alpha[o] * atan(1.0) / 45.0;
            hla[i] = make_double4(fields->hl_h_sing[o], fields->hl_coeff_1[o], fields->hl_coeff_2[o], 0.0);
            hlb[i] = make_double2(cos(a), sin(a));
        }
    }

    DevMesh& m = h->m;
    m.nc = (int)nc;
    m.ni = (int)ni;
    m.nb = (int)nb;
    int rc = SW2D_OK;
#define UP(vec, dst)                                        \
    do {                                                    \
        auto* tmp_ = (decltype(vec.data()))nullptr;         \
        rc = dev_upload(h, vec, &tmp_);                     \
        if (rc) return bail(rc);                            \
        dst = tmp_;                                         \
    } while (0)
    UP(st, m.st);
    UP(cst, m.cst);
    UP(cxy, m.cxy);
    if (!fric.empty()) UP(fric, m.fric);
    if (!hla.empty()) {
        UP(hla, m.hla);
        UP(hlb, m.hlb);
    }
    UP(zbv, m.zbv);
    UP(area, m.area);
    UP(coff, m.coff);
    UP(cint, m.cint);
    UP(eslot, m.eslot);
    UP(bslot, m.bslot);
    UP(lr, m.lr);
    UP(nxy, m.nxy);
    UP(mxy, m.mxy);
    UP(emc, m.emc);
    UP(len, m.len);
    UP(bcell, m.bcell);
    UP(bbc, m.bbc);
    double4* bgeo_d = nullptr;
    if ((rc = dev_upload(h, bgeo, &bgeo_d))) return bail(rc);
    m.bgeo = bgeo_d;
    if (dip) {
        std::vector<double> pgi(ni), pgb(nb);
        for (int64_t i = 0; i < ni; i++) pgi[i] = dip->phi_g_int[h->int_perm[i]];
        for (int64_t i = 0; i < nb; i++) pgb[i] = dip->phi_g_bnd[h->bnd_perm[i]];
        UP(pgi, m.phig);
        UP(pgb, m.phigb);
        if (dip->momentum_dissipation) {
            // swDip::setMomentumDissipationParameters (dip/swDip.cpp:1302-1334)
            std::vector<double4> mu(nc);
            for (int64_t i = 0; i < nc; i++) {
                const int o = h->cell_perm[i];
                double a = dip->mu_alpha[o] * atan(1.0) / 45.0;
                mu[i] = make_double4(dip->mu_1[o], dip->mu_2[o], cos(a), sin(a));
            }
            UP(mu, m.mu);
        }
    }
    UP(h->cell_perm, h->d_cell_perm);
    UP(h->int_perm, h->d_int_perm);
    UP(h->bnd_perm, h->d_bnd_perm);
    {
        std::vector<int> bct(bc->type, bc->type + bc->bc_nb);
        std::vector<long long> bco(bc->offset, bc->offset + bc->bc_nb + 1);
        const int64_t nrec = bc->offset[bc->bc_nb];
        std::vector<double> bt(bc->times, bc->times + nrec), bv(bc->values, bc->values + nrec);
        UP(bct, m.bctype);
        UP(bco, m.bcoff);
        UP(bt, m.bctimes);
        UP(bv, m.bcvals);
    }
#undef UP
    double2* coef_d = nullptr;
    if ((rc = dev_alloc(h, ni, &coef_d))) return bail(rc);
    m.coef = coef_d;
    // persistent balance slots start at zero, like the reference's resized flux vectors
    if ((rc = dev_alloc(h, nslot, &m.slot)) || (rc = dev_alloc(h, nslot, &m.slot_w)) ||
        (rc = dev_alloc(h, nc, &m.slope)) || (rc = dev_alloc(h, nc / 32 + grid_for(nc) + 2, &m.part)) ||
        (rc = dev_alloc(h, 3 * nc, &h->stage)))
        return bail(rc);
    m.flux = nullptr;
    m.bflux = nullptr;
    m.lmax = nullptr;
    m.lmaxb = nullptr;
    m.h_min = params->h_min;
    m.phi_min = ddp ? 0.0 : params->phi_min;
    m.cfl_max = params->cfl_max;
    m.dt_max = params->dt_max;
    m.dt_map = params->dt_map;
    m.v_max = params->v_max;
    m.fr_max = params->fr_max;
    m.neg_detect = params->negative_depth_detection ? 1 : 0;
    // constants of the dry-cell shortcuts, by the same IEEE operations the step would do
    {
        volatile double g = kGravity, sr = kSmallReal;
        m.dry.c0 = std::sqrt(g * sr);
        volatile double c0 = m.dry.c0;
        m.dry.r0 = std::sqrt(c0 * c0);
    }
    if (cudaMalloc(&h->ctrl, sizeof(Ctrl)) != cudaSuccess) return bail(fail(h, SW2D_E_CUDA, "cudaMalloc ctrl"));
    h->allocs.push_back(h->ctrl);
    if (cudaMallocHost(&h->ctrl_host, sizeof(Ctrl)) != cudaSuccess) return bail(fail(h, SW2D_E_CUDA, "cudaMallocHost"));
    m.ctrl = h->ctrl;
    Ctrl c0{};
    c0.t = params->t_0;
    c0.dt = 0.0;  // swSp.h:155
    c0.dmin = kDminEmpty;
    c0.t_max = params->t_max;
    *h->ctrl_host = c0;
    if (cudaMemcpyAsync(h->ctrl, h->ctrl_host, sizeof(Ctrl), cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
        return bail(fail(h, SW2D_E_CUDA, "ctrl upload"));
    k_edge_coefficients<<<grid_for(ni + nb), kBlock, 0, h->stream>>>(m, coef_d, bgeo_d);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess)
        return bail(fail(h, SW2D_E_CUDA, "initialisation kernels failed"));
    if ((rc = noalloc_prepare(h))) return bail(rc);
    if (!ddp) {
        // tables for the tiles of the fused step, which is an option ("fused_step"; the tiles
        // are built when it is first switched on).  The four-kernel step is the default, being
        // the faster form on B200 for both schemes: the step is bound by the latency of its FP64
        // instructions, not by HBM, and k_edges and k_slopes reach their operands through L1 at
        // a higher occupancy than the tile kernel, whose staging and barriers add instructions
        // and whose cross-tile edges are computed twice.
        h->tile_default = kDefaultTileCells;
        if (const char* env = std::getenv("SW2D_TILE_CELLS")) h->tile_default = std::atoi(env);
        h->h_coff = coff;
        h->h_cint = cint;
        h->h_lr = lr;
        h->h_bcell = bcell;
        h->fused = 0;
        h->err.clear();
    }
    if (ddp) {
        if ((rc = ddp_setup(h, mesh, fields, ddp, h0, q0, r0))) return bail(rc);
        CK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if ((rc = status_to_code(h, h->ctrl_host->status))) return bail(rc);
    }
    *out = h;
    return SW2D_OK;
}

}  // namespace

extern "C" {

int sw2d_step_n(sw2d_handle* h, int64_t n_steps, int64_t* steps_done)
{
    if (!h || n_steps < 0) return fail(h, SW2D_E_ARG, "invalid arguments");
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const long long before = h->ctrl_host->steps;
    if (h->result) {
        // chunks of at most half the frame ring, each drained to the writer thread; before a
        // chunk, the frames of the chunk before last are on file
        const int chunk = result_chunk(h);
        int64_t left = n_steps;
        while (left > 0) {
            const int64_t k = std::min<int64_t>(left, chunk);
            int rc = result_wait(h, chunk);
            if (rc) return rc;
            if (k == chunk) {
                if ((rc = ensure_graph(h, chunk))) return rc;
                CK(cudaGraphLaunch(h->graph, h->stream));
            } else {
                if ((rc = prepare_step(h))) return rc;
                for (int64_t i = 0; i < k; i++) launch_step(h);
            }
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            if ((rc = result_drain(h))) return rc;
            left -= k;
            if (h->ctrl_host->status || h->ctrl_host->steps - before < n_steps - left) break;
        }
        if (steps_done) *steps_done = h->ctrl_host->steps - before;
        return status_to_code(h, h->ctrl_host->status);
    }
    const int chunk = kGraphSteps;
    const int64_t full = n_steps / chunk, rem = n_steps % chunk;
    if (full > 0) {
        int st = ensure_graph(h, chunk);
        if (st) return st;
        for (int64_t i = 0; i < full; i++) CK(cudaGraphLaunch(h->graph, h->stream));
    }
    if (rem > 0) {
        int st = prepare_step(h);
        if (st) return st;
    }
    for (int64_t i = 0; i < rem; i++) launch_step(h);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (steps_done) *steps_done = h->ctrl_host->steps - before;
    return status_to_code(h, h->ctrl_host->status);
}

int sw2d_prepare_steps(sw2d_handle* h)
{
    if (!h) return fail(h, SW2D_E_ARG, "invalid handle");
    CK(cudaSetDevice(h->device));
    const int rc = ensure_graph(h, h->result ? result_chunk(h) : kGraphSteps);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->stream));
    return SW2D_OK;
}

int sw2d_execute(sw2d_handle* h, int64_t* steps_done)
{
    if (!h) return fail(h, SW2D_E_ARG, "invalid handle");
    // with a map file attached: the run's first map (swSp.cpp:504), once
    if (h->result && !result_started(h)) {
        CK(cudaSetDevice(h->device));
        const int rc = result_force(h);
        if (rc) return rc;
    }
    // passes of growing length (32 .. 1024 steps): a run that ends after a few steps does not
    // pay for a thousand launches that find the run over
    int64_t total = 0, chunk = 32;
    for (;;) {
        int64_t k = 0;
        int st = sw2d_step_n(h, chunk, &k);
        total += k;
        if (st) {
            if (steps_done) *steps_done = total;
            return st;
        }
        if (k < chunk) break;
        chunk = std::min<int64_t>(2 * chunk, 1024);
    }
    if (h->result) {  // the map after the loop (swSp.cpp:630), then every frame on file
        int rc = result_force(h);
        if (!rc) rc = result_wait(h, 0);
        if (rc) {
            if (steps_done) *steps_done = total;
            return rc;
        }
    }
    if (steps_done) *steps_done = total;
    return SW2D_OK;
}

int sw2d_phase_times(sw2d_handle* h, int64_t n_steps, double* ms, int capacity)
{
    if (!h || !ms || n_steps <= 0) return fail(h, SW2D_E_ARG, "invalid arguments");
    const int nph = (h->model == kModelDdp) ? 4 : n_phases(h);
    if (capacity < nph) return fail(h, SW2D_E_ARG, "capacity below the number of phases");
    CK(cudaSetDevice(h->device));
    {
        const int rc = prepare_step(h);
        if (rc) return rc;
    }
    cudaEvent_t ev[4 + 1];
    for (int i = 0; i <= nph; i++) CK(cudaEventCreate(&ev[i]));
    double acc[4] = {0, 0, 0, 0};
    for (int64_t s = 0; s < n_steps; s++) {
        for (int i = 0; i < nph; i++) {
            cudaEventRecord(ev[i], h->stream);
            launch_phase(h, i);
        }
        cudaEventRecord(ev[nph], h->stream);
        CK(cudaEventSynchronize(ev[nph]));
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

const char* sw2d_phase_label(sw2d_handle* h, int i)
{
    static const char* fused[] = {"k_flux", "k_update"};
    static const char* fused3[] = {"k_slopes", "k_flux", "k_update"};
    if (h && h->model != kModelDdp && h->fused) {
        if (slopes_first(h)) return (i >= 0 && i < 3) ? fused3[i] : "";
        return (i >= 0 && i < 2) ? fused[i] : "";
    }
    return sw2d_phase_name(i);
}

int sw2d_autotune(sw2d_handle* h, int iters, char* report, int capacity)
{
    if (!h || iters <= 0) return fail(h, SW2D_E_ARG, "invalid arguments");
    CK(cudaSetDevice(h->device));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    std::string rep;
    // The timed kernels recompute their outputs (slopes, balance slots, CFL contributions) from the
    // state, but k_flux and k_cfl also write the pending dt into the control block, which the
    // MUSCL-EVR reconstruction of the next step reads as the previous dt: the block is saved here
    // and put back once the timings are done, so the run continues as if nothing had been timed.
    Ctrl saved;
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(&saved, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    auto restore = [&]() -> int {
        CK(cudaStreamSynchronize(h->stream));
        CK(cudaMemcpy(h->ctrl, &saved, sizeof(Ctrl), cudaMemcpyHostToDevice));
        return SW2D_OK;
    };
    auto time_it = [&](auto&& launch) {
        launch();  // warm
        cudaEventRecord(e0, h->stream);
        for (int i = 0; i < iters; i++) launch();
        cudaEventRecord(e1, h->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return (double)ms / iters;
    };
    if (h->fused) {
        if (slopes_first(h)) {
            double bs = 1e300;
            for (int v = 0; v < kNumVariants; v++) {
                double ms = time_it([&] { launch_slopes(h, v); });
                rep += "k_slopes/" + std::to_string(kVariants[v].block) + "x" + std::to_string(kVariants[v].minb) + "=" +
                       std::to_string(ms) + "ms ";
                if (ms < bs) {
                    bs = ms;
                    h->slope_variant = v;
                }
            }
            launch_slopes(h, h->slope_variant);
        }
        double best = 1e300;
        for (int v = 0; v < flux_variants(); v++) {
            if (launch_flux(h, h->m, v, true) != cudaSuccess) continue;
            double ms = time_it([&] { launch_flux(h, h->m, v, false); });
            rep += "k_flux/" + flux_variant_label(v) + "=" + std::to_string(ms) + "ms ";
            if (ms < best) {
                best = ms;
                h->flux_variant = v;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        CK(cudaGetLastError());
        if (const int rc = restore()) return rc;
        if (h->graph) {
            cudaGraphExecDestroy(h->graph);
            h->graph = nullptr;
        }
        rep += "chosen k_flux/" + flux_variant_label(h->flux_variant) + " tile " + std::to_string(h->tiles.tile_cells);
        if (report && capacity > 0) {
            std::strncpy(report, rep.c_str(), (size_t)capacity - 1);
            report[capacity - 1] = '\0';
        }
        return SW2D_OK;
    }
    if (h->p.scheme == SW2D_SCHEME_MUSCL_EVR) {
        double best = 1e300;
        for (int v = 0; v < kNumVariants; v++) {
            double ms = time_it([&] { launch_slopes(h, v); });
            rep += "k_slopes/" + std::to_string(kVariants[v].block) + "x" + std::to_string(kVariants[v].minb) + "=" +
                   std::to_string(ms) + "ms ";
            if (ms < best) {
                best = ms;
                h->slope_variant = v;
            }
        }
        launch_slopes(h, h->slope_variant);
    }
    auto label = [&](int v) {
        int b = kVariants[v].block, mb = kVariants[v].minb;
        if (h->model == kModelDdp) ddp_variant(v, &b, &mb);
        return std::to_string(b) + "x" + std::to_string(mb);
    };
    double best = 1e300;
    for (int v = 0; v < kNumVariants; v++) {
        double ms = time_it([&] { launch_edges(h, v); });
        rep += std::string(h->model == kModelDdp ? "k_ddp_edges/" : "k_edges/") + label(v) + "=" + std::to_string(ms) +
               "ms ";
        if (ms < best) {
            best = ms;
            h->edge_variant = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CK(cudaGetLastError());
    if (const int rc = restore()) return rc;
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    rep += "chosen k_slopes/" + std::to_string(kVariants[h->slope_variant].block) + "x" +
           std::to_string(kVariants[h->slope_variant].minb) + (h->model == kModelDdp ? " k_ddp_edges/" : " k_edges/") +
           label(h->edge_variant);
    if (report && capacity > 0) {
        std::strncpy(report, rep.c_str(), (size_t)capacity - 1);
        report[capacity - 1] = '\0';
    }
    return SW2D_OK;
}

int sw2d_autotune_step(sw2d_handle* h, int iters, const int* tile_sizes, int n_tile_sizes, char* report,
                       int capacity)
{
    if (!h || iters <= 0 || n_tile_sizes < 0 || (n_tile_sizes && !tile_sizes))
        return fail(h, SW2D_E_ARG, "invalid arguments");
    if (h->model == kModelDdp) return sw2d_autotune(h, iters, report, capacity);
    CK(cudaSetDevice(h->device));
    static const int kDefaultTiles[] = {192, 256, 320, 384, 512};
    if (!n_tile_sizes) {
        tile_sizes = kDefaultTiles;
        n_tile_sizes = (int)(sizeof(kDefaultTiles) / sizeof(int));
    }
    // the timed kernels write the pending dt (read as the previous dt by the next MUSCL-EVR step):
    // the control block is put back at the end, as in sw2d_autotune
    Ctrl saved;
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(&saved, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto time_it = [&](auto&& launch) {
        launch();  // warm
        cudaEventRecord(e0, h->stream);
        for (int i = 0; i < iters; i++) launch();
        cudaEventRecord(e1, h->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return (double)ms / iters;
    };
    const bool muscl = h->p.scheme == SW2D_SCHEME_MUSCL_EVR;
    std::string rep;
    // k_slopes at its fastest launch variant (shared by the four-kernel step and the fused step
    // that computes the slopes first)
    double t_slopes = 0.0;
    int slope_v = h->slope_variant;
    if (muscl) {
        t_slopes = 1e300;
        for (int v = 0; v < kNumVariants; v++) {
            const double ms = time_it([&] { launch_slopes(h, v); });
            if (ms < t_slopes) {
                t_slopes = ms;
                slope_v = v;
            }
        }
        launch_slopes(h, slope_v);  // the slopes k_flux reads when it does not compute them
    }
    // four-kernel step: k_slopes + k_edges + k_cfl (k_update is the same in every form)
    double t_edges = 1e300;
    int edge_v = h->edge_variant;
    for (int v = 0; v < kNumVariants; v++) {
        const double ms = time_it([&] { launch_edges(h, v); });
        if (ms < t_edges) {
            t_edges = ms;
            edge_v = v;
        }
    }
    const double t_cfl = time_it([&] { k_cfl<false><<<cfl_grid(h, h->m.nc), kBlock, 0, h->stream>>>(h->m); });
    const double t_four = t_slopes + t_edges + t_cfl;
    rep += "four-kernel=" + std::to_string(t_four) + "ms ";
    // fused forms: for MUSCL-EVR both places of the slopes, every tile size
    struct Best {
        double ms;
        int fused, fused_slopes, tile, flux_v;
    } best{t_four, 0, h->fused_slopes, h->tiles.tile_cells, h->flux_variant};
    const int prev_fs = h->fused_slopes, prev_tile = h->tiles.tile_cells;
    for (int fs = muscl ? 0 : h->fused_slopes; fs <= (muscl ? 1 : h->fused_slopes); fs++) {
        h->fused_slopes = fs;
        for (int k = 0; k < n_tile_sizes; k++) {
            std::string why;
            if (tiles_build(h, h->h_coff, h->h_cint, h->h_lr, h->h_bcell, tile_sizes[k], why)) {
                rep += "tile " + std::to_string(tile_sizes[k]) + " refused ";
                continue;
            }
            const double pre = slopes_first(h) ? t_slopes : 0.0;
            double bf = 1e300;
            int bv = 0;
            for (int v = 0; v < flux_variants(); v++) {
                if (launch_flux(h, h->m, v, true) != cudaSuccess) continue;
                const double ms = time_it([&] { launch_flux(h, h->m, v, false); });
                if (ms < bf) {
                    bf = ms;
                    bv = v;
                }
            }
            rep += std::string(muscl ? (fs ? "fused" : "fused/slopes-first") : "fused") + "/tile" +
                   std::to_string(tile_sizes[k]) + "/" + flux_variant_label(bv) + "=" + std::to_string(pre + bf) +
                   "ms ";
            if (pre + bf < best.ms) best = {pre + bf, 1, fs, tile_sizes[k], bv};
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    // the chosen form (tiles rebuilt for it; the previous tiles, if any, when the four-kernel
    // step wins)
    h->fused_slopes = best.fused ? best.fused_slopes : prev_fs;
    if (best.fused || prev_tile > 0) {
        std::string why;
        const int rc = tiles_build(h, h->h_coff, h->h_cint, h->h_lr, h->h_bcell, best.fused ? best.tile : prev_tile, why);
        if (rc) {
            h->fused = 0;
            return fail(h, rc, "autotune_step: " + (why.empty() ? h->err : why));
        }
    }
    h->fused = best.fused;
    h->slope_variant = slope_v;
    h->edge_variant = edge_v;
    h->flux_variant = best.flux_v;
    CK(cudaMemcpy(h->ctrl, &saved, sizeof(Ctrl), cudaMemcpyHostToDevice));
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    if (best.fused)
        rep += "chosen fused" + std::string(muscl ? (best.fused_slopes ? "" : "/slopes-first") : "") + " tile " +
               std::to_string(best.tile) + " k_flux/" + flux_variant_label(best.flux_v);
    else
        rep += "chosen four-kernel k_slopes/" + std::to_string(kVariants[slope_v].block) + "x" +
               std::to_string(kVariants[slope_v].minb) + " k_edges/" + std::to_string(kVariants[edge_v].block) + "x" +
               std::to_string(kVariants[edge_v].minb);
    if (report && capacity > 0) {
        std::strncpy(report, rep.c_str(), (size_t)capacity - 1);
        report[capacity - 1] = '\0';
    }
    return SW2D_OK;
}

int sw2d_get_launch_config(sw2d_handle* h, int* slopes_variant, int* edges_variant)
{
    if (!h) return fail(h, SW2D_E_ARG, "invalid handle");
    if (slopes_variant) *slopes_variant = h->slope_variant;
    if (edges_variant) *edges_variant = h->edge_variant;
    return SW2D_OK;
}

int sw2d_set_launch_config(sw2d_handle* h, int slopes_variant, int edges_variant)
{
    if (!h || slopes_variant < 0 || slopes_variant >= kNumVariants || edges_variant < 0 ||
        edges_variant >= kNumVariants)
        return fail(h, SW2D_E_ARG, "invalid launch variant");
    h->slope_variant = slopes_variant;
    h->edge_variant = edges_variant;
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    return SW2D_OK;
}

int sw2d_set_option(sw2d_handle* h, const char* name, int64_t value)
{
    if (!h || !name) return fail(h, SW2D_E_ARG, "invalid arguments");
    CK(cudaSetDevice(h->device));
    if (std::strcmp(name, "record_wave_speeds") == 0) {
        if (value && !h->lmax_buf) {
            int rc = dev_alloc(h, h->ni, &h->lmax_buf);
            if (!rc) rc = dev_alloc(h, h->nb, &h->lmaxb_buf);
            if (rc) return rc;
        }
        h->m.lmax = value ? h->lmax_buf : nullptr;
        h->m.lmaxb = value ? h->lmaxb_buf : nullptr;
    } else if (std::strcmp(name, "record_fluxes") == 0) {
        // F1, F2, F3, S2L, S2R as the reference keeps them (swSp.h:183-193), for sw2d_get_array;
        // turn on before the first step so that edges left dry keep their (zero) initial values
        if (value && !h->flux_buf) {
            int rc = dev_alloc(h, 3 * h->ni, &h->flux_buf);
            if (!rc) rc = dev_alloc(h, h->nb, &h->bflux_buf);
            if (rc) return rc;
        }
        const bool keep = h->model == kModelDdp && h->m.div_corr == kDivCorrFlux;  // the correction scales them
        h->m.flux = (value || keep) ? h->flux_buf : nullptr;
        h->m.bflux = (value || keep) ? h->bflux_buf : nullptr;
    } else if (std::strcmp(name, "adjoint_flush_branch") == 0) {
        h->adj_flush_branch = value ? 1 : 0;
        return SW2D_OK;
    } else if (std::strcmp(name, "adjoint_store_states") == 0) {
        // 1 (default): the adjoint's segment recompute keeps each step's slopes and Riemann
        // states for the reverse steps when they fit in half of the free device memory; 0:
        // the reverse steps rebuild them (the same bits).  Takes effect at the next sw2d_record.
        h->adj_store_states = value ? 1 : 0;
        return SW2D_OK;
    } else if (std::strcmp(name, "adjoint_trace") == 0) {
        // 1: sw2d_adjoint records, after each reverse step, the non-finite entries and the largest
        // magnitudes of the state adjoint (sw2d_adjoint_trace)
        h->adj_trace = value ? 1 : 0;
        return SW2D_OK;
    } else if (std::strcmp(name, "adjoint_keep_nonfinite") == 0) {
        // 1: sw2d_adjoint counts its non-finite gradient entries but hands them back as they are
        // (to locate them) instead of zeroing them as the reference does
        h->adj_keep_nonfinite = value ? 1 : 0;
        return SW2D_OK;
    } else if (std::strcmp(name, "assim_sqrt_zero") == 0) {
        // reverse of sqrt at 0 in the assimilation sweep: 0 (subgradient 0, default) or 1
        // (IEEE: dy / (2 sqrt(0)), non-finite unless dy == 0, as source-transformation AD gives)
        h->assim_sqrt_zero = value ? 1 : 0;
        return SW2D_OK;
    } else if (std::strcmp(name, "assim_chained_recompute") == 0) {
        // where the gradient recomputes each segment: 0 from the dry run's checkpoints, as the
        // reference does; 1 from the replay's own states (the exact gradient of the replay cost)
        h->assim_chained = value ? 1 : 0;
        return SW2D_OK;
    } else if (std::strcmp(name, "closure_record") == 0) {
        // keep each step's closure features and network outputs (sw2d_closure_record)
        if (!h->closure) return fail(h, SW2D_E_ARG, "no closure attached");
        const int rc = closure_record(h, value ? 1 : 0);
        if (rc) return rc;
    } else if (std::strcmp(name, "closure_ctas_per_sm") == 0) {
        // launch shape of the closure's update kernel: CTAs per SM of its persistent grid (0:
        // as many as the kernel's registers and shared memory let reside)
        if (!h->closure) return fail(h, SW2D_E_ARG, "no closure attached");
        if (value < 0 || value > 8) return fail(h, SW2D_E_ARG, "closure_ctas_per_sm outside 0..8");
        closure_set_ctas(h, (int)value);
    } else if (std::strcmp(name, "fused_step") == 0) {
        // 1: the step as [k_slopes +] k_flux + k_update; 0 (the default): the four-kernel step
        // k_slopes, k_edges, k_cfl, k_update (the same results).  The tiles are built the first
        // time the fused step is switched on.
        if (value && !h->tiles.ntiles) {
            if (h->model == kModelDdp) return fail(h, SW2D_E_UNSUPPORTED, "the DDP model has no fused step");
            CK(cudaStreamSynchronize(h->stream));
            std::string why;
            const int rc = tiles_build(h, h->h_coff, h->h_cint, h->h_lr, h->h_bcell, h->tile_default, why);
            if (rc) return fail(h, rc, "fused_step: " + (why.empty() ? h->err : why));
        }
        h->fused = value ? 1 : 0;
    } else if (std::strcmp(name, "tile_cells") == 0) {
        // cells per tile of the fused step (32..8192): the tiles are rebuilt
        if (h->model == kModelDdp) return fail(h, SW2D_E_UNSUPPORTED, "the DDP model has no tiles");
        CK(cudaStreamSynchronize(h->stream));
        std::string why;
        const int rc = tiles_build(h, h->h_coff, h->h_cint, h->h_lr, h->h_bcell, (int)value, why);
        if (rc) {
            if (!h->tiles.ntiles) h->fused = 0;  // the previous tiles are kept unless they were released
            return fail(h, rc, "tile_cells: " + (why.empty() ? h->err : why));
        }
    } else if (std::strcmp(name, "fused_slopes") == 0) {
        // MUSCL-EVR fused step: 1 the slopes inside k_flux (ring 2 staged), 0 k_slopes first and
        // k_flux reading its output (the same results); the tiles are rebuilt
        if (h->model == kModelDdp) return fail(h, SW2D_E_UNSUPPORTED, "the DDP model has no tiles");
        CK(cudaStreamSynchronize(h->stream));
        const int prev = h->fused_slopes;
        h->fused_slopes = value ? 1 : 0;
        std::string why;
        const int tc = h->tiles.ntiles ? h->tiles.tile_cells : h->tile_default;
        const int rc = tiles_build(h, h->h_coff, h->h_cint, h->h_lr, h->h_bcell, tc, why);
        if (rc) {
            h->fused_slopes = prev;
            if (!h->tiles.ntiles) h->fused = 0;
            return fail(h, rc, "fused_slopes: " + (why.empty() ? h->err : why));
        }
    } else if (std::strcmp(name, "update_reverse") == 0) {
        // block order of the cell update: 1 from the last cells to the first (the same results)
        h->m.rev_update = value ? 1 : 0;
    } else if (std::strcmp(name, "flux_variant") == 0) {
        if (value < 0 || value >= flux_variants()) return fail(h, SW2D_E_ARG, "flux_variant outside the variants");
        h->flux_variant = (int)value;
    } else if (std::strcmp(name, "adjoint_edge_variant") == 0) {
        if (value < 0 || value > 4) return fail(h, SW2D_E_ARG, "adjoint_edge_variant outside 0..4");
        h->adj_edge_variant = (int)value;
        return SW2D_OK;
    } else {
        return fail(h, SW2D_E_ARG, std::string("unknown option ") + name);
    }
    if (h->graph) {  // the captured kernels hold the previous parameters
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    CK(cudaStreamSynchronize(h->stream));
    return SW2D_OK;
}

int sw2d_get_option(sw2d_handle* h, const char* name, int64_t* value)
{
    if (!h || !name || !value) return fail(h, SW2D_E_ARG, "invalid arguments");
    if (std::strcmp(name, "fused_step") == 0) *value = h->fused;
    else if (std::strcmp(name, "flux_variant") == 0) *value = h->flux_variant;
    else if (std::strcmp(name, "update_reverse") == 0) *value = h->m.rev_update;
    else if (std::strcmp(name, "fused_slopes") == 0) *value = h->fused_slopes;
    else if (std::strcmp(name, "tile_cells") == 0) *value = h->tiles.tile_cells;
    else if (std::strcmp(name, "record_fluxes") == 0) *value = h->m.flux != nullptr;
    else if (std::strcmp(name, "record_wave_speeds") == 0) *value = h->m.lmax != nullptr;
    else return fail(h, SW2D_E_ARG, std::string("option not readable: ") + name);
    return SW2D_OK;
}

int sw2d_get_state_device(sw2d_handle* h, double* dh, double* dq, double* dr)
{
    if (!h || !dh || !dq || !dr) return fail(h, SW2D_E_ARG, "invalid arguments");
    CK(cudaSetDevice(h->device));
    k_scatter_state<<<grid_for(h->nc), kBlock, 0, h->stream>>>(h->m.st, h->d_cell_perm, dh, dq, dr, (int)h->nc);
    CK(cudaGetLastError());
    return SW2D_OK;
}

int sw2d_set_state_device(sw2d_handle* h, const double* dh, const double* dq, const double* dr)
{
    if (!h || !dh || !dq || !dr) return fail(h, SW2D_E_ARG, "invalid arguments");
    CK(cudaSetDevice(h->device));
    k_gather_state<<<grid_for(h->nc), kBlock, 0, h->stream>>>(dh, dq, dr, h->d_cell_perm, h->m.cst, h->m.st, (int)h->nc);
    CK(cudaGetLastError());
    if (h->model == kModelDdp) return ddp_derive(h);  // z and the cell-table values of the new state
    return SW2D_OK;
}

int sw2d_get_state(sw2d_handle* h, double* wd, double* qx, double* qy)
{
    if (!h || !wd || !qx || !qy) return fail(h, SW2D_E_ARG, "invalid arguments");
    int st = sw2d_get_state_device(h, h->stage, h->stage + h->nc, h->stage + 2 * h->nc);
    if (st) return st;
    const size_t bytes = h->nc * sizeof(double);
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
    const size_t bytes = h->nc * sizeof(double);
    CK(cudaMemcpyAsync(h->stage, wd, bytes, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->stage + h->nc, qx, bytes, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->stage + 2 * h->nc, qy, bytes, cudaMemcpyHostToDevice, h->stream));
    int st = sw2d_set_state_device(h, h->stage, h->stage + h->nc, h->stage + 2 * h->nc);
    if (st) return st;
    CK(cudaStreamSynchronize(h->stream));
    return SW2D_OK;
}

// bytes of a saved point: the state records, the balance slots (they keep the fluxes of edges
// left dry from one step to the next) and the control block
static size_t point_bytes(const sw2d_handle* h, size_t* st, size_t* sl)
{
    *st = (size_t)h->nc * sizeof(double4);
    *sl = (size_t)h->h_coff.back().y * sizeof(Slot);
    return *st + *sl + sizeof(Ctrl);
}

int sw2d_save_point(sw2d_handle* h)
{
    if (!h) return fail(h, SW2D_E_ARG, "invalid handle");
    if (h->model == kModelDdp) return fail(h, SW2D_E_UNSUPPORTED, "save_point: the DDP model keeps more state");
    CK(cudaSetDevice(h->device));
    size_t st, sl;
    const size_t bytes = point_bytes(h, &st, &sl);
    if (!h->saved_point) CK(cudaMalloc(&h->saved_point, bytes));
    char* d = static_cast<char*>(h->saved_point);
    CK(cudaMemcpyAsync(d, h->m.st, st, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(d + st, h->m.slot, sl, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(d + st + sl, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return SW2D_OK;
}

int sw2d_restore_point(sw2d_handle* h)
{
    if (!h) return fail(h, SW2D_E_ARG, "invalid handle");
    if (!h->saved_point) return fail(h, SW2D_E_ARG, "restore_point: no point saved");
    CK(cudaSetDevice(h->device));
    size_t st, sl;
    point_bytes(h, &st, &sl);
    const char* d = static_cast<const char*>(h->saved_point);
    CK(cudaMemcpyAsync(h->m.st, d, st, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->m.slot, d + st, sl, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->ctrl, d + st + sl, sizeof(Ctrl), cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return SW2D_OK;
}

int sw2d_set_t_max(sw2d_handle* h, double t_max)
{
    if (!h) return fail(h, SW2D_E_ARG, "invalid handle");
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->ctrl_host->t_max = t_max;
    CK(cudaMemcpyAsync(h->ctrl, h->ctrl_host, sizeof(Ctrl), cudaMemcpyHostToDevice, h->stream));
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
    if (h->model == kModelDdp) {
        bool handled = false;
        const int64_t r = ddp_get_array(h, name, out, capacity, &handled);
        if (handled) return r;
    }
    if (h->fused && h->tiles.slopes_in && h->p.scheme == SW2D_SCHEME_MUSCL_EVR && !h->m.flux && !h->m.lmax &&
        (std::strcmp(name, "slope_x") == 0 || std::strcmp(name, "slope_y") == 0))
        return fail(h, SW2D_E_ARG, "the fused step keeps the slopes only with the option record_fluxes or "
                                   "record_wave_speeds on");
    struct Entry {
        const char* n;
        const double* p;
        int stride, offset;
        int64_t len;
        const int* perm;
    } tab[] = {
        {"F1_int", (const double*)h->m.flux, 6, 0, h->ni, h->d_int_perm},
        {"F2_int", (const double*)h->m.flux, 6, 1, h->ni, h->d_int_perm},
        {"F3_int", (const double*)h->m.flux, 6, 2, h->ni, h->d_int_perm},
        {"s2L_int", (const double*)h->m.flux, 6, 3, h->ni, h->d_int_perm},
        {"s2R_int", (const double*)h->m.flux, 6, 4, h->ni, h->d_int_perm},
        {"F1_bnd", (const double*)h->m.bflux, 4, 0, h->nb, h->d_bnd_perm},
        {"F2_bnd", (const double*)h->m.bflux, 4, 1, h->nb, h->d_bnd_perm},
        {"F3_bnd", (const double*)h->m.bflux, 4, 2, h->nb, h->d_bnd_perm},
        {"lambda_max_int", h->m.lmax, 1, 0, h->ni, h->d_int_perm},
        {"lambda_max_bnd", h->m.lmaxb, 1, 0, h->nb, h->d_bnd_perm},
        {"slope_x", (const double*)h->m.slope, 2, 0, h->nc, h->d_cell_perm},
        {"slope_y", (const double*)h->m.slope, 2, 1, h->nc, h->d_cell_perm},
    };
    for (const Entry& e : tab) {
        if (std::strcmp(e.n, name) != 0) continue;
        if (!e.p)
            return fail(h, SW2D_E_ARG, "recorded only with the option record_wave_speeds / record_fluxes");
        if (capacity < e.len) return fail(h, SW2D_E_ARG, "output buffer too small");
        CK(cudaSetDevice(h->device));
        double* tmp = nullptr;
        CK(cudaMalloc(&tmp, std::max<int64_t>(1, e.len) * sizeof(double)));
        k_scatter_strided<<<grid_for(e.len), kBlock, 0, h->stream>>>(e.p, e.stride, e.offset, e.perm, tmp, (int)e.len);
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

// ------------------------------------------------------------------------------------------
// Reading a per-edge or per-cell array without allocating.
//
// sw2d_get_array stages the array on the device in a buffer it allocates for the call
// (cudaMalloc/cudaFree).  Some callers must not allocate once their run has started: a
// forecasting service that reserves all device memory at start-up and must not fail with
// out-of-memory in the middle of an event, or an application whose memory pool forbids
// allocations from library code.  sw2d_get_array_noalloc does the same work with a fixed
// staging array compiled into the library instead (kNoAllocMaxDoubles doubles = 8 MiB, held by
// every GPU that loads the library until the process exits).
// ------------------------------------------------------------------------------------------
constexpr int64_t kNoAllocMaxDoubles = (int64_t)1 << 20;
static __device__ __align__(256) double g_noalloc_stage[kNoAllocMaxDoubles];

namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_stage on `device`, which must be the current device.  In host
// code the name g_noalloc_stage is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress, once per device, and is cached.
int noalloc_stage(sw2d_handle* h, int device, double** out)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (device < 0 || device >= kNoAllocMaxDevices) return fail(h, SW2D_E_ARG, "device ordinal out of range");
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_stage);
        if (e != cudaSuccess || !p)
            return fail(h, SW2D_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_noalloc_ptr[device] = static_cast<double*>(p);
    }
    *out = g_noalloc_ptr[device];
    return SW2D_OK;
}

}  // namespace

}  // extern "C"

namespace sw2d {

int noalloc_prepare(sw2d_handle* h)
{
    double* stage = nullptr;
    return noalloc_stage(h, h->device, &stage);
}

}  // namespace sw2d

extern "C" {

int64_t sw2d_get_array_noalloc(sw2d_handle* h, const char* name, double* out, int64_t capacity)
{
    if (!h || !name || !out) return fail(h, SW2D_E_ARG, "invalid arguments");
    if (h->model == kModelDdp) {  // the DDP model's map outputs, computed straight into the staging array
        CK(cudaSetDevice(h->device));
        double* stage = nullptr;
        const int st = noalloc_stage(h, h->device, &stage);
        if (st) return st;
        bool handled = false;
        const int64_t r = ddp_get_array_staged(h, name, out, capacity, stage, kNoAllocMaxDoubles, &handled);
        if (handled) return r;
    }
    if (h->fused && h->tiles.slopes_in && h->p.scheme == SW2D_SCHEME_MUSCL_EVR && !h->m.flux && !h->m.lmax &&
        (std::strcmp(name, "slope_x") == 0 || std::strcmp(name, "slope_y") == 0))
        return fail(h, SW2D_E_ARG, "the fused step keeps the slopes only with the option record_fluxes or "
                                   "record_wave_speeds on");
    struct Entry {
        const char* n;
        const double* p;
        int stride, offset;
        int64_t len;
        const int* perm;
    } tab[] = {
        {"F1_int", (const double*)h->m.flux, 6, 0, h->ni, h->d_int_perm},
        {"F2_int", (const double*)h->m.flux, 6, 1, h->ni, h->d_int_perm},
        {"F3_int", (const double*)h->m.flux, 6, 2, h->ni, h->d_int_perm},
        {"s2L_int", (const double*)h->m.flux, 6, 3, h->ni, h->d_int_perm},
        {"s2R_int", (const double*)h->m.flux, 6, 4, h->ni, h->d_int_perm},
        {"F1_bnd", (const double*)h->m.bflux, 4, 0, h->nb, h->d_bnd_perm},
        {"F2_bnd", (const double*)h->m.bflux, 4, 1, h->nb, h->d_bnd_perm},
        {"F3_bnd", (const double*)h->m.bflux, 4, 2, h->nb, h->d_bnd_perm},
        {"lambda_max_int", h->m.lmax, 1, 0, h->ni, h->d_int_perm},
        {"lambda_max_bnd", h->m.lmaxb, 1, 0, h->nb, h->d_bnd_perm},
        {"slope_x", (const double*)h->m.slope, 2, 0, h->nc, h->d_cell_perm},
        {"slope_y", (const double*)h->m.slope, 2, 1, h->nc, h->d_cell_perm},
    };
    for (const Entry& e : tab) {
        if (std::strcmp(e.n, name) != 0) continue;
        if (!e.p)
            return fail(h, SW2D_E_ARG, "recorded only with the option record_wave_speeds / record_fluxes");
        if (capacity < e.len) return fail(h, SW2D_E_ARG, "output buffer too small");
        if (e.len > kNoAllocMaxDoubles)
            return fail(h, SW2D_E_ARG, std::string("sw2d_get_array_noalloc: ") + name + " has " + std::to_string(e.len) +
                                           " values, more than the fixed staging array holds (" +
                                           std::to_string(kNoAllocMaxDoubles) + "); use sw2d_get_array");
        CK(cudaSetDevice(h->device));
        double* stage = nullptr;
        const int st = noalloc_stage(h, h->device, &stage);
        if (st) return st;
        // every element of [0, len) is written by the scatter (perm is a permutation), so the
        // previous call's contents need no clearing
        if (e.len > 0) {
            k_scatter_strided<<<grid_for(e.len), kBlock, 0, h->stream>>>(e.p, e.stride, e.offset, e.perm, stage,
                                                                          (int)e.len);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(out, stage, e.len * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        }
        CK(cudaStreamSynchronize(h->stream));
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
    if (h->model == kModelDdp) return ddp_kernels_per_step(h);
    if (h->fused) return n_phases(h);
    return h->p.scheme == SW2D_SCHEME_MUSCL_EVR ? 4 : 3;
}

int sw2d_eval_math(int device, int fn, const double* x, double* y, int64_t n)
{
    sw2d_handle* h = nullptr;
    if (!x || !y || n < 0 || fn < 0 || fn > 5) return fail(h, SW2D_E_ARG, "invalid arguments");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return fail(h, SW2D_E_NO_DEVICE, "no usable CUDA device");
    CK(cudaSetDevice(device));
    double *dx = nullptr, *dy = nullptr;
    CK(cudaMalloc(&dx, std::max<int64_t>(1, n) * sizeof(double)));
    if (cudaMalloc(&dy, std::max<int64_t>(1, n) * sizeof(double)) != cudaSuccess) {
        cudaFree(dx);
        return fail(h, SW2D_E_CUDA, "cudaMalloc");
    }
    cudaError_t e = cudaMemcpy(dx, x, n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n > 0) {
        k_eval_math<<<(unsigned)((n + kBlock - 1) / kBlock), kBlock>>>(fn, dx, dy, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(y, dy, n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dy);
    if (e != cudaSuccess) return fail(h, SW2D_E_CUDA, cudaGetErrorString(e));
    return SW2D_OK;
}

int sw2d_destroy(sw2d_handle* h)
{
    if (!h) return SW2D_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    adjoint_release(h);
    assim_release(h);
    ddp_release(h);
    closure_release(h);
    result_release(h);
    for (void* p : h->allocs) cudaFree(p);
    for (void* p : h->tile_allocs) cudaFree(p);
    if (h->saved_point) cudaFree(h->saved_point);
    if (h->ctrl_host) cudaFreeHost(h->ctrl_host);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return SW2D_OK;
}

const char* sw2d_last_error(sw2d_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

}  // extern "C"
