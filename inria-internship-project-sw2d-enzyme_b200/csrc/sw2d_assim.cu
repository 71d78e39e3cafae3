// sw2d_assim.cu — the reference's porosity-assimilation engine on the GPU.
//
// The reference (class swSpE, assim/swSpE*.cpp) runs its own variant of the SP step, the "_E"
// step, records a trajectory with it, replays that trajectory at frozen time steps to evaluate
// the cost J(m), and differentiates the replay with Enzyme.  Here:
//   record   swSpE::build_checkpoint_records (assim/swSpE_checkpoint.cpp:97-455): the CFL time
//            step of the _E step (swSpE_hyp.cpp:578-638) snapped onto the next observation time,
//            the observation triggers |t - t_obs| < 1e-6 and a checkpoint every `stride` steps,
//            all on the device (the host syncs once per segment);
//   replay   ckpt_segment_E (swSpE_checkpoint.cpp:584-715) over the segments, chained, with the
//            recorded dt and boundary times; replay_trajectory_cost (:1311-1427) from the window's
//            first checkpoint or per tile;
//   gradient get_spatial_gradient_checkpointed (:722-1281): the same segment loop in reverse, each
//            segment recomputed from its checkpoint (keeping each step's state and post-balance
//            state), then the hand-written reverse of its steps; the window, the tiles (adjoint
//            reset at each tile's end), the watermark and the early stop when the adjoint blows
//            up, and the final clean-up of non-finite entries, as the reference does them.
//
// Kernels of one step (forward):
//   k_slopes (MUSCL-EVR)  the limited free-surface slopes (shared with the native step)
//   k_e_edges             per edge: _E Riemann states, fluxes, balance slots {F1 or f F1, q, r
//                         terms, factor}, and (record) the CFL contributions lambda_max * length
//   k_e_cfl               (record) per cell swept sums -> grid minimum -> dt, t_max clip, 1e-6
//                         floor, observation snap
//   k_e_update            per cell: ordered gather of its slots, flush, clamp, friction, head loss
//   k_e_advance           (record) dt, t and trigger of the step; t += dt
// Reverse of one step:
//   k_obs_rev / k_e_gauge_rev   misfit gradient when the step ends on an observation
//   k_e_update_rev        per cell: reverse of the update -> adjoint of the raw post-balance state
//   k_slopes              recomputed slopes of the step (MUSCL-EVR)
//   k_e_edges_rev         per edge: fluxes recomputed, their adjoints from both cells' post-balance
//                         adjoints, the edge factors' adjoints (-> porosity), the reverse of the
//                         flux and of the Riemann states -> per-slot contributions
//   k_e_cells_rev         per cell: ordered gather of the slot contributions
//   k_limiter_rev, k_nbr_rev    reverse of the slope limiter (MUSCL-EVR)
// All sums run in a fixed order and no floating-point atomics are used: the gradient is
// bitwise reproducible.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "sw2d_internal.cuh"
#include "sp_adjoint.cuh"
#include "spe_math.cuh"
#include "adjoint_common.cuh"

using namespace sw2d;

namespace sw2d {

struct AssimSegment {
    double t_start = 0.0;
    int64_t j0 = 0;        // index of its first step
    int64_t n = 0;         // steps
};

struct AssimState {
    // configuration (assimConfig keys)
    sw2d_assim_params prm{};
    bool configured = false;
    double t0 = 0.0;                 // start of the trajectory
    double4* st0 = nullptr;          // nc: the state at the start (swSpE::save_initial_state)
    double4* slot4 = nullptr;        // nslot: balance slots of the differentiated step
    // control
    double* d_m = nullptr;           // nc (internal numbering)
    double* d_phi = nullptr;         // nc: phi = T(m)
    double2* d_coef = nullptr;       // ni: {coefL, coefR} = w / area / phi
    double* d_coefb = nullptr;       // nb
    double norm_lo = 0.0, norm_scale = 1.0;
    // observations
    int kind = SW2D_OBS_FRAMES;
    int64_t n_obs = 0, n_gauges = 0;
    std::vector<double> obs_t;
    double* d_obs_t = nullptr;
    int* d_ident = nullptr;          // FRAMES: 0 .. nc-1
    double *d_wh = nullptr, *d_wq = nullptr;
    double *d_hobs = nullptr, *d_qobs = nullptr, *d_robs = nullptr;   // [n_obs][nc] or [n_obs][ng]
    int* d_gcell = nullptr;          // GAUGES: gauge cells, internal numbering
    int64_t n_ucells = 0;            // distinct gauge cells (reverse: one thread each)
    int *d_ucell = nullptr, *d_uoff = nullptr, *d_ulist = nullptr;
    // trajectory
    int64_t stride = 0, n_steps = 0, cap = 0;
    std::vector<AssimSegment> segs;
    std::vector<double> dt_seq, t_seq;
    std::vector<int> trig;
    double *d_dt = nullptr, *d_t = nullptr;
    double* d_cost = nullptr;        // cost of the observation a step ends on (replays)
    int* d_trig = nullptr;
    std::vector<double4*> ck;        // state at the start of each segment
    std::vector<double4*> cs;        // the same states along the replay (option assim_chained_recompute)
    bool recorded = false;
    // window (get_spatial_gradient_checkpointed)
    int64_t first = 0, truncation = -1;
    std::vector<int64_t> tiles;
    // device control of the record
    Ctrl* ctrl = nullptr;
    Ctrl* ctrl_on = nullptr;         // always-active control (replay slopes, reverse kernels)
    int* d_obs_idx = nullptr;
    // reverse sweep
    int64_t nslot = 0, ncint = 0, seg_cap = 0;
    double4* seg_st = nullptr;       // (seg_cap + 1) * nc
    double4* seg_bal = nullptr;      // seg_cap * nc
    double4 *lam = nullptr, *lamb = nullptr, *ctb = nullptr;
    double2 *cts = nullptr, *sgb = nullptr;
    double *znb = nullptr, *gzb = nullptr;
    int* mirror = nullptr;
    double *g_phi = nullptr, *g_k1 = nullptr, *g_k2 = nullptr, *g_w = nullptr;   // g_w: watermark
    double* d_part = nullptr;        // reduction partials
    double* d_out = nullptr;         // small results
    unsigned long long* d_count = nullptr;
    double* stage = nullptr;         // 3 * nc doubles for transfers
    std::vector<void*> fixed_allocs, obs_allocs, traj_allocs, seg_allocs;
};

}  // namespace sw2d

namespace {

constexpr int kEUnroll = 4;

struct EView {
    const double* phi;       // nc
    const double2* coef;     // ni {coefL, coefR}
    const double* coefb;     // nb
    const double* dtp;       // the dt of the MUSCL-EVR reconstruction
    const double* tp;        // the time of the boundary values
};

// ------------------------------------------------------------------------------------------
// control
// ------------------------------------------------------------------------------------------

// phi = T(m) (swSpE::phi_correct, assim/swSpE.h:59-75)
__global__ void k_e_phi(const double* __restrict__ m, double* phi, int n, int kind, double lambda, double lo,
                        double scale)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) phi[i] = spe::phi_correct(kind, m[i], lambda, lo, scale);
}

// swSpE::computeEdgeFactors_E (assim/swSpE_hyp.cpp:277-333): w / area / phi, 0 where phi <= phi_min
__global__ void k_e_coef(DevMesh m, const double* __restrict__ phi, double2* coef, double* coefb)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m.ni) {
        const int2 lr = m.lr[i];
        const double w = m.len[i];
        const double pL = phi[lr.x], pR = phi[lr.y];
        const double aL = m.area[lr.x], aR = m.area[lr.y];
        const double sL = (pL > m.phi_min) ? pL : m.phi_min, sR = (pR > m.phi_min) ? pR : m.phi_min;
        coef[i] = make_double2((pL > m.phi_min) ? (w / aL / sL) : 0.0, (pR > m.phi_min) ? (w / aR / sR) : 0.0);
    } else if (i < m.ni + m.nb) {
        const int e = i - m.ni;
        const int c = m.bcell[e];
        const double p = phi[c];
        const double s = (p > m.phi_min) ? p : m.phi_min;
        coefb[e] = (p > m.phi_min) ? (m.bgeo[e].z / m.area[c] / s) : 0.0;
    }
}

// z = h + z_b of a state array
__global__ void k_refresh_z_e(double4* st, const double* __restrict__ zbv, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) st[i].w = st[i].x + zbv[i];
}

// ------------------------------------------------------------------------------------------
// forward step
// ------------------------------------------------------------------------------------------
template <int kScheme>
__device__ __forceinline__ void e_sides(const DevMesh& m, int e, int a, int b, double2 n, const double4& sa,
                                        const double4& sb, const double4& ca, const double4& cb, double dt,
                                        spe::ESide& SL, spe::ESide& SR)
{
    if (kScheme == SW2D_SCHEME_GODUNOV) {
        SL = spe::god_side(sa.x, sa.y, sa.z, ca.x, ca.y, n.x, n.y, m.h_min);
        SR = spe::god_side(sb.x, sb.y, sb.z, cb.x, cb.y, n.x, n.y, m.h_min);
    } else {
        const double4 d = ld(&m.emc[e]);
        const double2 ga = ld(&m.slope[a]), gb = ld(&m.slope[b]);
        SL = spe::evr_side(true, sa.x, sa.y, sa.z, ca.x, ca.y, sa.w, ga.x, ga.y, d.x, d.y, n.x, n.y, dt);
        SR = spe::evr_side(false, sb.x, sb.y, sb.z, cb.x, cb.y, sb.w, gb.x, gb.y, d.z, d.w, n.x, n.y, dt);
    }
}

template <int kScheme>
__device__ __forceinline__ spe::ESide e_bnd_side(const DevMesh& m, const double4& s, const double4& cs, double nx,
                                                 double ny)
{
    return (kScheme == SW2D_SCHEME_GODUNOV) ? spe::god_side(s.x, s.y, s.z, cs.x, cs.y, nx, ny, m.h_min)
                                            : spe::evr_bnd_side(s.x, s.y, s.z, cs.x, cs.y, nx, ny);
}

__device__ __forceinline__ double e_bc_value(const DevMesh& m, int e, double t, int* type)
{
    const int k = ld(&m.bbc[e]);
    const long long o0 = ld(&m.bcoff[k]), o1 = ld(&m.bcoff[k + 1]);
    *type = ld(&m.bctype[k]);
    return spe::bc_value_e(m.bctimes + o0, m.bcvals + o0, o1 - o0, t);
}

// hypComputeLRStates_E + hypComputeFluxes_E (assim/swSpE_hyp.cpp:396-505), the dt-free products of
// hypComputeBalance_E (:336-394) into the slots, and (kRecord) the CFL contributions of
// hypComputeTimeStep_E (:590-607): lambda_max * length for a wet cell, 0 otherwise.
template <int kScheme, bool kRecord>
__global__ void __launch_bounds__(kBlock) k_e_edges(DevMesh m, EView v)
{
    if (kRecord && !step_active(m.ctrl)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m.ni) {
        const int e = i;
        const int2 lr = ld(&m.lr[e]);
        const int a = lr.x, b = lr.y;
        const double2 n = ld(&m.nxy[e]);
        const double4 sa = ld(&m.st[a]), sb = ld(&m.st[b]);
        const double4 ca = ld(&m.cst[a]), cb = ld(&m.cst[b]);
        spe::ESide SL, SR;
        e_sides<kScheme>(m, e, a, b, n, sa, sb, ca, cb, (kScheme == SW2D_SCHEME_GODUNOV) ? 0.0 : *v.dtp, SL, SR);
        const int2 sl = ld(&m.eslot[e]);
        if (kRecord) {
            double lm;
            if (kScheme == SW2D_SCHEME_GODUNOV) {
                lm = max4(fabs(SL.lm), fabs(SL.lp), fabs(SR.lm), fabs(SR.lp));
            } else {
                const double m1 = smax(fabs(SL.lm), fabs(SL.lp)), m2 = smax(fabs(SR.lm), fabs(SR.lp));
                lm = smax(m1, m2);
            }
            const double lw = lm * ld(&m.len[e]);
            m.slot_w[sl.x] = (sa.x > m.h_min) ? lw : 0.0;
            m.slot_w[sl.y] = (sb.x > m.h_min) ? lw : 0.0;
        }
        const double phiL = ld(&v.phi[a]), phiR = ld(&v.phi[b]);
        const spe::EFlux f = spe::hllc(ca.y, cb.y, phiL, phiR, ca.x, cb.x, SL, SR, m.h_min, m.phi_min);
        const double2 cf = ld(&v.coef[e]);
        const double nx = n.x, ny = n.y;
        {
            const double c = cf.x;
            const double f1 = -c, f2F2 = -c * nx, f2F3 = +c * ny, f2S2 = +c * nx;
            const double f3F2 = -c * ny, f3F3 = -c * nx, f3S2 = +c * ny;
            m.slot4[sl.x] = make_double4(f.f1, f2F2 * f.f2 + f2S2 * f.sl + f2F3 * f.f3,
                                        f3F2 * f.f2 + f3S2 * f.sl + f3F3 * f.f3, f1);
        }
        {
            const double c = cf.y;
            const double f1 = +c, f2F2 = +c * nx, f2F3 = -c * ny, f2S2 = +c * nx;
            const double f3F2 = +c * ny, f3F3 = +c * nx, f3S2 = +c * ny;
            m.slot4[sl.y] = make_double4(f.f1, f2F2 * f.f2 + f2S2 * f.sr + f2F3 * f.f3,
                                        f3F2 * f.f2 + f3S2 * f.sr + f3F3 * f.f3, f1);
        }
    } else if (i < m.ni + m.nb) {
        const int e = i - m.ni;
        const int c = ld(&m.bcell[e]);
        const double4 s = ld(&m.st[c]);
        const double4 cs = ld(&m.cst[c]);
        const double4 g = ld(&m.bgeo[e]);
        const spe::ESide S = e_bnd_side<kScheme>(m, s, cs, g.x, g.y);
        const int sb = ld(&m.bslot[e]);
        if (kRecord) {
            const double lm = (kScheme == SW2D_SCHEME_GODUNOV) ? smax(fabs(S.lp), fabs(S.lm)) : smax(fabs(S.lm), fabs(S.lp));
            m.slot_w[sb] = (s.x > m.h_min) ? lm * g.z : 0.0;
        }
        int type;
        const double bcv = e_bc_value(m, e, *v.tp, &type);
        const spe::EBndFlux F = spe::boundary_flux(cs.y, ld(&v.phi[c]), cs.x, S, type, bcv, m.h_min, m.phi_min);
        const double cf = ld(&v.coefb[e]), nx = g.x, ny = g.y;
        const double fa = +cf, f2F2 = +cf * nx, f2F3 = -cf * ny, f2S2 = +cf * nx;
        const double f3F2 = +cf * ny, f3F3 = +cf * nx, f3S2 = +cf * ny;
        const double s2 = 0.0;  // source_right of hypBoundaryFlux_E (swSpE_hyp.cpp:167)
        m.slot4[sb] = make_double4(fa * F.f1, f2F2 * F.f2 + f2S2 * s2 + f2F3 * F.f3,
                                  f3F2 * F.f2 + f3S2 * s2 + f3F3 * F.f3, 1.0);
    }
}

__device__ __forceinline__ double e_min_keep(double a, double b) { return (b < a) ? b : a; }

// hypComputeTimeStep_E (assim/swSpE_hyp.cpp:578-638) and the observation snap of
// build_checkpoint_records (swSpE_checkpoint.cpp:228-250), on the device.
__global__ void __launch_bounds__(kBlock) k_e_cfl(DevMesh m, const double* __restrict__ obs_t, const int* obs_idx,
                                                  int n_obs)
{
    Ctrl* ctrl = m.ctrl;
    if (!step_active(ctrl)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) ctrl->go = 0;
        return;
    }
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double best = m.dt_max;
    if (c < m.nc) {
        const int k0 = ld(&m.coff[c].y), k1 = ld(&m.coff[c + 1].y);
        double sw = 0.0;
        for (int k = k0; k < k1; k++) sw += ld(&m.slot_w[k]);
        const double den = smax(sw, kSmallReal);
        const double x = m.cfl_max * (ld(&m.area[c]) / den);
        if (x < best) best = x;
    }
    for (int off = 16; off > 0; off >>= 1) best = e_min_keep(best, __shfl_down_sync(0xffffffffu, best, off));
    __shared__ double wmin[kBlock / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) wmin[wid] = best;
    __syncthreads();
    if (wid == 0) {
        best = (lane < kBlock / 32) ? wmin[lane] : m.dt_max;
        for (int off = 16; off > 0; off >>= 1) best = e_min_keep(best, __shfl_down_sync(0xffffffffu, best, off));
        if (lane == 0) {
            m.part[blockIdx.x] = best;
            __threadfence();
            const unsigned done = atomicAdd(&ctrl->blocks_done, 1u);
            last = (done == gridDim.x - 1);
        }
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double b2 = m.dt_max;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) b2 = e_min_keep(b2, ((volatile double*)m.part)[i]);
    for (int off = 16; off > 0; off >>= 1) b2 = e_min_keep(b2, __shfl_down_sync(0xffffffffu, b2, off));
    if (lane == 0) wmin[wid] = b2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double dt = m.dt_max;
        for (int w = 0; w < kBlock / 32; w++)
            if (wmin[w] < dt) dt = wmin[w];
        const double t = ctrl->t, t_max = ctrl->t_max;
        if ((t + dt) > t_max) dt = t_max - t;
        if (dt < spe::kDtFloor) dt = spe::kDtFloor;
        double dt_target = m.dt_max;
        const int k = *obs_idx;
        if (k < n_obs) {
            const double to = obs_t[k] - t;
            if (to - 10e-6 > 0.0 && to < dt_target) dt_target = to;
        }
        double cur = (dt < dt_target) ? dt : dt_target;
        if ((t + cur) > t_max) cur = t_max - t;
        if (cur < spe::kDtFloor) cur = spe::kDtFloor;
        ctrl->dt = cur;
        ctrl->go = 1;
        ctrl->blocks_done = 0;
    }
}

// hypComputeBalance_E (swSpE_hyp.cpp:336-394) from the cell's slots in the reference's order,
// then the dry-cell floor, friction and head loss (swSpE_checkpoint.cpp:675-702).
template <int kFriction, bool kHeadLoss, bool kStore>
__global__ void __launch_bounds__(kBlock) k_e_update(DevMesh m, const double* __restrict__ dtp, const int* go)
{
    if (go && !*go) return;
    const double dt = *dtp;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const double4 s0 = m.st[c];
    double hh = s0.x, qq = s0.y, rr = s0.z;
    const int k0 = ld(&m.coff[c].y), k1 = ld(&m.coff[c + 1].y);
    if (k1 - k0 <= kEUnroll) {
        double4 v[kEUnroll];
#pragma unroll
        for (int i = 0; i < kEUnroll; i++)
            if (i < k1 - k0) v[i] = m.slot4[k0 + i];
#pragma unroll
        for (int i = 0; i < kEUnroll; i++)
            if (i < k1 - k0) {
                hh += v[i].w * (v[i].x * dt);
                qq += v[i].y * dt;
                rr += v[i].z * dt;
            }
    } else {
        for (int k = k0; k < k1; k++) {
            const double4 v = m.slot4[k];
            hh += v.w * (v.x * dt);
            qq += v.y * dt;
            rr += v.z * dt;
        }
    }
    if (kStore) m.bal[c] = make_double4(hh, qq, rr, 0.0);
    spe::ECellParams p;
    p.friction = kFriction != SW2D_FRICTION_NONE;
    p.head_loss = kHeadLoss;
    p.h_min = m.h_min;
    if (kFriction != SW2D_FRICTION_NONE) {
        const double4 fr = ld(&m.fric[c]);
        p.k1 = fr.x;
        p.k2 = fr.y;
        p.ca = fr.z;
        p.sa = fr.w;
    }
    if (kHeadLoss) {
        const double4 hl = ld(&m.hla[c]);
        const double2 cs = ld(&m.hlb[c]);
        p.hs = hl.x;
        p.hk1 = hl.y;
        p.hk2 = hl.z;
        p.hca = cs.x;
        p.hsa = cs.y;
    }
    spe::cell_update(hh, qq, rr, p, dt);
    m.st[c] = make_double4(hh, qq, rr, hh + ld(&m.zbv[c]));
}

// The step's bookkeeping in build_checkpoint_records (swSpE_checkpoint.cpp:315-377): keep dt and
// t of the step, t += dt, pass observations already overtaken, trigger the one landed on.
__global__ void k_e_advance(Ctrl* ctrl, int* obs_idx, const double* __restrict__ obs_t, int n_obs, double* dt_seq,
                            double* t_seq, int* trig, long long cap)
{
    if (!ctrl->go) return;
    const long long j = ctrl->steps;
    const double t0 = ctrl->t, dt = ctrl->dt;
    const double t = t0 + dt;
    int k = *obs_idx;
    while (k < n_obs && t > obs_t[k] + 1e-6) k++;
    int tr = -1;
    if (k < n_obs && fabs(t - obs_t[k]) < 1e-6) {
        tr = k;
        k++;
    }
    if (j < cap) {
        dt_seq[j] = dt;
        t_seq[j] = t0;
        trig[j] = tr;
    }
    *obs_idx = k;
    ctrl->t = t;
    ctrl->steps = j + 1;
    ctrl->go = 0;
}

// the cost of an observation: per-block partials (fixed tree), then one thread adds them in
// block order and divides by the number of frames when costs are normalised
__global__ void k_e_obs_finish(const double* part, int nblocks, double divisor, double* out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < nblocks; b++) s += part[b];
        *out = (divisor > 0.0) ? s / divisor : s;
    }
}

// ------------------------------------------------------------------------------------------
// reverse step
// ------------------------------------------------------------------------------------------

// gauge misfit gradient, one thread per distinct gauge cell (its gauges in order)
__global__ void k_e_gauge_rev(const int* __restrict__ ucell, const int* __restrict__ uoff, const int* __restrict__ ulist,
                              const double* __restrict__ w, const double* __restrict__ hobs, const double4* st,
                              double4* lam, double scale, int n)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    const int c = ucell[u];
    const double h = st[c].x;
    double g = 0.0;
    for (int k = uoff[u]; k < uoff[u + 1]; k++) {
        const int gi = ulist[k];
        g += 2.0 * w[gi] * (h - hobs[gi]) * scale;
    }
    lam[c].x += g;
}

template <int kFriction, bool kHeadLoss>
__global__ void __launch_bounds__(kBlock) k_e_update_rev(DevMesh m, const double4* __restrict__ bal, double4* lam,
                                                         double4* lamb, double* gk1, double* gk2, double dt)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const double4 l = lam[c];
    const double4 b = bal[c];
    spe::ECellParams p;
    p.friction = kFriction != SW2D_FRICTION_NONE;
    p.head_loss = kHeadLoss;
    p.h_min = m.h_min;
    if (kFriction != SW2D_FRICTION_NONE) {
        const double4 fr = ld(&m.fric[c]);
        p.k1 = fr.x;
        p.k2 = fr.y;
        p.ca = fr.z;
        p.sa = fr.w;
    }
    if (kHeadLoss) {
        const double4 hl = ld(&m.hla[c]);
        const double2 cs = ld(&m.hlb[c]);
        p.hs = hl.x;
        p.hk1 = hl.y;
        p.hk2 = hl.z;
        p.hca = cs.x;
        p.hsa = cs.y;
    }
    double hb = l.x, qb = l.y, rb = l.z, k1b = 0.0, k2b = 0.0;
    spe::cell_update_rev(b.x, b.y, b.z, p, dt, hb, qb, rb, k1b, k2b);
    if (kFriction != SW2D_FRICTION_NONE) {
        gk1[c] += k1b;
        gk2[c] += k2b;
    }
    const double4 o = make_double4(hb, qb, rb, 0.0);
    lamb[c] = o;
    lam[c] = o;
}

// Per edge: the adjoints of its fluxes and factors from the post-balance adjoints of its cells
// (the balance adds w (F1 dt), (...) dt to each side), the factors' adjoints to the porosity
// (coef = w / area / phi), then the reverse of the flux and of both Riemann states.  Each side's
// contribution goes to its slot: ctb = {h, q, r, phi} adjoints of that cell, cts = its slope's.
template <int kScheme>
__global__ void __launch_bounds__(kBlock) k_e_edges_rev(DevMesh m, EView v, const double4* __restrict__ lamb,
                                                        double4* ctb, double2* cts, double dt, int ieee)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m.ni) {
        const int e = i;
        const int2 lr = ld(&m.lr[e]);
        const int a = lr.x, b = lr.y;
        const double2 n = ld(&m.nxy[e]);
        const double4 sa = ld(&m.st[a]), sb = ld(&m.st[b]);
        const double4 ca = ld(&m.cst[a]), cb = ld(&m.cst[b]);
        spe::ESide SL, SR;
        e_sides<kScheme>(m, e, a, b, n, sa, sb, ca, cb, dt, SL, SR);
        const double phiL = ld(&v.phi[a]), phiR = ld(&v.phi[b]);
        const spe::EFlux f = spe::hllc(ca.y, cb.y, phiL, phiR, ca.x, cb.x, SL, SR, m.h_min, m.phi_min);
        const double4 lL = ld(&lamb[a]), lR = ld(&lamb[b]);
        const double2 cf = ld(&v.coef[e]);
        const double cL = cf.x, cR = cf.y, nx = n.x, ny = n.y;
        spe::EFlux fb;
        fb.f1 = dt * (-cL * lL.x + cR * lR.x);
        fb.f2 = dt * (cL * (-nx * lL.y - ny * lL.z) + cR * (nx * lR.y + ny * lR.z));
        fb.f3 = dt * (cL * (ny * lL.y - nx * lL.z) + cR * (-ny * lR.y + nx * lR.z));
        fb.sl = dt * cL * (nx * lL.y + ny * lL.z);
        fb.sr = dt * cR * (nx * lR.y + ny * lR.z);
        const double cLb = dt * (-f.f1 * lL.x + (-nx * f.f2 + nx * f.sl + ny * f.f3) * lL.y +
                                 (-ny * f.f2 + ny * f.sl - nx * f.f3) * lL.z);
        const double cRb = dt * (f.f1 * lR.x + (nx * f.f2 + nx * f.sr - ny * f.f3) * lR.y +
                                 (ny * f.f2 + ny * f.sr + nx * f.f3) * lR.z);
        double pLb = (phiL > m.phi_min) ? -cLb * cL / phiL : 0.0;
        double pRb = (phiR > m.phi_min) ? -cRb * cR / phiR : 0.0;
        spe::ESideBar Lb{0, 0, 0, 0, 0}, Rb{0, 0, 0, 0, 0};
        spe::hllc_rev(ca.y, cb.y, phiL, phiR, ca.x, cb.x, SL, SR, m.h_min, m.phi_min, fb, pLb, pRb, Lb, Rb);
        const int2 sl = ld(&m.eslot[e]);
        double hb = 0, qb = 0, rb = 0;
        if (kScheme == SW2D_SCHEME_GODUNOV) {
            spe::god_side_rev(sa.x, sa.y, sa.z, ca.y, nx, ny, m.h_min, Lb, hb, qb, rb, ieee);
            ctb[sl.x] = make_double4(hb, qb, rb, pLb);
            hb = qb = rb = 0.0;
            spe::god_side_rev(sb.x, sb.y, sb.z, cb.y, nx, ny, m.h_min, Rb, hb, qb, rb, ieee);
            ctb[sl.y] = make_double4(hb, qb, rb, pRb);
        } else {
            const double4 d = ld(&m.emc[e]);
            const double2 ga = ld(&m.slope[a]), gb = ld(&m.slope[b]);
            double zcb = 0, sxb = 0, syb = 0;
            spe::evr_side_rev(true, sa.x, sa.y, sa.z, ca.x, ca.y, sa.w, ga.x, ga.y, d.x, d.y, nx, ny, dt, Lb, hb, qb, rb,
                              zcb, sxb, syb, ieee);
            ctb[sl.x] = make_double4(hb + zcb, qb, rb, pLb);
            cts[sl.x] = make_double2(sxb, syb);
            hb = qb = rb = zcb = sxb = syb = 0.0;
            spe::evr_side_rev(false, sb.x, sb.y, sb.z, cb.x, cb.y, sb.w, gb.x, gb.y, d.z, d.w, nx, ny, dt, Rb, hb, qb, rb,
                              zcb, sxb, syb, ieee);
            ctb[sl.y] = make_double4(hb + zcb, qb, rb, pRb);
            cts[sl.y] = make_double2(sxb, syb);
        }
    } else if (i < m.ni + m.nb) {
        const int e = i - m.ni;
        const int c = ld(&m.bcell[e]);
        const double4 s = ld(&m.st[c]);
        const double4 cs = ld(&m.cst[c]);
        const double4 g = ld(&m.bgeo[e]);
        const spe::ESide S = e_bnd_side<kScheme>(m, s, cs, g.x, g.y);
        int type;
        const double bcv = e_bc_value(m, e, *v.tp, &type);
        const double phi = ld(&v.phi[c]);
        const spe::EBndFlux F = spe::boundary_flux(cs.y, phi, cs.x, S, type, bcv, m.h_min, m.phi_min);
        const double4 l = ld(&lamb[c]);
        const double cf = ld(&v.coefb[e]), nx = g.x, ny = g.y;
        const double f1b = cf * dt * l.x;
        const double f2b = dt * cf * (nx * l.y + ny * l.z);
        const double f3b = dt * cf * (-ny * l.y + nx * l.z);
        const double cfb = dt * (F.f1 * l.x + (nx * F.f2 - ny * F.f3) * l.y + (ny * F.f2 + nx * F.f3) * l.z);
        double pb = (phi > m.phi_min) ? -cfb * cf / phi : 0.0;
        spe::ESideBar Sb{0, 0, 0, 0, 0};
        spe::boundary_flux_rev(cs.y, phi, cs.x, S, type, bcv, m.h_min, m.phi_min, f1b, f2b, f3b, pb, Sb);
        double hb = 0, qb = 0, rb = 0;
        if (kScheme == SW2D_SCHEME_GODUNOV) spe::god_side_rev(s.x, s.y, s.z, cs.y, nx, ny, m.h_min, Sb, hb, qb, rb, ieee);
        else spe::evr_bnd_side_rev(s.x, s.y, s.z, cs.y, nx, ny, Sb, hb, qb, rb, ieee);
        const int sb = ld(&m.bslot[e]);
        ctb[sb] = make_double4(hb, qb, rb, pb);
        if (kScheme != SW2D_SCHEME_GODUNOV) cts[sb] = make_double2(0.0, 0.0);
    }
}

// ordered gather of the slot contributions of each cell
template <bool kMuscl>
__global__ void __launch_bounds__(kBlock) k_e_cells_rev(DevMesh m, double4* lam, const double4* __restrict__ ctb,
                                                        const double2* __restrict__ cts, double* gphi, double2* sgb)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const int k0 = ld(&m.coff[c].y), k1 = ld(&m.coff[c + 1].y);
    double4 l = lam[c];
    double gp = 0.0, sx = 0.0, sy = 0.0;
    for (int k = k0; k < k1; k++) {
        const double4 v = ld(&ctb[k]);
        l.x += v.x;
        l.y += v.y;
        l.z += v.z;
        gp += v.w;
        if (kMuscl) {
            const double2 s = ld(&cts[k]);
            sx += s.x;
            sy += s.y;
        }
    }
    lam[c] = l;
    gphi[c] += gp;
    if (kMuscl) sgb[c] = make_double2(sx, sy);
}

// sum of squares of the h adjoint: per-block partials in a fixed tree
__global__ void __launch_bounds__(kBlock) k_e_norm2(const double4* __restrict__ lam, int n, double* part)
{
    __shared__ double sh[kBlock];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double x = lam[i].x;
        acc += x * x;
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kBlock / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// dJ/dm = dJ/dphi * dphi/dm, then the reference's clean-up (swSpE_checkpoint.cpp:1181-1210):
// non-finite -> 0 (counts[0]); with mask_wall, phi <= phi_min -> 0 (counts[1]).  The friction
// and state adjoints are cleaned the same way (counts[2]).
__global__ void k_e_finish(const double* __restrict__ gphi, const double* __restrict__ mv, const double* __restrict__ phi,
                           double* gm, double* gk1, double* gk2, double4* lam, int n, int kind, double lambda,
                           double scale, int mask_wall, double phi_min, unsigned long long* counts)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double g = gphi[i] * spe::dphi_dm(kind, mv[i], lambda, scale);
    if (!isfinite(g)) {
        g = 0.0;
        atomicAdd(counts, 1ull);
    } else if (mask_wall && !(phi[i] > phi_min)) {
        g = 0.0;
        atomicAdd(counts + 1, 1ull);
    }
    gm[i] = g;
    unsigned long long other = 0;
    if (!isfinite(gk1[i])) gk1[i] = 0.0, other++;
    if (!isfinite(gk2[i])) gk2[i] = 0.0, other++;
    double4 l = lam[i];
    if (!isfinite(l.x)) l.x = 0.0, other++;
    if (!isfinite(l.y)) l.y = 0.0, other++;
    if (!isfinite(l.z)) l.z = 0.0, other++;
    lam[i] = l;
    if (other) atomicAdd(counts + 2, other);
}

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
template <class T>
int dev_upload_list(sw2d_handle* h, std::vector<void*>& list, const std::vector<T>& v, T** out)
{
    int rc = adj_alloc(h, list, v.size(), out);
    if (rc) return rc;
    if (!v.empty()) CK(cudaMemcpyAsync(*out, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, h->stream));
    return SW2D_OK;
}

AssimState* ensure_state(sw2d_handle* h)
{
    if (!h->assim) h->assim = new AssimState();
    return h->assim;
}

DevMesh view_with(sw2d_handle* h, Ctrl* ctrl)
{
    DevMesh m = h->m;
    m.ctrl = ctrl;
    m.slot4 = h->assim ? h->assim->slot4 : nullptr;
    return m;
}

int fixed_buffers(sw2d_handle* h)
{
    AssimState* a = h->assim;
    if (!a->fixed_allocs.empty()) return SW2D_OK;
    int2 last{0, 0};
    CK(cudaMemcpyAsync(&last, h->m.coff + h->nc, sizeof(int2), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    a->ncint = last.x;
    a->nslot = last.y;
    const int64_t nc = h->nc;
    auto& L = a->fixed_allocs;
    int rc = SW2D_OK;
    if ((rc = adj_alloc(h, L, nc, &a->st0)) || (rc = adj_alloc(h, L, nc, &a->d_m)) || (rc = adj_alloc(h, L, nc, &a->d_phi)) ||
        (rc = adj_alloc(h, L, h->ni, &a->d_coef)) || (rc = adj_alloc(h, L, h->nb, &a->d_coefb)) ||
        (rc = adj_alloc(h, L, 1, &a->ctrl)) || (rc = adj_alloc(h, L, 1, &a->ctrl_on)) ||
        (rc = adj_alloc(h, L, 1, &a->d_obs_idx)) || (rc = adj_alloc(h, L, nc, &a->lam)) ||
        (rc = adj_alloc(h, L, nc, &a->lamb)) || (rc = adj_alloc(h, L, a->nslot, &a->ctb)) ||
        (rc = adj_alloc(h, L, a->nslot, &a->cts)) || (rc = adj_alloc(h, L, nc, &a->sgb)) ||
        (rc = adj_alloc(h, L, a->ncint, &a->znb)) || (rc = adj_alloc(h, L, nc, &a->gzb)) ||
        (rc = adj_alloc(h, L, a->ncint, &a->mirror)) || (rc = adj_alloc(h, L, nc, &a->g_phi)) ||
        (rc = adj_alloc(h, L, nc, &a->g_k1)) || (rc = adj_alloc(h, L, nc, &a->g_k2)) ||
        (rc = adj_alloc(h, L, nc, &a->g_w)) || (rc = adj_alloc(h, L, kCostBlocks, &a->d_part)) ||
        (rc = adj_alloc(h, L, 8, &a->d_out)) || (rc = adj_alloc(h, L, 4, &a->d_count)) ||
        (rc = adj_alloc(h, L, 3 * nc, &a->stage)) || (rc = adj_alloc(h, L, a->nslot, &a->slot4)))
        return rc;
    Ctrl on{};
    on.t = 0.0;
    on.t_max = 1.0;
    CK(cudaMemcpyAsync(a->ctrl_on, &on, sizeof(Ctrl), cudaMemcpyHostToDevice, h->stream));
    if (nc > 0) k_mirror<<<grid_for(nc), kBlock, 0, h->stream>>>(h->m.coff, h->m.cint, a->mirror, (int)nc);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    return SW2D_OK;
}

// m (caller numbering, host) -> d_m, phi, edge factors.  In the normalize mode, `bounds`
// first sets the bounds to those of m over all cells (update_phi_norm_bounds,
// swSpE_core.cpp:229-266, with every cell free), as the reference does before a record; a replay
// keeps the recorded bounds.
int set_control(sw2d_handle* h, const double* m_host, bool bounds)
{
    AssimState* a = h->assim;
    const int64_t nc = h->nc;
    if (bounds && a->prm.phi_transform == SW2D_PHI_NORMALIZE) {
        double lo = HUGE_VAL, hi = -HUGE_VAL;
        for (int64_t i = 0; i < nc; i++) {
            lo = std::min(lo, m_host[i]);
            hi = std::max(hi, m_host[i]);
        }
        if (hi - lo < 1e-12) {  // (quasi) uniform map: phi = m
            a->norm_lo = 0.0;
            a->norm_scale = 1.0;
        } else {
            a->norm_lo = lo;
            a->norm_scale = 1.0 / (hi - lo);
        }
    }
    CK(cudaMemcpyAsync(a->stage, m_host, nc * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    k_gather_component<<<grid_for(nc), kBlock, 0, h->stream>>>(a->stage, h->d_cell_perm, a->d_m, 1, 0, (int)nc);
    k_e_phi<<<grid_for(nc), kBlock, 0, h->stream>>>(a->d_m, a->d_phi, (int)nc, a->prm.phi_transform, a->prm.lambda_tanh,
                                                      a->norm_lo, a->norm_scale);
    const int64_t ne = h->ni + h->nb;
    if (ne > 0) k_e_coef<<<grid_for(ne), kBlock, 0, h->stream>>>(h->m, a->d_phi, a->d_coef, a->d_coefb);
    CK(cudaGetLastError());
    return SW2D_OK;
}

EView eview(const AssimState* a, const double* dtp, const double* tp)
{
    EView v;
    v.phi = a->d_phi;
    v.coef = a->d_coef;
    v.coefb = a->d_coefb;
    v.dtp = dtp;
    v.tp = tp;
    return v;
}

template <bool kRecord>
void launch_edges(sw2d_handle* h, const DevMesh& m, const EView& v)
{
    const unsigned g = grid_for(h->ni + h->nb);
    if (g == 0) return;
    if (h->p.scheme == SW2D_SCHEME_GODUNOV) k_e_edges<SW2D_SCHEME_GODUNOV, kRecord><<<g, kBlock, 0, h->stream>>>(m, v);
    else k_e_edges<SW2D_SCHEME_MUSCL_EVR, kRecord><<<g, kBlock, 0, h->stream>>>(m, v);
}

template <int kF>
void launch_update_f(sw2d_handle* h, const DevMesh& m, const double* dtp, const int* go, bool store)
{
    const unsigned g = grid_for(h->nc);
    if (h->p.singular_head_loss) {
        if (store) k_e_update<kF, true, true><<<g, kBlock, 0, h->stream>>>(m, dtp, go);
        else k_e_update<kF, true, false><<<g, kBlock, 0, h->stream>>>(m, dtp, go);
    } else {
        if (store) k_e_update<kF, false, true><<<g, kBlock, 0, h->stream>>>(m, dtp, go);
        else k_e_update<kF, false, false><<<g, kBlock, 0, h->stream>>>(m, dtp, go);
    }
}

// The _E friction is sourceFrictionStrickler_E whenever a friction law is set: one kernel form.
void launch_update(sw2d_handle* h, const DevMesh& m, const double* dtp, const int* go, bool store)
{
    if (h->p.friction != SW2D_FRICTION_NONE) launch_update_f<SW2D_FRICTION_STRICKLER>(h, m, dtp, go, store);
    else launch_update_f<SW2D_FRICTION_NONE>(h, m, dtp, go, store);
}

void launch_update_rev(sw2d_handle* h, const DevMesh& m, const double4* bal, double dt)
{
    AssimState* a = h->assim;
    const unsigned g = grid_for(h->nc);
    const bool fr = h->p.friction != SW2D_FRICTION_NONE, hl = h->p.singular_head_loss != 0;
    if (fr && hl) k_e_update_rev<SW2D_FRICTION_STRICKLER, true><<<g, kBlock, 0, h->stream>>>(m, bal, a->lam, a->lamb, a->g_k1, a->g_k2, dt);
    else if (fr) k_e_update_rev<SW2D_FRICTION_STRICKLER, false><<<g, kBlock, 0, h->stream>>>(m, bal, a->lam, a->lamb, a->g_k1, a->g_k2, dt);
    else if (hl) k_e_update_rev<SW2D_FRICTION_NONE, true><<<g, kBlock, 0, h->stream>>>(m, bal, a->lam, a->lamb, a->g_k1, a->g_k2, dt);
    else k_e_update_rev<SW2D_FRICTION_NONE, false><<<g, kBlock, 0, h->stream>>>(m, bal, a->lam, a->lamb, a->g_k1, a->g_k2, dt);
}

int64_t obs_width(const AssimState* a, const sw2d_handle* h)
{
    return a->kind == SW2D_OBS_FRAMES ? h->nc : a->n_gauges;
}

ObsView make_view(const AssimState* a, const sw2d_handle* h, int k)
{
    const int64_t w = obs_width(a, h);
    ObsView o;
    o.pts = a->kind == SW2D_OBS_FRAMES ? a->d_ident : a->d_gcell;
    o.wh = a->d_wh;
    o.wq = a->kind == SW2D_OBS_FRAMES ? a->d_wq : nullptr;
    o.hobs = a->d_hobs + (size_t)k * w;
    o.qobs = a->d_qobs ? a->d_qobs + (size_t)k * w : nullptr;
    o.robs = a->d_robs ? a->d_robs + (size_t)k * w : nullptr;
    o.n = (int)w;
    o.scale = (a->prm.cost_normalize && a->n_obs > 0) ? 1.0 / (double)a->n_obs : 1.0;
    o.wdh = a->kind == SW2D_OBS_GAUGES;
    return o;
}

// cost of observation k on state st into d_out[slot]
void cost_at(sw2d_handle* h, int k, const double4* st, double* out)
{
    AssimState* a = h->assim;
    const ObsView o = make_view(a, h, k);
    const int nb = std::max(1, std::min(kCostBlocks, (int)grid_for(o.n)));
    k_obs_cost<<<nb, kBlock, 0, h->stream>>>(o, st, a->d_part);
    const double div = (a->prm.cost_normalize && a->n_obs > 0) ? (double)a->n_obs : 0.0;
    k_e_obs_finish<<<1, 32, 0, h->stream>>>(a->d_part, nb, div, out);
}

void obs_rev_at(sw2d_handle* h, int k, const double4* st)
{
    AssimState* a = h->assim;
    const ObsView o = make_view(a, h, k);
    if (a->kind == SW2D_OBS_FRAMES) {
        if (o.n > 0) k_obs_rev<<<grid_for(o.n), kBlock, 0, h->stream>>>(o, st, a->lam);
    } else if (a->n_ucells > 0) {
        k_e_gauge_rev<<<grid_for(a->n_ucells), kBlock, 0, h->stream>>>(a->d_ucell, a->d_uoff, a->d_ulist, a->d_wh, o.hobs, st,
                                                                      a->lam, o.scale, (int)a->n_ucells);
    }
}

void free_steps(AssimState* a)
{
    if (a->d_dt) cudaFree(a->d_dt);
    if (a->d_t) cudaFree(a->d_t);
    if (a->d_cost) cudaFree(a->d_cost);
    if (a->d_trig) cudaFree(a->d_trig);
    a->d_dt = a->d_t = a->d_cost = nullptr;
    a->d_trig = nullptr;
    a->cap = 0;
}

int ensure_steps(sw2d_handle* h, int64_t need)
{
    AssimState* a = h->assim;
    if (need <= a->cap) return SW2D_OK;
    int64_t cap = std::max<int64_t>(need, 2 * a->cap + 1024);
    double *dt = nullptr, *t = nullptr, *cost = nullptr;
    int* tr = nullptr;
    CK(cudaMalloc(&dt, cap * sizeof(double)));
    CK(cudaMalloc(&t, cap * sizeof(double)));
    CK(cudaMalloc(&cost, cap * sizeof(double)));
    CK(cudaMalloc(&tr, cap * sizeof(int)));
    if (a->cap > 0) {
        CK(cudaMemcpyAsync(dt, a->d_dt, a->cap * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(t, a->d_t, a->cap * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(tr, a->d_trig, a->cap * sizeof(int), cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        free_steps(a);
    }
    a->d_dt = dt;
    a->d_t = t;
    a->d_cost = cost;
    a->d_trig = tr;
    a->cap = cap;
    return SW2D_OK;
}

void free_checkpoints(AssimState* a)
{
    for (double4* p : a->ck) cudaFree(p);
    a->ck.clear();
    for (double4* p : a->cs) cudaFree(p);
    a->cs.clear();
}


// Window and tiles of the gradient (swSpE_checkpoint.cpp:781-951).
void compute_window(AssimState* a, double t_max)
{
    const int64_t K = (int64_t)a->segs.size();
    int64_t first = 0;
    a->truncation = -1;
    a->tiles.clear();
    const sw2d_assim_params& p = a->prm;
    if (p.windowed && K > 0) {
        if (p.window_steps > 0) {
            int64_t acc = 0;
            for (int64_t k = K - 1; k >= 0; --k) {
                acc += a->segs[k].n;
                if (acc >= p.window_steps) {
                    first = k;
                    break;
                }
            }
        } else if (p.window_duration > 0.) {
            const double tw = t_max - p.window_duration;
            for (int64_t k = 0; k < K; ++k) {
                if (a->segs[k].t_start <= tw + 1e-9) first = k;
                else break;
            }
        } else if (p.t_state_assimilation > a->t0) {
            for (int64_t k = 0; k < K; ++k) {
                if (a->segs[k].t_start <= p.t_state_assimilation + 1e-9) first = k;
                else break;
            }
        }
        if (first > 0) a->truncation = first - 1;
    }
    if (p.forced_first_segment >= 0 && K > 0) {
        first = std::min<int64_t>(p.forced_first_segment, K - 1);
        a->truncation = first - 1;
    }
    a->first = first;
    if (p.n_windows > 1 && first < K) {
        const int64_t M = K - first;
        const int64_t n = std::min<int64_t>(p.n_windows, M);
        for (int64_t t = 0; t < n; ++t) a->tiles.push_back(first + (t * M) / n);
    }
}

// build_checkpoint_records: from the start state, CFL steps until t_max, a checkpoint at the
// start of every segment of `stride` steps.
int record(sw2d_handle* h, int64_t stride)
{
    AssimState* a = h->assim;
    const int64_t nc = h->nc;
    free_checkpoints(a);
    a->segs.clear();
    a->recorded = false;
    a->stride = stride;
    Ctrl c0{};
    c0.t = a->t0;
    c0.dt = h->p.dt_max;   // reset_to_start (swSpE_spAD.cpp:110-111)
    c0.t_max = h->p.t_max;
    CK(cudaMemcpyAsync(a->ctrl, &c0, sizeof(Ctrl), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(a->d_obs_idx, 0, sizeof(int), h->stream));
    CK(cudaMemcpyAsync(h->m.st, a->st0, nc * sizeof(double4), cudaMemcpyDeviceToDevice, h->stream));
    const DevMesh m = view_with(h, a->ctrl);
    const EView v = eview(a, &a->ctrl->dt, &a->ctrl->t);
    const bool muscl = h->p.scheme == SW2D_SCHEME_MUSCL_EVR;
    const unsigned gc = grid_for(nc);
    int64_t done = 0;
    double t_host = a->t0;
    Ctrl ch{};
    while (t_host < h->p.t_max) {
        int rc = ensure_steps(h, done + stride);
        if (rc) return rc;
        double4* ck = nullptr;
        CK(cudaMalloc(&ck, std::max<int64_t>(1, nc) * sizeof(double4)));
        a->ck.push_back(ck);
        CK(cudaMemcpyAsync(ck, h->m.st, nc * sizeof(double4), cudaMemcpyDeviceToDevice, h->stream));
        for (int64_t j = 0; j < stride; j++) {
            if (muscl) launch_slopes_on(h, m);
            launch_edges<true>(h, m, v);
            if (gc > 0) k_e_cfl<<<gc, kBlock, 0, h->stream>>>(m, a->d_obs_t, a->d_obs_idx, (int)a->n_obs);
            launch_update(h, m, &a->ctrl->dt, &a->ctrl->go, false);
            k_e_advance<<<1, 1, 0, h->stream>>>(a->ctrl, a->d_obs_idx, a->d_obs_t, (int)a->n_obs, a->d_dt, a->d_t,
                                                 a->d_trig, (long long)a->cap);
        }
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(&ch, a->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        const int64_t n = ch.steps - done;
        if (n <= 0) {
            cudaFree(a->ck.back());
            a->ck.pop_back();
            break;
        }
        AssimSegment s;
        s.t_start = t_host;
        s.j0 = done;
        s.n = n;
        a->segs.push_back(s);
        done = ch.steps;
        t_host = ch.t;
        if (nc == 0) break;
    }
    a->n_steps = done;
    a->dt_seq.resize(done);
    a->t_seq.resize(done);
    a->trig.resize(done);
    if (done > 0) {
        CK(cudaMemcpyAsync(a->dt_seq.data(), a->d_dt, done * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(a->t_seq.data(), a->d_t, done * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(a->trig.data(), a->d_trig, done * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    compute_window(a, h->p.t_max);
    a->recorded = true;
    return SW2D_OK;
}

// One replayed step j of ckpt_segment_E on the handle's state (dt and boundary time frozen);
// with bal, the raw post-balance state is kept there.
void replay_step(sw2d_handle* h, int64_t j, double4* bal)
{
    AssimState* a = h->assim;
    DevMesh m = view_with(h, a->ctrl_on);
    m.bal = bal;
    const EView v = eview(a, a->d_dt + j, a->d_t + j);
    if (h->p.scheme == SW2D_SCHEME_MUSCL_EVR) launch_slopes_on(h, m);
    launch_edges<false>(h, m, v);
    launch_update(h, m, a->d_dt + j, nullptr, bal != nullptr);
}

// replays segments s0 .. s1 chained from the state in the handle; the cost of the observation
// a step ends on goes to d_cost[j]
void replay_segments(sw2d_handle* h, int64_t s0, int64_t s1)
{
    AssimState* a = h->assim;
    for (int64_t s = s0; s <= s1; s++) {
        const AssimSegment& sg = a->segs[s];
        for (int64_t j = sg.j0; j < sg.j0 + sg.n; j++) {
            replay_step(h, j, nullptr);
            if (a->trig[j] >= 0 && a->trig[j] < a->n_obs) cost_at(h, a->trig[j], h->m.st, a->d_cost + j);
        }
    }
}

// replay_trajectory_cost: per segment the sum of its observations' costs in step order (from 0),
// added to the total segment by segment, as ckpt_segment_E returns them
// the chains replay_trajectory_cost replays: (first segment, last segment) from each tile's
// checkpoint, or from the one after the truncation
std::vector<std::pair<int64_t, int64_t>> replay_runs(const AssimState* a)
{
    const int64_t K = (int64_t)a->segs.size();
    std::vector<std::pair<int64_t, int64_t>> runs;
    if (!a->tiles.empty()) {
        for (size_t ti = 0; ti < a->tiles.size(); ti++)
            runs.emplace_back(a->tiles[ti], (ti + 1 < a->tiles.size()) ? a->tiles[ti + 1] - 1 : K - 1);
    } else {
        int64_t s0 = 0;
        if (a->truncation >= 0 && a->truncation + 1 < K) s0 = a->truncation + 1;
        runs.emplace_back(s0, K - 1);
    }
    return runs;
}

// The segment-start states along the replay's chains (cs[k]; for the first segment of a chain,
// its checkpoint).  With the MUSCL-EVR scheme they differ from the dry run's checkpoints: the dry
// run reconstructs with the previous step's dt (build_checkpoint_records calls
// hypComputeLRStates_E before setting this->dt, swSpE_checkpoint.cpp:236-246), the replay with
// the step's own (ckpt_segment_E, :640-641).
int chain_states(sw2d_handle* h)
{
    AssimState* a = h->assim;
    const int64_t K = (int64_t)a->segs.size(), nc = h->nc;
    while ((int64_t)a->cs.size() < K) {
        double4* p = nullptr;
        CK(cudaMalloc(&p, std::max<int64_t>(1, nc) * sizeof(double4)));
        a->cs.push_back(p);
    }
    for (const auto& r : replay_runs(a)) {
        CK(cudaMemcpyAsync(h->m.st, a->ck[r.first], nc * sizeof(double4), cudaMemcpyDeviceToDevice, h->stream));
        for (int64_t s = r.first; s <= r.second; s++) {
            CK(cudaMemcpyAsync(a->cs[s], h->m.st, nc * sizeof(double4), cudaMemcpyDeviceToDevice, h->stream));
            for (int64_t j = a->segs[s].j0; j < a->segs[s].j0 + a->segs[s].n; j++) replay_step(h, j, nullptr);
        }
    }
    CK(cudaGetLastError());
    return SW2D_OK;
}

int replay_cost(sw2d_handle* h, double* J)
{
    AssimState* a = h->assim;
    const auto runs = replay_runs(a);
    for (const auto& r : runs) {
        CK(cudaMemcpyAsync(h->m.st, a->ck[r.first], h->nc * sizeof(double4), cudaMemcpyDeviceToDevice, h->stream));
        replay_segments(h, r.first, r.second);
    }
    CK(cudaGetLastError());
    std::vector<double> cost(a->n_steps, 0.0);
    if (a->n_steps > 0)
        CK(cudaMemcpyAsync(cost.data(), a->d_cost, a->n_steps * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    double total = 0.0;
    for (const auto& r : runs)
        for (int64_t s = r.first; s <= r.second; s++) {
            double seg = 0.0;
            for (int64_t j = a->segs[s].j0; j < a->segs[s].j0 + a->segs[s].n; j++)
                if (a->trig[j] >= 0 && a->trig[j] < a->n_obs) seg += cost[j];
            total += seg;
        }
    *J = total;
    return SW2D_OK;
}

int seg_buffers(sw2d_handle* h)
{
    AssimState* a = h->assim;
    int64_t longest = 0;
    for (const auto& s : a->segs) longest = std::max(longest, s.n);
    if (longest <= a->seg_cap) return SW2D_OK;
    free_list(a->seg_allocs);
    a->seg_cap = 0;
    int rc = SW2D_OK;
    if ((rc = adj_alloc(h, a->seg_allocs, (longest + 1) * h->nc, &a->seg_st)) ||
        (rc = adj_alloc(h, a->seg_allocs, longest * h->nc, &a->seg_bal)))
        return rc;
    a->seg_cap = longest;
    return SW2D_OK;
}

double norm_h(sw2d_handle* h, int* rc)
{
    AssimState* a = h->assim;
    const int nb = std::max(1, std::min(kCostBlocks, (int)grid_for(h->nc)));
    k_e_norm2<<<nb, kBlock, 0, h->stream>>>(a->lam, (int)h->nc, a->d_part);
    std::vector<double> p(nb);
    if (cudaMemcpyAsync(p.data(), a->d_part, nb * sizeof(double), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
        *rc = fail(h, SW2D_E_CUDA, "adjoint norm");
        return 0.0;
    }
    double s = 0.0;
    for (double x : p) s += x;
    return std::sqrt(s);
}

// Reverse of segment k (recompute from its checkpoint, or from its state along the replay with
// the option assim_chained_recompute, then the steps backwards).
int reverse_segment(sw2d_handle* h, int64_t k)
{
    AssimState* a = h->assim;
    const AssimSegment& sg = a->segs[k];
    const int64_t nc = h->nc;
    const bool muscl = h->p.scheme == SW2D_SCHEME_MUSCL_EVR;
    const double4* start = (h->assim_chained && k < (int64_t)a->cs.size()) ? a->cs[k] : a->ck[k];
    CK(cudaMemcpyAsync(h->m.st, start, nc * sizeof(double4), cudaMemcpyDeviceToDevice, h->stream));
    for (int64_t j = sg.j0; j < sg.j0 + sg.n; j++) {
        CK(cudaMemcpyAsync(a->seg_st + (j - sg.j0) * nc, h->m.st, nc * sizeof(double4), cudaMemcpyDeviceToDevice,
                           h->stream));
        replay_step(h, j, a->seg_bal + (j - sg.j0) * nc);
    }
    CK(cudaMemcpyAsync(a->seg_st + sg.n * nc, h->m.st, nc * sizeof(double4), cudaMemcpyDeviceToDevice, h->stream));
    const unsigned gc = grid_for(nc);
    const unsigned ge = grid_for(h->ni + h->nb);
    for (int64_t j = sg.j0 + sg.n - 1; j >= sg.j0; j--) {
        const int64_t r = j - sg.j0;
        if (a->trig[j] >= 0 && a->trig[j] < a->n_obs) obs_rev_at(h, a->trig[j], a->seg_st + (r + 1) * nc);
        DevMesh mr = view_with(h, a->ctrl_on);
        mr.st = a->seg_st + r * nc;
        const double dt = a->dt_seq[j];
        if (gc > 0) launch_update_rev(h, mr, a->seg_bal + r * nc, dt);
        if (muscl) launch_slopes_on(h, mr);
        const EView v = eview(a, a->d_dt + j, a->d_t + j);
        if (ge > 0) {
            const int ieee = h->assim_sqrt_zero;
            if (muscl)
                k_e_edges_rev<SW2D_SCHEME_MUSCL_EVR><<<ge, kBlock, 0, h->stream>>>(mr, v, a->lamb, a->ctb, a->cts, dt, ieee);
            else k_e_edges_rev<SW2D_SCHEME_GODUNOV><<<ge, kBlock, 0, h->stream>>>(mr, v, a->lamb, a->ctb, a->cts, dt, ieee);
        }
        if (gc > 0) {
            if (muscl) {
                k_e_cells_rev<true><<<gc, kBlock, 0, h->stream>>>(mr, a->lam, a->ctb, a->cts, a->g_phi, a->sgb);
                k_limiter_rev<<<gc, kBlock, 0, h->stream>>>(mr, a->sgb, a->lam, a->gzb, a->znb);
                k_nbr_rev<<<gc, kBlock, 0, h->stream>>>(mr, a->mirror, a->znb, a->lam, a->gzb);
            } else {
                k_e_cells_rev<false><<<gc, kBlock, 0, h->stream>>>(mr, a->lam, a->ctb, a->cts, a->g_phi, a->sgb);
            }
        }
    }
    CK(cudaGetLastError());
    return SW2D_OK;
}

int scatter(sw2d_handle* h, const double* src, int stride, int offset, double* out)
{
    if (!out) return SW2D_OK;
    AssimState* a = h->assim;
    k_scatter_cells<<<grid_for(h->nc), kBlock, 0, h->stream>>>(src, stride, offset, h->d_cell_perm, a->stage, (int)h->nc);
    CK(cudaMemcpyAsync(out, a->stage, h->nc * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return SW2D_OK;
}

int require(sw2d_handle* h, bool need_record)
{
    if (!h) return SW2D_E_ARG;
    if (h->model != kModelSp) return fail(h, SW2D_E_UNSUPPORTED, "the assimilation engine runs the SP model only");
    if (!h->assim || !h->assim->configured) return fail(h, SW2D_E_ARG, "call sw2d_assim_configure first");
    if (need_record && !h->assim->recorded) return fail(h, SW2D_E_ARG, "no recorded trajectory (sw2d_assim_record)");
    return SW2D_OK;
}

}  // namespace

namespace sw2d {

void assim_release(sw2d_handle* h)
{
    if (!h || !h->assim) return;
    AssimState* a = h->assim;
    free_checkpoints(a);
    free_steps(a);
    free_list(a->seg_allocs);
    free_list(a->traj_allocs);
    free_list(a->obs_allocs);
    free_list(a->fixed_allocs);
    delete a;
    h->assim = nullptr;
}

}  // namespace sw2d

// ------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------
extern "C" {

int sw2d_assim_configure(sw2d_handle* h, const sw2d_assim_params* params)
{
    if (!h || !params) return fail(h, SW2D_E_ARG, "invalid arguments");
    if (h->model != kModelSp) return fail(h, SW2D_E_UNSUPPORTED, "the assimilation engine runs the SP model only");
    if (params->phi_transform < SW2D_PHI_NONE || params->phi_transform > SW2D_PHI_NORMALIZE)
        return fail(h, SW2D_E_ARG, "unknown phi_transform");
    if (params->n_windows < 1) return fail(h, SW2D_E_ARG, "n_windows must be >= 1");
    CK(cudaSetDevice(h->device));
    AssimState* a = ensure_state(h);
    int rc = fixed_buffers(h);
    if (rc) return rc;
    const bool first = !a->configured;
    a->prm = *params;
    if (first) {
        // the start of the trajectory: the handle's current state and time
        CK(cudaMemcpyAsync(a->st0, h->m.st, h->nc * sizeof(double4), cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        a->t0 = h->ctrl_host->t;
    }
    a->configured = true;
    if (a->recorded) compute_window(a, h->p.t_max);
    return SW2D_OK;
}

int sw2d_assim_set_observations(sw2d_handle* h, const sw2d_assim_obs* obs)
{
    int rc = require(h, false);
    if (rc) return rc;
    if (!obs || obs->n_obs < 0 || (obs->n_obs > 0 && !obs->times)) return fail(h, SW2D_E_ARG, "invalid observations");
    if (obs->kind != SW2D_OBS_FRAMES && obs->kind != SW2D_OBS_GAUGES) return fail(h, SW2D_E_ARG, "unknown observation kind");
    for (int32_t k = 1; k < obs->n_obs; k++)
        if (!(obs->times[k] > obs->times[k - 1])) return fail(h, SW2D_E_ARG, "observation times must increase");
    CK(cudaSetDevice(h->device));
    AssimState* a = h->assim;
    free_list(a->obs_allocs);
    a->d_ident = a->d_gcell = a->d_ucell = a->d_uoff = a->d_ulist = nullptr;
    a->d_wh = a->d_wq = a->d_hobs = a->d_qobs = a->d_robs = a->d_obs_t = nullptr;
    a->kind = obs->kind;
    a->n_obs = obs->n_obs;
    a->obs_t.assign(obs->times, obs->times + obs->n_obs);
    auto& L = a->obs_allocs;
    const int64_t nc = h->nc, nk = obs->n_obs;
    if ((rc = adj_alloc(h, L, std::max<int64_t>(1, nk), &a->d_obs_t))) return rc;
    if (nk > 0) CK(cudaMemcpyAsync(a->d_obs_t, obs->times, nk * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (obs->kind == SW2D_OBS_FRAMES) {
        if (nk > 0 && !obs->frames) return fail(h, SW2D_E_ARG, "frames missing");
        a->n_gauges = 0;
        if ((rc = adj_alloc(h, L, nc, &a->d_ident)) || (rc = adj_alloc(h, L, nc, &a->d_wh)) ||
            (rc = adj_alloc(h, L, nc, &a->d_wq)) || (rc = adj_alloc(h, L, nk * nc, &a->d_hobs)) ||
            (rc = adj_alloc(h, L, nk * nc, &a->d_qobs)) || (rc = adj_alloc(h, L, nk * nc, &a->d_robs)))
            return rc;
        std::vector<int> ident(nc);
        for (int64_t i = 0; i < nc; i++) ident[i] = (int)i;
        CK(cudaMemcpyAsync(a->d_ident, ident.data(), nc * sizeof(int), cudaMemcpyHostToDevice, h->stream));
        // weights: caller numbering -> internal
        const double* wsrc[2] = {obs->h_weight, obs->q_weight};
        double* wdst[2] = {a->d_wh, a->d_wq};
        std::vector<double> ones(nc, 1.0);
        for (int w = 0; w < 2; w++) {
            CK(cudaMemcpyAsync(a->stage, wsrc[w] ? wsrc[w] : ones.data(), nc * sizeof(double), cudaMemcpyHostToDevice,
                               h->stream));
            k_gather_component<<<grid_for(nc), kBlock, 0, h->stream>>>(a->stage, h->d_cell_perm, wdst[w], 1, 0, (int)nc);
            CK(cudaStreamSynchronize(h->stream));
        }
        for (int64_t k = 0; k < nk; k++) {
            CK(cudaMemcpyAsync(a->stage, obs->frames + (size_t)k * 3 * nc, 3 * nc * sizeof(double), cudaMemcpyHostToDevice,
                               h->stream));
            double* dst[3] = {a->d_hobs + k * nc, a->d_qobs + k * nc, a->d_robs + k * nc};
            for (int q = 0; q < 3; q++)
                k_gather_component<<<grid_for(nc), kBlock, 0, h->stream>>>(a->stage + q * nc, h->d_cell_perm, dst[q], 1, 0,
                                                                          (int)nc);
            CK(cudaStreamSynchronize(h->stream));
        }
    } else {
        const int64_t ng = obs->n_gauges;
        if (ng < 0 || (ng > 0 && (!obs->gauge_cells || !obs->gauge_weight || (nk > 0 && !obs->gauge_h))))
            return fail(h, SW2D_E_ARG, "invalid gauges");
        a->n_gauges = ng;
        std::vector<int> inv(nc);
        for (int64_t i = 0; i < nc; i++) inv[h->cell_perm[i]] = (int)i;
        std::vector<int> gc(ng);
        for (int64_t g = 0; g < ng; g++) {
            if (obs->gauge_cells[g] < 0 || obs->gauge_cells[g] >= nc) return fail(h, SW2D_E_ARG, "gauge cell out of range");
            gc[g] = inv[obs->gauge_cells[g]];
        }
        // distinct cells with their gauges, for the reverse
        std::vector<int> order(ng);
        for (int64_t g = 0; g < ng; g++) order[g] = (int)g;
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return gc[x] < gc[y]; });
        std::vector<int> ucell, uoff{0};
        for (int64_t q = 0; q < ng; q++) {
            if (q == 0 || gc[order[q]] != gc[order[q - 1]]) {
                if (q > 0) uoff.push_back((int)q);
                ucell.push_back(gc[order[q]]);
            }
        }
        uoff.push_back((int)ng);
        if (ng == 0) uoff.assign(1, 0);
        a->n_ucells = (int64_t)ucell.size();
        std::vector<double> hv((size_t)std::max<int64_t>(1, nk * ng));
        if (nk * ng > 0) std::memcpy(hv.data(), obs->gauge_h, nk * ng * sizeof(double));
        std::vector<double> wv(obs->gauge_weight, obs->gauge_weight + ng);
        if ((rc = dev_upload_list(h, L, gc, &a->d_gcell)) || (rc = dev_upload_list(h, L, ucell, &a->d_ucell)) ||
            (rc = dev_upload_list(h, L, uoff, &a->d_uoff)) || (rc = dev_upload_list(h, L, order, &a->d_ulist)) ||
            (rc = dev_upload_list(h, L, wv, &a->d_wh)) || (rc = dev_upload_list(h, L, hv, &a->d_hobs)))
            return rc;
        CK(cudaStreamSynchronize(h->stream));
    }
    CK(cudaGetLastError());
    return SW2D_OK;
}

int sw2d_assim_record(sw2d_handle* h, const double* m, int64_t stride, int64_t* n_steps, int64_t* n_segments)
{
    int rc = require(h, false);
    if (rc) return rc;
    if (!m || stride <= 0) return fail(h, SW2D_E_ARG, "invalid arguments");
    CK(cudaSetDevice(h->device));
    if ((rc = set_control(h, m, true)) || (rc = record(h, stride))) return rc;
    if (n_steps) *n_steps = h->assim->n_steps;
    if (n_segments) *n_segments = (int64_t)h->assim->segs.size();
    return SW2D_OK;
}

int sw2d_assim_replay_cost(sw2d_handle* h, const double* m, double* J)
{
    int rc = require(h, true);
    if (rc) return rc;
    if (!m || !J) return fail(h, SW2D_E_ARG, "invalid arguments");
    if (h->assim->segs.empty()) {
        *J = 0.0;
        return SW2D_OK;
    }
    CK(cudaSetDevice(h->device));
    if ((rc = set_control(h, m, false))) return rc;
    return replay_cost(h, J);
}

int sw2d_assim_gradient(sw2d_handle* h, const double* m, int64_t stride, double* dJ_dm, double* dJ_dk1, double* dJ_dk2,
                        double* dJ_dstate, sw2d_assim_info* info)
{
    int rc = require(h, false);
    if (rc) return rc;
    if (!m || !dJ_dm || stride <= 0) return fail(h, SW2D_E_ARG, "invalid arguments");
    CK(cudaSetDevice(h->device));
    AssimState* a = h->assim;
    const int64_t nc = h->nc;
    if ((rc = set_control(h, m, true)) || (rc = record(h, stride))) return rc;
    sw2d_assim_info inf{};
    inf.grad_argmax = -1;
    inf.exploded_segment = -1;
    const int64_t K = (int64_t)a->segs.size();
    CK(cudaMemsetAsync(a->lam, 0, nc * sizeof(double4), h->stream));
    CK(cudaMemsetAsync(a->g_phi, 0, nc * sizeof(double), h->stream));
    CK(cudaMemsetAsync(a->g_k1, 0, nc * sizeof(double), h->stream));
    CK(cudaMemsetAsync(a->g_k2, 0, nc * sizeof(double), h->stream));
    CK(cudaMemsetAsync(a->g_w, 0, nc * sizeof(double), h->stream));
    CK(cudaMemsetAsync(a->gzb, 0, nc * sizeof(double), h->stream));
    if (K > 0 && (rc = seg_buffers(h))) return rc;
    if (K > 0 && h->assim_chained && (rc = chain_states(h))) return rc;
    // tiles: tile_top[k] = the last segment of a tile (the adjoint restarts from 0 before it)
    std::vector<char> tile_top(K, 0);
    const bool tiled = !a->tiles.empty();
    for (size_t t = 0; t < a->tiles.size(); t++) {
        const int64_t e = (t + 1 < a->tiles.size()) ? a->tiles[t + 1] - 1 : K - 1;
        tile_top[e] = 1;
    }
    int64_t watermark_seg = K - 1, kept_start = K;
    double ref_norm = -1.0, dh_peak = 0.0;
    const bool forced = a->prm.forced_first_segment >= 0;
    for (int64_t k = K - 1; k >= a->first; k--) {
        if (tiled && tile_top[k]) {
            CK(cudaMemsetAsync(a->lam, 0, nc * sizeof(double4), h->stream));
            CK(cudaMemcpyAsync(a->g_w, a->g_phi, nc * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
            kept_start = k + 1;
        }
        if ((rc = reverse_segment(h, k))) return rc;
        const double norm = norm_h(h, &rc);
        if (rc) return rc;
        if (norm > dh_peak) dh_peak = norm;
        if (ref_norm < 0.0 && norm > 0.0) ref_norm = norm;
        const AssimSegment& sg = a->segs[k];
        bool has_obs = false;
        for (int64_t j = sg.j0; j < sg.j0 + sg.n; j++) has_obs = has_obs || a->trig[j] >= 0;
        const bool milestone = (k % 50 == 0) || (k == K - 1) || (k == 0);
        const bool blown = !forced && ref_norm > 0.0 && norm > 1e8 * ref_norm;
        if (!tiled) {
            if (milestone || has_obs) {
                CK(cudaMemcpyAsync(a->g_w, a->g_phi, nc * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
                watermark_seg = k;
            }
            if (blown) {
                CK(cudaMemcpyAsync(a->g_phi, a->g_w, nc * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
                a->truncation = watermark_seg - 1;
                inf.exploded_segment = k;
                break;
            }
        } else if (blown) {
            CK(cudaMemcpyAsync(a->g_phi, a->g_w, nc * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
            a->truncation = kept_start - 1;
            while (!a->tiles.empty() && a->tiles.front() < kept_start) a->tiles.erase(a->tiles.begin());
            inf.exploded_segment = k;
            break;
        }
    }
    // dJ/dm and the clean-up
    CK(cudaMemsetAsync(a->d_count, 0, 4 * sizeof(unsigned long long), h->stream));
    double* gm = a->gzb;  // reused as the output buffer
    if (nc > 0)
        k_e_finish<<<grid_for(nc), kBlock, 0, h->stream>>>(a->g_phi, a->d_m, a->d_phi, gm, a->g_k1, a->g_k2, a->lam, (int)nc,
                                                             a->prm.phi_transform, a->prm.lambda_tanh, a->norm_scale,
                                                             a->prm.mask_wall_gradient, h->p.phi_min, a->d_count);
    CK(cudaGetLastError());
    unsigned long long cnt[4];
    CK(cudaMemcpyAsync(cnt, a->d_count, sizeof(cnt), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if ((rc = scatter(h, gm, 1, 0, dJ_dm))) return rc;
    if ((rc = scatter(h, a->g_k1, 1, 0, dJ_dk1)) || (rc = scatter(h, a->g_k2, 1, 0, dJ_dk2))) return rc;
    if (dJ_dstate) {
        const double* ls = reinterpret_cast<const double*>(a->lam);
        if ((rc = scatter(h, ls, 4, 0, dJ_dstate)) || (rc = scatter(h, ls, 4, 1, dJ_dstate + nc)) ||
            (rc = scatter(h, ls, 4, 2, dJ_dstate + 2 * nc)))
            return rc;
    }
    double gl2 = 0.0, gmax = 0.0;
    int64_t gidx = 0;
    for (int64_t i = 0; i < nc; i++) {
        const double g = dJ_dm[i];
        gl2 += g * g;
        if (std::fabs(g) > std::fabs(gmax)) {
            gmax = g;
            gidx = i;
        }
    }
    // the cost of the function whose gradient this is
    double J = 0.0;
    if (K > 0 && (rc = replay_cost(h, &J))) return rc;
    inf.J = J;
    inf.grad_l2 = std::sqrt(gl2);
    inf.grad_max = gmax;
    inf.grad_argmax = gidx;
    inf.dh_peak = dh_peak;
    inf.n_steps = a->n_steps;
    inf.n_segments = K;
    inf.first_segment = a->first;
    inf.truncation_segment = a->truncation;
    inf.n_tiles = (int64_t)a->tiles.size();
    inf.n_nonfinite = (int64_t)cnt[0];
    inf.n_masked = (int64_t)(cnt[0] + cnt[1]);
    if (info) *info = inf;
    return SW2D_OK;
}

int sw2d_assim_segments(sw2d_handle* h, double* t_start, int64_t* n_steps, int64_t capacity)
{
    int rc = require(h, true);
    if (rc) return rc;
    const AssimState* a = h->assim;
    if ((int64_t)a->segs.size() > capacity) return fail(h, SW2D_E_ARG, "capacity too small");
    for (size_t k = 0; k < a->segs.size(); k++) {
        if (t_start) t_start[k] = a->segs[k].t_start;
        if (n_steps) n_steps[k] = a->segs[k].n;
    }
    return SW2D_OK;
}

int sw2d_assim_steps(sw2d_handle* h, double* dt, int32_t* obs_trig, int64_t capacity)
{
    int rc = require(h, true);
    if (rc) return rc;
    const AssimState* a = h->assim;
    if (a->n_steps > capacity) return fail(h, SW2D_E_ARG, "capacity too small");
    for (int64_t j = 0; j < a->n_steps; j++) {
        if (dt) dt[j] = a->dt_seq[j];
        if (obs_trig) obs_trig[j] = a->trig[j];
    }
    return SW2D_OK;
}

int sw2d_assim_set_start(sw2d_handle* h, const double* water_depth, const double* unit_discharge_x,
                         const double* unit_discharge_y)
{
    int rc = require(h, false);
    if (rc) return rc;
    if (!water_depth || !unit_discharge_x || !unit_discharge_y) return fail(h, SW2D_E_ARG, "invalid arguments");
    CK(cudaSetDevice(h->device));
    AssimState* a = h->assim;
    const int64_t nc = h->nc;
    const double* src[3] = {water_depth, unit_discharge_x, unit_discharge_y};
    double* st0 = reinterpret_cast<double*>(a->st0);
    for (int q = 0; q < 3; q++) {
        CK(cudaMemcpyAsync(a->stage, src[q], nc * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        k_gather_component<<<grid_for(nc), kBlock, 0, h->stream>>>(a->stage, h->d_cell_perm, st0, 4, q, (int)nc);
        CK(cudaStreamSynchronize(h->stream));
    }
    k_refresh_z_e<<<grid_for(nc), kBlock, 0, h->stream>>>(a->st0, h->m.zbv, (int)nc);
    if (a->recorded && !a->ck.empty())
        CK(cudaMemcpyAsync(a->ck[0], a->st0, nc * sizeof(double4), cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    return SW2D_OK;
}

int sw2d_assim_trigger_states(sw2d_handle* h, const double* m, double* water_depth, double* unit_discharge_x,
                              double* unit_discharge_y, int64_t n_obs_capacity, int64_t* n_written)
{
    int rc = require(h, true);
    if (rc) return rc;
    if (!m || !water_depth || !unit_discharge_x || !unit_discharge_y || n_obs_capacity < 0)
        return fail(h, SW2D_E_ARG, "invalid arguments");
    AssimState* a = h->assim;
    if (n_obs_capacity < a->n_obs) return fail(h, SW2D_E_ARG, "capacity below the number of observations");
    CK(cudaSetDevice(h->device));
    if ((rc = set_control(h, m, false))) return rc;
    const int64_t nc = h->nc;
    // the recorded trajectory from its start state (swSpE::reset_to_start), step by step with the
    // frozen dt and boundary times; the state after a step that lands on observation k is what
    // storeReferenceMap writes at that time (swSpE_checkpoint.cpp:360-375)
    CK(cudaMemcpyAsync(h->m.st, a->st0, nc * sizeof(double4), cudaMemcpyDeviceToDevice, h->stream));
    int64_t written = 0;
    for (const AssimSegment& sg : a->segs)
        for (int64_t j = sg.j0; j < sg.j0 + sg.n; j++) {
            replay_step(h, j, nullptr);
            const int k = a->trig[j];
            if (k < 0 || k >= a->n_obs) continue;
            const double* src = reinterpret_cast<const double*>(h->m.st);
            if ((rc = scatter(h, src, 4, 0, water_depth + k * nc)) ||
                (rc = scatter(h, src, 4, 1, unit_discharge_x + k * nc)) ||
                (rc = scatter(h, src, 4, 2, unit_discharge_y + k * nc)))
                return rc;
            written++;
        }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    if (n_written) *n_written = written;
    return SW2D_OK;
}

int sw2d_assim_checkpoint(sw2d_handle* h, int64_t k, double* water_depth, double* unit_discharge_x,
                          double* unit_discharge_y)
{
    int rc = require(h, true);
    if (rc) return rc;
    AssimState* a = h->assim;
    if (k < 0 || k >= (int64_t)a->ck.size()) return fail(h, SW2D_E_ARG, "no such checkpoint");
    CK(cudaSetDevice(h->device));
    const double* src = reinterpret_cast<const double*>(a->ck[k]);
    if ((rc = scatter(h, src, 4, 0, water_depth)) || (rc = scatter(h, src, 4, 1, unit_discharge_x)) ||
        (rc = scatter(h, src, 4, 2, unit_discharge_y)))
        return rc;
    return SW2D_OK;
}

}  // extern "C"
