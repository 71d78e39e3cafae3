// sw2d_adjoint.cu — reverse mode of the SP step on the B200: recorded trajectories with
// checkpoints, frozen-dt replays, the observation misfit J and its gradient with respect to the
// per-cell friction coefficients (Manning n for the Manning law), the initial state and the
// bed elevation.
//
// What is differentiated.  As in the reference's assimilation (assim/swSpE_checkpoint.cpp:
// 1436-1453, `ckpt_segment_E` with a frozen dt sequence, assim/swSpE.h:237-251), the time
// steps and the boundary values are those of a recorded run: J(m) is the cost of replaying the
// recorded dt sequence with controls m.  J sums, over observation steps, weighted squared
// misfits of h (and optionally q, r) at observed cells (compute_cost_gauges_ptr,
// assim/swSpE_gauges.cpp:166-179; compute_cost_frame_ptr, assim/swSpE_ad.cpp:273-308),
// optionally divided by the number of observations (cost_normalize).
//
// Checkpointing.  sw2d_record runs the CFL-driven step and keeps the dt sequence; the state,
// the balance slots and the control block are stored every K steps.  The reverse sweep walks
// the segments backwards: it restores a checkpoint, recomputes the K forward steps storing each
// step's state and post-balance state, then runs the reverse kernels step by step:
//
//   k_obs_rev       per observed cell   misfit gradient at an observation step
//   k_update_rev    per cell            reverse of flush / clamp / friction / head loss / velocity
//                                       cap; friction-coefficient gradient; slot adjoints
//                                       sigma += dt * (adjoint of the post-balance state)
//   k_slopes        per cell            forward slopes of the step (recomputed)
//   k_edges_rev     per edge            Riemann states recomputed, reverse of the HLLC flux (internal
//                                       edges: adjoints of the two Riemann states per slot) or of the
//                                       boundary flux and state (boundary edges: final contributions),
//                                       for the edges whose flux the step computed; those slots'
//                                       adjoints reset
//   k_cells_rev     per cell            ordered gather over the cell's slots, with the reverse of the
//                                       cell's reconstruction on each internal slot
//   k_limiter_rev   per cell            reverse of the cell's slope limiter (per-neighbour
//                                       contributions) (MUSCL-EVR)
//   k_nbr_rev       per cell            ordered gather of the neighbours' slope contributions
//
// Edges left dry keep their previous balance terms in the forward step (swSpHyp.cpp:339), so a
// slot's adjoint carries over to the previous step until a step that computed that flux.  All
// sums run in a fixed order; no floating-point atomics are used, so gradients are bitwise
// reproducible and independent of the checkpoint interval.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "sw2d_internal.cuh"
#include "sp_adjoint.cuh"
#include "adjoint_common.cuh"

using namespace sw2d;

namespace sw2d {

struct AdjointState {
    int64_t nslot = 0, ncint = 0;
    // trajectory
    int64_t n_requested = 0, n_steps = 0, every = 0, n_ck = 0;
    long long base_steps = 0;
    double dt_before = 0.0;              // dt of the step before the trajectory (MUSCL-EVR uses it)
    std::vector<double> dt_seq, t_seq;   // dt_j and the time at the start of step j
    double* d_dt_seq = nullptr;
    double* d_t_seq = nullptr;
    // checkpoints k = 0 .. n_ck-1 at step k*every, and the end of the trajectory
    double4* ck_st = nullptr;            // (n_ck + 1) * nc
    Slot* ck_slot = nullptr;             // (n_ck + 1) * nslot
    Ctrl* ck_ctrl = nullptr;             // n_ck + 1
    bool ck_valid = false;
    // one segment of recomputed steps
    double4* seg_st = nullptr;           // (every + 1) * nc
    double4* seg_bal = nullptr;          // every * nc
    double2* seg_slope = nullptr;        // every * nc: each step's MUSCL-EVR slopes
    double2* seg_rs = nullptr;           // every * ni * 5: each step's Riemann states (when memory allows)
    double2* eside = nullptr;            // 3 * ni: {z_b}, {b}, {phi} of each internal edge's (L, R) cells
    // adjoint buffers
    double4* lam = nullptr;              // nc: adjoint of the state {h, q, r, -}
    double4* sig = nullptr;              // nslot: adjoint of the balance slots {a, b, c, -}
    double4* ctb = nullptr;              // nslot: per-slot contributions {h, q, r, z_b}
    double2* cts = nullptr;              // nslot: per-slot slope contributions {sx, sy}
    double* znb = nullptr;               // ncint: per-neighbour-entry z contributions
    double2* sgb = nullptr;              // nc: adjoint of each cell's limited slope
    int* mirror = nullptr;               // ncint: entry of the same edge in the neighbour's list
    double4* sgeo = nullptr;             // ncint: {nx, ny, midpoint - centroid} of each entry's edge
    double* g_zb = nullptr;
    double* g_k1 = nullptr;
    double* g_k2 = nullptr;
    Ctrl* ctrl_rev = nullptr;            // control block that keeps recomputed slopes active
    double* d_Jobs = nullptr;            // n_obs: cost of each observation
    double* d_part = nullptr;
    double* stage = nullptr;             // nc doubles for parameter transfers
    unsigned long long* d_nonfinite = nullptr;  // 6 counters of the last gradient's clean-up
    int64_t nonfinite[6] = {0, 0, 0, 0, 0, 0};
    // option "adjoint_trace": per reverse step j, after its kernels, {non-finite entries of the
    // state adjoint, bits of max |adjoint of h|, bits of max |adjoint of q, r|, first cell with a
    // non-finite entry}
    unsigned long long* d_trace = nullptr;
    int64_t trace_steps = 0;
    // observations
    int64_t n_pts = 0, n_obs = 0;
    int normalize = 0;
    std::vector<int64_t> obs_steps;
    std::vector<int> obs_at;             // [n_steps + 1] observation index of a step, or -1
    int* d_pts = nullptr;
    double *d_wh = nullptr, *d_wq = nullptr, *d_hobs = nullptr, *d_qobs = nullptr, *d_robs = nullptr;
    std::vector<void*> traj_allocs, obs_allocs, fixed_allocs;
};

}  // namespace sw2d

namespace {

// ------------------------------------------------------------------------------------------
// small kernels of the record / replay loop
// ------------------------------------------------------------------------------------------

// after k_cfl in a recorded run: keep dt_j and t_j of the step about to be taken
__global__ void k_note_dt(const Ctrl* ctrl, double* dt_seq, double* t_seq, long long base)
{
    if (ctrl->go) {
        const long long j = ctrl->steps - base;
        dt_seq[j] = ctrl->dt;
        t_seq[j] = ctrl->t;
    }
}

// in place of k_cfl in a replay: the recorded dt of step j (the host launches exactly the
// recorded number of steps, so j stays inside dt_seq)
__global__ void k_frozen_dt(Ctrl* ctrl, const double* dt_seq, long long base)
{
    const long long j = ctrl->steps - base;
    ctrl->dt = dt_seq[j];
    ctrl->go = 1;
}

// z = h + z_b of a state array after a change of z_b
__global__ void k_refresh_z(double4* st, const double* zbv, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        double4 s = st[i];
        s.w = s.x + zbv[i];
        st[i] = s;
    }
}

// out[p] = st[pts[p]]: the state at sampled cells
__global__ void k_sample(const double4* __restrict__ st, const int* __restrict__ pts, double4* out, int n)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) out[p] = st[pts[p]];
}

// ------------------------------------------------------------------------------------------
// reverse kernels
// ------------------------------------------------------------------------------------------

// The side table of k_edges_rev: per internal edge, {z_b}, {b}, {phi} of its (L, R) cells, in
// three planes of ni double2 (rebuilt at each reverse sweep from the current cell constants)
__global__ void k_edge_sides(DevMesh m, double2* eside)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.ni) return;
    const size_t ni = (size_t)m.ni;
    const int2 lr = ld(&m.lr[e]);
    const double4 ca = ld(&m.cst[lr.x]), cb = ld(&m.cst[lr.y]);
    eside[e] = make_double2(ca.x, cb.x);
    eside[ni + e] = make_double2(ca.y, cb.y);
    eside[2 * ni + e] = make_double2(ca.z, cb.z);
}

// The slot adjoints, which k_update_rev accumulates and k_edges_rev resets, are loaded and
// stored through volatile asms on the coherent path, in the order they stand (ld_now, in
// sw2d_internal.cuh, covers the read-only tables).  Only {x, y, z} of a slot adjoint is used.
__device__ __forceinline__ double4 ld_sig(const double4* p)
{
    double4 v;
    asm volatile("ld.global.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    asm volatile("ld.global.f64 %0, [%1+16];" : "=d"(v.z) : "l"(p));
    v.w = 0.0;
    return v;
}
__device__ __forceinline__ void st_sig(double4* p, double x, double y, double z)
{
    asm volatile("st.global.v2.f64 [%0], {%1, %2};\n\tst.global.f64 [%0+16], %3;" ::"l"(p), "d"(x), "d"(y), "d"(z));
}
__device__ __forceinline__ void st_sig_zero(double4* p) { st_sig(p, 0.0, 0.0, 0.0); }

// Reverse of k_update for one step: lam holds the adjoint of the state after the step and
// becomes the adjoint of the state before it (balance part); the slots' adjoints gain
// dt * (adjoint of the post-balance state); friction-coefficient gradients accumulate.
template <int kFriction, bool kHeadLoss>
__global__ void __launch_bounds__(kBlock) k_update_rev(DevMesh m, const double4* __restrict__ bal, double4* lam,
                                                       double4* sig, double* gk1, double* gk2, double dt,
                                                       int flush_branch)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    UpdateParams p;
    p.friction = kFriction;
    p.head_loss = kHeadLoss;
    p.clamp_negative = !m.neg_detect;
    p.flush_branch = flush_branch != 0;
    p.h_min = m.h_min;
    p.v_max = m.v_max;
    p.fr_max = m.fr_max;
    p.dt = dt;
    p.k1 = p.k2 = 0.0;
    p.fcos = 1.0;
    p.fsin = 0.0;
    p.hs = p.hk1 = p.hk2 = 0.0;
    p.hcos = 1.0;
    p.hsin = 0.0;
    if (kFriction != SW2D_FRICTION_NONE) {
        const double4 f = ld(&m.fric[c]);
        p.k1 = f.x;
        p.k2 = f.y;
        p.fcos = f.z;
        p.fsin = f.w;
    }
    if (kHeadLoss) {
        const double4 a = ld(&m.hla[c]);
        const double2 b = ld(&m.hlb[c]);
        p.hs = a.x;
        p.hk1 = a.y;
        p.hk2 = a.z;
        p.hcos = b.x;
        p.hsin = b.y;
    }
    const double4 B = bal[c];
    const double4 l = lam[c];
    // bal.w: h^(-4/3) of the recomputed step's friction stage, its sign bit set where the
    // velocity cap acted
    p.P_given = true;
    p.P = fabs(B.w);
    p.cap_given = true;
    p.cap_acted = signbit(B.w);
    // the adjoints of the cell's first kPre slots, in flight during the cell's reverse
    constexpr int kPre = 4;
    const int k0 = ld(&m.coff[c].y), k1 = ld(&m.coff[c + 1].y);
    double4 s[kPre];
#pragma unroll
    for (int i = 0; i < kPre; i++)
        if (k0 + i < k1) s[i] = ld_sig(&sig[k0 + i]);
    double hb, qb, rb, k1b = 0.0, k2b = 0.0;
    update_cell_rev(p, B.x, B.y, B.z, l.x, l.y, l.z, hb, qb, rb, k1b, k2b);
    if (kFriction != SW2D_FRICTION_NONE) {
        gk1[c] += k1b;
        gk2[c] += k2b;
    }
    lam[c] = make_double4(hb, qb, rb, 0.0);
    const double a = hb * dt, b = qb * dt, cc = rb * dt;
#pragma unroll
    for (int i = 0; i < kPre; i++)
        if (k0 + i < k1) st_sig(&sig[k0 + i], s[i].x + a, s[i].y + b, s[i].z + cc);
    for (int k = k0 + kPre; k < k1; k++) {
        const double4 t = ld_sig(&sig[k]);
        st_sig(&sig[k], t.x + a, t.y + b, t.z + cc);
    }
}

// Flux adjoints of one balance slot {a, b, c} = {f1 F1, f2F2 F2 + f2S2 S + f2F3 F3,
// f3F2 F2 + f3S2 S + f3F3 F3} (factors of swSp::computeEdgeFactors, swSp.cpp:398-427)
struct SlotFactors {
    double f1, f2F2, f2F3, f2S2, f3F2, f3F3, f3S2;
};

__device__ __forceinline__ void slot_rev(const SlotFactors& f, const double4& s, double& F1b, double& F2b, double& F3b,
                                         double& Sb)
{
    F1b += f.f1 * s.x;
    F2b += f.f2F2 * s.y + f.f3F2 * s.z;
    F3b += f.f2F3 * s.y + f.f3F3 * s.z;
    Sb += f.f2S2 * s.y + f.f3S2 * s.z;
}

// kStored: the two Riemann states of the step come from the segment's forward recompute
// (rs, 5 planes of ni double2) and the constants of the two cells from the side table (eside,
// 3 planes of ni double2: {z_b}, {b}, {phi} of (L, R)), so that no load of an internal edge
// depends on another one but the two slot adjoints (on the edge's slots); otherwise the states
// are rebuilt here from the cells.
template <int kScheme, bool kBlending, int kB, int kMinB, bool kStored>
__global__ void __launch_bounds__(kB, kMinB) k_edges_rev(DevMesh m, double4* sig, double4* ctb, double2* cts, double t,
                                                         double dtp, const double2* __restrict__ rs,
                                                         const double2* __restrict__ eside)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m.ni) {
        const int e = i;
        SideState SL, SR;
        double zbL, zbR, bL, bR, phL, phR;
        int2 sl;
        double2 n, cf;
        double4 sa, sb;
        if (kStored) {
            const size_t ni = (size_t)m.ni;
            sl = ld_now(&m.eslot[e]);
            const double2 r0 = ld_now(rs + e), r1 = ld_now(rs + ni + e), r2 = ld_now(rs + 2 * ni + e);
            const double2 r3 = ld_now(rs + 3 * ni + e), r4 = ld_now(rs + 4 * ni + e);
            const double2 z = ld_now(eside + e), bb = ld_now(eside + ni + e), ph = ld_now(eside + 2 * ni + e);
            n = ld_now(&m.nxy[e]);
            cf = ld_now(&m.coef[e]);
            sa = ld_sig(&sig[sl.x]);
            sb = ld_sig(&sig[sl.y]);
            SL.z = r0.x;
            SL.q = r0.y;
            SL.r = r1.x;
            SL.lm = r1.y;
            SL.lp = r2.x;
            SR.z = r2.y;
            SR.q = r3.x;
            SR.r = r3.y;
            SR.lm = r4.x;
            SR.lp = r4.y;
            zbL = z.x;
            zbR = z.y;
            bL = bb.x;
            bR = bb.y;
            phL = ph.x;
            phR = ph.y;
        } else {
            const int2 lr = ld(&m.lr[e]);
            const int a = lr.x, b = lr.y;
            n = ld(&m.nxy[e]);
            sl = ld(&m.eslot[e]);
            const double4 ca = ld(&m.cst[a]), cb = ld(&m.cst[b]);
            const double4 qa = ld(&m.st[a]), qb = ld(&m.st[b]);
            if (kScheme == SW2D_SCHEME_GODUNOV) {
                SL = godunov_side(qa.x, qa.y, qa.z, ca.x, ca.y, n.x, n.y);
                SR = godunov_side(qb.x, qb.y, qb.z, cb.x, cb.y, n.x, n.y);
            } else {
                const double4 d = ld(&m.emc[e]);
                const double2 ga = m.slope[a], gb = m.slope[b];
                SL = evr_side(true, qa.x, qa.y, qa.z, ca.x, ca.y, qa.w, ga.x, ga.y, d.x, d.y, n.x, n.y, dtp, m.dry);
                SR = evr_side(false, qb.x, qb.y, qb.z, cb.x, cb.y, qb.w, gb.x, gb.y, d.z, d.w, n.x, n.y, dtp, m.dry);
            }
            zbL = ca.x;
            zbR = cb.x;
            bL = ca.y;
            bR = cb.y;
            phL = ca.z;
            phR = cb.z;
        }
        const double hL = SL.z - zbL, hR = SR.z - zbR;
        if (!((hL > m.h_min) || (hR > m.h_min))) {
            // flux not computed at this step: the slots keep their values and their adjoints
            ctb[sl.x] = make_double4(0.0, 0.0, 0.0, 0.0);
            ctb[sl.y] = make_double4(0.0, 0.0, 0.0, 0.0);
            cts[sl.x] = make_double2(0.0, 0.0);
            cts[sl.y] = make_double2(0.0, 0.0);
            return;
        }
        if (!kStored) {
            cf = ld(&m.coef[e]);
            sa = ld_sig(&sig[sl.x]);
            sb = ld_sig(&sig[sl.y]);
        }
        const double nx = n.x, ny = n.y;
        EdgeFlux fb;
        fb.f1 = fb.f2 = fb.f3 = fb.sl = fb.sr = 0.0;
        fb.bad = 0;
        {
            const double c = cf.x;
            const SlotFactors f{-c, -c * nx, +c * ny, +c * nx, -c * ny, -c * nx, +c * ny};
            slot_rev(f, sa, fb.f1, fb.f2, fb.f3, fb.sl);
        }
        {
            const double c = cf.y;
            const SlotFactors f{+c, +c * nx, -c * ny, +c * nx, +c * ny, +c * nx, +c * ny};
            slot_rev(f, sb, fb.f1, fb.f2, fb.f3, fb.sr);
        }
        st_sig_zero(&sig[sl.x]);
        st_sig_zero(&sig[sl.y]);
        SideBar Lb{0, 0, 0, 0, 0}, Rb{0, 0, 0, 0, 0};
        double zbLb = 0.0, zbRb = 0.0;
        hllc_rev(kBlending, bL, bR, phL, phR, zbL, zbR, SL, SR, m.h_min, m.phi_min, fb, Lb, Rb, zbLb, zbRb);
        // adjoints of the two Riemann states; k_cells_rev takes them back through the
        // reconstruction of each side
        ctb[sl.x] = make_double4(Lb.z, Lb.q, Lb.r, Lb.lm);
        cts[sl.x] = make_double2(Lb.lp, zbLb);
        ctb[sl.y] = make_double4(Rb.z, Rb.q, Rb.r, Rb.lm);
        cts[sl.y] = make_double2(Rb.lp, zbRb);
    } else if (i < m.ni + m.nb) {
        const int e = i - m.ni;
        const int c = ld(&m.bcell[e]);
        const double4 s = ld(&m.st[c]);
        const double4 cs = ld(&m.cst[c]);
        const double4 g = ld(&m.bgeo[e]);
        const SideState S = godunov_side(s.x, s.y, s.z, cs.x, cs.y, g.x, g.y);
        const int k = ld(&m.bbc[e]);
        const long long o0 = ld(&m.bcoff[k]), o1 = ld(&m.bcoff[k + 1]);
        const double v = bc_value(m.bctimes + o0, m.bcvals + o0, o1 - o0, t);
        const int sb = ld(&m.bslot[e]);
        const double cf = g.w, nx = g.x, ny = g.y;
        const SlotFactors f{+cf, +cf * nx, -cf * ny, +cf * nx, +cf * ny, +cf * nx, +cf * ny};
        double F1b = 0.0, F2b = 0.0, F3b = 0.0, Sb = 0.0;
        slot_rev(f, sig[sb], F1b, F2b, F3b, Sb);
        sig[sb] = make_double4(0.0, 0.0, 0.0, 0.0);
        SideBar sbar{0, 0, 0, 0, 0};
        double zbb = 0.0;
        boundary_flux_rev(cs.y, cs.z, cs.x, S, ld(&m.bctype[k]), v, m.h_min, F1b, F2b, F3b, sbar, zbb);
        CellBar A{0, 0, 0, 0, 0, 0, 0};
        godunov_side_rev(s.x, s.y, s.z, cs.y, nx, ny, sbar, A);
        ctb[sb] = make_double4(A.h, A.q, A.r, A.zb + zbb);
        cts[sb] = make_double2(0.0, 0.0);
    }
}

// The slot geometry of k_cells_rev: per entry k of the cells' neighbour lists (cint), the
// normal of the entry's edge and the midpoint - centroid offset of the cell on that edge
// {nx, ny, dx, dy}, so that a cell's loads all depend on its offsets alone
__global__ void k_slot_geom(DevMesh m, double4* sgeo, int n)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int e0 = ld(&m.coff[c].x), e1 = ld(&m.coff[c + 1].x);
    for (int k = e0; k < e1; k++) {
        const int2 en = ld(&m.cint[k]);
        const int e = en.x >> 1;
        const double2 nn = ld(&m.nxy[e]);
        const double4 d = ld(&m.emc[e]);
        const bool left = (en.x & 1) == 0;
        sgeo[k] = make_double4(nn.x, nn.y, left ? d.x : d.z, left ? d.y : d.w);
    }
}

__device__ __forceinline__ double4 ld_now4(const double4* p)
{
    const double2 a = ld_now(reinterpret_cast<const double2*>(p)), b = ld_now(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// One internal slot of k_cells_rev: the reverse of the cell's reconstruction on that slot,
// added to the cell's sums (skipped when the slot's adjoints are all zero)
template <bool kMuscl>
__device__ __forceinline__ void cell_slot_rev(const double4& a, const double2& b, int entry, const double4& geo,
                                              const double4& s, const double4& cs, const double2& g, double dtp,
                                              double& hb, double& qb, double& rb, double& zbb, double& sxb,
                                              double& syb)
{
    if (a.x == 0.0 && a.y == 0.0 && a.z == 0.0 && a.w == 0.0 && b.x == 0.0 && b.y == 0.0) return;
    const SideBar sb{a.x, a.y, a.z, a.w, b.x};
    CellBar cb{0, 0, 0, 0, 0, 0, 0};
    if (kMuscl) {
        const bool left = (entry & 1) == 0;
        evr_side_rev(left, s.x, s.y, s.z, cs.x, cs.y, s.w, g.x, g.y, geo.z, geo.w, geo.x, geo.y, dtp, sb, cb);
    } else {
        godunov_side_rev(s.x, s.y, s.z, cs.y, geo.x, geo.y, sb, cb);
    }
    // z_c = h + z_b of the cell
    hb += cb.h + cb.zc;
    qb += cb.q;
    rb += cb.r;
    zbb += cb.zb + b.y + cb.zc;
    sxb += cb.sx;
    syb += cb.sy;
}

// Ordered gather, over the slots of each cell in the reference's order: boundary slots hold
// their final contributions; internal slots hold the adjoints of this cell's Riemann state,
// taken back here through the cell's reconstruction (godunov_side / evr_side).  For MUSCL-EVR
// the adjoint of the cell's limited slope goes to sgb for k_limiter_rev.  The adjoints of the
// first kPre internal slots are loaded together, ahead of the boundary sums; a slot's geometry
// only when its adjoints are not all zero.
template <int kScheme>
__global__ void __launch_bounds__(kBlock) k_cells_rev(DevMesh m, double4* lam, const double4* __restrict__ ctb,
                                                      const double2* __restrict__ cts, double* gzb, double2* sgb,
                                                      double dtp, const double4* __restrict__ sgeo)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    constexpr bool kMuscl = kScheme == SW2D_SCHEME_MUSCL_EVR;
    constexpr int kPre = 3;
    const int2 o0 = ld(&m.coff[c]), o1 = ld(&m.coff[c + 1]);
    const int k0 = o0.y, k1 = o1.y, e0 = o0.x, e1 = o1.x;
    const int nint = e1 - e0, nbnd = (k1 - k0) - nint;
    double4 A[kPre];
    double2 Bv[kPre];
#pragma unroll
    for (int i = 0; i < kPre; i++)
        if (i < nint) {
            A[i] = ld_now4(&ctb[k0 + nbnd + i]);
            Bv[i] = ld_now(&cts[k0 + nbnd + i]);
        }
    double hb = 0.0, qb = 0.0, rb = 0.0, zbb = 0.0, sxb = 0.0, syb = 0.0;
    for (int k = k0; k < k0 + nbnd; k++) {
        const double4 v = ctb[k];
        hb += v.x;
        qb += v.y;
        rb += v.z;
        zbb += v.w;
    }
    const double4 s = m.st[c];
    const double4 cs = ld(&m.cst[c]);
    double2 g = make_double2(0.0, 0.0);
    if (kMuscl) g = m.slope[c];
#pragma unroll
    for (int i = 0; i < kPre; i++)
        if (i < nint) {
            const double4 a = A[i];
            const double2 b = Bv[i];
            if (a.x == 0.0 && a.y == 0.0 && a.z == 0.0 && a.w == 0.0 && b.x == 0.0 && b.y == 0.0) continue;
            cell_slot_rev<kMuscl>(a, b, ld(&m.cint[e0 + i]).x, ld(&sgeo[e0 + i]), s, cs, g, dtp, hb, qb, rb, zbb, sxb, syb);
        }
    for (int i = kPre; i < nint; i++) {
        const int k = k0 + nbnd + i;
        cell_slot_rev<kMuscl>(ctb[k], cts[k], ld(&m.cint[e0 + i]).x, sgeo[e0 + i], s, cs, g, dtp, hb, qb, rb, zbb,
                              sxb, syb);
    }
    if (kMuscl) sgb[c] = make_double2(sxb, syb);
    double4 l = lam[c];
    l.x += hb;
    l.y += qb;
    l.z += rb;
    lam[c] = l;
    gzb[c] += zbb;
}

// one reverse step of the trace: non-finite entries of the state adjoint (count, first cell)
// and the largest finite magnitudes (order-preserving bits of non-negative doubles)
__global__ void k_trace(const double4* __restrict__ lam, int n, unsigned long long* out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const double4 l = lam[c];
    if (!isfinite(l.x) || !isfinite(l.y) || !isfinite(l.z)) {
        atomicAdd(out, 1ull);
        atomicMin(out + 3, (unsigned long long)c);
        return;
    }
    atomicMax(out + 1, (unsigned long long)__double_as_longlong(fabs(l.x)));
    atomicMax(out + 2, (unsigned long long)__double_as_longlong(fmax(fabs(l.y), fabs(l.z))));
}

__global__ void k_sanitize(double4* lam, double* gzb, double* gk1, double* gk2, unsigned long long* counts, int n,
                           int with_friction, int keep)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    double4 l = lam[c];
    clean(l.x, counts + 0, keep);
    clean(l.y, counts + 1, keep);
    clean(l.z, counts + 2, keep);
    lam[c] = l;
    clean(gzb[c], counts + 3, keep);
    if (with_friction) {
        clean(gk1[c], counts + 4, keep);
        clean(gk2[c], counts + 5, keep);
    }
}

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------

// buffers that depend only on the mesh
int adjoint_fixed(sw2d_handle* h)
{
    if (h->adj) return SW2D_OK;
    AdjointState* a = new AdjointState();
    h->adj = a;
    int2 last{0, 0};
    CK(cudaMemcpyAsync(&last, h->m.coff + h->nc, sizeof(int2), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    a->ncint = last.x;
    a->nslot = last.y;
    int rc = SW2D_OK;
    auto& L = a->fixed_allocs;
    if ((rc = adj_alloc(h, L, h->nc, &a->lam)) || (rc = adj_alloc(h, L, a->nslot, &a->sig)) ||
        (rc = adj_alloc(h, L, a->nslot, &a->ctb)) || (rc = adj_alloc(h, L, a->nslot, &a->cts)) ||
        (rc = adj_alloc(h, L, a->ncint, &a->znb)) || (rc = adj_alloc(h, L, h->nc, &a->sgb)) || (rc = adj_alloc(h, L, a->ncint, &a->mirror)) ||
        (rc = adj_alloc(h, L, h->nc, &a->g_zb)) || (rc = adj_alloc(h, L, h->nc, &a->g_k1)) ||
        (rc = adj_alloc(h, L, h->nc, &a->g_k2)) || (rc = adj_alloc(h, L, 1, &a->ctrl_rev)) ||
        (rc = adj_alloc(h, L, kCostBlocks, &a->d_part)) ||
        (rc = adj_alloc(h, L, h->nc, &a->stage)) || (rc = adj_alloc(h, L, 6, &a->d_nonfinite)) ||
        (rc = adj_alloc(h, L, a->ncint, &a->sgeo)))
        return rc;
    Ctrl cr{};
    cr.t = 0.0;
    cr.t_max = 1.0;
    CK(cudaMemcpyAsync(a->ctrl_rev, &cr, sizeof(Ctrl), cudaMemcpyHostToDevice, h->stream));
    if (h->nc > 0) k_mirror<<<grid_for(h->nc), kBlock, 0, h->stream>>>(h->m.coff, h->m.cint, a->mirror, (int)h->nc);
    if (h->nc > 0) k_slot_geom<<<grid_for(h->nc), kBlock, 0, h->stream>>>(h->m, a->sgeo, (int)h->nc);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    return SW2D_OK;
}

int require_trajectory(sw2d_handle* h)
{
    if (!h->adj || h->adj->n_steps <= 0) return fail(h, SW2D_E_ARG, "no recorded trajectory (call sw2d_record first)");
    return SW2D_OK;
}

// copies of the state, the slots and the control block into / out of checkpoint k
int ck_save(sw2d_handle* h, int64_t k)
{
    AdjointState* a = h->adj;
    CK(cudaMemcpyAsync(a->ck_st + k * h->nc, h->m.st, h->nc * sizeof(double4), cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(a->ck_slot + k * a->nslot, h->m.slot, a->nslot * sizeof(Slot), cudaMemcpyDeviceToDevice,
                       h->stream));
    CK(cudaMemcpyAsync(a->ck_ctrl + k, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToDevice, h->stream));
    return SW2D_OK;
}

int ck_load(sw2d_handle* h, int64_t k)
{
    AdjointState* a = h->adj;
    CK(cudaMemcpyAsync(h->m.st, a->ck_st + k * h->nc, h->nc * sizeof(double4), cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->m.slot, a->ck_slot + k * a->nslot, a->nslot * sizeof(Slot), cudaMemcpyDeviceToDevice,
                       h->stream));
    CK(cudaMemcpyAsync(h->ctrl, a->ck_ctrl + k, sizeof(Ctrl), cudaMemcpyDeviceToDevice, h->stream));
    return SW2D_OK;
}

ObsView obs_view(const AdjointState* a, int k)
{
    ObsView o;
    o.pts = a->d_pts;
    o.wh = a->d_wh;
    o.wq = a->d_wq;
    o.hobs = a->d_hobs + (size_t)k * a->n_pts;
    o.qobs = a->d_qobs ? a->d_qobs + (size_t)k * a->n_pts : nullptr;
    o.robs = a->d_robs ? a->d_robs + (size_t)k * a->n_pts : nullptr;
    o.n = (int)a->n_pts;
    o.scale = (a->normalize && a->n_obs > 0) ? 1.0 / (double)a->n_obs : 1.0;
    o.wdh = 0;
    return o;
}

void cost_at(sw2d_handle* h, int k, const double4* st)
{
    AdjointState* a = h->adj;
    const ObsView o = obs_view(a, k);
    const int nb = std::max(1, std::min(kCostBlocks, (int)grid_for(a->n_pts)));
    k_obs_cost<<<nb, kBlock, 0, h->stream>>>(o, st, a->d_part);
    k_obs_finish<<<1, 32, 0, h->stream>>>(a->d_part, nb, o.scale, a->d_Jobs + k);
}

int obs_index(const AdjointState* a, int64_t step)
{
    if (a->n_obs == 0 || step < 0 || step >= (int64_t)a->obs_at.size()) return -1;
    return a->obs_at[step];
}

// Forward over the recorded trajectory from checkpoint 0 with the recorded dt (replay) or the
// CFL dt (record), storing checkpoints; `at_step(j)` is called with the state after j steps
// (j = 0 .. n_steps) in the model's state buffer.
template <class F>
int run_trajectory(sw2d_handle* h, bool record, F&& at_step)
{
    AdjointState* a = h->adj;
    int rc = ck_load(h, 0);
    if (rc) return rc;
    at_step(0);
    for (int64_t j = 0; j < a->n_steps; j++) {
        if (j % a->every == 0 && j > 0 && (rc = ck_save(h, j / a->every))) return rc;
        launch_slopes_on(h, h->m);
        launch_edges_on(h, h->m);
        if (record) {
            launch_cfl_on(h, h->m);
            k_note_dt<<<1, 1, 0, h->stream>>>(h->ctrl, a->d_dt_seq, a->d_t_seq, a->base_steps);
        } else {
            k_frozen_dt<<<1, 1, 0, h->stream>>>(h->ctrl, a->d_dt_seq, a->base_steps);
        }
        launch_update_on(h, h->m, false);
        at_step(j + 1);
    }
    if ((rc = ck_save(h, a->n_ck))) return rc;
    CK(cudaGetLastError());
    return SW2D_OK;
}

int run_trajectory(sw2d_handle* h, bool record) { return run_trajectory(h, record, [](int64_t) {}); }

// replay adding the cost of every observation step
int replay_with_cost(sw2d_handle* h)
{
    AdjointState* a = h->adj;
    return run_trajectory(h, false, [&](int64_t j) {
        const int k = obs_index(a, j);
        if (k >= 0) cost_at(h, k, h->m.st);
    });
}

int read_status(sw2d_handle* h)
{
    CK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return status_to_code(h, h->ctrl_host->status);
}

template <int kF>
void launch_update_rev_f(sw2d_handle* h, const double4* bal, double dt)
{
    AdjointState* a = h->adj;
    const unsigned g = grid_for(h->nc);
    if (h->p.singular_head_loss)
        k_update_rev<kF, true><<<g, kBlock, 0, h->stream>>>(h->m, bal, a->lam, a->sig, a->g_k1, a->g_k2, dt,
                                                            h->adj_flush_branch);
    else
        k_update_rev<kF, false><<<g, kBlock, 0, h->stream>>>(h->m, bal, a->lam, a->sig, a->g_k1, a->g_k2, dt,
                                                             h->adj_flush_branch);
}

void launch_update_rev(sw2d_handle* h, const double4* bal, double dt)
{
    switch (h->p.friction) {
        case SW2D_FRICTION_CHEZY: launch_update_rev_f<SW2D_FRICTION_CHEZY>(h, bal, dt); break;
        case SW2D_FRICTION_MANNING: launch_update_rev_f<SW2D_FRICTION_MANNING>(h, bal, dt); break;
        case SW2D_FRICTION_STRICKLER: launch_update_rev_f<SW2D_FRICTION_STRICKLER>(h, bal, dt); break;
        default: launch_update_rev_f<SW2D_FRICTION_NONE>(h, bal, dt); break;
    }
}

// Launch variants {threads per block, minimum resident blocks per SM} of k_edges_rev (its
// register cap); the option "adjoint_edge_variant" selects one.
struct RevVariant {
    int block, minb;
};
constexpr RevVariant kRevVariants[] = {{128, 3}, {256, 1}, {256, 2}, {128, 4}, {256, 3}};
constexpr int kNumRevVariants = sizeof(kRevVariants) / sizeof(kRevVariants[0]);

template <int kScheme, bool kBlending, int V>
void launch_edges_rev_v(sw2d_handle* h, const DevMesh& m, double t, double dtp, const double2* rs)
{
    constexpr int B = kRevVariants[V].block, M = kRevVariants[V].minb;
    AdjointState* a = h->adj;
    const unsigned n = (unsigned)(m.ni + m.nb);
    if (rs)
        k_edges_rev<kScheme, kBlending, B, M, true><<<(n + B - 1) / B, B, 0, h->stream>>>(m, a->sig, a->ctb, a->cts, t,
                                                                                          dtp, rs, a->eside);
    else
        k_edges_rev<kScheme, kBlending, B, M, false><<<(n + B - 1) / B, B, 0, h->stream>>>(m, a->sig, a->ctb, a->cts, t,
                                                                                           dtp, rs, nullptr);
}

template <int kScheme, bool kBlending>
void launch_edges_rev_s(sw2d_handle* h, const DevMesh& m, double t, double dtp, const double2* rs)
{
    switch (h->adj_edge_variant) {
        case 1: launch_edges_rev_v<kScheme, kBlending, 1>(h, m, t, dtp, rs); break;
        case 2: launch_edges_rev_v<kScheme, kBlending, 2>(h, m, t, dtp, rs); break;
        case 3: launch_edges_rev_v<kScheme, kBlending, 3>(h, m, t, dtp, rs); break;
        case 4: launch_edges_rev_v<kScheme, kBlending, 4>(h, m, t, dtp, rs); break;
        default: launch_edges_rev_v<kScheme, kBlending, 0>(h, m, t, dtp, rs); break;
    }
}

// rs: the step's stored Riemann states, or nullptr to rebuild them
void launch_edges_rev(sw2d_handle* h, const DevMesh& m, double t, double dtp, const double2* rs)
{
    const bool bl = h->p.topo == SW2D_TOPO_BLENDING;
    if (h->p.scheme == SW2D_SCHEME_GODUNOV) {
        if (bl) launch_edges_rev_s<SW2D_SCHEME_GODUNOV, true>(h, m, t, dtp, rs);
        else launch_edges_rev_s<SW2D_SCHEME_GODUNOV, false>(h, m, t, dtp, rs);
    } else {
        if (bl) launch_edges_rev_s<SW2D_SCHEME_MUSCL_EVR, true>(h, m, t, dtp, rs);
        else launch_edges_rev_s<SW2D_SCHEME_MUSCL_EVR, false>(h, m, t, dtp, rs);
    }
}

int scatter_cells(sw2d_handle* h, const double* src, int stride, int offset, double* out)
{
    if (!out) return SW2D_OK;
    AdjointState* a = h->adj;
    k_scatter_cells<<<grid_for(h->nc), kBlock, 0, h->stream>>>(src, stride, offset, h->d_cell_perm, a->stage,
                                                                       (int)h->nc);
    CK(cudaMemcpyAsync(out, a->stage, h->nc * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return SW2D_OK;
}

}  // namespace

namespace {

// sum of the per-observation costs, in observation order
int total_cost(sw2d_handle* h, double* J)
{
    AdjointState* a = h->adj;
    std::vector<double> v(a->n_obs, 0.0);
    if (a->n_obs > 0)
        CK(cudaMemcpyAsync(v.data(), a->d_Jobs, a->n_obs * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    double s = 0.0;
    for (double x : v) s += x;
    if (J) *J = s;
    return SW2D_OK;
}

int check_observations(sw2d_handle* h)
{
    AdjointState* a = h->adj;
    if (a->n_obs <= 0) return fail(h, SW2D_E_ARG, "no observations (call sw2d_set_observations)");
    if (a->obs_steps.back() > a->n_steps)
        return fail(h, SW2D_E_ARG, "an observation step lies beyond the recorded trajectory");
    a->obs_at.assign(a->n_steps + 1, -1);
    for (int64_t k = 0; k < a->n_obs; k++) a->obs_at[a->obs_steps[k]] = (int)k;
    return SW2D_OK;
}

// Reverse sweep over the segments (checkpoints must be valid).  Leaves the gradients in lam,
// g_zb, g_k1, g_k2, the per-observation costs in d_Jobs, and the model at the trajectory's end.
int reverse_sweep(sw2d_handle* h)
{
    AdjointState* a = h->adj;
    const int64_t nc = h->nc;
    const bool muscl = h->p.scheme == SW2D_SCHEME_MUSCL_EVR;
    CK(cudaMemsetAsync(a->lam, 0, nc * sizeof(double4), h->stream));
    CK(cudaMemsetAsync(a->sig, 0, a->nslot * sizeof(double4), h->stream));
    CK(cudaMemsetAsync(a->g_zb, 0, nc * sizeof(double), h->stream));
    CK(cudaMemsetAsync(a->g_k1, 0, nc * sizeof(double), h->stream));
    CK(cudaMemsetAsync(a->g_k2, 0, nc * sizeof(double), h->stream));
    const unsigned gc = grid_for(nc);
    if (a->seg_rs && h->ni) k_edge_sides<<<grid_for(h->ni), kBlock, 0, h->stream>>>(h->m, a->eside);
    int rc = SW2D_OK;
    if (h->adj_trace) {
        if (a->trace_steps != a->n_steps) {
            cudaFree(a->d_trace);
            a->d_trace = nullptr;
            CK(cudaMalloc(&a->d_trace, 4 * a->n_steps * sizeof(unsigned long long)));
            a->trace_steps = a->n_steps;
        }
        std::vector<unsigned long long> init(4 * a->n_steps, 0ull);
        for (int64_t j = 0; j < a->n_steps; j++) init[4 * j + 3] = ~0ull;
        CK(cudaMemcpy(a->d_trace, init.data(), init.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice));
    } else if (a->d_trace) {
        cudaFree(a->d_trace);
        a->d_trace = nullptr;
        a->trace_steps = 0;
    }
    for (int64_t s = a->n_ck - 1; s >= 0; s--) {
        const int64_t j0 = s * a->every, j1 = std::min(a->n_steps, j0 + a->every);
        if ((rc = ck_load(h, s))) return rc;
        // recompute the segment, keeping each step's state and post-balance state: step j reads
        // seg_st[j - j0] and writes seg_st[j + 1 - j0]; its dt is frozen, so the CFL
        // contributions are not written
        CK(cudaMemcpyAsync(a->seg_st, h->m.st, nc * sizeof(double4), cudaMemcpyDeviceToDevice, h->stream));
        for (int64_t j = j0; j < j1; j++) {
            DevMesh mj = h->m;
            mj.st = a->seg_st + (j - j0) * nc;
            mj.st_out = a->seg_st + (j + 1 - j0) * nc;
            mj.slot_w = nullptr;
            mj.bal = a->seg_bal + (j - j0) * nc;
            if (a->seg_slope) mj.slope = a->seg_slope + (j - j0) * nc;
            if (a->seg_rs) mj.rstate = a->seg_rs + (j - j0) * 5 * h->ni;
            launch_slopes_on(h, mj);
            launch_edges_on(h, mj);
            k_frozen_dt<<<1, 1, 0, h->stream>>>(h->ctrl, a->d_dt_seq, a->base_steps);
            launch_update_on(h, mj, true);
            const int k = obs_index(a, j + 1);
            if (k >= 0) cost_at(h, k, mj.st_out);
        }
        // reverse steps
        for (int64_t j = j1 - 1; j >= j0; j--) {
            const int k = obs_index(a, j + 1);
            if (k >= 0 && a->n_pts > 0)
                k_obs_rev<<<grid_for(a->n_pts), kBlock, 0, h->stream>>>(obs_view(a, k), a->seg_st + (j + 1 - j0) * nc,
                                                                        a->lam);
            launch_update_rev(h, a->seg_bal + (j - j0) * nc, a->dt_seq[j]);
            DevMesh mr = h->m;
            mr.st = a->seg_st + (j - j0) * nc;
            if (muscl) {
                if (a->seg_slope) {
                    mr.slope = a->seg_slope + (j - j0) * nc;  // kept by the segment's recompute
                } else {
                    DevMesh ms = mr;
                    ms.ctrl = a->ctrl_rev;  // always active: recompute the slopes of step j
                    launch_slopes_on(h, ms);
                }
            }
            launch_edges_rev(h, mr, a->t_seq[j], j > 0 ? a->dt_seq[j - 1] : a->dt_before,
                             a->seg_rs ? a->seg_rs + (j - j0) * 5 * h->ni : nullptr);
            const double dtp = j > 0 ? a->dt_seq[j - 1] : a->dt_before;
            if (muscl) {
                k_cells_rev<SW2D_SCHEME_MUSCL_EVR><<<gc, kBlock, 0, h->stream>>>(mr, a->lam, a->ctb, a->cts, a->g_zb,
                                                                                  a->sgb, dtp, a->sgeo);
                k_limiter_rev<<<gc, kBlock, 0, h->stream>>>(mr, a->sgb, a->lam, a->g_zb, a->znb);
                k_nbr_rev<<<gc, kBlock, 0, h->stream>>>(mr, a->mirror, a->znb, a->lam, a->g_zb);
            } else {
                k_cells_rev<SW2D_SCHEME_GODUNOV><<<gc, kBlock, 0, h->stream>>>(mr, a->lam, a->ctb, a->cts, a->g_zb,
                                                                                a->sgb, dtp, a->sgeo);
            }
            if (a->d_trace && j < a->trace_steps)
                k_trace<<<gc, kBlock, 0, h->stream>>>(a->lam, (int)nc, a->d_trace + 4 * j);
        }
        CK(cudaGetLastError());
    }
    const int k0 = obs_index(a, 0);
    if (k0 >= 0 && a->n_pts > 0) {
        k_obs_rev<<<grid_for(a->n_pts), kBlock, 0, h->stream>>>(obs_view(a, k0), a->ck_st, a->lam);
        cost_at(h, k0, a->ck_st);
    }
    CK(cudaMemsetAsync(a->d_nonfinite, 0, 6 * sizeof(unsigned long long), h->stream));
    k_sanitize<<<gc, kBlock, 0, h->stream>>>(a->lam, a->g_zb, a->g_k1, a->g_k2, a->d_nonfinite, (int)nc,
                                              h->p.friction != SW2D_FRICTION_NONE, h->adj_keep_nonfinite);
    unsigned long long cnt[6];
    CK(cudaMemcpyAsync(cnt, a->d_nonfinite, sizeof(cnt), cudaMemcpyDeviceToHost, h->stream));
    if ((rc = ck_load(h, a->n_ck))) return rc;
    CK(cudaStreamSynchronize(h->stream));
    for (int k = 0; k < 6; k++) a->nonfinite[k] = (int64_t)cnt[k];
    CK(cudaGetLastError());
    return SW2D_OK;
}

int alloc_trajectory(sw2d_handle* h, int64_t n_steps, int64_t every)
{
    AdjointState* a = h->adj;
    free_list(a->traj_allocs);
    a->ck_valid = false;
    a->n_requested = 0;
    a->n_steps = n_steps;
    a->every = every;
    a->n_ck = (n_steps + every - 1) / every;
    const int64_t nc = h->nc, seg = std::min(every, n_steps);
    auto& L = a->traj_allocs;
    int rc = SW2D_OK;
    if ((rc = adj_alloc(h, L, (a->n_ck + 1) * nc, &a->ck_st)) ||
        (rc = adj_alloc(h, L, (a->n_ck + 1) * a->nslot, &a->ck_slot)) ||
        (rc = adj_alloc(h, L, a->n_ck + 1, &a->ck_ctrl)) || (rc = adj_alloc(h, L, (seg + 1) * nc, &a->seg_st)) ||
        (rc = adj_alloc(h, L, seg * nc, &a->seg_bal)) || (rc = adj_alloc(h, L, n_steps, &a->d_dt_seq)) ||
        (rc = adj_alloc(h, L, n_steps, &a->d_t_seq))) {
        free_list(a->traj_allocs);
        a->n_steps = 0;
        return rc;
    }
    // each step's slopes and Riemann states, kept by the segment's forward recompute for the
    // reverse steps, when they fit in half of the free device memory (else rebuilt there)
    a->seg_slope = nullptr;
    a->seg_rs = nullptr;
    a->eside = nullptr;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
        const size_t sl_b = h->p.scheme == SW2D_SCHEME_MUSCL_EVR ? (size_t)seg * nc * sizeof(double2) : 0;
        const size_t rs_b = (size_t)seg * h->ni * 5 * sizeof(double2);
        if (h->adj_store_states && sl_b + rs_b < free_b / 2) {
            if (sl_b && adj_alloc(h, L, seg * nc, &a->seg_slope)) a->seg_slope = nullptr;
            if (h->ni && (adj_alloc(h, L, seg * h->ni * 5, &a->seg_rs) || adj_alloc(h, L, 3 * h->ni, &a->eside))) {
                a->seg_rs = nullptr;
                a->eside = nullptr;
            }
            h->err.clear();
        }
    }
    a->n_requested = n_steps;
    return SW2D_OK;
}

// The CFL-driven run from checkpoint 0 that fixes the trajectory's dt sequence (sw2d_record,
// and sw2d_rerecord at new parameters); stops early at t_max.
int record_from_start(sw2d_handle* h, int64_t* steps_done)
{
    AdjointState* a = h->adj;
    const int64_t n_steps = a->n_requested, every = a->every;
    a->n_steps = n_steps;
    a->n_ck = (n_steps + every - 1) / every;
    a->ck_valid = false;
    int rc = run_trajectory(h, true);
    if (rc) {
        a->n_steps = 0;
        return rc;
    }
    CK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const int64_t done = h->ctrl_host->steps - a->base_steps;
    if (steps_done) *steps_done = done;
    if ((rc = status_to_code(h, h->ctrl_host->status))) {
        a->n_steps = 0;
        return rc;
    }
    if (done <= 0) {
        a->n_steps = 0;
        return fail(h, SW2D_E_ARG, "no step recorded: the run is already at t_max");
    }
    if (done < n_steps) {  // t_max reached: the trajectory ends there
        a->n_steps = done;
        a->n_ck = (done + every - 1) / every;
        if ((rc = ck_save(h, a->n_ck))) return rc;
    }
    a->dt_seq.resize(a->n_steps);
    a->t_seq.resize(a->n_steps);
    CK(cudaMemcpyAsync(a->dt_seq.data(), a->d_dt_seq, a->n_steps * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(a->t_seq.data(), a->d_t_seq, a->n_steps * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    a->ck_valid = true;
    return SW2D_OK;
}

}  // namespace

namespace sw2d {

void adjoint_release(sw2d_handle* h)
{
    if (!h || !h->adj) return;
    cudaFree(h->adj->d_trace);
    free_list(h->adj->traj_allocs);
    free_list(h->adj->obs_allocs);
    free_list(h->adj->fixed_allocs);
    delete h->adj;
    h->adj = nullptr;
}

void adjoint_invalidate(sw2d_handle* h)
{
    if (h && h->adj) h->adj->ck_valid = false;
}

}  // namespace sw2d

// ------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------
extern "C" {

int sw2d_record(sw2d_handle* h, int64_t n_steps, int64_t checkpoint_every, int64_t* steps_done)
{
    if (!h || n_steps <= 0 || checkpoint_every <= 0) return fail(h, SW2D_E_ARG, "invalid arguments");
    if (n_steps >= (int64_t)1 << 31) return fail(h, SW2D_E_ARG, "trajectory too long");
    if (h->model != kModelSp) return fail(h, SW2D_E_UNSUPPORTED, "the adjoint covers the SP model only");
    CK(cudaSetDevice(h->device));
    int rc = adjoint_fixed(h);
    if (rc) return rc;
    AdjointState* a = h->adj;
    if ((rc = alloc_trajectory(h, n_steps, checkpoint_every))) return rc;
    CK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (h->ctrl_host->status) return status_to_code(h, h->ctrl_host->status);
    a->base_steps = h->ctrl_host->steps;
    a->dt_before = h->ctrl_host->dt;
    if ((rc = ck_save(h, 0))) return rc;
    return record_from_start(h, steps_done);
}

int sw2d_rerecord(sw2d_handle* h, int64_t* steps_done)
{
    if (!h) return fail(h, SW2D_E_ARG, "invalid handle");
    if (!h->adj || h->adj->n_requested <= 0)
        return fail(h, SW2D_E_ARG, "no recorded trajectory (call sw2d_record first)");
    CK(cudaSetDevice(h->device));
    return record_from_start(h, steps_done);
}

int sw2d_trajectory_info(sw2d_handle* h, int64_t* n_steps, int64_t* checkpoint_every, double* t_start, double* t_end)
{
    if (!h) return fail(h, SW2D_E_ARG, "invalid handle");
    int rc = require_trajectory(h);
    if (rc) return rc;
    const AdjointState* a = h->adj;
    if (n_steps) *n_steps = a->n_steps;
    if (checkpoint_every) *checkpoint_every = a->every;
    if (t_start) *t_start = a->t_seq.front();
    if (t_end) *t_end = a->t_seq.back() + a->dt_seq.back();
    return SW2D_OK;
}

int sw2d_get_trajectory_dt(sw2d_handle* h, double* dt, int64_t capacity)
{
    if (!h || !dt) return fail(h, SW2D_E_ARG, "invalid arguments");
    int rc = require_trajectory(h);
    if (rc) return rc;
    if (capacity < h->adj->n_steps) return fail(h, SW2D_E_ARG, "output buffer too small");
    std::memcpy(dt, h->adj->dt_seq.data(), h->adj->n_steps * sizeof(double));
    return SW2D_OK;
}

int sw2d_set_trajectory_start(sw2d_handle* h, const double* h0, const double* q0, const double* r0)
{
    if (!h || !h0 || !q0 || !r0) return fail(h, SW2D_E_ARG, "invalid arguments");
    int rc = require_trajectory(h);
    if (rc) return rc;
    CK(cudaSetDevice(h->device));
    AdjointState* a = h->adj;
    const int64_t nc = h->nc;
    const size_t bytes = nc * sizeof(double);
    double* ck0 = reinterpret_cast<double*>(a->ck_st);
    const double* src[3] = {h0, q0, r0};
    for (int c = 0; c < 3; c++) {
        CK(cudaMemcpyAsync(a->stage, src[c], bytes, cudaMemcpyHostToDevice, h->stream));
        k_gather_component<<<grid_for(nc), kBlock, 0, h->stream>>>(a->stage, h->d_cell_perm, ck0, 4, c, (int)nc);
    }
    k_refresh_z<<<grid_for(nc), kBlock, 0, h->stream>>>(a->ck_st, h->m.zbv, (int)nc);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    a->ck_valid = false;
    return SW2D_OK;
}

int sw2d_set_param(sw2d_handle* h, const char* name, const double* values)
{
    if (!h || !name || !values) return fail(h, SW2D_E_ARG, "invalid arguments");
    CK(cudaSetDevice(h->device));
    const int64_t nc = h->nc;
    double* dst = nullptr;
    int stride = 0, off = 0;
    const bool f1 = std::strcmp(name, "friction_1") == 0, f2 = std::strcmp(name, "friction_2") == 0;
    const bool fb = std::strcmp(name, "friction") == 0, zb = std::strcmp(name, "z_b") == 0;
    if (f1 || f2 || fb) {
        if (h->p.friction == SW2D_FRICTION_NONE) return fail(h, SW2D_E_ARG, "the model has no friction law");
        dst = reinterpret_cast<double*>(const_cast<double4*>(h->m.fric));
        stride = 4;
        off = f2 ? 1 : 0;
    } else if (zb) {
        dst = reinterpret_cast<double*>(const_cast<double4*>(h->m.cst));
        stride = 4;
        off = 0;
    } else {
        return fail(h, SW2D_E_ARG, std::string("unknown parameter ") + name);
    }
    CK(cudaMemcpyAsync(h->stage, values, nc * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    k_gather_component<<<grid_for(nc), kBlock, 0, h->stream>>>(h->stage, h->d_cell_perm, dst, stride, off, (int)nc);
    if (fb)
        k_gather_component<<<grid_for(nc), kBlock, 0, h->stream>>>(h->stage, h->d_cell_perm, dst, stride, 1, (int)nc);
    if (zb) {
        k_gather_component<<<grid_for(nc), kBlock, 0, h->stream>>>(h->stage, h->d_cell_perm, const_cast<double*>(h->m.zbv),
                                                                   1, 0, (int)nc);
        // z = h + z_b of the current state and of the trajectory's initial state
        k_refresh_z<<<grid_for(nc), kBlock, 0, h->stream>>>(h->m.st, h->m.zbv, (int)nc);
        if (h->adj && h->adj->n_steps > 0)
            k_refresh_z<<<grid_for(nc), kBlock, 0, h->stream>>>(h->adj->ck_st, h->m.zbv, (int)nc);
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    adjoint_invalidate(h);
    return SW2D_OK;
}

int sw2d_get_param(sw2d_handle* h, const char* name, double* values)
{
    if (!h || !name || !values) return fail(h, SW2D_E_ARG, "invalid arguments");
    CK(cudaSetDevice(h->device));
    const double* src = nullptr;
    int off = 0;
    if (std::strcmp(name, "friction_1") == 0 || std::strcmp(name, "friction_2") == 0) {
        if (h->p.friction == SW2D_FRICTION_NONE) return fail(h, SW2D_E_ARG, "the model has no friction law");
        src = reinterpret_cast<const double*>(h->m.fric);
        off = name[9] == '2' ? 1 : 0;
    } else if (std::strcmp(name, "z_b") == 0) {
        src = reinterpret_cast<const double*>(h->m.cst);
    } else {
        return fail(h, SW2D_E_ARG, std::string("unknown parameter ") + name);
    }
    k_scatter_cells<<<grid_for(h->nc), kBlock, 0, h->stream>>>(src, 4, off, h->d_cell_perm, h->stage, (int)h->nc);
    CK(cudaMemcpyAsync(values, h->stage, h->nc * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return SW2D_OK;
}

int sw2d_set_observations(sw2d_handle* h, const sw2d_obs* obs)
{
    if (!h || !obs) return fail(h, SW2D_E_ARG, "invalid arguments");
    if (obs->n_points < 0 || obs->n_times <= 0 || (obs->n_points > 0 && (!obs->cells || !obs->w_h || !obs->h_obs)) ||
        !obs->steps)
        return fail(h, SW2D_E_ARG, "incomplete observation set");
    if (obs->w_q && (!obs->q_obs || !obs->r_obs)) return fail(h, SW2D_E_ARG, "w_q given without q_obs / r_obs");
    CK(cudaSetDevice(h->device));
    int rc = adjoint_fixed(h);
    if (rc) return rc;
    AdjointState* a = h->adj;
    const int64_t np = obs->n_points, nt = obs->n_times;
    std::vector<int> inv(h->nc), pts(np);
    for (int64_t i = 0; i < h->nc; i++) inv[h->cell_perm[i]] = (int)i;
    std::vector<char> seen(h->nc, 0);
    for (int64_t i = 0; i < np; i++) {
        const int64_t c = obs->cells[i];
        if (c < 0 || c >= h->nc) return fail(h, SW2D_E_ARG, "observed cell out of range");
        if (seen[c]) return fail(h, SW2D_E_ARG, "an observed cell appears twice");
        seen[c] = 1;
        pts[i] = inv[c];
    }
    for (int64_t k = 0; k < nt; k++)
        if (obs->steps[k] < 0 || (k > 0 && obs->steps[k] <= obs->steps[k - 1]))
            return fail(h, SW2D_E_ARG, "observation steps must be non-negative and increasing");
    free_list(a->obs_allocs);
    a->n_pts = 0;
    a->n_obs = 0;
    auto& L = a->obs_allocs;
    a->d_wq = a->d_qobs = a->d_robs = nullptr;
    if ((rc = adj_alloc(h, L, np, &a->d_pts)) || (rc = adj_alloc(h, L, np, &a->d_wh)) ||
        (rc = adj_alloc(h, L, np * nt, &a->d_hobs)) || (rc = adj_alloc(h, L, nt, &a->d_Jobs)))
        return rc;
    if (obs->w_q && ((rc = adj_alloc(h, L, np, &a->d_wq)) || (rc = adj_alloc(h, L, np * nt, &a->d_qobs)) ||
                     (rc = adj_alloc(h, L, np * nt, &a->d_robs))))
        return rc;
    if (np > 0) {
        CK(cudaMemcpyAsync(a->d_pts, pts.data(), np * sizeof(int), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(a->d_wh, obs->w_h, np * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(a->d_hobs, obs->h_obs, np * nt * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        if (obs->w_q) {
            CK(cudaMemcpyAsync(a->d_wq, obs->w_q, np * sizeof(double), cudaMemcpyHostToDevice, h->stream));
            CK(cudaMemcpyAsync(a->d_qobs, obs->q_obs, np * nt * sizeof(double), cudaMemcpyHostToDevice, h->stream));
            CK(cudaMemcpyAsync(a->d_robs, obs->r_obs, np * nt * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        }
    }
    CK(cudaStreamSynchronize(h->stream));
    a->n_pts = np;
    a->n_obs = nt;
    a->normalize = obs->normalize ? 1 : 0;
    a->obs_steps.assign(obs->steps, obs->steps + nt);
    return SW2D_OK;
}

int sw2d_replay_cost(sw2d_handle* h, double* J)
{
    if (!h) return fail(h, SW2D_E_ARG, "invalid handle");
    int rc = require_trajectory(h);
    if (rc) return rc;
    CK(cudaSetDevice(h->device));
    if ((rc = check_observations(h))) return rc;
    if ((rc = replay_with_cost(h))) return rc;
    if ((rc = read_status(h))) return rc;
    h->adj->ck_valid = true;
    return total_cost(h, J);
}

int sw2d_replay_sample(sw2d_handle* h, int64_t n_points, const int64_t* cells, int64_t n_times, const int64_t* steps,
                       double* h_out, double* q_out, double* r_out)
{
    if (!h || n_points <= 0 || n_times <= 0 || !cells || !steps || !h_out)
        return fail(h, SW2D_E_ARG, "invalid arguments");
    int rc = require_trajectory(h);
    if (rc) return rc;
    CK(cudaSetDevice(h->device));
    AdjointState* a = h->adj;
    std::vector<int> at(a->n_steps + 1, -1);
    for (int64_t k = 0; k < n_times; k++) {
        if (steps[k] < 0 || steps[k] > a->n_steps) return fail(h, SW2D_E_ARG, "sample step outside the trajectory");
        if (k > 0 && steps[k] <= steps[k - 1]) return fail(h, SW2D_E_ARG, "sample steps must be increasing");
        at[steps[k]] = (int)k;
    }
    std::vector<int> inv(h->nc), pts(n_points);
    for (int64_t i = 0; i < h->nc; i++) inv[h->cell_perm[i]] = (int)i;
    for (int64_t p = 0; p < n_points; p++) {
        if (cells[p] < 0 || cells[p] >= h->nc) return fail(h, SW2D_E_ARG, "sampled cell out of range");
        pts[p] = inv[cells[p]];
    }
    std::vector<void*> tmp;
    int* d_pts = nullptr;
    double4* d_out = nullptr;
    auto release = [&] { free_list(tmp); };
    if ((rc = adj_alloc(h, tmp, n_points, &d_pts)) || (rc = adj_alloc(h, tmp, n_points * n_times, &d_out))) {
        release();
        return rc;
    }
    if (cudaMemcpyAsync(d_pts, pts.data(), n_points * sizeof(int), cudaMemcpyHostToDevice, h->stream) != cudaSuccess) {
        release();
        return fail(h, SW2D_E_CUDA, "sample upload");
    }
    const unsigned g = grid_for(n_points);
    rc = run_trajectory(h, false, [&](int64_t j) {
        if (at[j] >= 0)
            k_sample<<<g, kBlock, 0, h->stream>>>(h->m.st, d_pts, d_out + (size_t)at[j] * n_points, (int)n_points);
    });
    std::vector<double4> out(n_points * n_times);
    if (!rc && cudaMemcpyAsync(out.data(), d_out, out.size() * sizeof(double4), cudaMemcpyDeviceToHost, h->stream) !=
                   cudaSuccess)
        rc = fail(h, SW2D_E_CUDA, "sample read-back");
    if (!rc && cudaStreamSynchronize(h->stream) != cudaSuccess) rc = fail(h, SW2D_E_CUDA, "sample synchronise");
    release();
    if (rc) return rc;
    if ((rc = read_status(h))) return rc;
    a->ck_valid = true;
    for (size_t i = 0; i < out.size(); i++) {
        h_out[i] = out[i].x;
        if (q_out) q_out[i] = out[i].y;
        if (r_out) r_out[i] = out[i].z;
    }
    return SW2D_OK;
}

int sw2d_adjoint(sw2d_handle* h, double* J, const sw2d_gradient* grad)
{
    if (!h) return fail(h, SW2D_E_ARG, "invalid handle");
    int rc = require_trajectory(h);
    if (rc) return rc;
    CK(cudaSetDevice(h->device));
    AdjointState* a = h->adj;
    if ((rc = check_observations(h))) return rc;
    if (!a->ck_valid) {
        if ((rc = run_trajectory(h, false))) return rc;
        if ((rc = read_status(h))) return rc;
        a->ck_valid = true;
    }
    if ((rc = reverse_sweep(h))) return rc;
    if ((rc = read_status(h))) return rc;
    if ((rc = total_cost(h, J))) return rc;
    if (grad) {
        const double* lam = reinterpret_cast<const double*>(a->lam);
        if ((rc = scatter_cells(h, lam, 4, 0, grad->h0)) || (rc = scatter_cells(h, lam, 4, 1, grad->q0)) ||
            (rc = scatter_cells(h, lam, 4, 2, grad->r0)) || (rc = scatter_cells(h, a->g_zb, 1, 0, grad->z_b)))
            return rc;
        if (h->p.friction != SW2D_FRICTION_NONE) {
            if ((rc = scatter_cells(h, a->g_k1, 1, 0, grad->friction_1)) ||
                (rc = scatter_cells(h, a->g_k2, 1, 0, grad->friction_2)))
                return rc;
        } else {
            if (grad->friction_1) std::memset(grad->friction_1, 0, h->nc * sizeof(double));
            if (grad->friction_2) std::memset(grad->friction_2, 0, h->nc * sizeof(double));
        }
    }
    return SW2D_OK;
}

int sw2d_adjoint_trace(sw2d_handle* h, int64_t* nonfinite, double* max_h, double* max_qr, int64_t* first_cell,
                       int64_t capacity)
{
    if (!h || capacity < 0) return fail(h, SW2D_E_ARG, "invalid arguments");
    if (!h->adj || !h->adj->d_trace) return fail(h, SW2D_E_ARG, "no traced gradient (option adjoint_trace)");
    AdjointState* a = h->adj;
    const int64_t n = std::min(capacity, a->trace_steps);
    std::vector<unsigned long long> t(4 * a->trace_steps);
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpy(t.data(), a->d_trace, t.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    for (int64_t j = 0; j < n; j++) {
        if (nonfinite) nonfinite[j] = (int64_t)t[4 * j];
        if (max_h) max_h[j] = __builtin_bit_cast(double, t[4 * j + 1]);
        if (max_qr) max_qr[j] = __builtin_bit_cast(double, t[4 * j + 2]);
        if (first_cell) first_cell[j] = t[4 * j + 3] == ~0ull ? -1 : h->cell_perm[t[4 * j + 3]];
    }
    return (int)std::min<int64_t>(a->trace_steps, INT32_MAX);
}

int sw2d_adjoint_nonfinite(sw2d_handle* h, int64_t* counts)
{
    if (!h || !counts) return fail(h, SW2D_E_ARG, "invalid arguments");
    if (!h->adj) return fail(h, SW2D_E_ARG, "no gradient computed yet");
    for (int k = 0; k < 6; k++) counts[k] = h->adj->nonfinite[k];
    return SW2D_OK;
}

}  // extern "C"
