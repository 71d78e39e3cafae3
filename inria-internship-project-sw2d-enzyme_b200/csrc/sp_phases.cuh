// sp_phases.cuh — the per-element bodies of the SP/DIP step's phases, shared by the step kernels
// (k_slopes, k_edges, k_cfl, k_update in sw2d_sp.cu) and the ensemble work-queue kernel
// (sw2d_queue.cu), so that both compute the same bits.
//
//   slopes_cell     one cell's limited free-surface slope      swSpHypMusclEvr.cpp:11-115
//   edge_internal   one internal edge: Riemann states, CFL     swSpHypGodunov.cpp, swSpHypMusclEvr.cpp:119-277,
//                   contributions, HLLC, balance slots         swSpHyp.cpp:276-402,664-998
//   edge_boundary   one boundary edge                          swSpHyp.cpp:13-135
//   cfl_cell        one cell's CFL bound                       swSpHyp.cpp:430-495
//   dt_finalize     dt_map snap and t_max clip of the grid dt  swSpHyp.cpp:496-512
//   update_cell     one cell's balance, flush, clamp, sources  swSpHyp.cpp:184-273, swSpSourceFriction.cpp
//
// The load policy L says how a body reads the arrays that the step itself writes (states,
// slopes, balance slots, CFL contributions, the control block).  LdNc: the step kernels, where
// those arrays were written by an earlier kernel, through the read-only path.  LdL2: through L2
// only.  LdCo: plain (coherent, L1-cached) loads, for the work-queue kernel, where other CTAs of
// the same launch wrote the arrays: each item starts after a gpu-scope acquire of the counter
// its prerequisites released, followed by a CTA barrier, and the memory model then orders its
// plain loads after those writes (the read-only path gives no such guarantee).  The arithmetic
// is the same under every policy.
#pragma once

#include "sw2d_internal.cuh"

namespace sw2d {

// loads through L2 only (ld.global.cg)
template <class T>
__device__ __forceinline__ T ldl2(const T* p) { return __ldcg(p); }

__device__ __forceinline__ double4 ldl2(const double4* p)
{
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = __ldcg(q), b = __ldcg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ Slot ldl2(const Slot* p)
{
    const double* q = reinterpret_cast<const double*>(p);
    return make_slot(__ldcg(q), __ldcg(q + 1), __ldcg(q + 2));
}

struct LdNc {
    // an array written by an earlier kernel
    template <class T>
    static __device__ __forceinline__ T in(const T* p) { return ld(p); }
    // an array this thread reads and then writes (the update's own state and slots)
    template <class T>
    static __device__ __forceinline__ T own(const T* p) { return *p; }
    static __device__ __forceinline__ double ctl(const double* p) { return *p; }
};

struct LdL2 {
    template <class T>
    static __device__ __forceinline__ T in(const T* p) { return ldl2(p); }
    template <class T>
    static __device__ __forceinline__ T own(const T* p) { return ldl2(p); }
    static __device__ __forceinline__ double ctl(const double* p) { return __ldcg(p); }
};

struct LdCo {
    template <class T>
    static __device__ __forceinline__ T in(const T* p) { return *p; }
    template <class T>
    static __device__ __forceinline__ T own(const T* p) { return *p; }
    static __device__ __forceinline__ double ctl(const double* p) { return *p; }
};

// ------------------------------------------------------------------------------------------
// slopes_cell: swSp::computeMusclSlopes (swSpHypMusclEvr.cpp:11-115) for one cell.  Step 1 sums
// the neighbour contributions in increasing internal-edge order; step 2 applies, edge after
// edge in the same order, the under/overshoot rescaling of this cell's slope (that rescaling
// only reads this cell's slope, so the reference's global edge loop decomposes exactly per
// cell).  Cells with up to kUnrollSlopes neighbours issue all their neighbour loads up front.
// ------------------------------------------------------------------------------------------
constexpr int kUnroll = 4;        // balance slots handled without a loop (cell degree)
constexpr int kUnrollSlopes = 3;  // neighbours gathered up front in slopes_cell (triangles)

__device__ __forceinline__ void limit_slope(double zc, double zj, bool is_r, double2 mp, double2 xy, double& sx,
                                            double& sy)
{
    const double zL = is_r ? zj : zc;
    const double zR = is_r ? zc : zj;
    const double fmx = smax(zL, zR);
    const double fmn = smin(zL, zR);
    const double rec = zc + (mp.x - xy.x) * sx + (mp.y - xy.y) * sy;
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

__device__ __forceinline__ void grad_term(double zc, double zj, double2 xy, double2 xj, double& sx, double& sy,
                                          double& wsum)
{
    double dx = xj.x - xy.x;
    double dy = xj.y - xy.y;
    double dist = sqrt(dx * dx + dy * dy);
    double w = 1.0 / dist;
    sx += (zj - zc) * dx / dist / dist * w;
    sy += (zj - zc) * dy / dist / dist * w;
    wsum += w;
}

template <class L>
__device__ __forceinline__ void slopes_cell(const DevMesh& m, int c)
{
    const double zc = L::in(&m.st[c].w);
    const double2 xy = ld(&m.cxy[c]);
    const int k0 = ld(&m.coff[c].x), k1 = ld(&m.coff[c + 1].x);
    const int cnt = k1 - k0;
    double sx = 0.0, sy = 0.0, wsum = 0.0;
    if (cnt <= kUnrollSlopes) {
        int2 en[kUnrollSlopes];
        double zj[kUnrollSlopes];
        double2 xj[kUnrollSlopes];
#pragma unroll
        for (int i = 0; i < kUnrollSlopes; i++)
            if (i < cnt) en[i] = ld(&m.cint[k0 + i]);
#pragma unroll
        for (int i = 0; i < kUnrollSlopes; i++)
            if (i < cnt) {
                zj[i] = L::in(&m.st[en[i].y].w);
                xj[i] = ld(&m.cxy[en[i].y]);
            }
        if (cnt > 1) {
#pragma unroll
            for (int i = 0; i < kUnrollSlopes; i++)
                if (i < cnt) grad_term(zc, zj[i], xy, xj[i], sx, sy, wsum);
            sx /= wsum;
            sy /= wsum;
        }
#pragma unroll
        for (int i = 0; i < kUnrollSlopes; i++)
            if (i < cnt) limit_slope(zc, zj[i], en[i].x & 1, ld(&m.mxy[en[i].x >> 1]), xy, sx, sy);
    } else {
        for (int k = k0; k < k1; k++) {
            const int j = ld(&m.cint[k]).y;
            grad_term(zc, L::in(&m.st[j].w), xy, ld(&m.cxy[j]), sx, sy, wsum);
        }
        sx /= wsum;
        sy /= wsum;
        for (int k = k0; k < k1; k++) {
            const int2 en = ld(&m.cint[k]);
            limit_slope(zc, L::in(&m.st[en.y].w), en.x & 1, ld(&m.mxy[en.x >> 1]), xy, sx, sy);
        }
    }
    m.slope[c] = make_double2(sx, sy);
}

// ------------------------------------------------------------------------------------------
// edge_internal: one internal edge.  Writes the balance terms {a, b, c} of the edge into the
// slots of its cells (when the flux is computed) and, every step, the CFL contributions
// lambda_max * length that hypComputeTimeStep adds (swSpHyp.cpp:437-477: the L cell counts it
// when it is wet; the R cell when L or R is wet, because the reference carries `lambda` over
// from the L test).  Returns the status bits of the edge.
// ------------------------------------------------------------------------------------------
template <int kScheme, bool kBlending, int kModel, class L>
__device__ __forceinline__ unsigned edge_internal(const DevMesh& m, int e)
{
    constexpr bool kDip = kModel == kModelDip;
    unsigned bad = 0;
    const int2 lr = ld(&m.lr[e]);
    const int a = lr.x, b = lr.y;
    const double2 n = ld(&m.nxy[e]);
    // the edge's own tables, in flight with the cell gathers (else the slots and factors are
    // loaded after the Riemann solve, which then waits for them)
    const int2 sl = ld_now(&m.eslot[e]);
    const double2 cf = ld_now(&m.coef[e]);
    const double len_e = ld(&m.len[e]);
    const double4 emc_e = (kScheme != SW2D_SCHEME_GODUNOV) ? ld(&m.emc[e]) : make_double4(0.0, 0.0, 0.0, 0.0);
    const double4 sa = L::in(&m.st[a]), sb = L::in(&m.st[b]);
    const double4 ca = ld(&m.cst[a]), cb = ld(&m.cst[b]);
    SideState SL, SR;
    double phiG = 0.0, xL = 1.0, xR = 1.0;
    if (kDip) {
        phiG = ld(&m.phig[e]);
        xL = dip_x(ca.z, phiG);
        xR = dip_x(cb.z, phiG);
    }
    if (kScheme == SW2D_SCHEME_GODUNOV) {
        if (kDip) {
            SL = godunov_side_dip(sa.x, sa.y, sa.z, ca.x, ca.y, xL, n.x, n.y);
            SR = godunov_side_dip(sb.x, sb.y, sb.z, cb.x, cb.y, xR, n.x, n.y);
        } else {
            SL = godunov_side(sa.x, sa.y, sa.z, ca.x, ca.y, n.x, n.y);
            SR = godunov_side(sb.x, sb.y, sb.z, cb.x, cb.y, n.x, n.y);
        }
    } else {
        const double dtp = L::ctl(&m.ctrl->dt);
        const double4 d = emc_e;  // midpoint - centroid of L and R
        const double2 ga = L::in(&m.slope[a]), gb = L::in(&m.slope[b]);
        if (kDip) {
            SL = evr_side_dip(true, sa.x, sa.y, sa.z, ca.x, ca.y, xL, sa.w, ga.x, ga.y, d.x, d.y, n.x, n.y, dtp);
            SR = evr_side_dip(false, sb.x, sb.y, sb.z, cb.x, cb.y, xR, sb.w, gb.x, gb.y, d.z, d.w, n.x, n.y, dtp);
        } else {
            SL = evr_side(true, sa.x, sa.y, sa.z, ca.x, ca.y, sa.w, ga.x, ga.y, d.x, d.y, n.x, n.y, dtp, m.dry);
            SR = evr_side(false, sb.x, sb.y, sb.z, cb.x, cb.y, sb.w, gb.x, gb.y, d.z, d.w, n.x, n.y, dtp, m.dry);
        }
    }
    const double lm = max4(fabs(SL.lm), fabs(SL.lp), fabs(SR.lm), fabs(SR.lp));
    if (m.lmax) m.lmax[e] = lm;
    if (m.rstate) {
        // five planes of ni double2 each, so that a warp's stores and the reverse's loads are
        // contiguous
        const size_t ni = (size_t)m.ni;
        double2* p = m.rstate + e;
        p[0] = make_double2(SL.z, SL.q);
        p[ni] = make_double2(SL.r, SL.lm);
        p[2 * ni] = make_double2(SL.lp, SR.z);
        p[3 * ni] = make_double2(SR.q, SR.r);
        p[4 * ni] = make_double2(SR.lm, SR.lp);
    }
    const double lw = lm * len_e;
    const bool wetL = sa.x > m.h_min, wetR = sb.x > m.h_min;
    if (m.slot_w) {
        m.slot_w[sl.x] = wetL ? lw : 0.0;
        m.slot_w[sl.y] = (wetL || wetR) ? lw : 0.0;
    }
    const double hL = SL.z - ca.x, hR = SR.z - cb.x;
    if ((hL > m.h_min) || (hR > m.h_min)) {
        EdgeFlux f = kDip ? hllc_dip(kBlending, ca.y, cb.y, phiG, ca.z, cb.z, ca.x, cb.x, SL, SR, m.h_min, m.phi_min)
                          : hllc(kBlending, ca.y, cb.y, ca.z, cb.z, ca.x, cb.x, SL, SR, m.h_min, m.phi_min);
        bad |= f.bad;
        if (isnan(f.f1)) bad |= kStatusNanFlux;
        if (m.flux) {
            double2* fp = m.flux + 3 * (size_t)e;
            fp[0] = make_double2(f.f1, f.f2);
            fp[1] = make_double2(f.f3, f.sl);
            fp[2] = make_double2(f.sr, 0.0);
        }
        // factors of swSp::computeEdgeFactors (swSp.cpp:398-427) and the dt-free products of
        // hypComputeBalance (swSpHyp.cpp:237-262)
        const double nx = n.x, ny = n.y;
        {
            const double c = cf.x;
            const double f1 = -c, f2F2 = -c * nx, f2F3 = +c * ny, f2S2 = +c * nx;
            const double f3F2 = -c * ny, f3F3 = -c * nx, f3S2 = +c * ny;
            m.slot[sl.x] = make_slot(f1 * f.f1, f2F2 * f.f2 + f2S2 * f.sl + f2F3 * f.f3,
                                     f3F2 * f.f2 + f3S2 * f.sl + f3F3 * f.f3);
        }
        {
            const double c = cf.y;
            const double f1 = +c, f2F2 = +c * nx, f2F3 = -c * ny, f2S2 = +c * nx;
            const double f3F2 = +c * ny, f3F3 = +c * nx, f3S2 = +c * ny;
            m.slot[sl.y] = make_slot(f1 * f.f1, f2F2 * f.f2 + f2S2 * f.sr + f2F3 * f.f3,
                                     f3F2 * f.f2 + f3S2 * f.sr + f3F3 * f.f3);
        }
    }
    return bad;
}

// edge_boundary: one boundary edge (hypBoundaryFlux); returns the status bits of the edge
template <int kScheme, int kModel, class L>
__device__ __forceinline__ unsigned edge_boundary(const DevMesh& m, int e)
{
    constexpr bool kDip = kModel == kModelDip;
    const int c = ld(&m.bcell[e]);
    const double4 s = L::in(&m.st[c]);
    const double4 cs = ld(&m.cst[c]);
    const double4 g = ld(&m.bgeo[e]);
    const double phiGb = kDip ? ld(&m.phigb[e]) : 0.0;
    SideState S = kDip ? godunov_side_dip(s.x, s.y, s.z, cs.x, cs.y, dip_x(cs.z, phiGb), g.x, g.y)
                       : godunov_side(s.x, s.y, s.z, cs.x, cs.y, g.x, g.y);
    const double lm = (kScheme == SW2D_SCHEME_GODUNOV) ? smax(fabs(S.lp), fabs(S.lm)) : smax(fabs(S.lm), fabs(S.lp));
    if (m.lmaxb) m.lmaxb[e] = lm;
    const int sb = ld(&m.bslot[e]);
    if (m.slot_w) m.slot_w[sb] = (s.x > m.h_min) ? lm * g.z : 0.0;
    const int k = ld(&m.bbc[e]);
    const long long o0 = ld(&m.bcoff[k]), o1 = ld(&m.bcoff[k + 1]);
    const double v = bc_value(m.bctimes + o0, m.bcvals + o0, o1 - o0, L::ctl(&m.ctrl->t));
    double f1, f2, f3;
    const unsigned bad = kDip ? boundary_flux_dip(cs.y, phiGb, cs.z, cs.x, S, ld(&m.bctype[k]), v, m.h_min, &f1, &f2, &f3)
                              : boundary_flux(cs.y, cs.z, cs.x, S, ld(&m.bctype[k]), v, m.h_min, &f1, &f2, &f3);
    if (m.bflux) m.bflux[e] = make_double4(f1, f2, f3, 0.0);
    const double cf = g.w, nx = g.x, ny = g.y;
    const double fa = +cf, f2F2 = +cf * nx, f2F3 = -cf * ny, f2S2 = +cf * nx;
    const double f3F2 = +cf * ny, f3F3 = +cf * nx, f3S2 = +cf * ny;
    const double s2 = 0.0;  // boundary geometric source: never set by hypBoundaryFlux
    m.slot[sb] = make_slot(fa * f1, f2F2 * f2 + f2S2 * s2 + f2F3 * f3, f3F2 * f2 + f3S2 * s2 + f3F3 * f3);
    return bad;
}

// ------------------------------------------------------------------------------------------
// cfl_cell: the CFL bound cfl * area / max(swept, 1e-16) of one cell (swSpHyp.cpp:430-495).
// swept sums the cell's slot contributions in the reference's order; a skipped contribution
// is stored as 0, and adding +0 to the (non-negative) sum changes no bit.
// ------------------------------------------------------------------------------------------
template <class L>
__device__ __forceinline__ double cfl_cell(const DevMesh& m, int c)
{
    const int k0 = ld(&m.coff[c].y), k1 = ld(&m.coff[c + 1].y);
    double sw = 0.0;
    if (k1 - k0 <= kUnroll) {
        double w[kUnroll];
#pragma unroll
        for (int i = 0; i < kUnroll; i++) w[i] = (i < k1 - k0) ? L::in(&m.slot_w[k0 + i]) : 0.0;
#pragma unroll
        for (int i = 0; i < kUnroll; i++)
            if (i < k1 - k0) sw += w[i];
    } else {
        for (int k = k0; k < k1; k++) sw += L::in(&m.slot_w[k]);
    }
    return m.cfl_max * (ld(&m.area[c]) / smax(sw, kSmallReal));
}

// minimum that keeps a when b is not smaller (a NaN candidate b never wins)
__device__ __forceinline__ double min_keep(double a, double b) { return (b < a) ? b : a; }

// dt_finalize: the grid minimum dt (at most dt_max), snapped to the next storage time
// (swSpHyp.cpp:496-504) and clipped at t_max; sets the control block's dt, go and store_map.
// kDdpSnap: the DDP model's form of the snap, which truncates t and t + dt to integers before
// dividing by dt_map (swDdpHyp.cpp:588-600: `(int)t / dt_map`).
template <bool kDdpSnap, class L = LdNc>
__device__ __forceinline__ void dt_finalize(const DevMesh& m, Ctrl* ctrl, double dt)
{
    const double t = L::ctl(&ctrl->t);
    const double t_max = L::ctl(&ctrl->t_max);
    int store = m.dt_map <= -kSmallReal ? 1 : 0;
    if (m.dt_map > kSmallReal) {
        int now, later;
        if (kDdpSnap) {
            now = (int)((double)(int)t / m.dt_map);
            later = (int)((double)(int)(t + dt) / m.dt_map);
        } else {
            now = (int)(t / m.dt_map);
            later = (int)((t + dt) / m.dt_map);
        }
        if (later > now) {
            dt = later * m.dt_map - t;
            store = 1;
        }
    }
    if ((t + dt) > t_max) dt = t_max - t;
    ctrl->store_map = store;
    ctrl->dt = dt;
    ctrl->go = 1;
}

// ------------------------------------------------------------------------------------------
// update_cell: balance + sources of one cell (the step's time advance t += dt is the caller's).
// ------------------------------------------------------------------------------------------
template <int kFriction, bool kHeadLoss, bool kStoreB, bool kDissip, class L>
__device__ __forceinline__ void update_cell(const DevMesh& m, int c, double dt)
{
    const double4 s0 = L::own(&m.st[c]);
    // a cell wet at the start of the step loads its friction coefficients with its slots (one
    // round trip less); dry cells, which mostly stay dry, leave them unread
    const bool fr_early = kFriction != SW2D_FRICTION_NONE && s0.x > smax(m.h_min, kSmallReal);
    double4 fr = make_double4(0.0, 0.0, 0.0, 0.0);
    if (fr_early) fr = ld(&m.fric[c]);
    double hh = s0.x, qq = s0.y, rr = s0.z;
    // hypComputeBalance (swSpHyp.cpp:214-273): h += (factor*F1)*dt, q += (...)*dt, r += (...)*dt
    // over the cell's slots, in the reference's order
    const int k0 = ld(&m.coff[c].y), k1 = ld(&m.coff[c + 1].y);
    if (k1 - k0 <= kUnroll) {
        Slot v[kUnroll];
#pragma unroll
        for (int i = 0; i < kUnroll; i++)
            if (i < k1 - k0) v[i] = L::own(&m.slot[k0 + i]);
#pragma unroll
        for (int i = 0; i < kUnroll; i++)
            if (i < k1 - k0) {
                hh += v[i].a * dt;
                qq += v[i].b * dt;
                rr += v[i].c * dt;
            }
    } else {
        for (int k = k0; k < k1; k++) {
            const Slot v = L::own(&m.slot[k]);
            hh += v.a * dt;
            qq += v.b * dt;
            rr += v.c * dt;
        }
    }
    if (kDissip) {  // DIP momentum dissipation, before the round-off flush (dip/swDipHyp.cpp:295-324)
        const double4 mu = ld(&m.mu[c]);
        momentum_dissipation(mu.x, mu.y, mu.z, mu.w, s0.x, s0.y, s0.z, hh, qq, rr);
    }
    const double hB = hh, qB = qq, rB = rr;  // the post-balance state, kept for the reverse sweep
    if (fabs(hh) < kSmallReal) hh = 0.;
    if (fabs(qq) < kSmallReal) qq = 0.;
    if (fabs(rr) < kSmallReal) rr = 0.;
    // negative depth (swSpHyp.cpp:182-210)
    if (m.neg_detect) {
        if (hh < 0) atomicOr(&m.ctrl->status, kStatusNegDepth);
    } else if (hh < 0.) {
        hh = 0.;
        qq = 0.;
        rr = 0.;
    }
    double P = 0.0;
    bool capped = false;
    cell_sources<kFriction, kHeadLoss>(m, c, dt, hh, qq, rr, kStoreB ? &P : nullptr, fr_early ? &fr : nullptr,
                                       kStoreB ? &capped : nullptr);
    // with the friction stage's h^(-4/3) >= 0, its sign bit set where the velocity cap acted
    if (kStoreB) m.bal[c] = make_double4(hB, qB, rB, capped ? -P : P);
    // z = h + z_b of the new state, as the next step's reconstruction computes it
    // (swSpHypMusclEvr.cpp:129, swSpHypGodunov.cpp:23)
    (m.st_out ? m.st_out : m.st)[c] = make_double4(hh, qq, rr, hh + ld(&m.zbv[c]));
}

}  // namespace sw2d
