// sw2d_ddp.cu — SW2D depth-dependent porosity (DDP) explicit step on the B200 (sm_100a), FP64.
//
// The step is the body of swDdp::execute's loop (src/sw2dSolver/models/ddp/swDdp.cpp:595-690):
// Godunov Riemann states, time step, HLLC and boundary fluxes, balance, momentum dissipation,
// divergence correction, negative-volume clamp, friction, singular head loss, velocity cap.
// The state of a cell is its stored volume thetaW and momentum thetaW*u, thetaW*v; the free
// surface z = zOfThetaW(thetaW) is kept beside it (st.w), with the cell's porosity, volume and
// pressure force at that level (dv), so that the edge kernel reads them instead of scanning the
// cell's table once per adjacent edge.
//
//   k_ddp_edges    per edge   Riemann states, wave speeds, the edge-table    swDdpHypGodunov.cpp:8-162,
//                             lookups, HLLC / boundary fluxes, CFL share      swDdpHyp.cpp:13-135,370-485,821-1007
//   k_cfl<true>    per cell   swept length, dt, the DDP map-storage snap      swDdpHyp.cpp:522-636
//   k_ddp_update   per cell   balance, dissipation, clamp, sources, then     swDdpHyp.cpp:142-349,
//                             z = zOfThetaW and the cell-table values        swDdpSourceFriction.cpp, swDdp.cpp:527-561
//
// With a divergence correction the update splits: k_ddp_balance keeps the pre-balance state,
// then either the time-step limitation (k_dc_ts_scan, k_dc_ts_min: swDdpHyp.cpp:723-768) or the
// flux limitation (k_lf_*: swDdpHyp.cpp:668-720, up to n_it_div_max + 1 passes, each pass
// predicated on the device), and k_ddp_finish does the rest.  Every kernel reads the loop
// control on the device, so a CUDA graph of many steps runs without the host.
//
// Tables live in HBM as levels {z, phi} (16 bytes each; the cumulated volume is rebuilt on the
// fly by the recurrence that built it), cells and internal edges in the internal numbering with
// CSR offsets; boundary-edge tables are read and checked but the step
// never uses them (swDdpHyp.cpp:38-48 and swDdpHypGodunov.cpp:39-42 force phiG = phiW there).
// Balance slots, their order and their persistence are the SP step's (sw2d_sp.cu): the DDP
// edge factors are w / area (swDdp.cpp:399-489), the SP ones with phi = 1.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "sw2d_internal.cuh"

using namespace sw2d;
using ddp::Lvl;
using ddp::PhiTheta;

namespace sw2d {

// Device loop control of the divergence correction.
struct DdpCtrl {
    int active;            // limit_flux: another pass runs
    int nbiter;            // limit_flux: passes done
    int ndry;              // limit_flux: cells with thetaW < 0 in this pass
    int n_sel;             // limit_flux: length of the ordered dry-cell list
    int any_dry;           // limit_timestep: some cell has thetaW <= 0
    int k_nan;             // limit_timestep: largest original index whose candidate is NaN
    unsigned blocks_done;  // limit_timestep: last-block reduction
    int pad;
    double ratio;          // limit_timestep: dt / dt_initial
};

struct DdpTables {
    // per record (original numbering): levels [off[k], off[k+1]) of z, phi, theta
    std::vector<int64_t> off;
    std::vector<double> z, phi, theta;
    int64_t levels(int64_t k) const { return off[k + 1] - off[k]; }
};

struct DdpState {
    DdpTables cell, eint, ebnd;
    int div_corr = kDivCorrNone;
    int n_it_div_max = 10;
    DdpCtrl* dctl = nullptr;
    // limit_flux: per original cell its ratio, internal- and boundary-edge counts; the dry list
    int* inv_cell = nullptr;  // original -> internal cell
    int* nint_o = nullptr;
    int* nbnd_o = nullptr;
    double* ratio = nullptr;
    int* blockcnt = nullptr;
    int* blockoff = nullptr;
    int* list = nullptr;
    int maxdeg = 0;           // largest per-cell count of internal or of boundary edges
    int* dc_int_e = nullptr;  // internal index of the original internal edges 0 .. maxdeg-1 (-1 if none)
    int* dc_bnd_e = nullptr;  // internal index of the original boundary edges 0 .. maxdeg-1
    // limit_timestep: per-block (value, original index) partial minima
    double2* part2 = nullptr;
    double* outbuf = nullptr;  // 3 * nc, derived output arrays
};

}  // namespace sw2d

namespace {

constexpr int kUnroll = 4;
constexpr int kFlagBlock = 256;

// ------------------------------------------------------------------------------------------
// Per-cell derived values: z = zOfThetaW(theta) and, at z, phiW, thetaW and the pressure force
// against the cell (swDdp.cpp:3368-3388, 1074-1097, 2708-2736, 1245-1273).
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ double derive_cell(const DevMesh& m, int c, double th, unsigned& bad)
{
    const int o = ld(&m.ctoff[c]), n = ld(&m.ctoff[c + 1]) - o;
    const Lvl* t = m.ctab + o;
    const double z = ddp::z_of_theta(t, n, th, bad);
    const double zq[1] = {z};
    PhiTheta pt[1];
    double p[1];
    ddp::table_pass<1, 1>(t, n, zq, pt, zq, p, bad);
    m.dv[c] = make_double4(pt[0].phi, pt[0].theta, p[0], 0.0);
    return z;
}

// dt-free balance terms of an internal edge for its L and R cells (swDdp.cpp:399-489 factors,
// swDdpHyp.cpp:274-297 products), as the SP step lays them out
__device__ __forceinline__ void put_int_slots(const DevMesh& m, int e, double nx, double ny, int2 sl, double f1,
                                              double f2, double f3, double sL, double sR, double2 cf)
{
    {
        const double c = cf.x;
        const double a1 = -c, f2F2 = -c * nx, f2F3 = +c * ny, f2S2 = +c * nx;
        const double f3F2 = -c * ny, f3F3 = -c * nx, f3S2 = +c * ny;
        m.slot[sl.x] = make_slot(a1 * f1, f2F2 * f2 + f2S2 * sL + f2F3 * f3, f3F2 * f2 + f3S2 * sL + f3F3 * f3);
    }
    {
        const double c = cf.y;
        const double a1 = +c, f2F2 = +c * nx, f2F3 = -c * ny, f2S2 = +c * nx;
        const double f3F2 = +c * ny, f3F3 = +c * nx, f3S2 = +c * ny;
        m.slot[sl.y] = make_slot(a1 * f1, f2F2 * f2 + f2S2 * sR + f2F3 * f3, f3F2 * f2 + f3S2 * sR + f3F3 * f3);
    }
}

// the same for a boundary edge (swDdpHyp.cpp:259-272)
__device__ __forceinline__ void put_bnd_slot(const DevMesh& m, double4 g, int sb, double f1, double f2, double f3,
                                             double s2)
{
    const double cf = g.w, nx = g.x, ny = g.y;
    const double fa = +cf, f2F2 = +cf * nx, f2F3 = -cf * ny, f2S2 = +cf * nx;
    const double f3F2 = +cf * ny, f3F3 = +cf * nx, f3S2 = +cf * ny;
    m.slot[sb] = make_slot(fa * f1, f2F2 * f2 + f2S2 * s2 + f2F3 * f3, f3F2 * f2 + f3S2 * s2 + f3F3 * f3);
}

// ------------------------------------------------------------------------------------------
// k_ddp_edges.  Internal edges: swDdp::hypGodunovComputeLRStates (swDdpHypGodunov.cpp:57-159)
// for both sides, lambda_max and the CFL shares of hypTimeStep (swDdpHyp.cpp:540-566: the L
// cell counts the edge when its own depth above z_tab[0] exceeds h_min, the R cell when either
// side does, since the reference carries `lambda` over), then, when either side is deeper than
// h_min above its cell's bottom z_b (swDdpHyp.cpp:426), hypHllc.  An edge left out keeps its
// previous slots, as the reference keeps its previous fluxes.  Boundary edges: the Riemann state
// of swDdpHypGodunov.cpp:16-54 (theta_riemann_bnd holds the depth there, and the flux velocity
// divides by it, swDdpHyp.cpp:372-377) and hypBoundaryFlux.
// ------------------------------------------------------------------------------------------
template <int kB, int kMinB>
__global__ void __launch_bounds__(kB, kMinB) k_ddp_edges(DevMesh m)
{
    if (!step_active(m.ctrl)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned bad = 0;
    if (i < m.ni) {
        const int e = i;
        const int2 lr = ld(&m.lr[e]);
        const int a = lr.x, b = lr.y;
        const double2 n = ld(&m.nxy[e]);
        // the edge's slots, factors and length and the two cells' table offsets, in flight with
        // the cell gathers (else loaded after the Riemann states, which they then wait for)
        const int2 sl = ld_now(&m.eslot[e]);
        const double2 cf = ld_now(&m.coef[e]);
        const double len_e = ld(&m.len[e]);
        const int ao = ld_now(&m.ctoff[a]), an = ld_now(&m.ctoff[a + 1]) - ao;
        const int bo = ld_now(&m.ctoff[b]), bn = ld_now(&m.ctoff[b + 1]) - bo;
        const double4 sa = ld(&m.st[a]), sb = ld(&m.st[b]);   // {theta, theta u, theta v, z}
        const double2 va = ld(reinterpret_cast<const double2*>(&m.dv[a]));  // {phiW, thetaW} at z
        const double2 vb = ld(reinterpret_cast<const double2*>(&m.dv[b]));
        const double2 ca = ld(reinterpret_cast<const double2*>(&m.cst[a]));  // {z_b, boussinesq}
        const double2 cb = ld(reinterpret_cast<const double2*>(&m.cst[b]));
        const double ta0 = ld(&m.cst[a].z), tb0 = ld(&m.cst[b].z);  // lowest table levels
        const int eo = ld(&m.etoff[e]), en = ld(&m.etoff[e + 1]) - eo;
        const Lvl* et = m.etab + eo;
        // the edge's table at both sides' levels: phiG, thetaG and the pressure force on the edge
        const double zs[2] = {sa.w, sb.w};
        PhiTheta gs[2];
        double fg[2];
        ddp::table_pass<2, 2>(et, en, zs, gs, zs, fg, bad);
        const PhiTheta oL{va.x, va.y}, oR{vb.x, vb.y};
        const ddp::Side SL = ddp::lr_side(
            sa.x, sa.y, sa.z, sa.w, ta0, ca.y, n.x, n.y, oL, gs[0],
            [&](PhiTheta& om, PhiTheta& gm) {
                const double4 ma = ld(&m.dcs[a]), e0 = ld(&m.des[2 * e]);
                om = PhiTheta{ma.x, ma.y};
                gm = PhiTheta{e0.z, e0.w};
            },
            m.h_min);
        const ddp::Side SR = ddp::lr_side(
            sb.x, sb.y, sb.z, sb.w, tb0, cb.y, n.x, n.y, oR, gs[1],
            [&](PhiTheta& om, PhiTheta& gm) {
                const double4 mb = ld(&m.dcs[b]), e1 = ld(&m.des[2 * e + 1]);
                om = PhiTheta{mb.z, mb.w};
                gm = PhiTheta{e1.x, e1.y};
            },
            m.h_min);
        const double lm = max4(fabs(SL.lm), fabs(SL.lp), fabs(SR.lm), fabs(SR.lp));
        if (m.lmax) m.lmax[e] = lm;
        const double lw = lm * len_e;
        const bool wetL = sa.w - ta0 > m.h_min, wetR = sb.w - tb0 > m.h_min;
        m.slot_w[sl.x] = wetL ? lw : 0.0;
        m.slot_w[sl.y] = (wetL || wetR) ? lw : 0.0;
        const double hL = sa.w - ca.x, hR = sb.w - cb.x;
        if ((hL > m.h_min) || (hR > m.h_min)) {
            ddp::HllcIn in;
            in.bL = ca.y;
            in.bR = cb.y;
            in.zL = sa.w;
            in.zR = sb.w;
            in.uL = 0.0;
            in.vL = 0.0;
            if (sa.x > kSmallReal) {
                in.uL = SL.tu / sa.x;
                in.vL = SL.tv / sa.x;
            }
            in.uR = 0.0;
            in.vR = 0.0;
            if (sb.x > kSmallReal) {
                in.uR = SR.tu / sb.x;
                in.vR = SR.tv / sb.x;
            }
            in.omega_L = oL;
            in.omega_R = oR;
            in.gamma_L = gs[0];
            in.gamma_R = gs[1];
            in.theta_RL = ddp::phi_theta(m.ctab + bo, bn, sa.w, bad).theta;
            in.theta_LR = ddp::phi_theta(m.ctab + ao, an, sb.w, bad).theta;
            in.force_omega_L = ld(&m.dv[a].z);
            in.force_omega_R = ld(&m.dv[b].z);
            in.force_gamma_L = fg[0];
            in.force_gamma_R = fg[1];
            const double2 e0 = ld(reinterpret_cast<const double2*>(&m.des[2 * e]));
            in.theta_gamma_hmin = e0.x;
            in.z_gamma_min = e0.y;
            const ddp::Flux f = ddp::hllc(in, m.h_min, m.chi_phi_max);
            bad |= f.bad;
            if (isnan(f.f1)) bad |= kStatusNanFlux;
            if (m.flux) {
                double2* fp = m.flux + 3 * (size_t)e;
                fp[0] = make_double2(f.f1, f.f2);
                fp[1] = make_double2(f.f3, f.sl);
                fp[2] = make_double2(f.sr, 0.0);
            }
            put_int_slots(m, e, n.x, n.y, sl, f.f1, f.f2, f.f3, f.sl, f.sr, cf);
        }
    } else if (i < m.ni + m.nb) {
        const int e = i - m.ni;
        const int c = ld(&m.bcell[e]);
        const double4 s = ld(&m.st[c]);
        const double4 v = ld(&m.dv[c]);
        const double4 cs = ld(&m.cst[c]);
        const double4 g = ld(&m.bgeo[e]);  // {nx, ny, length, w / area}
        const double theta_in = s.x, z_in = s.w;
        const double h_in = smax(z_in - cs.z, 0.);
        double tu = s.y * g.x + s.z * g.y;
        double tv = -s.y * g.y + s.z * g.x;
        if (h_in < m.h_min) {
            tu = 0.;
            tv = 0.;
        }
        const double c_in = ddp::celerity(theta_in, v.x);
        const double u_in = tu / smax(theta_in, kSmallReal);
        const double lp = ddp::lam_plus(u_in, c_in, 1.0, 1.0, cs.y);
        const double lmn = ddp::lam_minus(u_in, c_in, 1.0, 1.0, cs.y);
        const double lmb = smax(fabs(lp), fabs(lmn));
        if (m.lmaxb) m.lmaxb[e] = lmb;
        const int sb = ld(&m.bslot[e]);
        m.slot_w[sb] = (z_in - cs.z > m.h_min) ? lmb * g.z : 0.0;
        double uR = 0.0, vR = 0.0;
        if (h_in > kSmallReal) {
            uR = tu / h_in;
            vR = tv / h_in;
        }
        const int k = ld(&m.bbc[e]);
        const long long o0 = ld(&m.bcoff[k]), o1 = ld(&m.bcoff[k + 1]);
        const double val = bc_value(m.bctimes + o0, m.bcvals + o0, o1 - o0, m.ctrl->t);
        const int type = ld(&m.bctype[k]);
        double theta_bc = 0.0;
        if (type == SW2D_BC_H || type == SW2D_BC_Z) {
            const int co = ld(&m.ctoff[c]), cn = ld(&m.ctoff[c + 1]) - co;
            theta_bc = ddp::phi_theta(m.ctab + co, cn, ddp::boundary_level(type, val, cs.z), bad).theta;
        }
        double f1, f2, f3;
        bad |= ddp::boundary_flux(cs.y, uR, vR, PhiTheta{v.x, v.y}, v.z, type, val, theta_bc, &f1, &f2, &f3);
        if (m.bflux) m.bflux[e] = make_double4(f1, f2, f3, 0.0);
        put_bnd_slot(m, g, sb, f1, f2, f3, 0.0);  // source_right: never set by hypBoundaryFlux
    }
    if (bad) atomicOr(&m.ctrl->status, bad);
}

// hypComputeBalance (swDdpHyp.cpp:256-297) over the cell's slots in the reference's order
__device__ __forceinline__ void slot_balance(const DevMesh& m, int c, double dt, double& hh, double& qq, double& rr)
{
    const int k0 = ld(&m.coff[c].y), k1 = ld(&m.coff[c + 1].y);
    if (k1 - k0 <= kUnroll) {
        Slot v[kUnroll];
#pragma unroll
        for (int i = 0; i < kUnroll; i++)
            if (i < k1 - k0) v[i] = m.slot[k0 + i];
#pragma unroll
        for (int i = 0; i < kUnroll; i++)
            if (i < k1 - k0) {
                hh += v[i].a * dt;
                qq += v[i].b * dt;
                rr += v[i].c * dt;
            }
    } else {
        for (int k = k0; k < k1; k++) {
            const Slot v = m.slot[k];
            hh += v.a * dt;
            qq += v.b * dt;
            rr += v.c * dt;
        }
    }
}

// after the balance (and any divergence correction): the negative-volume clamp or detection
// (swDdpHyp.cpp:203-229), friction, singular head loss, velocity cap, then z and the cell-table
// values of the new state
template <int kF, bool kHL>
__device__ __forceinline__ void finish_cell(const DevMesh& m, int c, double dt, double th, double qq, double rr,
                                            unsigned& bad)
{
    if (m.neg_detect) {
        if (th < 0) bad |= kStatusNegDepth;
    } else if (th < 0.) {
        th = 0.;
        qq = 0.;
        rr = 0.;
    }
    cell_sources<kF, kHL>(m, c, dt, th, qq, rr);
    const double z = derive_cell(m, c, th, bad);
    m.st[c] = make_double4(th, qq, rr, z);
}

// k_ddp_update: the whole cell update when no divergence correction is selected
template <int kF, bool kHL, bool kDissip>
__global__ void __launch_bounds__(kBlock, 3) k_ddp_update(DevMesh m)
{
    Ctrl* ctrl = m.ctrl;
    if (!ctrl->go) return;
    const double dt = ctrl->dt;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0) {
        ctrl->t = ctrl->t + dt;  // swDdp.cpp:669
        ctrl->steps += 1;
    }
    if (c >= m.nc) return;
    const double4 s0 = m.st[c];
    double th = s0.x, qq = s0.y, rr = s0.z;
    slot_balance(m, c, dt, th, qq, rr);
    if (kDissip) {  // swDdpHyp.cpp:300-325
        const double4 mu = ld(&m.mu[c]);
        momentum_dissipation(mu.x, mu.y, mu.z, mu.w, s0.x, s0.y, s0.z, th, qq, rr);
    }
    unsigned bad = 0;
    finish_cell<kF, kHL>(m, c, dt, th, qq, rr, bad);
    if (bad) atomicOr(&ctrl->status, bad);
}

// k_ddp_balance: the balance and dissipation with a divergence correction to follow; keeps the
// pre-balance state (swDdpHyp.cpp:176-182) and resets the correction's loop control
__global__ void __launch_bounds__(kBlock) k_ddp_balance(DevMesh m, bool dissip)
{
    Ctrl* ctrl = m.ctrl;
    if (!ctrl->go) return;
    const double dt = ctrl->dt;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0) {
        DdpCtrl* d = m.dctl;
        d->active = 1;
        d->nbiter = 0;
        d->ndry = 0;
        d->n_sel = 0;
        d->any_dry = 0;
        d->k_nan = -1;
        d->blocks_done = 0;
        d->ratio = 1.0;
    }
    if (c >= m.nc) return;
    const double4 s0 = m.st[c];
    double th = s0.x, qq = s0.y, rr = s0.z;
    slot_balance(m, c, dt, th, qq, rr);
    if (dissip) {
        const double4 mu = ld(&m.mu[c]);
        momentum_dissipation(mu.x, mu.y, mu.z, mu.w, s0.x, s0.y, s0.z, th, qq, rr);
    }
    m.old[c] = s0;
    m.st[c] = make_double4(th, qq, rr, s0.w);
}

// ------------------------------------------------------------------------------------------
// limit_timestep: swDdp::hypDivCorrTimeStep (swDdpHyp.cpp:723-768).  Over the cells in their
// original order, every cell with thetaW <= 0 offers dt * (old - new) / new and the reference
// folds them with std::min(candidate, running): a NaN candidate (old = new = 0) replaces the
// running value, which the next candidate then replaces.  The fold therefore equals the
// minimum over the candidates after the last NaN one (NaN if none follows it), or over all of
// them and the CFL dt when none is NaN; ties go to the later cell.  Two reductions compute
// exactly that: the largest original index of a NaN candidate, then the minimum over the later
// ones.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_dc_ts_scan(DevMesh m, const int* __restrict__ perm)
{
    if (!m.ctrl->go) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const double th = m.st[c].x;
    if (th <= 0.0) {
        const double dt = m.ctrl->dt;
        m.dctl->any_dry = 1;
        const double cand = dt * (m.old[c].x - th) / th;
        if (cand != cand) atomicMax(&m.dctl->k_nan, ld(&perm[c]));
    }
}

__device__ __forceinline__ double2 better(double2 a, double2 b)
{
    // (value, original index): the smaller value; on a tie the later cell (index -1: none)
    if (b.y < 0) return a;
    if (a.y < 0) return b;
    if (b.x < a.x) return b;
    if (a.x < b.x) return a;
    return (b.y > a.y) ? b : a;
}

__global__ void __launch_bounds__(kBlock) k_dc_ts_min(DevMesh m, const int* __restrict__ perm, double2* part)
{
    Ctrl* ctrl = m.ctrl;
    if (!ctrl->go) return;
    DdpCtrl* d = m.dctl;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const double dt = ctrl->dt;
    const int k_nan = *((volatile int*)&d->k_nan);
    double2 best = make_double2(0.0, -1.0);
    if (c < m.nc) {
        const double th = m.st[c].x;
        const int o = ld(&perm[c]);
        if (th <= 0.0 && o > k_nan) {
            const double cand = dt * (m.old[c].x - th) / th;
            if (cand == cand) best = make_double2(cand, (double)o);
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        double2 o;
        o.x = __shfl_down_sync(0xffffffffu, best.x, off);
        o.y = __shfl_down_sync(0xffffffffu, best.y, off);
        best = better(best, o);
    }
    __shared__ double2 wbest[kBlock / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) wbest[wid] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 bb = wbest[0];
        for (int w = 1; w < kBlock / 32; w++) bb = better(bb, wbest[w]);
        part[blockIdx.x] = bb;
        __threadfence();
        const unsigned done = atomicAdd(&d->blocks_done, 1u);
        last = (done == gridDim.x - 1);
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double2 bb = make_double2(0.0, -1.0);
    for (unsigned b = 0; b < gridDim.x; b++) {
        const volatile double2* p = part + b;
        bb = better(bb, make_double2(p->x, p->y));
    }
    if (!*((volatile int*)&d->any_dry)) return;  // nothing changes
    double dt_avoid;
    if (k_nan >= 0)
        dt_avoid = (bb.y < 0) ? ddp::quiet_nan() : bb.x;
    else
        dt_avoid = (bb.y < 0) ? dt : smin(dt, bb.x);
    const double dt_new = smin(dt, dt_avoid);
    d->ratio = dt_new / dt;
    ctrl->dt = dt_new;
}

// ------------------------------------------------------------------------------------------
// limit_flux: swDdp::hypDivCorrFluxes (swDdpHyp.cpp:668-720), pass by pass.  For each cell with
// thetaW < 0, in original order, the reference multiplies by old / (old - new) the fluxes of the
// boundary edges 0 .. n_b - 1 and of the internal edges 0 .. n_i - 1 (n_b, n_i: the cell's
// boundary- and internal-edge counts; the loop indexes the global arrays with its local
// counter), then re-assigns every cell touched by an internal edge from its pre-balance state
// and that edge's fluxes alone, edge after edge, so that the last internal edge of a cell (by
// original index) decides its value and boundary fluxes drop out.  Passes repeat while cells
// stay dry, at most n_it_div_max + 1 times.  Here: the dry cells are listed in original order
// (flag, block scan, scatter), one thread per affected edge applies the ratios in that order,
// and the cell's last internal slot re-assigns it.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kFlagBlock) k_lf_flag(DevMesh m, const int* __restrict__ inv, int* blockcnt,
                                                        double* ratio)
{
    if (!m.ctrl->go || !m.dctl->active) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // original cell index
    bool dry = false;
    if (i < m.nc) {
        const int c = ld(&inv[i]);
        const double th = m.st[c].x;
        if (th < 0.0) {
            dry = true;
            const double o = m.old[c].x;
            ratio[i] = o / (o - th);
        }
    }
    const int cnt = __syncthreads_count(dry);
    if (threadIdx.x == 0) {
        blockcnt[blockIdx.x] = cnt;
        if (cnt) atomicAdd(&m.dctl->ndry, cnt);
    }
}

__global__ void __launch_bounds__(1024) k_lf_scan(DevMesh m, const int* __restrict__ blockcnt, int* blockoff, int nblk)
{
    if (!m.ctrl->go || !m.dctl->active) return;
    __shared__ int wsum[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int base = 0; base < nblk; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = (i < nblk) ? blockcnt[i] : 0;
        int x = v;
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x += y;
        }
        if (lane == 31) wsum[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int w = wsum[lane];
            for (int off = 1; off < 32; off <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, w, off);
                if (lane >= off) w += y;
            }
            wsum[lane] = w;  // inclusive over warps
        }
        __syncthreads();
        const int before = carry + (wid > 0 ? wsum[wid - 1] : 0) + x - v;
        if (i < nblk) blockoff[i] = before;
        __syncthreads();
        if (threadIdx.x == 0) carry += wsum[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) m.dctl->n_sel = carry;
}

__global__ void __launch_bounds__(kFlagBlock) k_lf_scatter(DevMesh m, const int* __restrict__ inv,
                                                           const int* __restrict__ blockoff, int* list)
{
    if (!m.ctrl->go || !m.dctl->active) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool dry = false;
    if (i < m.nc) dry = m.st[ld(&inv[i])].x < 0.0;
    __shared__ int wcnt[kFlagBlock / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned ballot = __ballot_sync(0xffffffffu, dry);
    if (lane == 0) wcnt[wid] = __popc(ballot);
    __syncthreads();
    if (dry) {
        int pos = blockoff[blockIdx.x];
        for (int w = 0; w < wid; w++) pos += wcnt[w];
        pos += __popc(ballot & ((1u << lane) - 1u));
        list[pos] = i;
    }
}

// one thread per affected internal edge (tid < 32) and boundary edge (tid >= 32)
__global__ void k_lf_chain(DevMesh m, const int* __restrict__ list, const double* __restrict__ ratio,
                           const int* __restrict__ nint_o, const int* __restrict__ nbnd_o,
                           const int* __restrict__ int_e, const int* __restrict__ bnd_e, int maxdeg)
{
    if (!m.ctrl->go || !m.dctl->active) return;
    const int n = m.dctl->n_sel;
    const int tid = threadIdx.x;
    const bool is_int = tid < 32;
    const int j = is_int ? tid : tid - 32;
    if (j >= maxdeg) return;
    const int e = is_int ? int_e[j] : bnd_e[j];
    if (e < 0) return;
    double f[5];
    if (is_int) {
        const double2* fp = m.flux + 3 * (size_t)e;
        f[0] = fp[0].x; f[1] = fp[0].y; f[2] = fp[1].x; f[3] = fp[1].y; f[4] = fp[2].x;
    } else {
        const double4 b = m.bflux[e];
        f[0] = b.x; f[1] = b.y; f[2] = b.z; f[3] = b.w; f[4] = 0.0;
    }
    bool scaled = false;
    for (int k = 0; k < n; k++) {
        const int id = list[k];
        const int cnt = is_int ? nint_o[id] : nbnd_o[id];
        if (cnt > j) {
            const double r = ratio[id];
#pragma unroll
            for (int q = 0; q < 5; q++) f[q] *= r;
            scaled = true;
        }
    }
    if (!scaled) return;
    if (is_int) {
        double2* fp = m.flux + 3 * (size_t)e;
        fp[0] = make_double2(f[0], f[1]);
        fp[1] = make_double2(f[2], f[3]);
        fp[2] = make_double2(f[4], 0.0);
        const double2 nn = m.nxy[e];
        put_int_slots(m, e, nn.x, nn.y, m.eslot[e], f[0], f[1], f[2], f[3], f[4], ld(&m.coef[e]));
    } else {
        m.bflux[e] = make_double4(f[0], f[1], f[2], f[3]);
        put_bnd_slot(m, m.bgeo[e], m.bslot[e], f[0], f[1], f[2], f[3]);
    }
}

// re-assignment of hypDivCorrFluxes (swDdpHyp.cpp:693-716): the cell's last internal slot
__global__ void __launch_bounds__(kBlock) k_lf_recompute(DevMesh m)
{
    if (!m.ctrl->go || !m.dctl->active) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const int2 a = ld(&m.coff[c]), b = ld(&m.coff[c + 1]);
    if (b.x - a.x <= 0) return;  // no internal edge
    const double dt = m.ctrl->dt;
    const Slot v = m.slot[b.y - 1];
    const double4 o = m.old[c];
    const double4 s = m.st[c];
    m.st[c] = make_double4(o.x + v.a * dt, o.y + v.b * dt, o.z + v.c * dt, s.w);
}

__global__ void k_lf_next(DevMesh m)
{
    DdpCtrl* d = m.dctl;
    if (!m.ctrl->go || !d->active) return;
    d->nbiter += 1;
    if ((d->ndry == 0) || (d->nbiter > m.n_it_div_max)) d->active = 0;
    d->ndry = 0;
}

// k_ddp_finish: after a divergence correction (time-step limitation: re-weights the state when
// some cell dries, swDdpHyp.cpp:756-766), the rest of the step with the final dt
template <int kF, bool kHL, bool kTs>
__global__ void __launch_bounds__(kBlock, 3) k_ddp_finish(DevMesh m)
{
    Ctrl* ctrl = m.ctrl;
    if (!ctrl->go) return;
    const double dt = ctrl->dt;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0) {
        ctrl->t = ctrl->t + dt;
        ctrl->steps += 1;
    }
    if (c >= m.nc) return;
    const double4 s = m.st[c];
    double th = s.x, qq = s.y, rr = s.z;
    if (kTs && m.dctl->any_dry) {
        const double r = m.dctl->ratio;
        const double4 o = m.old[c];
        th = o.x * (1.0 - r) + th * r;
        qq = o.y * (1.0 - r) + qq * r;
        rr = o.z * (1.0 - r) + rr * r;
    }
    unsigned bad = 0;
    finish_cell<kF, kHL>(m, c, dt, th, qq, rr, bad);
    if (bad) atomicOr(&ctrl->status, bad);
}

// ------------------------------------------------------------------------------------------
// set-up kernels
// ------------------------------------------------------------------------------------------
// per-cell statics at the shallow levels z_tab[0] + h_min and z_tab[1] + h_min, the lowest level
// into cst.z, per-edge statics (thetaG at z_tab[0] + h_min_ddp: swDdp.cpp:2232-2234)
__global__ void k_ddp_statics(DevMesh m, double h_min_ddp, double4* dcs, double4* des, double4* cst)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned bad = 0;
    if (i < m.nc) {
        const int o = m.ctoff[i], n = m.ctoff[i + 1] - o;
        const Lvl* t = m.ctab + o;
        const PhiTheta p0 = ddp::phi_theta(t, n, t[0].z + m.h_min, bad);
        const PhiTheta p1 = ddp::phi_theta(t, n, t[1].z + m.h_min, bad);
        dcs[i] = make_double4(p0.phi, p0.theta, p1.phi, p1.theta);
        double4 c = cst[i];
        c.z = t[0].z;
        cst[i] = c;
    } else if (i < m.nc + m.ni) {
        const int e = i - m.nc;
        const int o = m.etoff[e], n = m.etoff[e + 1] - o;
        const Lvl* t = m.etab + o;
        const int2 lr = m.lr[e];
        const Lvl* ta = m.ctab + m.ctoff[lr.x];
        const Lvl* tb = m.ctab + m.ctoff[lr.y];
        const double th_hmin = ddp::phi_theta(t, n, t[0].z + h_min_ddp, bad).theta;
        const PhiTheta gl = ddp::phi_theta(t, n, ta[0].z + m.h_min, bad);
        const PhiTheta gr = ddp::phi_theta(t, n, tb[1].z + m.h_min, bad);
        des[2 * e] = make_double4(th_hmin, t[0].z, gl.phi, gl.theta);
        des[2 * e + 1] = make_double4(gr.phi, gr.theta, 0.0, 0.0);
    }
    if (bad) atomicOr(&m.ctrl->status, bad);
}

// swDdp::setInitialConditions (swDdp.cpp:1608-1726): thetaW from h (above z_tab[0]) or z, the
// momentum from q (theta q / max(1e-16, z(theta) - z_tab[0])) or u (theta u); then z and the
// cell-table values.  Inputs in the caller's numbering.
__global__ void k_ddp_ic(DevMesh m, const double* __restrict__ lv, const double* __restrict__ xv,
                         const double* __restrict__ yv, int cols, const int* __restrict__ perm)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    unsigned bad = 0;
    const int p = perm[c];
    const int o = m.ctoff[c], n = m.ctoff[c + 1] - o;
    const Lvl* t = m.ctab + o;
    const double zs = (cols & SW2D_DDP_IC_LEVEL_Z) ? lv[p] : lv[p] + t[0].z;
    const double th = ddp::phi_theta(t, n, zs, bad).theta;
    double tu, tv;
    if (cols & SW2D_DDP_IC_X_VELOCITY) {
        tu = th * xv[p];
    } else {
        const double h = smax(kSmallReal, ddp::z_of_theta(t, n, th, bad) - t[0].z);
        tu = th * xv[p] / h;
    }
    if (cols & SW2D_DDP_IC_Y_VELOCITY) {
        tv = th * yv[p];
    } else {
        const double h = smax(kSmallReal, ddp::z_of_theta(t, n, th, bad) - t[0].z);
        tv = th * yv[p] / h;
    }
    const double z = derive_cell(m, c, th, bad);
    m.st[c] = make_double4(th, tu, tv, z);
    if (bad) atomicOr(&m.ctrl->status, bad);
}

__global__ void k_ddp_derive(DevMesh m)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    unsigned bad = 0;
    double4 s = m.st[c];
    s.w = derive_cell(m, c, s.x, bad);
    m.st[c] = s;
    if (bad) atomicOr(&m.ctrl->status, bad);
}

// storeResultMaps outputs (swDdp.cpp:2489-2513): h = max(0, z - z_tab[0]), q = u h, r = v h
// with u = theta u / theta when theta > 1e-16 (else 0); and z itself
__global__ void k_ddp_outputs(DevMesh m, double* out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const double4 s = m.st[c];
    const double4 cs = m.cst[c];
    const double h = smax(0.0, s.w - cs.z);
    double u = 0.0, v = 0.0;
    if (s.x > kSmallReal) {
        u = s.y / s.x;
        v = s.z / s.x;
    }
    out[c] = h;
    out[m.nc + c] = u * h;
    out[2 * m.nc + c] = v * h;
    out[3 * m.nc + c] = s.w;
}

// one storeResultMaps output of k_ddp_outputs (0 h, 1 q, 2 r, 3 z) per cell, written straight to
// the caller's numbering: out[perm[c]]
__global__ void k_ddp_output_field(DevMesh m, int which, const int* __restrict__ perm, double* out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const double4 s = m.st[c];
    const double4 cs = m.cst[c];
    const double h = smax(0.0, s.w - cs.z);
    double u = 0.0, v = 0.0;
    if (s.x > kSmallReal) {
        u = s.y / s.x;
        v = s.z / s.x;
    }
    out[perm[c]] = which == 0 ? h : which == 1 ? u * h : which == 2 ? v * h : s.w;
}

// out[perm[i]] = src[i * stride + offset]
__global__ void k_scatter_field(const double* __restrict__ src, int stride, int offset, const int* __restrict__ perm,
                                double* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[perm[i]] = src[(size_t)i * stride + offset];
}

// ------------------------------------------------------------------------------------------
// launches
// ------------------------------------------------------------------------------------------
struct Variant {
    int block, minb;
};
constexpr Variant kDdpVariants[] = {{256, 2}, {128, 4}, {256, 3}, {192, 3}, {128, 5}, {512, 1}};

template <int V>
void launch_edges_v(sw2d_handle* h, const DevMesh& m)
{
    constexpr int B = kDdpVariants[V].block, M = kDdpVariants[V].minb;
    const unsigned n = (unsigned)(m.ni + m.nb);
    k_ddp_edges<B, M><<<(n + B - 1) / B, B, 0, h->stream>>>(m);
}

template <int kF, bool kHL>
void launch_tail_f(sw2d_handle* h, const DevMesh& m)
{
    const unsigned g = grid_for(m.nc);
    DdpState* d = h->ddp;
    if (d->div_corr == kDivCorrNone) {
        if (h->dissipation) k_ddp_update<kF, kHL, true><<<g, kBlock, 0, h->stream>>>(m);
        else k_ddp_update<kF, kHL, false><<<g, kBlock, 0, h->stream>>>(m);
        return;
    }
    k_ddp_balance<<<g, kBlock, 0, h->stream>>>(m, h->dissipation != 0);
    if (d->div_corr == kDivCorrTimestep) {
        k_dc_ts_scan<<<g, kBlock, 0, h->stream>>>(m, h->d_cell_perm);
        k_dc_ts_min<<<g, kBlock, 0, h->stream>>>(m, h->d_cell_perm, d->part2);
        k_ddp_finish<kF, kHL, true><<<g, kBlock, 0, h->stream>>>(m);
    } else {
        const unsigned gf = (unsigned)((m.nc + kFlagBlock - 1) / kFlagBlock);
        for (int it = 0; it <= d->n_it_div_max; it++) {
            k_lf_flag<<<gf, kFlagBlock, 0, h->stream>>>(m, d->inv_cell, d->blockcnt, d->ratio);
            k_lf_scan<<<1, 1024, 0, h->stream>>>(m, d->blockcnt, d->blockoff, (int)gf);
            k_lf_scatter<<<gf, kFlagBlock, 0, h->stream>>>(m, d->inv_cell, d->blockoff, d->list);
            k_lf_chain<<<1, 64, 0, h->stream>>>(m, d->list, d->ratio, d->nint_o, d->nbnd_o, d->dc_int_e, d->dc_bnd_e,
                                                d->maxdeg);
            k_lf_recompute<<<g, kBlock, 0, h->stream>>>(m);
            k_lf_next<<<1, 1, 0, h->stream>>>(m);
        }
        k_ddp_finish<kF, kHL, false><<<g, kBlock, 0, h->stream>>>(m);
    }
}

template <int kF>
void launch_tail_h(sw2d_handle* h, const DevMesh& m)
{
    if (h->p.singular_head_loss) launch_tail_f<kF, true>(h, m);
    else launch_tail_f<kF, false>(h, m);
}

void launch_tail(sw2d_handle* h, const DevMesh& m)
{
    switch (h->p.friction) {
        case SW2D_FRICTION_CHEZY: launch_tail_h<SW2D_FRICTION_CHEZY>(h, m); break;
        case SW2D_FRICTION_MANNING: launch_tail_h<SW2D_FRICTION_MANNING>(h, m); break;
        case SW2D_FRICTION_STRICKLER: launch_tail_h<SW2D_FRICTION_STRICKLER>(h, m); break;
        default: launch_tail_h<SW2D_FRICTION_NONE>(h, m); break;
    }
}

// ------------------------------------------------------------------------------------------
// host: the porosity laws of swDdp::setPorosityCellMap / EdgeBndMap / EdgeIntMap
// (swDdp.cpp:1787-2238) and swDdp::tabulatePorosity (swDdp.cpp:2596-2645), on the records as
// swDdp::readPorosityFile reads them (law type, count, parameters; lengths checked as
// swDdp::porosityLineSize does, swDdp.cpp:1099-1211).
// ------------------------------------------------------------------------------------------
bool tabulate(size_t ntab, const std::vector<double>& z, const std::vector<double>& phi, std::vector<double>& z_tab,
              std::vector<double>& phi_tab, std::string& why)
{
    const size_t nv = z.size();
    if (ntab < 2 || nv < 2) {
        why = "a re-tabulated porosity law needs n_por_tab_max >= 2 and two points";
        return false;
    }
    phi_tab.assign(ntab, 0.0);
    z_tab.assign(ntab, 0.0);
    const double dz = (z[nv - 1] - z[0]) / (double)(ntab - 1);
    for (size_t level = 0; level < ntab; ++level) z_tab[level] = z[0] + (double)level * dz;
    std::vector<double> phi_interp(ntab, 0.0);
    phi_interp[0] = 0;
    size_t index = 0;
    for (size_t level = 1; level < ntab; ++level) {
        while (z_tab[level] > z[index]) {
            ++index;
            if (index >= nv) {
                // the reference reads past the end of its point list here
                why = "porosity law: a tabulated level lies above the last point (n_por_tab_max rounding)";
                return false;
            }
        }
        if (index == 0) {
            why = "porosity law: points not increasing";
            return false;
        }
        phi_interp[level] =
            phi[index - 1] + (phi[index] - phi[index - 1]) * (z_tab[level] - z[index - 1]) / (z[index] - z[index - 1]);
    }
    for (size_t level = 0; level < ntab - 1; ++level) phi_tab[level] = (phi_interp[level + 1] + phi_interp[level]) * 0.5;
    phi_tab[ntab - 1] = phi[nv - 1];
    return true;
}

// one record -> its table; `base` is the cell's bottom or the edge's midpoint elevation
bool law_table(const double* rec, int64_t len, double base, size_t ntab, std::vector<double>& z_tab,
               std::vector<double>& phi_tab, std::string& why)
{
    if (len < 2) {
        why = "porosity record shorter than its law type and count";
        return false;
    }
    const double law = rec[0];
    z_tab.clear();
    phi_tab.clear();
    if (law == -2 || law == -1) {
        const int64_t nc = (int64_t)(int)rec[1];
        if (nc < 1 || len != 2 * nc + 2) {
            why = "porosity record (law -2/-1): length is not 2 n + 2";
            return false;
        }
        std::vector<double> zr, pr;
        for (int64_t l = 0; l < nc; l++) {
            zr.push_back(base + rec[2 + 2 * l]);
            pr.push_back(rec[3 + 2 * l]);
        }
        if (law == -2) {
            z_tab = zr;
            phi_tab = pr;
            return true;
        }
        return tabulate(ntab, zr, pr, z_tab, phi_tab, why);
    }
    if (law == 0) {
        const int64_t nl = (int64_t)(int)rec[1];
        if (nl < 2 || len != nl + 2) {
            why = "porosity record (law 0): length is not n + 2";
            return false;
        }
        std::vector<double> zr, pr;
        for (int64_t l = 0; l < nl; l++) {
            zr.push_back(base + rec[2 + l]);
            pr.push_back((double)l * 1.0 / (double)(nl - 1));
        }
        return tabulate(ntab, zr, pr, z_tab, phi_tab, why);
    }
    if (law == 1) {
        if (len != 4) {
            why = "porosity record (law 1): length is not 4";
            return false;
        }
        const double z = base + rec[2];
        const double phi = rec[3];
        std::vector<double> zr = {z, z + 1.0}, pr = {phi, phi};
        if (!tabulate(ntab, zr, pr, z_tab, phi_tab, why)) return false;
        phi_tab[0] = phi;
        return true;
    }
    if (law == 2 || law == 3) {
        if (len != (law == 2 ? 6 : 7)) {
            why = "porosity record (law 2/3): length is not 6/7";
            return false;
        }
        if (ntab < 2) {
            why = "n_por_tab_max < 2";
            return false;
        }
        const double z0 = base + rec[2];
        const double z1 = base + rec[4];
        const double phi0 = rec[3];
        const double phi1 = rec[5];
        const double dz = (z1 - z0) / (double)(ntab - 1);
        const double dphi = (phi1 - phi0) / (double)(ntab - 1);
        z_tab.assign(ntab, 0.0);
        phi_tab.assign(ntab, 0.0);
        for (size_t l = 0; l < ntab - 1; ++l) {
            z_tab[l] = z0 + (double)l * dz;
            phi_tab[l] = phi0 + ((double)l + 0.5) * dphi;
        }
        z_tab[ntab - 1] = z1;
        phi_tab[ntab - 1] = (law == 2) ? phi1 : rec[6];
        return true;
    }
    why = "porosity law type not in {-2, -1, 0, 1, 2, 3}";
    return false;
}

bool build_tables(int64_t n, const sw2d_ddp_records& rec, const double* base, size_t ntab, DdpTables& out,
                  std::string& why)
{
    out.off.assign(n + 1, 0);
    out.z.clear();
    out.phi.clear();
    out.theta.clear();
    if (n > 0 && (!rec.offset || !rec.values || !base)) {
        why = "porosity records or base elevations missing";
        return false;
    }
    std::vector<double> zt, pt;
    for (int64_t k = 0; k < n; k++) {
        const int64_t a = rec.offset[k], b = rec.offset[k + 1];
        if (b < a) {
            why = "porosity record offsets decrease";
            return false;
        }
        if (!law_table(rec.values + a, b - a, base[k], ntab, zt, pt, why)) {
            why += " (record " + std::to_string(k) + ")";
            return false;
        }
        // thetaW_tab (swDdp.cpp:1921-1929): theta_0 = 0, theta_l += (z_l - z_(l-1)) phi_(l-1)
        double theta = 0;
        out.z.push_back(zt[0]);
        out.phi.push_back(pt[0]);
        out.theta.push_back(0.0);
        for (size_t l = 1; l < zt.size(); l++) {
            theta += (zt[l] - zt[l - 1]) * pt[l - 1];
            out.z.push_back(zt[l]);
            out.phi.push_back(pt[l]);
            out.theta.push_back(theta);
        }
        out.off[k + 1] = (int64_t)out.z.size();
    }
    return true;
}

std::vector<Lvl> levels_in_order(const DdpTables& t, const std::vector<int>& perm, std::vector<int>& off)
{
    std::vector<Lvl> lv;
    off.assign(perm.size() + 1, 0);
    lv.reserve(t.z.size());
    for (size_t i = 0; i < perm.size(); i++) {
        const int64_t o = perm[i];
        for (int64_t k = t.off[o]; k < t.off[o + 1]; k++) lv.push_back(Lvl{t.z[k], t.phi[k]});
        off[i + 1] = (int)lv.size();
    }
    return lv;
}

}  // namespace

namespace sw2d {

void launch_ddp_edges(sw2d_handle* h, const DevMesh& m, int v)
{
    switch (v) {
        case 1: launch_edges_v<1>(h, m); break;
        case 2: launch_edges_v<2>(h, m); break;
        case 3: launch_edges_v<3>(h, m); break;
        case 4: launch_edges_v<4>(h, m); break;
        case 5: launch_edges_v<5>(h, m); break;
        default: launch_edges_v<0>(h, m); break;
    }
}

void ddp_variant(int v, int* block, int* minb)
{
    const Variant x = kDdpVariants[(v >= 0 && v < 6) ? v : 0];
    *block = x.block;
    *minb = x.minb;
}

void launch_ddp_phase(sw2d_handle* h, int i)
{
    switch (i) {
        case 0: break;  // no reconstruction: the DDP step is Godunov only (swDdpHyp.cpp:496-516)
        case 1: launch_ddp_edges(h, h->m, h->edge_variant); break;
        case 2: launch_cfl_ddp_on(h, h->m); break;
        default: launch_tail(h, h->m); break;
    }
}

void launch_ddp_step(sw2d_handle* h)
{
    for (int i = 1; i < 4; i++) launch_ddp_phase(h, i);
}

int ddp_kernels_per_step(sw2d_handle* h)
{
    if (!h->ddp) return 0;
    if (h->ddp->div_corr == kDivCorrNone) return 3;
    if (h->ddp->div_corr == kDivCorrTimestep) return 6;
    return 4 + 6 * (h->ddp->n_it_div_max + 1);
}

int ddp_derive(sw2d_handle* h)
{
    k_ddp_derive<<<grid_for(h->nc), kBlock, 0, h->stream>>>(h->m);
    CK(cudaGetLastError());
    return SW2D_OK;
}

int ddp_check(const sw2d_mesh* mesh, const sw2d_ddp_fields* ddp, std::string& why)
{
    if (!ddp) {
        why = "DDP fields missing";
        return SW2D_E_ARG;
    }
    if (ddp->n_por_tab_max < 2 || ddp->n_por_tab_max > 100000) {
        why = "n_por_tab_max must be in [2, 100000]";
        return SW2D_E_ARG;
    }
    if (ddp->div_corr < kDivCorrNone || ddp->div_corr > kDivCorrTimestep) {
        why = "divergence correction not in {none, limit_flux, limit_timestep}";
        return SW2D_E_ARG;
    }
    if (ddp->div_corr == kDivCorrFlux && (ddp->n_it_div_max <= 0 || ddp->n_it_div_max > 1000)) {
        why = "n_it_div_max must be in [1, 1000] with limit_flux (swSolverParam.cpp:32-36)";
        return SW2D_E_ARG;
    }
    if (!(ddp->chi_phi_max >= 1.0)) {
        why = "ddp_chi_phi_max must be >= 1 (swSolverParam.cpp:1094-1098)";
        return SW2D_E_ARG;
    }
    if ((mesh->edge_int_nb && !ddp->edge_int_mz) || (mesh->edge_bnd_nb && !ddp->edge_bnd_mz)) {
        why = "edge midpoint elevations missing";
        return SW2D_E_ARG;
    }
    if (ddp->momentum_dissipation && (!ddp->mu_1 || !ddp->mu_2 || !ddp->mu_alpha)) {
        why = "momentum dissipation map missing";
        return SW2D_E_ARG;
    }
    return SW2D_OK;
}

int ddp_setup(sw2d_handle* h, const sw2d_mesh* mesh, const sw2d_cell_fields* fields, const sw2d_ddp_fields* ddp,
              const double* ic_level, const double* ic_x, const double* ic_y)
{
    (void)fields;
    DdpState* d = new DdpState();
    h->ddp = d;
    h->edge_variant = 0;  // {256, 2}: the DDP edge kernel's registers without spills
    d->div_corr = ddp->div_corr;
    d->n_it_div_max = (int)ddp->n_it_div_max;
    const int64_t nc = h->nc, ni = h->ni, nb = h->nb;
    const size_t ntab = (size_t)ddp->n_por_tab_max;
    std::string why;
    if (!build_tables(nc, ddp->cell, mesh->cell_z_b, ntab, d->cell, why) ||
        !build_tables(ni, ddp->edge_int, ddp->edge_int_mz, ntab, d->eint, why) ||
        !build_tables(nb, ddp->edge_bnd, ddp->edge_bnd_mz, ntab, d->ebnd, why))
        return fail(h, SW2D_E_ARG, why);
    // swDdp::checkParameterConsistency (swDdp.cpp:129-215): porosities in [0, 1], an edge's
    // porosity not above its cells' at the same level
    auto in01 = [](const DdpTables& t) {
        for (double p : t.phi)
            if ((p < 0.0) || (p > 1.0)) return false;
        return true;
    };
    if (!in01(d->cell)) return fail(h, SW2D_E_ARG, "cell porosity should belong to [0,1]");
    if (!in01(d->eint)) return fail(h, SW2D_E_ARG, "internal edge porosity should belong to [0,1]");
    if (!in01(d->ebnd)) return fail(h, SW2D_E_ARG, "boundary edge porosity should belong to [0,1]");
    for (int64_t c = 0; c < nc; c++)
        if (d->cell.levels(c) < 2)
            return fail(h, SW2D_E_ARG, "a cell porosity table needs two levels (the Riemann states read z_tab[1])");
    auto below = [&](const DdpTables& t, int64_t e, int64_t cell) {
        const int64_t ne = t.levels(e);
        if (ne > d->cell.levels(cell)) return false;  // the reference would read past the cell's table
        for (int64_t l = 0; l < ne; l++)
            if (t.phi[t.off[e] + l] > d->cell.phi[d->cell.off[cell] + l]) return false;
        return true;
    };
    for (int64_t e = 0; e < nb; e++)
        if (!below(d->ebnd, e, mesh->edge_bnd_cell[e]))
            return fail(h, SW2D_E_ARG, "boundary edge porosity larger than its cell's (or more levels)");
    for (int64_t e = 0; e < ni; e++) {
        if (d->eint.levels(e) < 1) return fail(h, SW2D_E_ARG, "empty internal edge porosity table");
        if (!below(d->eint, e, mesh->edge_int_cells[2 * e]) || !below(d->eint, e, mesh->edge_int_cells[2 * e + 1]))
            return fail(h, SW2D_E_ARG, "internal edge porosity larger than an adjacent cell's (or more levels)");
    }

    DevMesh& m = h->m;
    int rc = SW2D_OK;
    std::vector<int> coff, eoff;
    std::vector<Lvl> clv = levels_in_order(d->cell, h->cell_perm, coff);
    std::vector<Lvl> elv = levels_in_order(d->eint, h->int_perm, eoff);
    {
        Lvl* p = nullptr;
        if ((rc = dev_upload(h, clv, &p))) return rc;
        m.ctab = p;
        if ((rc = dev_upload(h, elv, &p))) return rc;
        m.etab = p;
        int* q = nullptr;
        if ((rc = dev_upload(h, coff, &q))) return rc;
        m.ctoff = q;
        if ((rc = dev_upload(h, eoff, &q))) return rc;
        m.etoff = q;
    }
    double4 *dcs = nullptr, *des = nullptr;
    if ((rc = dev_alloc(h, nc, &m.dv)) || (rc = dev_alloc(h, nc, &dcs)) || (rc = dev_alloc(h, 2 * ni, &des)))
        return rc;
    m.dcs = dcs;
    m.des = des;
    if (ddp->momentum_dissipation) {
        // swDdp::setMomentumDissipationParameters (swDdp.cpp:1729-1762)
        std::vector<double4> mu(nc);
        for (int64_t i = 0; i < nc; i++) {
            const int o = h->cell_perm[i];
            double a = ddp->mu_alpha[o] * atan(1.0) / 45.0;
            mu[i] = make_double4(ddp->mu_1[o], ddp->mu_2[o], cos(a), sin(a));
        }
        double4* p = nullptr;
        if ((rc = dev_upload(h, mu, &p))) return rc;
        m.mu = p;
    }
    if ((rc = dev_alloc(h, 1, &d->dctl))) return rc;
    m.dctl = d->dctl;
    m.chi_phi_max = ddp->chi_phi_max;
    m.div_corr = ddp->div_corr;
    m.n_it_div_max = (int)ddp->n_it_div_max;
    if (ddp->div_corr != kDivCorrNone) {
        if ((rc = dev_alloc(h, nc, &m.old))) return rc;
    }
    if (ddp->div_corr == kDivCorrTimestep) {
        if ((rc = dev_alloc(h, grid_for(nc) + 1, &d->part2))) return rc;
    }
    if (ddp->div_corr == kDivCorrFlux) {
        // the correction scales stored fluxes: keep them per edge
        if (!h->flux_buf) {
            if ((rc = dev_alloc(h, 3 * ni, &h->flux_buf)) || (rc = dev_alloc(h, nb, &h->bflux_buf))) return rc;
        }
        m.flux = h->flux_buf;
        m.bflux = h->bflux_buf;
        std::vector<int> inv(nc), nint(nc, 0), nbnd(nc, 0);
        for (int64_t i = 0; i < nc; i++) inv[h->cell_perm[i]] = (int)i;
        for (int64_t e = 0; e < ni; e++) {
            nint[mesh->edge_int_cells[2 * e]]++;
            nint[mesh->edge_int_cells[2 * e + 1]]++;
        }
        for (int64_t e = 0; e < nb; e++) nbnd[mesh->edge_bnd_cell[e]]++;
        int maxdeg = 0;
        for (int64_t c = 0; c < nc; c++) maxdeg = std::max(maxdeg, std::max(nint[c], nbnd[c]));
        if (maxdeg > 32) return fail(h, SW2D_E_UNSUPPORTED, "limit_flux: a cell with more than 32 edges of one kind");
        d->maxdeg = maxdeg;
        std::vector<int> inv_int(ni), inv_bnd(nb);
        for (int64_t i = 0; i < ni; i++) inv_int[h->int_perm[i]] = (int)i;
        for (int64_t i = 0; i < nb; i++) inv_bnd[h->bnd_perm[i]] = (int)i;
        std::vector<int> ie(std::max(1, maxdeg), -1), be(std::max(1, maxdeg), -1);
        for (int j = 0; j < maxdeg; j++) {
            if (j < ni) ie[j] = inv_int[j];
            if (j < nb) be[j] = inv_bnd[j];
        }
        const int64_t nblk = (nc + kFlagBlock - 1) / kFlagBlock;
        if ((rc = dev_upload(h, inv, &d->inv_cell)) || (rc = dev_upload(h, nint, &d->nint_o)) ||
            (rc = dev_upload(h, nbnd, &d->nbnd_o)) || (rc = dev_upload(h, ie, &d->dc_int_e)) ||
            (rc = dev_upload(h, be, &d->dc_bnd_e)) || (rc = dev_alloc(h, nc, &d->ratio)) ||
            (rc = dev_alloc(h, nblk, &d->blockcnt)) || (rc = dev_alloc(h, nblk, &d->blockoff)) ||
            (rc = dev_alloc(h, nc, &d->list)))
            return rc;
    }
    k_ddp_statics<<<grid_for(nc + ni), kBlock, 0, h->stream>>>(m, ddp->h_min_ddp, dcs, des, const_cast<double4*>(m.cst));
    CK(cudaGetLastError());
    // initial conditions from the caller's arrays
    double* tmp = nullptr;
    CK(cudaMalloc(&tmp, 3 * std::max<int64_t>(1, nc) * sizeof(double)));
    cudaError_t ce = cudaMemcpyAsync(tmp, ic_level, nc * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(tmp + nc, ic_x, nc * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(tmp + 2 * nc, ic_y, nc * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (ce == cudaSuccess) {
        k_ddp_ic<<<grid_for(nc), kBlock, 0, h->stream>>>(m, tmp, tmp + nc, tmp + 2 * nc, ddp->ic_columns,
                                                         h->d_cell_perm);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->stream);
    cudaFree(tmp);
    if (ce != cudaSuccess) return fail(h, SW2D_E_CUDA, std::string("DDP initialisation: ") + cudaGetErrorString(ce));
    return SW2D_OK;
}

void ddp_release(sw2d_handle* h)
{
    if (h->ddp && h->ddp->outbuf) cudaFree(h->ddp->outbuf);
    delete h->ddp;
    h->ddp = nullptr;
}

// DDP per-cell outputs of storeResultMaps ("water_depth", "unit_discharge_x",
// "unit_discharge_y", "surface_elevation") and the per-edge "thetaG_int_hmin", in the caller's
// numbering.  *handled is false for any other name.
int64_t ddp_get_array(sw2d_handle* h, const char* name, double* out, int64_t capacity, bool* handled)
{
    *handled = false;
    static const char* names[] = {"water_depth", "unit_discharge_x", "unit_discharge_y", "surface_elevation"};
    int which = -1;
    for (int i = 0; i < 4; i++)
        if (std::strcmp(name, names[i]) == 0) which = i;
    const bool hmin = std::strcmp(name, "thetaG_int_hmin") == 0;
    if (which < 0 && !hmin) return 0;
    *handled = true;
    const int64_t len = hmin ? h->ni : h->nc;
    if (capacity < len) return fail(h, SW2D_E_ARG, "output buffer too small");
    CK(cudaSetDevice(h->device));
    DdpState* d = h->ddp;
    const int64_t span = std::max<int64_t>(1, std::max(h->nc, h->ni));
    if (!d->outbuf) CK(cudaMalloc(&d->outbuf, 5 * span * sizeof(double)));
    double* stage = d->outbuf + 4 * span;
    if (hmin) {
        k_scatter_field<<<grid_for(h->ni), kBlock, 0, h->stream>>>(reinterpret_cast<const double*>(h->m.des), 8, 0,
                                                                    h->d_int_perm, stage, (int)h->ni);
    } else {
        k_ddp_outputs<<<grid_for(h->nc), kBlock, 0, h->stream>>>(h->m, d->outbuf);
        k_scatter_field<<<grid_for(h->nc), kBlock, 0, h->stream>>>(d->outbuf + which * h->nc, 1, 0, h->d_cell_perm,
                                                                    stage, (int)h->nc);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, stage, len * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return len;
}

// ddp_get_array through a device staging buffer the caller supplies (stage_cap doubles), with no
// allocation; arrays longer than stage_cap are rejected.
int64_t ddp_get_array_staged(sw2d_handle* h, const char* name, double* out, int64_t capacity, double* stage,
                             int64_t stage_cap, bool* handled)
{
    *handled = false;
    static const char* names[] = {"water_depth", "unit_discharge_x", "unit_discharge_y", "surface_elevation"};
    int which = -1;
    for (int i = 0; i < 4; i++)
        if (std::strcmp(name, names[i]) == 0) which = i;
    const bool hmin = std::strcmp(name, "thetaG_int_hmin") == 0;
    if (which < 0 && !hmin) return 0;
    *handled = true;
    const int64_t len = hmin ? h->ni : h->nc;
    if (capacity < len) return fail(h, SW2D_E_ARG, "output buffer too small");
    if (len > stage_cap)
        return fail(h, SW2D_E_ARG, std::string("sw2d_get_array_noalloc: ") + name + " has " + std::to_string(len) +
                                       " values, more than the fixed staging array holds (" +
                                       std::to_string(stage_cap) + "); use sw2d_get_array");
    CK(cudaSetDevice(h->device));
    if (len > 0) {
        if (hmin)
            k_scatter_field<<<grid_for(h->ni), kBlock, 0, h->stream>>>(reinterpret_cast<const double*>(h->m.des), 8, 0,
                                                                        h->d_int_perm, stage, (int)h->ni);
        else
            k_ddp_output_field<<<grid_for(h->nc), kBlock, 0, h->stream>>>(h->m, which, h->d_cell_perm, stage);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out, stage, len * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    return len;
}

// Porosity table of one record in the caller's numbering: which 0 cells, 1 internal edges,
// 2 boundary edges.  Returns the level count (copies min(count, capacity) levels).
int64_t ddp_get_table(sw2d_handle* h, int which, int64_t record, double* z, double* phi, double* theta,
                      int64_t capacity)
{
    if (!h->ddp) return fail(h, SW2D_E_ARG, "not a DDP handle");
    const DdpTables* t = which == 0 ? &h->ddp->cell : which == 1 ? &h->ddp->eint : which == 2 ? &h->ddp->ebnd : nullptr;
    if (!t) return fail(h, SW2D_E_ARG, "table kind not in {0 cells, 1 internal edges, 2 boundary edges}");
    if (record < 0 || record + 1 >= (int64_t)t->off.size()) return fail(h, SW2D_E_ARG, "record out of range");
    const int64_t a = t->off[record], n = t->off[record + 1] - a;
    for (int64_t l = 0; l < std::min(n, capacity); l++) {
        if (z) z[l] = t->z[a + l];
        if (phi) phi[l] = t->phi[a + l];
        if (theta) theta[l] = t->theta[a + l];
    }
    return n;
}

}  // namespace sw2d
