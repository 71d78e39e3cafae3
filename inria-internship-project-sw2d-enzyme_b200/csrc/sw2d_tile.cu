// sw2d_tile.cu — the flux half of the fused SP/DIP time step: one kernel per step that does
// everything of the step up to the time step itself, tile by tile of the Hilbert-ordered cells.
//
// The step is two kernels:
//   k_flux     per cell tile (one CTA)     slopes + limiter (MUSCL-EVR), Riemann states, HLLC and
//                                          boundary fluxes, the dt-free balance terms of the tile's
//                                          cells, their swept lengths and CFL bound, block minimum,
//                                          then the grid minimum, dt_map snap and t_max clip in the
//                                          last CTA done
//   k_update   per cell (sw2d_sp.cu)       balance in the reference's order, flush, clamp, sources
//
// Reference routines restated, per cell of a tile: swSp::computeMusclSlopes
// (sp/swSpHypMusclEvr.cpp:11-115), hypMusclEvrComputeLRStates / hypGodunovComputeLRStates
// (swSpHypMusclEvr.cpp:119-277, swSpHypGodunov.cpp:9-84), hypComputeFluxes and hypHllc
// (swSpHyp.cpp:276-402, 664-998), hypBoundaryFlux (swSpHyp.cpp:13-135), the dt-free products of
// hypComputeBalance (swSpHyp.cpp:214-273) and hypComputeTimeStep (swSpHyp.cpp:430-512); for the
// DIP model the same routines of dip/swDipHyp.cpp.
//
// A tile is a run of consecutive cells in the internal (Hilbert) numbering.  Its CTA stages in
// shared memory the state and statics of the tile's cells and of the cells one edge away (ring
// 1), and the free-surface elevation and centroid of the cells two edges away (ring 2), which
// the slopes of ring 1 need.  It then computes
//   * the limited slope of every tile and ring-1 cell (ring-1 slopes are recomputed by each
//     neighbouring tile: a few tenths of a slope per cell);
//   * every internal edge with at least one cell in the tile: the edges whose lower cell is in
//     the tile ("owned", a contiguous range of the edge numbering) and the edges that come in
//     from a lower tile (computed again there, for that tile's own cell);
//   * the tile's boundary edges;
// and writes the balance terms only for its own cells' slots, which lie in one contiguous slot
// range: the writes stay inside the tile, and nothing computed by the tile is read back from
// memory by the tile.  The CFL contributions of the edges stay in shared memory.
//
// Every arithmetic step is the one of the four-kernel step (k_slopes, k_edges, k_cfl), with the
// same operands in the same order, so the two give identical bits; only where the operands live
// changes.  Each per-cell sum runs over the cell's slots in the reference's order (boundary
// edges, then internal edges by increasing original index).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "sw2d_internal.cuh"

using namespace sw2d;

namespace {

// Asynchronous global -> shared copies (cp.async, sm_80+): every copy of a tile is issued before
// the first is waited for, so the loads of a tile are in flight together.
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cpa16(void* s, const void* g)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cpa8(void* s, const void* g)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cpa4(void* s, const void* g)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cpa_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// A tile's stage in shared memory, in the global records' own layouts (byte offsets computed on
// the host, TileMesh::o_*): per staged cell its state {h, q, r, z} and centroid {x, y}; per tile
// and ring-1 cell its statics {z_b, b, phi, area} and limited slope {sx, sy}; per tile cell its
// slot offsets; per tile slot the CFL contribution; per flux edge {nx, ny}, {coefL, coefR},
// length, {slot L, slot R} (and phiG for DIP); per tile edge {mx, my} and the local {L, R}; the
// neighbour lists of the tile and ring-1 cells.
struct Stage {
    double4* st;
    double4* cst;
    double2* xy;
    double2* sl;
    int2* coff;
    double* lam;
    double2* en;
    double2* ecf;
    double* elen;
    int2* esl;
    double* epg;
    double2* em;
    ushort2* ell;
    unsigned* ent;
    unsigned* so;
};

__device__ __forceinline__ Stage stage_of(const TileMesh& tm)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Stage v;
    v.st = reinterpret_cast<double4*>(smem_raw + tm.o_st);
    v.cst = reinterpret_cast<double4*>(smem_raw + tm.o_cst);
    v.xy = reinterpret_cast<double2*>(smem_raw + tm.o_xy);
    v.sl = reinterpret_cast<double2*>(smem_raw + tm.o_sl);
    v.coff = reinterpret_cast<int2*>(smem_raw + tm.o_coff);
    v.lam = reinterpret_cast<double*>(smem_raw + tm.o_lam);
    v.en = reinterpret_cast<double2*>(smem_raw + tm.o_en);
    v.ecf = reinterpret_cast<double2*>(smem_raw + tm.o_ecf);
    v.elen = reinterpret_cast<double*>(smem_raw + tm.o_elen);
    v.esl = reinterpret_cast<int2*>(smem_raw + tm.o_esl);
    v.epg = reinterpret_cast<double*>(smem_raw + tm.o_epg);
    v.em = reinterpret_cast<double2*>(smem_raw + tm.o_em);
    v.ell = reinterpret_cast<ushort2*>(smem_raw + tm.o_ell);
    v.ent = reinterpret_cast<unsigned*>(smem_raw + tm.o_ent);
    v.so = reinterpret_cast<unsigned*>(smem_raw + tm.o_so);
    return v;
}

// the slope of one cell from its neighbour list (entries: local neighbour | tile edge << 16 |
// side << 31), the same two passes as k_slopes: the gradient over the neighbours in the
// reference's order (divided by the weight sum; none with a single neighbour), then the limiter
// edge by edge in the same order
__device__ __forceinline__ double2 tile_slope(const Stage& sv, int k0, int k1, double zc, double xc, double yc)
{
    const int cnt = k1 - k0;
    double sx = 0.0, sy = 0.0, wsum = 0.0;
    if (cnt == 3) {
        // triangles: the three neighbours' terms are independent until they are summed, in the
        // same order as below
        unsigned en[3];
        double zj[3];
        double2 xj[3];
#pragma unroll
        for (int i = 0; i < 3; i++) {
            en[i] = sv.ent[k0 + i];
            const int j = (int)(en[i] & 0xffffu);
            xj[i] = sv.xy[j];
            zj[i] = sv.st[j].w;
        }
        double tx[3], ty[3], w[3];
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const double dx = xj[i].x - xc;
            const double dy = xj[i].y - yc;
            const double dist = sqrt(dx * dx + dy * dy);
            w[i] = 1.0 / dist;
            tx[i] = (zj[i] - zc) * dx / dist / dist * w[i];
            ty[i] = (zj[i] - zc) * dy / dist / dist * w[i];
        }
#pragma unroll
        for (int i = 0; i < 3; i++) {
            sx += tx[i];
            sy += ty[i];
            wsum += w[i];
        }
        sx /= wsum;
        sy /= wsum;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const int te = (int)((en[i] >> 16) & 0x7fffu);
            const bool is_r = (en[i] >> 31) != 0;
            const double2 mp = sv.em[te];
            const double zL = is_r ? zj[i] : zc;
            const double zR = is_r ? zc : zj[i];
            const double fmx = smax(zL, zR);
            const double fmn = smin(zL, zR);
            const double rec = zc + (mp.x - xc) * sx + (mp.y - yc) * sy;
            if (rec < fmn) {
                const double fac = (fmn - zc) / (rec - zc);
                sx *= fac;
                sy *= fac;
            }
            if (rec > fmx) {
                const double fac = (fmx - zc) / (rec - zc);
                sx *= fac;
                sy *= fac;
            }
        }
        return make_double2(sx, sy);
    }
    if (cnt > 1) {
        for (int k = k0; k < k1; k++) {
            const int j = (int)(sv.ent[k] & 0xffffu);
            const double2 xj = sv.xy[j];
            const double zj = sv.st[j].w;
            const double dx = xj.x - xc;
            const double dy = xj.y - yc;
            const double dist = sqrt(dx * dx + dy * dy);
            const double w = 1.0 / dist;
            sx += (zj - zc) * dx / dist / dist * w;
            sy += (zj - zc) * dy / dist / dist * w;
            wsum += w;
        }
        sx /= wsum;
        sy /= wsum;
    }
    for (int k = k0; k < k1; k++) {
        const unsigned en = sv.ent[k];
        const int j = (int)(en & 0xffffu);
        const int te = (int)((en >> 16) & 0x7fffu);
        const bool is_r = (en >> 31) != 0;
        const double2 mp = sv.em[te];
        const double zj = sv.st[j].w;
        const double zL = is_r ? zj : zc;
        const double zR = is_r ? zc : zj;
        const double fmx = smax(zL, zR);
        const double fmn = smin(zL, zR);
        const double rec = zc + (mp.x - xc) * sx + (mp.y - yc) * sy;
        if (rec < fmn) {
            const double fac = (fmn - zc) / (rec - zc);
            sx *= fac;
            sy *= fac;
        }
        if (rec > fmx) {
            const double fac = (fmx - zc) / (rec - zc);
            sx *= fac;
            sy *= fac;
        }
    }
    return make_double2(sx, sy);
}

__device__ __forceinline__ double min_keep_t(double a, double b) { return (b < a) ? b : a; }

#define TI(field) __ldg(&tm.info[blockIdx.x].field)

template <int kScheme, bool kBlending, int kModel, int kThreads, int kMinB>
__global__ void __launch_bounds__(kThreads, kMinB) k_flux(DevMesh m, TileMesh tm)
{
    constexpr bool kMuscl = kScheme == SW2D_SCHEME_MUSCL_EVR;
    constexpr bool kDip = kModel == kModelDip;
    Ctrl* ctrl = m.ctrl;
    if (!step_active(ctrl)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) ctrl->go = 0;
        return;
    }
    const Stage sv = stage_of(tm);

    // ---- stage the tile (contiguous), its rings (gathered) and its edges, all copies in flight
    {
        const int c0 = TI(c0), nt = TI(nt), hoff = TI(hoff);
        const bool own_slopes = kMuscl && tm.slopes_in;
        const int nf = nt + TI(nh1), nl = own_slopes ? nf + TI(nh2) : nf;
        for (int l = threadIdx.x; l < nl; l += kThreads) {
            const int g = (l < nt) ? c0 + l : ld(&tm.halo[hoff + l - nt]);
            const double2* sg = reinterpret_cast<const double2*>(m.st + g);
            cpa16(reinterpret_cast<double2*>(sv.st + l), sg);
            cpa16(reinterpret_cast<double2*>(sv.st + l) + 1, sg + 1);
            if (kMuscl) cpa16(sv.xy + l, m.cxy + g);
            if (l < nf) {
                const double2* cg = reinterpret_cast<const double2*>(m.cst + g);
                cpa16(reinterpret_cast<double2*>(sv.cst + l), cg);
                cpa16(reinterpret_cast<double2*>(sv.cst + l) + 1, cg + 1);
                if (kMuscl && !own_slopes) cpa16(sv.sl + l, m.slope + g);
            }
        }
        for (int l = threadIdx.x; l <= nt; l += kThreads) cpa8(sv.coff + l, m.coff + c0 + l);
        const int e0 = TI(e0), ne_own = TI(ne_own), xoff = TI(xoff), loff = TI(loff);
        const int nflux = ne_own + TI(nx_flux), nall = own_slopes ? nflux + TI(nx_slope) : nflux;
        for (int j = threadIdx.x; j < nall; j += kThreads) {
            const int e = (j < ne_own) ? e0 + j : ld(&tm.xe[xoff + j - ne_own]);
            cpa4(sv.ell + j, tm.eloc + loff + j);
            if (kMuscl) cpa16(sv.em + j, m.mxy + e);
            if (j < nflux) {
                cpa16(sv.en + j, m.nxy + e);
                cpa16(sv.ecf + j, m.coef + e);
                cpa8(sv.elen + j, m.len + e);
                cpa8(sv.esl + j, m.eslot + e);
                if (kDip) cpa8(sv.epg + j, m.phig + e);
            }
        }
        if (own_slopes) {
            const int soff = TI(soff), so_off = TI(so_off), nent = TI(nent);
            for (int k = threadIdx.x; k < nent; k += kThreads) cpa4(sv.ent + k, tm.scsr + soff + k);
            for (int l = threadIdx.x; l <= nf; l += kThreads) cpa4(sv.so + l, tm.soffs + so_off + l);
        }
        cpa_wait_all();
    }
    __syncthreads();

    // ---- slopes of the tile and ring-1 cells (computeMusclSlopes), unless k_slopes computed them
    if (kMuscl && tm.slopes_in) {
        const int c0 = TI(c0), nt = TI(nt), nf = nt + TI(nh1);
        const bool keep = m.flux != nullptr || m.lmax != nullptr;
        for (int l = threadIdx.x; l < nf; l += kThreads) {
            const double2 xy = sv.xy[l];
            const double2 g = tile_slope(sv, (int)sv.so[l], (int)sv.so[l + 1], sv.st[l].w, xy.x, xy.y);
            sv.sl[l] = g;
            if (keep && l < nt) m.slope[c0 + l] = g;
        }
        __syncthreads();
    }

    // ---- internal edges of the tile: owned, then incoming
    unsigned bad = 0;
    {
        const double dtp = ctrl->dt;
        const int nt = TI(nt), s0 = TI(s0);
        const int ne_own = TI(ne_own);
        const int nflux = ne_own + TI(nx_flux);
        const bool rec = m.flux != nullptr || m.lmax != nullptr;
        for (int j = threadIdx.x; j < nflux; j += kThreads) {
            const ushort2 ll = sv.ell[j];
            const int a = ll.x, b = ll.y;
            const double2 n = sv.en[j];
            const double4 Sa = sv.st[a], Sb = sv.st[b];
            const double4 Ka = sv.cst[a], Kb = sv.cst[b];
            SideState SL, SR;
            double phiG = 0.0, xL = 1.0, xR = 1.0;
            if (kDip) {
                phiG = sv.epg[j];
                xL = dip_x(Ka.z, phiG);
                xR = dip_x(Kb.z, phiG);
            }
            if (!kMuscl) {
                if (kDip) {
                    SL = godunov_side_dip(Sa.x, Sa.y, Sa.z, Ka.x, Ka.y, xL, n.x, n.y);
                    SR = godunov_side_dip(Sb.x, Sb.y, Sb.z, Kb.x, Kb.y, xR, n.x, n.y);
                } else {
                    SL = godunov_side(Sa.x, Sa.y, Sa.z, Ka.x, Ka.y, n.x, n.y);
                    SR = godunov_side(Sb.x, Sb.y, Sb.z, Kb.x, Kb.y, n.x, n.y);
                }
            } else {
                const double2 mp = sv.em[j];
                const double2 ca = sv.xy[a], cb = sv.xy[b];
                const double2 ga = sv.sl[a], gb = sv.sl[b];
                const double dax = mp.x - ca.x, day = mp.y - ca.y;
                const double dbx = mp.x - cb.x, dby = mp.y - cb.y;
                if (kDip) {
                    SL = evr_side_dip(true, Sa.x, Sa.y, Sa.z, Ka.x, Ka.y, xL, Sa.w, ga.x, ga.y, dax, day, n.x, n.y, dtp);
                    SR = evr_side_dip(false, Sb.x, Sb.y, Sb.z, Kb.x, Kb.y, xR, Sb.w, gb.x, gb.y, dbx, dby, n.x, n.y, dtp);
                } else {
                    SL = evr_side(true, Sa.x, Sa.y, Sa.z, Ka.x, Ka.y, Sa.w, ga.x, ga.y, dax, day, n.x, n.y, dtp, m.dry);
                    SR = evr_side(false, Sb.x, Sb.y, Sb.z, Kb.x, Kb.y, Sb.w, gb.x, gb.y, dbx, dby, n.x, n.y, dtp, m.dry);
                }
            }
            const double lm = max4(fabs(SL.lm), fabs(SL.lp), fabs(SR.lm), fabs(SR.lp));
            const int e = rec ? ((j < ne_own) ? TI(e0) + j : ld(&tm.xe[TI(xoff) + j - ne_own])) : 0;
            if (m.lmax) m.lmax[e] = lm;
            const double lw = lm * sv.elen[j];
            const bool wetL = Sa.x > m.h_min, wetR = Sb.x > m.h_min;
            const int2 sl = sv.esl[j];
            const bool ownL = a < nt, ownR = b < nt;
            if (ownL) sv.lam[sl.x - s0] = wetL ? lw : 0.0;
            if (ownR) sv.lam[sl.y - s0] = (wetL || wetR) ? lw : 0.0;
            const double hL = SL.z - Ka.x, hR = SR.z - Kb.x;
            if ((hL > m.h_min) || (hR > m.h_min)) {
                EdgeFlux f = kDip ? hllc_dip(kBlending, Ka.y, Kb.y, phiG, Ka.z, Kb.z, Ka.x, Kb.x, SL, SR, m.h_min, m.phi_min)
                                  : hllc(kBlending, Ka.y, Kb.y, Ka.z, Kb.z, Ka.x, Kb.x, SL, SR, m.h_min, m.phi_min);
                bad |= f.bad;
                if (isnan(f.f1)) bad |= kStatusNanFlux;
                if (m.flux) {
                    double2* fp = m.flux + 3 * (size_t)e;
                    fp[0] = make_double2(f.f1, f.f2);
                    fp[1] = make_double2(f.f3, f.sl);
                    fp[2] = make_double2(f.sr, 0.0);
                }
                const double2 cf = sv.ecf[j];
                const double nx = n.x, ny = n.y;
                if (ownL) {
                    const double c = cf.x;
                    const double f1 = -c, f2F2 = -c * nx, f2F3 = +c * ny, f2S2 = +c * nx;
                    const double f3F2 = -c * ny, f3F3 = -c * nx, f3S2 = +c * ny;
                    m.slot[sl.x] = make_slot(f1 * f.f1, f2F2 * f.f2 + f2S2 * f.sl + f2F3 * f.f3,
                                             f3F2 * f.f2 + f3S2 * f.sl + f3F3 * f.f3);
                }
                if (ownR) {
                    const double c = cf.y;
                    const double f1 = +c, f2F2 = +c * nx, f2F3 = -c * ny, f2S2 = +c * nx;
                    const double f3F2 = +c * ny, f3F3 = +c * nx, f3S2 = +c * ny;
                    m.slot[sl.y] = make_slot(f1 * f.f1, f2F2 * f.f2 + f2S2 * f.sr + f2F3 * f.f3,
                                             f3F2 * f.f2 + f3S2 * f.sr + f3F3 * f.f3);
                }
            }
        }
    }

    // ---- the tile's boundary edges (hypBoundaryFlux)
    {
        const double tnow = ctrl->t;
        const int c0 = TI(c0), b0 = TI(b0), nbe = TI(b1) - b0, s0 = TI(s0);
        for (int j = threadIdx.x; j < nbe; j += kThreads) {
            const int e = b0 + j;
            const int l = ld(&m.bcell[e]) - c0;
            const double4 g = ld(&m.bgeo[e]);
            const double4 Sl = sv.st[l], Kl = sv.cst[l];
            const double phiGb = kDip ? ld(&m.phigb[e]) : 0.0;
            SideState S = kDip ? godunov_side_dip(Sl.x, Sl.y, Sl.z, Kl.x, Kl.y, dip_x(Kl.z, phiGb), g.x, g.y)
                               : godunov_side(Sl.x, Sl.y, Sl.z, Kl.x, Kl.y, g.x, g.y);
            const double lm = kMuscl ? smax(fabs(S.lm), fabs(S.lp)) : smax(fabs(S.lp), fabs(S.lm));
            if (m.lmaxb) m.lmaxb[e] = lm;
            const int sbi = ld(&m.bslot[e]);
            sv.lam[sbi - s0] = (Sl.x > m.h_min) ? lm * g.z : 0.0;
            const int k = ld(&m.bbc[e]);
            const long long o0 = ld(&m.bcoff[k]), o1 = ld(&m.bcoff[k + 1]);
            const double v = bc_value(m.bctimes + o0, m.bcvals + o0, o1 - o0, tnow);
            double f1, f2, f3;
            bad |= kDip ? boundary_flux_dip(Kl.y, phiGb, Kl.z, Kl.x, S, ld(&m.bctype[k]), v, m.h_min, &f1, &f2, &f3)
                        : boundary_flux(Kl.y, Kl.z, Kl.x, S, ld(&m.bctype[k]), v, m.h_min, &f1, &f2, &f3);
            if (m.bflux) m.bflux[e] = make_double4(f1, f2, f3, 0.0);
            const double cf = g.w, nx = g.x, ny = g.y;
            const double fa = +cf, f2F2 = +cf * nx, f2F3 = -cf * ny, f2S2 = +cf * nx;
            const double f3F2 = +cf * ny, f3F3 = +cf * nx, f3S2 = +cf * ny;
            const double s2 = 0.0;  // boundary geometric source: never set by hypBoundaryFlux
            m.slot[sbi] = make_slot(fa * f1, f2F2 * f2 + f2S2 * s2 + f2F3 * f3, f3F2 * f2 + f3S2 * s2 + f3F3 * f3);
        }
    }
    if (bad) atomicOr(&ctrl->status, bad);
    __syncthreads();

    // ---- swept length and CFL bound of the tile's cells (hypComputeTimeStep)
    double best = m.dt_max;
    {
        const int nt = TI(nt), s0 = TI(s0);
        for (int l = threadIdx.x; l < nt; l += kThreads) {
            const int k0 = sv.coff[l].y - s0, k1 = sv.coff[l + 1].y - s0;
            double sw = 0.0;
            for (int k = k0; k < k1; k++) sw += sv.lam[k];
            const double x = m.cfl_max * (sv.cst[l].w / smax(sw, kSmallReal));
            if (x < best) best = x;
        }
    }
    // warp -> block minimum; the grid minimum by an integer atomicMin on the order-preserving key
    // (the minimum does not depend on the order it is taken in; no candidate is NaN: a NaN bound
    // never replaces best); dt_map snap and t_max clip in the last CTA done
    for (int off = 16; off > 0; off >>= 1) best = min_keep_t(best, __shfl_down_sync(0xffffffffu, best, off));
    __shared__ double wmin[kThreads / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) wmin[wid] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kThreads / 32; w++) best = min_keep_t(best, wmin[w]);
        atomicMin(&ctrl->dmin, dmin_key((unsigned long long)__double_as_longlong(best)));
        __threadfence();
        const unsigned done = atomicAdd(&ctrl->blocks_done, 1u);
        last = (done == gridDim.x - 1);
        if (last) {
            __threadfence();
            const unsigned long long key = atomicExch(&ctrl->dmin, kDminEmpty);
            double dt = __longlong_as_double((long long)dmin_bits(key));
            const double t = ctrl->t;
            int store = m.dt_map <= -kSmallReal ? 1 : 0;
            if (m.dt_map > kSmallReal) {
                const int now = (int)(t / m.dt_map);
                const int later = (int)((t + dt) / m.dt_map);
                if (later > now) {
                    dt = later * m.dt_map - t;
                    store = 1;
                }
            }
            if ((t + dt) > ctrl->t_max) dt = ctrl->t_max - t;
            ctrl->store_map = store;
            ctrl->dt = dt;
            ctrl->go = 1;
            ctrl->blocks_done = 0;
        }
    }
}

#undef TI

// Launch variants {threads per CTA, minimum resident CTAs per SM (register cap)}.
struct FluxVariant {
    int threads, minb;
};
constexpr FluxVariant kFluxVariants[] = {{256, 2}, {256, 3}, {192, 3}, {320, 2}, {256, 4}, {128, 8}};
constexpr int kNumFluxVariants = sizeof(kFluxVariants) / sizeof(kFluxVariants[0]);

// The stage's byte layout (every section 16-byte aligned) for the largest tile; returns its size.
size_t stage_layout(TileMesh& tm, bool muscl, bool slopes_read, bool dip)
{
    size_t o = 0;
    auto sec = [&](int* off, size_t bytes) {
        *off = (int)o;
        o += (bytes + 15) & ~(size_t)15;
    };
    const bool evr = muscl || slopes_read;
    sec(&tm.o_st, 32 * (size_t)tm.nl_max);
    sec(&tm.o_cst, 32 * (size_t)tm.nf_max);
    sec(&tm.o_xy, evr ? 16 * (size_t)tm.nl_max : 0);
    sec(&tm.o_sl, evr ? 16 * (size_t)tm.nf_max : 0);
    sec(&tm.o_coff, 8 * ((size_t)tm.nt_max + 1));
    sec(&tm.o_lam, 8 * (size_t)tm.ns_max);
    sec(&tm.o_en, 16 * (size_t)tm.ne_max);
    sec(&tm.o_ecf, 16 * (size_t)tm.ne_max);
    sec(&tm.o_elen, 8 * (size_t)tm.ne_max);
    sec(&tm.o_esl, 8 * (size_t)tm.ne_max);
    sec(&tm.o_epg, dip ? 8 * (size_t)tm.ne_max : 0);
    sec(&tm.o_em, evr ? 16 * (size_t)tm.na_max : 0);
    sec(&tm.o_ell, 4 * (size_t)tm.na_max);
    sec(&tm.o_ent, muscl ? 4 * (size_t)tm.nent_max : 0);
    sec(&tm.o_so, muscl ? 4 * ((size_t)tm.nf_max + 1) : 0);
    tm.smem = (int)o;
    return o;
}

size_t flux_smem(const TileMesh& tm, bool) { return (size_t)tm.smem; }

template <int kScheme, bool kBlending, int kModel, int V>
cudaError_t launch_flux_v(sw2d_handle* h, const DevMesh& m, bool attr_only)
{
    constexpr int T = kFluxVariants[V].threads, B = kFluxVariants[V].minb;
    auto kern = k_flux<kScheme, kBlending, kModel, T, B>;
    const size_t smem = flux_smem(h->tiles, kScheme == SW2D_SCHEME_MUSCL_EVR);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess || attr_only) return e;
    kern<<<(unsigned)h->tiles.ntiles, T, smem, h->stream>>>(m, h->tiles);
    return cudaSuccess;
}

template <int kScheme, bool kBlending, int kModel>
cudaError_t launch_flux_s(sw2d_handle* h, const DevMesh& m, int v, bool attr_only)
{
    switch (v) {
        case 1: return launch_flux_v<kScheme, kBlending, kModel, 1>(h, m, attr_only);
        case 2: return launch_flux_v<kScheme, kBlending, kModel, 2>(h, m, attr_only);
        case 3: return launch_flux_v<kScheme, kBlending, kModel, 3>(h, m, attr_only);
        case 4: return launch_flux_v<kScheme, kBlending, kModel, 4>(h, m, attr_only);
        case 5: return launch_flux_v<kScheme, kBlending, kModel, 5>(h, m, attr_only);
        default: return launch_flux_v<kScheme, kBlending, kModel, 0>(h, m, attr_only);
    }
}

template <int kModel>
cudaError_t launch_flux_m(sw2d_handle* h, const DevMesh& m, int v, bool attr_only)
{
    const bool bl = h->p.topo == SW2D_TOPO_BLENDING;
    if (h->p.scheme == SW2D_SCHEME_GODUNOV) {
        return bl ? launch_flux_s<SW2D_SCHEME_GODUNOV, true, kModel>(h, m, v, attr_only)
                  : launch_flux_s<SW2D_SCHEME_GODUNOV, false, kModel>(h, m, v, attr_only);
    }
    return bl ? launch_flux_s<SW2D_SCHEME_MUSCL_EVR, true, kModel>(h, m, v, attr_only)
              : launch_flux_s<SW2D_SCHEME_MUSCL_EVR, false, kModel>(h, m, v, attr_only);
}

}  // namespace

namespace sw2d {

int flux_variants() { return kNumFluxVariants; }

std::string flux_variant_label(int v)
{
    if (v < 0 || v >= kNumFluxVariants) return "?";
    return std::to_string(kFluxVariants[v].threads) + "x" + std::to_string(kFluxVariants[v].minb);
}

cudaError_t launch_flux(sw2d_handle* h, const DevMesh& m, int v, bool attr_only)
{
    if (h->model == kModelDip) return launch_flux_m<kModelDip>(h, m, v, attr_only);
    return launch_flux_m<kModelSp>(h, m, v, attr_only);
}

// Host-side construction of the tiles (see the top of this file).  Inputs are in the internal
// numbering: per cell, its internal-neighbour entries {edge * 2 + side, neighbour} in the
// reference's order (coff.x ranges of cint) and its first balance slot (coff.y); per internal
// edge its {L, R} cells; edges are ordered by their lower cell, boundary edges by their cell.
int tiles_build(sw2d_handle* h, const std::vector<int2>& coff, const std::vector<int2>& cint,
                const std::vector<int2>& lr, const std::vector<int>& bcell, int tile_cells, std::string& why)
{
    // ring 2, the ring-1 slope edges and the neighbour lists serve the slopes k_flux computes
    const bool muscl = h->p.scheme == SW2D_SCHEME_MUSCL_EVR && h->fused_slopes;
    const bool slopes_read = h->p.scheme == SW2D_SCHEME_MUSCL_EVR && !h->fused_slopes;
    const int nc = (int)h->nc, ni = (int)h->ni, nb = (int)h->nb;
    if (tile_cells < 32 || tile_cells > 8192) {
        why = "tile size outside 32..8192 cells";
        return SW2D_E_ARG;
    }
    const int ntiles = (nc + tile_cells - 1) / tile_cells;
    // first edge of each lower cell (edges are sorted by their lower cell)
    std::vector<int> efirst(nc + 1, 0);
    for (int e = 0; e < ni; e++) efirst[std::min(lr[e].x, lr[e].y) + 1]++;
    for (int c = 0; c < nc; c++) efirst[c + 1] += efirst[c];
    for (int e = 1; e < ni; e++)
        if (std::min(lr[e].x, lr[e].y) < std::min(lr[e - 1].x, lr[e - 1].y)) {
            why = "internal edges not ordered by their lower cell";
            return SW2D_E_ARG;
        }
    std::vector<int> bfirst(nc + 1, 0);
    for (int e = 0; e < nb; e++) bfirst[bcell[e] + 1]++;
    for (int c = 0; c < nc; c++) bfirst[c + 1] += bfirst[c];

    std::vector<TileInfo> info(ntiles);
    std::vector<int> halo, xe;
    std::vector<ushort2> eloc;
    std::vector<unsigned> scsr;
    std::vector<unsigned> soffs;
    halo.reserve((size_t)nc / 2);
    std::vector<int> cstamp(nc, -1), clid(nc, 0), estamp(ni, -1), elid(ni, 0);
    int nl_max = 0, nf_max = 0, ns_max = 0, ne_max = 0, na_max = 0, nent_max = 0, nt_max = 0;
    std::vector<int> h1, h2, xin, xsl;
    for (int t = 0; t < ntiles; t++) {
        TileInfo& ti = info[t];
        const int c0 = t * tile_cells, nt = std::min(tile_cells, nc - c0), c1 = c0 + nt;
        auto in_tile = [&](int c) { return c >= c0 && c < c1; };
        h1.clear();
        h2.clear();
        xin.clear();
        xsl.clear();
        for (int c = c0; c < c1; c++)
            for (int k = coff[c].x; k < coff[c + 1].x; k++) {
                const int j = cint[k].y;
                if (!in_tile(j) && cstamp[j] != t) {
                    cstamp[j] = t;
                    clid[j] = nt + (int)h1.size();
                    h1.push_back(j);
                }
            }
        if (muscl)
            for (int hc : h1)
                for (int k = coff[hc].x; k < coff[hc + 1].x; k++) {
                    const int j = cint[k].y;
                    if (!in_tile(j) && cstamp[j] != t) {
                        cstamp[j] = t;
                        clid[j] = nt + (int)h1.size() + (int)h2.size();
                        h2.push_back(j);
                    }
                }
        auto lid = [&](int c) { return in_tile(c) ? c - c0 : clid[c]; };
        // owned edges [e0, e1): lower cell in the tile
        const int e0 = efirst[c0], e1 = efirst[c1];
        // incoming edges: an internal edge of a tile cell whose other cell lies below the tile
        for (int c = c0; c < c1; c++)
            for (int k = coff[c].x; k < coff[c + 1].x; k++)
                if (cint[k].y < c0) xin.push_back(cint[k].x >> 1);
        std::sort(xin.begin(), xin.end());
        const int ne_own = e1 - e0, nx_flux = (int)xin.size();
        for (int i = 0; i < nx_flux; i++) {
            estamp[xin[i]] = t;
            elid[xin[i]] = ne_own + i;
        }
        // slope-only edges: ring-1 cell to a ring-1 or ring-2 cell
        if (muscl)
            for (int hc : h1)
                for (int k = coff[hc].x; k < coff[hc + 1].x; k++) {
                    const int e = cint[k].x >> 1;
                    const int j = cint[k].y;
                    if (in_tile(j) || estamp[e] == t) continue;
                    estamp[e] = t;
                    elid[e] = ne_own + nx_flux + (int)xsl.size();
                    xsl.push_back(e);
                }
        auto tedge = [&](int e) { return (e >= e0 && e < e1) ? e - e0 : elid[e]; };
        const int nh1 = (int)h1.size(), nh2 = (int)h2.size();
        const int nf = nt + nh1, nl = nf + (muscl ? nh2 : 0);
        const int nedges = ne_own + nx_flux + (int)xsl.size();
        if (nl > 0xffff || nedges > 0x7fff) {
            why = "a tile's rings or edges exceed the 16-bit local indices";
            return SW2D_E_UNSUPPORTED;
        }
        ti.c0 = c0;
        ti.nt = nt;
        ti.nh1 = nh1;
        ti.nh2 = muscl ? nh2 : 0;
        ti.hoff = (int)halo.size();
        halo.insert(halo.end(), h1.begin(), h1.end());
        if (muscl) halo.insert(halo.end(), h2.begin(), h2.end());
        ti.e0 = e0;
        ti.ne_own = ne_own;
        ti.xoff = (int)xe.size();
        ti.nx_flux = nx_flux;
        ti.nx_slope = (int)xsl.size();
        xe.insert(xe.end(), xin.begin(), xin.end());
        xe.insert(xe.end(), xsl.begin(), xsl.end());
        ti.loff = (int)eloc.size();
        for (int e = e0; e < e1; e++) eloc.push_back(make_ushort2((unsigned short)lid(lr[e].x), (unsigned short)lid(lr[e].y)));
        for (int e : xin) eloc.push_back(make_ushort2((unsigned short)lid(lr[e].x), (unsigned short)lid(lr[e].y)));
        for (int e : xsl) eloc.push_back(make_ushort2((unsigned short)lid(lr[e].x), (unsigned short)lid(lr[e].y)));
        ti.soff = (int)scsr.size();
        ti.so_off = (int)soffs.size();
        ti.nent = 0;
        if (muscl) {
            int cnt = 0;
            for (int l = 0; l < nf; l++) {
                soffs.push_back((unsigned)cnt);
                const int g = l < nt ? c0 + l : h1[l - nt];
                for (int k = coff[g].x; k < coff[g + 1].x; k++) {
                    const int e = cint[k].x >> 1, side = cint[k].x & 1;
                    scsr.push_back((unsigned)lid(cint[k].y) | ((unsigned)tedge(e) << 16) | ((unsigned)side << 31));
                    cnt++;
                }
                if (cnt > 0xffff) {
                    why = "a tile's neighbour lists exceed the 16-bit offsets";
                    return SW2D_E_UNSUPPORTED;
                }
            }
            soffs.push_back((unsigned)cnt);
            ti.nent = cnt;
        }
        ti.b0 = bfirst[c0];
        ti.b1 = bfirst[c1];
        ti.s0 = coff[c0].y;
        nl_max = std::max(nl_max, nl);
        nf_max = std::max(nf_max, nf);
        nt_max = std::max(nt_max, nt);
        ns_max = std::max(ns_max, coff[c1].y - coff[c0].y);
        ne_max = std::max(ne_max, ne_own + nx_flux);
        na_max = std::max(na_max, nedges);
        nent_max = std::max(nent_max, ti.nent);
    }
    TileMesh& tm = h->tiles;
    TileMesh probe;
    probe.nl_max = nl_max;
    probe.nf_max = nf_max;
    probe.nt_max = nt_max;
    probe.ns_max = ns_max;
    probe.ne_max = ne_max;
    probe.na_max = na_max;
    probe.nent_max = nent_max;
    probe.slopes_in = muscl ? 1 : 0;
    const size_t smem = stage_layout(probe, muscl, slopes_read, h->model == kModelDip);
    if (smem > 200 * 1024) {
        why = "a tile's shared-memory stage exceeds 200 KB";
        return SW2D_E_UNSUPPORTED;
    }
    // replace the previous tiles' arrays
    for (void* p : h->tile_allocs) cudaFree(p);
    h->tile_allocs.clear();
    tm = probe;
    tm.ntiles = ntiles;
    tm.tile_cells = tile_cells;
    auto up = [&](const auto& vec, auto** dst) -> int {
        using T = typename std::remove_reference<decltype(vec)>::type::value_type;
        void* p = nullptr;
        const size_t bytes = std::max<size_t>(1, vec.size()) * sizeof(T);
        if (cudaMalloc(&p, bytes) != cudaSuccess) return fail(h, SW2D_E_CUDA, "cudaMalloc (tiles)");
        h->tile_allocs.push_back(p);
        if (!vec.empty() && cudaMemcpyAsync(p, vec.data(), vec.size() * sizeof(T), cudaMemcpyHostToDevice, h->stream) !=
                                cudaSuccess)
            return fail(h, SW2D_E_CUDA, "tile upload");
        *dst = static_cast<T*>(p);
        return SW2D_OK;
    };
    TileInfo* d_info = nullptr;
    int *d_halo = nullptr, *d_xe = nullptr;
    ushort2* d_eloc = nullptr;
    unsigned* d_scsr = nullptr;
    unsigned* d_soffs = nullptr;
    int rc = up(info, &d_info);
    if (!rc) rc = up(halo, &d_halo);
    if (!rc) rc = up(xe, &d_xe);
    if (!rc) rc = up(eloc, &d_eloc);
    if (!rc) rc = up(scsr, &d_scsr);
    if (!rc) rc = up(soffs, &d_soffs);
    if (!rc && cudaStreamSynchronize(h->stream) != cudaSuccess) rc = fail(h, SW2D_E_CUDA, "tile upload");
    if (rc) {
        for (void* p : h->tile_allocs) cudaFree(p);
        h->tile_allocs.clear();
        tm = TileMesh{};
        return rc;
    }
    tm.info = d_info;
    tm.halo = d_halo;
    tm.xe = d_xe;
    tm.eloc = d_eloc;
    tm.scsr = d_scsr;
    tm.soffs = d_soffs;
    return SW2D_OK;
}

}  // namespace sw2d
