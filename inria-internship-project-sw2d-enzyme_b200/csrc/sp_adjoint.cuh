// sp_adjoint.cuh — hand-written reverse mode of the SP step's arithmetic (sp_math.cuh).
//
// Each *_rev function recomputes the forward intermediates of its forward twin and
// propagates output adjoints ("bars") back to the inputs that are controls or states:
// water depth h, unit discharges q, r, free surface z, bed level z_b, limited slopes and the
// friction coefficients.  Porosity, Boussinesq coefficients, geometry and dt are constants
// (dt is frozen along the recorded trajectory, as the reference's assimilation does,
// assim/swSpE_checkpoint.cpp:1436-1453).
//
// Branches follow the forward evaluation (wet/dry tests, HLLC configuration, limiter
// triggers, max/min selections): the derivative is that of the branch taken.  Where the
// forward takes sqrt of exactly 0 (a dry cell's celerity) or the norm of a zero velocity,
// the subgradient 0 is used instead of an infinite derivative.
#pragma once

#include "sp_math.cuh"

namespace sw2d {

struct SideBar {
    double z, q, r, lm, lp;
};

struct CellBar {
    double h, q, r, zb, zc, sx, sy;
};

SW2D_HD double dsqrt_bar(double y, double ybar) { return (y > 0.0) ? ybar * 0.5 / y : 0.0; }

// ---- godunov_side (swSpHypGodunov.cpp:17-35)
SW2D_HD void godunov_side_rev(double h, double q, double r, double b, double nx, double ny, const SideBar& sb,
                              CellBar& cb)
{
    const double sq = q * nx + r * ny;
    const double d = smax(h, kSmallReal);
    const double u = sq / d;
    const double c = sqrt(kGravity * h);
    const double X = (b - 1.0) * b * u * u + c * c;
    const double root = sqrt(X);
    const double bu_bar = sb.lm + sb.lp;
    const double root_bar = sb.lp - sb.lm;
    const double X_bar = dsqrt_bar(root, root_bar);
    const double u_bar = bu_bar * b + X_bar * (b - 1.0) * b * 2.0 * u;
    const double c_bar = X_bar * 2.0 * c;
    double h_bar = sb.z;                          // z = h + z_b
    cb.zb += sb.z;
    h_bar += dsqrt_bar(c, c_bar) * kGravity;      // c = sqrt(g h)
    const double sq_bar = sb.q + u_bar / d;
    if (!(h < kSmallReal)) h_bar += -u_bar * u / d;   // d = h
    const double sr_bar = sb.r;                   // sr = -q ny + r nx
    cb.h += h_bar;
    cb.q += sq_bar * nx - sr_bar * ny;
    cb.r += sq_bar * ny + sr_bar * nx;
}

// ---- evr_side (swSpHypMusclEvr.cpp:176-272).  zc = h + z_b of the cell, (sx, sy) its slopes.
SW2D_HD void evr_side_rev(bool left, double h, double q, double r, double zb, double b, double zc, double sx,
                          double sy, double dmx, double dmy, double nx, double ny, double dt,
                          const SideBar& sb, CellBar& cb)
{
    // forward recomputation
    const double ql = q * nx + r * ny;
    const double rl = r * nx - q * ny;
    const double hd = smax(kSmallReal, h);
    const double cl = sqrt(kGravity * hd);
    const double ul = ql / hd;
    const double vl = rl / hd;
    const double X1 = (b - 1.0) * b * ul * ul + cl * cl;
    const double root1 = sqrt(X1);
    const double lmv = b * ul - root1;
    const double lpv = b * ul + root1;
    const double l1 = left ? smax(0.0, lmv) : smin(0.0, lmv);
    const double dx1 = dmx - 0.5 * l1 * dt * nx;
    const double dy1 = dmy - 0.5 * l1 * dt * ny;
    const double z1 = zc + dx1 * sx + dy1 * sy;
    const double l2 = left ? smax(0.0, lpv) : smin(0.0, lpv);
    const double dx2 = dmx - 0.5 * l2 * dt * nx;
    const double dy2 = dmy - 0.5 * l2 * dt * ny;
    const double z2 = zc + dx2 * sx + dy2 * sy;
    const double h1 = smax(0.0, z1 - zb);
    const double h2 = smax(0.0, z2 - zb);
    const double hr = 0.5 * (h1 + h2);
    const double sq = hr * ul;
    const double d2 = smax(hr, kSmallReal);
    const double u = sq / d2;
    const double c = sqrt(kGravity * hr);
    const double X = (b - 1.0) * b * u * u + c * c;
    const double root = sqrt(X);
    // reverse (the derivative terms multiply by the reciprocals of the two denominators)
    const double rd2 = 1.0 / d2, rhd = 1.0 / hd;
    const double bu_bar = sb.lm + sb.lp;
    const double root_bar = sb.lp - sb.lm;
    const double X_bar = dsqrt_bar(root, root_bar);
    const double u_bar = bu_bar * b + X_bar * (b - 1.0) * b * 2.0 * u;
    const double c_bar = X_bar * 2.0 * c;
    double hr_bar = dsqrt_bar(c, c_bar) * kGravity;
    const double sq_bar = sb.q + u_bar * rd2;
    if (!(hr < kSmallReal)) hr_bar += -u_bar * u * rd2;
    hr_bar += sb.z;                               // z = hr + z_b
    double zb_bar = sb.z;
    hr_bar += sq_bar * ul;
    double ul_bar = sq_bar * hr;
    hr_bar += sb.r * vl;                          // sr = hr vl
    const double vl_bar = sb.r * hr;
    const double h1_bar = 0.5 * hr_bar, h2_bar = 0.5 * hr_bar;
    double zc_bar = 0.0, sx_bar = 0.0, sy_bar = 0.0, lmv_bar = 0.0, lpv_bar = 0.0;
    {  // h2 = max(0, z2 - zb)
        const double e = (0.0 < z2 - zb) ? h2_bar : 0.0;
        zb_bar -= e;
        zc_bar += e;
        sx_bar += e * dx2;
        sy_bar += e * dy2;
        const double l2_bar = -(e * sx) * 0.5 * dt * nx - (e * sy) * 0.5 * dt * ny;
        if (left ? (0.0 < lpv) : (lpv < 0.0)) lpv_bar += l2_bar;
    }
    {  // h1 = max(0, z1 - zb)
        const double e = (0.0 < z1 - zb) ? h1_bar : 0.0;
        zb_bar -= e;
        zc_bar += e;
        sx_bar += e * dx1;
        sy_bar += e * dy1;
        const double l1_bar = -(e * sx) * 0.5 * dt * nx - (e * sy) * 0.5 * dt * ny;
        if (left ? (0.0 < lmv) : (lmv < 0.0)) lmv_bar += l1_bar;
    }
    ul_bar += b * (lmv_bar + lpv_bar);
    const double root1_bar = lpv_bar - lmv_bar;
    const double X1_bar = dsqrt_bar(root1, root1_bar);
    ul_bar += X1_bar * (b - 1.0) * b * 2.0 * ul;
    const double cl_bar = X1_bar * 2.0 * cl;
    const double ql_bar = ul_bar * rhd;
    const double rl_bar = vl_bar * rhd;
    double hd_bar = -ul_bar * ul * rhd - vl_bar * vl * rhd + dsqrt_bar(cl, cl_bar) * kGravity;
    if (kSmallReal < h) cb.h += hd_bar;
    cb.q += ql_bar * nx - rl_bar * ny;
    cb.r += ql_bar * ny + rl_bar * nx;
    cb.zb += zb_bar;
    cb.zc += zc_bar;
    cb.sx += sx_bar;
    cb.sy += sy_bar;
}

// ---- hllc (swSpHyp.cpp:664-998): flux bars -> side bars and bed bars.  Returns false when the
// forward configuration is the one the reference rejects.
SW2D_HD void hllc_rev(bool blending, double bL, double bR, double phiL, double phiR, double zbL, double zbR,
                      const SideState& L, const SideState& R, double h_min, double phi_min, const EdgeFlux& fb,
                      SideBar& Lb, SideBar& Rb, double& zbL_bar, double& zbR_bar)
{
    double hL, hR;
    bool selL = true, selR = true;  // whether h = z - z_b (not the 0 of the max)
    if (blending) {
        hL = L.z - zbL;
        hR = R.z - zbR;
    } else {
        selL = 0.0 < L.z - zbL;
        selR = 0.0 < R.z - zbR;
        hL = selL ? L.z - zbL : 0.0;
        hR = selR ? R.z - zbR : 0.0;
    }
    bool both = false, lhs = false, rhs = false, none = false;
    if (((hL <= h_min) && (hR <= h_min)) || ((phiL <= phi_min) && (phiR <= phi_min))) {
        none = true;
    } else {
        both = true;
        if ((phiR <= phi_min) || ((phiR > phi_min) && (hR <= h_min) && (L.z <= zbR + h_min))) { lhs = true; both = false; }
        if ((phiL <= phi_min) || ((phiL > phi_min) && (hL <= h_min) && (R.z <= zbL + h_min))) { rhs = true; both = false; }
    }
    double hL_bar = 0.0, hR_bar = 0.0;
    if ((int)both + (int)lhs + (int)rhs + (int)none != 1 || none) {
        // no flux depends on the states
    } else if (rhs && !lhs) {
        hR_bar += fb.sr * phiR * kGravity * hR;    // sr = phiR 0.5 g hR^2
    } else if (lhs && !rhs) {
        hL_bar += -fb.sl * phiL * kGravity * hL;   // sl = -phiL 0.5 g hL^2
    } else {
        // ---- forward recomputation of the "both" branch
        const double duL = blending ? smax(hL, kSmallReal) : smax(kSmallReal, hL);
        const double duR = blending ? smax(hR, kSmallReal) : smax(kSmallReal, hR);
        const bool duL_h = blending ? !(hL < kSmallReal) : (kSmallReal < hL);
        const bool duR_h = blending ? !(hR < kSmallReal) : (kSmallReal < hR);
        const double uL = L.q / duL, uR = R.q / duR;
        const double mR = smin(R.lm, 0.);
        const double L1 = smin(L.lm, mR);
        const double m2 = smax(R.lp, 0.);
        const double L2 = smax(L.lp, m2);
        const double dLL = L2 - L1;
        const double den = smax(dLL, kSmallReal);
        const double phiLR = smin(phiL, phiR);
        const double pm = smin(phiL, phiR);
        double alpha = 0.0, ratio = 0.0, dzb = zbL - zbR;
        bool alpha_free = false;
        double F1h = 0, F1z = 0, f1, s2a, s2z = 0, s2h = 0;
        const double fact = 0.5 * pm * (hL + hR);
        if (blending) {
            if (fabs(dzb) > kSmallReal) {
                ratio = (L.z - R.z) / dzb;
                const double inner = smin(1.0, ratio);
                alpha = smax(0.0, inner);
                alpha_free = (0.0 < inner) && (ratio < 1.0);
            }
            F1h = phiLR * (L2 * L.q - L1 * R.q + L1 * L2 * (hR - hL)) / den;
            F1z = phiLR * (L2 * L.q - L1 * R.q + L1 * L2 * (R.z - L.z)) / den;
            f1 = alpha * F1h + (1.0 - alpha) * F1z;
            s2z = (phiR * hR * hR - phiL * hL * hL) * 0.5 + fact * (L.z - R.z);
            s2h = (zbL > zbR) ? phiR * hR * (zbL - zbR) : phiL * hL * (zbL - zbR);
            s2a = alpha * s2h + (1.0 - alpha) * s2z;
        } else {
            f1 = phiLR * (L2 * L.q - L1 * R.q + L1 * L2 * (R.z - L.z)) / den;
            s2a = (phiR * hR * hR - phiL * hL * hL) * 0.5 + fact * (L.z - R.z);
        }
        const double s2 = s2a * kGravity / den;
        const double sl = -L1 * s2, sr = L2 * s2;
        const double FL = spec_force(bL, phiL, hL, uL);
        const double FR = spec_force(bR, phiR, hR, uR);
        const double P = phiR * R.q - phiL * L.q;
        const double N2 = L2 * (FL + sl) - L1 * (FR - sr) + L1 * L2 * P;
        const double f2 = N2 / den;
        const double dvL = smax(hL, kSmallReal), dvR = smax(hR, kSmallReal);
        const double vL = L.r / dvL, vR = R.r / dvR;
        // ---- reverse.  The derivative terms divide by the reciprocal of each denominator, taken
        // once (the forward values above, which decide the branches, keep the forward's divisions)
        const double rden = 1.0 / den, rdvL = 1.0 / dvL, rdvR = 1.0 / dvR, rduL = 1.0 / duL, rduR = 1.0 / duR;
        double f1_bar = fb.f1, L1_bar = 0, L2_bar = 0, den_bar = 0;
        double Lq_bar = 0, Rq_bar = 0, Lz_bar = 0, Rz_bar = 0, Lr_bar = 0, Rr_bar = 0;
        double uL_bar = 0, uR_bar = 0;
        if (f1 >= 0) {
            f1_bar += fb.f3 * bL * vL;
            const double vL_bar = fb.f3 * bL * f1;
            Lr_bar += vL_bar * rdvL;
            if (!(hL < kSmallReal)) hL_bar += -vL_bar * vL * rdvL;
        } else {
            f1_bar += fb.f3 * bR * vR;
            const double vR_bar = fb.f3 * bR * f1;
            Rr_bar += vR_bar * rdvR;
            if (!(hR < kSmallReal)) hR_bar += -vR_bar * vR * rdvR;
        }
        const double N2_bar = fb.f2 * rden;
        den_bar += -fb.f2 * f2 * rden;
        L2_bar += N2_bar * (FL + sl) + N2_bar * L1 * P;
        const double FL_bar = N2_bar * L2;
        double sl_bar = fb.sl + N2_bar * L2;
        L1_bar += -N2_bar * (FR - sr) + N2_bar * L2 * P;
        const double FR_bar = -N2_bar * L1;
        double sr_bar = fb.sr + N2_bar * L1;
        Rq_bar += N2_bar * L1 * L2 * phiR;
        Lq_bar -= N2_bar * L1 * L2 * phiL;
        // F = phi (b h u^2 + 0.5 g h^2)
        hL_bar += FL_bar * phiL * (bL * uL * uL + kGravity * hL);
        uL_bar += FL_bar * phiL * bL * hL * 2.0 * uL;
        hR_bar += FR_bar * phiR * (bR * uR * uR + kGravity * hR);
        uR_bar += FR_bar * phiR * bR * hR * 2.0 * uR;
        L1_bar += -sl_bar * s2;
        double s2_bar = -sl_bar * L1 + sr_bar * L2;
        L2_bar += sr_bar * s2;
        const double s2a_bar = s2_bar * kGravity * rden;
        den_bar += -s2_bar * s2 * rden;
        double fact_bar = 0.0, alpha_bar = 0.0;
        if (blending) {
            alpha_bar += s2a_bar * (s2h - s2z);
            const double s2h_bar = s2a_bar * alpha;
            const double s2z_bar = s2a_bar * (1.0 - alpha);
            if (zbL > zbR) {
                hR_bar += s2h_bar * phiR * (zbL - zbR);
                zbL_bar += s2h_bar * phiR * hR;
                zbR_bar -= s2h_bar * phiR * hR;
            } else {
                hL_bar += s2h_bar * phiL * (zbL - zbR);
                zbL_bar += s2h_bar * phiL * hL;
                zbR_bar -= s2h_bar * phiL * hL;
            }
            hR_bar += s2z_bar * phiR * hR;
            hL_bar -= s2z_bar * phiL * hL;
            fact_bar += s2z_bar * (L.z - R.z);
            Lz_bar += s2z_bar * fact;
            Rz_bar -= s2z_bar * fact;
            // f1 = alpha F1h + (1 - alpha) F1z
            alpha_bar += f1_bar * (F1h - F1z);
            const double F1h_bar = f1_bar * alpha, F1z_bar = f1_bar * (1.0 - alpha);
            const double Nh_bar = F1h_bar * phiLR * rden, Nz_bar = F1z_bar * phiLR * rden;
            den_bar += -F1h_bar * F1h * rden - F1z_bar * F1z * rden;
            const double Ns_bar = Nh_bar + Nz_bar;  // the shared part L2 qL - L1 qR
            L2_bar += Ns_bar * L.q + Nh_bar * L1 * (hR - hL) + Nz_bar * L1 * (R.z - L.z);
            L1_bar += -Ns_bar * R.q + Nh_bar * L2 * (hR - hL) + Nz_bar * L2 * (R.z - L.z);
            Lq_bar += Ns_bar * L2;
            Rq_bar -= Ns_bar * L1;
            hR_bar += Nh_bar * L1 * L2;
            hL_bar -= Nh_bar * L1 * L2;
            Rz_bar += Nz_bar * L1 * L2;
            Lz_bar -= Nz_bar * L1 * L2;
            if (alpha_free) {
                const double ratio_bar = alpha_bar;
                Lz_bar += ratio_bar / dzb;
                Rz_bar -= ratio_bar / dzb;
                const double dzb_bar = -ratio_bar * ratio / dzb;
                zbL_bar += dzb_bar;
                zbR_bar -= dzb_bar;
            }
        } else {
            hR_bar += s2a_bar * phiR * hR;
            hL_bar -= s2a_bar * phiL * hL;
            fact_bar += s2a_bar * (L.z - R.z);
            Lz_bar += s2a_bar * fact;
            Rz_bar -= s2a_bar * fact;
            const double N1_bar = f1_bar * phiLR * rden;
            den_bar += -f1_bar * f1 * rden;
            L2_bar += N1_bar * (L.q + L1 * (R.z - L.z));
            L1_bar += N1_bar * (-R.q + L2 * (R.z - L.z));
            Lq_bar += N1_bar * L2;
            Rq_bar -= N1_bar * L1;
            Rz_bar += N1_bar * L1 * L2;
            Lz_bar -= N1_bar * L1 * L2;
        }
        hL_bar += fact_bar * 0.5 * pm;
        hR_bar += fact_bar * 0.5 * pm;
        if (!(dLL < kSmallReal)) {
            L2_bar += den_bar;
            L1_bar -= den_bar;
        }
        // L1 = min(L.lm, min(R.lm, 0)), L2 = max(L.lp, max(R.lp, 0))
        if (mR < L.lm) {
            if (!(0. < R.lm)) Rb.lm += L1_bar;
        } else {
            Lb.lm += L1_bar;
        }
        if (L.lp < m2) {
            if (!(R.lp < 0.)) Rb.lp += L2_bar;
        } else {
            Lb.lp += L2_bar;
        }
        Lq_bar += uL_bar * rduL;
        if (duL_h) hL_bar += -uL_bar * uL * rduL;
        Rq_bar += uR_bar * rduR;
        if (duR_h) hR_bar += -uR_bar * uR * rduR;
        Lb.q += Lq_bar;
        Rb.q += Rq_bar;
        Lb.r += Lr_bar;
        Rb.r += Rr_bar;
        Lb.z += Lz_bar;
        Rb.z += Rz_bar;
    }
    // h = z - z_b (blending) or max(0, z - z_b)
    if (selL) {
        Lb.z += hL_bar;
        zbL_bar -= hL_bar;
    }
    if (selR) {
        Rb.z += hR_bar;
        zbR_bar -= hR_bar;
    }
}

// ---- boundary_flux (swSpHyp.cpp:13-135): flux bars -> side bar and bed bar
SW2D_HD void boundary_flux_rev(double bR, double phiR, double zbR, const SideState& S, int type, double bcv,
                               double h_min, double f1b, double f2b, double f3b, SideBar& sb, double& zb_bar)
{
    const double hR0 = S.z - zbR;
    const bool dry = hR0 < h_min;
    const double hR = dry ? 0. : hR0;
    const double q1 = dry ? 0. : S.q, r1 = dry ? 0. : S.r;
    const double dR = smax(hR, kSmallReal);
    const double cR = sqrt(kGravity * dR);
    const double uR = q1 / dR;
    const bool lsel = 0.0 < S.lp;
    const double L1 = lsel ? S.lp : 0.0;
    // forward flux1 (needed by the f3 branch and by flux2)
    double flux1 = 0.0;
    int path = 0;  // 1: fr, 2: h/z wet, 3: h/z dry, 4: q (bc value), 5: q (critical inflow)
    double c_fr = 0, cpre = 0, hc = 0;
    if (type == 3) {
        cpre = (uR - 2. * cR) / (-bcv - 2.);
        c_fr = smax(cpre, 0.);
        const double u = -bcv * c_fr;
        const double h = c_fr * c_fr / kGravity;
        flux1 = phiR * u * h;
        path = 1;
    } else if (type == 1 || type == 2) {
        const double h_bc = (type == 1) ? smax(bcv, 0.) : smax(bcv - zbR, 0.);
        if (hR > h_min) {
            flux1 = phiR * (q1 + L1 * (h_bc - hR));
            path = 2;
        } else {
            flux1 = phiR * h_bc * sqrt(kGravity * h_bc);
            path = 3;
        }
    } else if (type == 0) {
        flux1 = bcv;
        hc = h_critical(phiR, bcv);
        path = 4;
        if (hc >= hR) {
            flux1 = phiR * 1.5 * sqrt(kGravity * hc) * hc;
            path = 5;
        }
    }
    // reverse
    double flux1_bar = f1b, hR_bar = 0.0, q1_bar = 0.0, r1_bar = 0.0, uR_bar = 0.0, L1_bar = 0.0, cR_bar = 0.0;
    double zbR_bar_local = 0.0;
    if (!(flux1 > 0)) {  // flux3 = flux1 * r1 / max(hR, small)
        const double dv = smax(hR, kSmallReal);
        const double vR = r1 / dv;
        flux1_bar += f3b * vR;
        const double vR_bar = f3b * flux1;
        r1_bar += vR_bar / dv;
        if (!(hR < kSmallReal)) hR_bar += -vR_bar * vR / dv;
    }
    double flux2R_bar = 0.0;
    if (path == 1 || path == 2 || path == 4 || path == 5) {  // flux2 = flux2R + (flux1 - q1 phiR) L1
        flux2R_bar += f2b;
        flux1_bar += f2b * L1;
        q1_bar += -f2b * L1 * phiR;
        L1_bar += f2b * (flux1 - q1 * phiR);
    }
    // path 3: flux2 = spec_force(bR, phiR, h_bc, c) depends only on the boundary value (and z_b for 'z')
    if (path == 3 && type == 2) {
        const double hbc0 = bcv - zbR;
        if (!(hbc0 < 0.)) {
            const double h_bc = hbc0;
            const double c = sqrt(kGravity * h_bc);
            // flux1 = phiR h_bc c ; flux2 = phiR (bR h_bc c^2 + 0.5 g h_bc^2)
            double hbc_bar = flux1_bar * phiR * c + f2b * phiR * (bR * c * c + kGravity * h_bc);
            const double c_bar = flux1_bar * phiR * h_bc + f2b * phiR * bR * h_bc * 2.0 * c;
            hbc_bar += dsqrt_bar(c, c_bar) * kGravity;
            zbR_bar_local -= hbc_bar;
        }
        flux1_bar = 0.0;
    }
    if (path == 1) {
        // flux1 = phiR u h, u = -bcv c, h = c^2/g, c = max(cpre, 0)
        const double c_bar = flux1_bar * phiR * ((-bcv) * (c_fr * c_fr / kGravity) + (-bcv * c_fr) * 2.0 * c_fr / kGravity);
        if (!(cpre < 0.)) {
            const double cpre_bar = c_bar;
            uR_bar += cpre_bar / (-bcv - 2.);
            cR_bar += -2. * cpre_bar / (-bcv - 2.);
        }
    } else if (path == 2) {
        const double h_bc = (type == 1) ? smax(bcv, 0.) : smax(bcv - zbR, 0.);
        q1_bar += flux1_bar * phiR;
        L1_bar += flux1_bar * phiR * (h_bc - hR);
        hR_bar -= flux1_bar * phiR * L1;
        if (type == 2 && !(bcv - zbR < 0.)) zbR_bar_local -= flux1_bar * phiR * L1;
    } else if (path == 5) {
        // flux1 = phiR 1.5 sqrt(g hc) hc: hc depends on the boundary value only
    }
    // flux2R = spec_force(bR, phiR, hR, uR)
    hR_bar += flux2R_bar * phiR * (bR * uR * uR + kGravity * hR);
    uR_bar += flux2R_bar * phiR * bR * hR * 2.0 * uR;
    // uR = q1 / dR ; cR = sqrt(g dR)
    q1_bar += uR_bar / dR;
    double dR_bar = -uR_bar * uR / dR + dsqrt_bar(cR, cR_bar) * kGravity;
    if (!(hR < kSmallReal)) hR_bar += dR_bar;
    if (lsel) sb.lp += L1_bar;
    if (!dry) {
        sb.q += q1_bar;
        sb.r += r1_bar;
        sb.z += hR_bar;      // hR = z - z_b
        zbR_bar_local -= hR_bar;
    }
    zb_bar += zbR_bar_local;
}

// ---- k_update's per-cell part (swSpHyp.cpp:197-209, swSpSourceFriction.cpp:39-219, swSp.cpp:447-479).
// Forward from the post-balance state (hB, qB, rB); reverse gives the bars of the post-balance
// state and of the two friction coefficients.
struct UpdateParams {
    int friction;        // 0 none, 1 chezy, 2 manning, 3 strickler
    bool head_loss;
    bool clamp_negative; // negative_depth_detection off: h < 0 -> (0, 0, 0)
    bool flush_branch;   // round-off flush |x| < 1e-16 -> 0: zero derivative (the branch taken)
                         // instead of the identity
    double h_min, v_max, fr_max, dt;
    double k1, k2, fcos, fsin;           // friction
    double hs, hk1, hk2, hcos, hsin;     // head loss
    bool P_given = false;                // P = friction_power(h) of the friction stage is known
    double P = 0.0;                      // (the forward recompute keeps it)
    bool cap_given = false;              // whether the velocity cap acted is known (cap_acted)
    bool cap_acted = false;
};

// Reverse of friction_factor: f is the forward factor, P = exp(-4/3 log h) (Manning, Strickler),
// rh = 1 / h (the derivative terms multiply by it)
SW2D_HD void friction_factor_rev(int model, double k, double h, double un, double dt, double P, double f,
                                 double f_bar, double& k_bar, double& h_bar, double& un_bar, double rh)
{
    if (model == 1) {
        if ((h > kSmallReal) && (k > kSmallReal)) {
            const double A_bar = f_bar * f * dt;
            un_bar += A_bar * (-kGravity / k / k / h);
            k_bar += A_bar * 2.0 * kGravity * un / (k * k * k) / h;
            h_bar += A_bar * kGravity * un / k / k * (1.0 / (h * h));
        }
    } else if (model == 2) {
        if (h > kSmallReal) {
            const double A_bar = f_bar * f * dt;
            un_bar += A_bar * (-kGravity * k * k * P);
            k_bar += A_bar * (-kGravity * un * 2.0 * k * P);
            h_bar += A_bar * (-kGravity * un * k * k) * P * (-4.0 / 3.0) * rh;
        }
    } else {
        if ((h > kSmallReal) && (k > kSmallReal)) {
            const double A_bar = f_bar * f * dt;
            un_bar += A_bar * (-kGravity / k / k * P);
            k_bar += A_bar * 2.0 * kGravity * un / (k * k * k) * P;
            h_bar += A_bar * (-kGravity * un / k / k) * P * (-4.0 / 3.0) * rh;
        }
    }
}

// out = U(in); (ho, qo, ro) = out bars -> (hb, qb, rb) = in bars, k1b, k2b = coefficient bars
SW2D_HD void update_cell_rev(const UpdateParams& p, double hB, double qB, double rB, double ho, double qo, double ro,
                             double& hb, double& qb, double& rb, double& k1b, double& k2b)
{
    // ---- forward, keeping what the reverse needs
    double hh = hB, qq = qB, rr = rB;
    const bool fh = fabs(hh) < kSmallReal, fq = fabs(qq) < kSmallReal, fr_ = fabs(rr) < kSmallReal;
    if (fh) hh = 0.;
    if (fq) qq = 0.;
    if (fr_) rr = 0.;
    const bool neg = p.clamp_negative && hh < 0.;
    if (neg) { hh = 0.; qq = 0.; rr = 0.; }
    const double hthr = smax(p.h_min, kSmallReal);
    // friction
    const double h_f = hh, q_f = qq, r_f = rr;   // inputs of the friction stage
    bool fr_wet = false;
    double u = 0, v = 0, ul0 = 0, vl0 = 0, un = 0, f1 = 1, f2 = 1, P = 0;
    if (p.friction != 0) {
        if (hh > hthr) {
            fr_wet = true;
            u = qq / hh;
            v = rr / hh;
            ul0 = u * p.fcos + v * p.fsin;
            vl0 = -u * p.fsin + v * p.fcos;
            un = sqrt(u * u + v * v);
            if (p.friction != 1 && hh > kSmallReal) P = p.P_given ? p.P : friction_power(hh);
            f1 = friction_factor_p(p.friction, p.k1, hh, un, p.dt, P);
            f2 = (p.k2 == p.k1) ? f1 : friction_factor_p(p.friction, p.k2, hh, un, p.dt, P);
            const double ul = ul0 * f1, vl = vl0 * f2;
            qq = (ul * p.fcos - vl * p.fsin) * hh;
            rr = (ul * p.fsin + vl * p.fcos) * hh;
        } else {
            qq = 0.;
            rr = 0.;
        }
    }
    // head loss
    const double q_h = qq, r_h = rr;
    double qx0 = 0, qy0 = 0, ax = 0, ay = 0, ex = 1, ey = 1, nq = 0;
    bool hl_wet = false, hl_act = false;
    if (p.head_loss) {
        qx0 = qq * p.hcos + rr * p.hsin;
        qy0 = -qq * p.hsin + rr * p.hcos;
        double qx = qx0, qy = qy0;
        if (hh > hthr) {
            hl_wet = true;
            if (hh > p.hs) {
                hl_act = true;
                nq = sqrt(qx * qx + qy * qy);
                ax = nq * p.hk1 / hh;
                ay = nq * p.hk2 / hh;
            }
            ex = sw2d_exp(-ax * p.dt);
            ey = sw2d_exp(-ay * p.dt);
            qx = qx * ex;
            qy = qy * ey;
        } else {
            qx = 0.;
            qy = 0.;
        }
        qq = qx * p.hcos - qy * p.hsin;
        rr = qx * p.hsin + qy * p.hcos;
    }
    // velocity cap
    const double q_c = qq, r_c = rr;
    bool capped = false;
    double qn = 0, cc = 0, fact = 0;
    bool fact_from_v = false;
    if (hh > p.h_min && (!p.cap_given || p.cap_acted)) {  // the cap's test, unless known to be off
        qn = sqrt(qq * qq + rr * rr);
        cc = sqrt(kGravity * hh);
        const double Fr = qn / cc / hh;
        const double a = qn / (hh * p.v_max), b = Fr / p.fr_max;
        fact = smax(a, b);
        fact_from_v = !(a < b);
        if (fact > 1.0) capped = true;
    }
    // ---- reverse
    double h_bar = ho, q_bar = qo, r_bar = ro;
    if (capped) {
        // qo = q_c / fact, ro = r_c / fact
        const double fact_bar = -q_bar * q_c / (fact * fact) - r_bar * r_c / (fact * fact);
        q_bar = q_bar / fact;
        r_bar = r_bar / fact;
        double qn_bar = 0.0;
        if (fact_from_v) {  // fact = qn / (h vmax)
            qn_bar += fact_bar / (hh * p.v_max);
            h_bar += -fact_bar * qn / (hh * hh * p.v_max);
        } else {            // fact = qn / cc / h / frmax
            qn_bar += fact_bar / cc / hh / p.fr_max;
            const double cc_bar = -fact_bar * qn / (cc * cc) / hh / p.fr_max;
            h_bar += -fact_bar * qn / cc / (hh * hh) / p.fr_max;
            h_bar += dsqrt_bar(cc, cc_bar) * kGravity;
        }
        if (qn > 0.0) {
            q_bar += qn_bar * q_c / qn;
            r_bar += qn_bar * r_c / qn;
        }
    }
    if (p.head_loss) {
        // qq = qx cos - qy sin ; rr = qx sin + qy cos
        double qx_bar = q_bar * p.hcos + r_bar * p.hsin;
        double qy_bar = -q_bar * p.hsin + r_bar * p.hcos;
        double qx0_bar = 0.0, qy0_bar = 0.0;
        if (hl_wet) {
            qx0_bar = qx_bar * ex;
            qy0_bar = qy_bar * ey;
            if (hl_act) {
                const double ax_bar = qx_bar * qx0 * ex * (-p.dt);
                const double ay_bar = qy_bar * qy0 * ey * (-p.dt);
                const double nq_bar = ax_bar * p.hk1 / hh + ay_bar * p.hk2 / hh;
                h_bar += -ax_bar * ax / hh - ay_bar * ay / hh;
                if (nq > 0.0) {
                    qx0_bar += nq_bar * qx0 / nq;
                    qy0_bar += nq_bar * qy0 / nq;
                }
            }
        }
        // qx0 = q cos + r sin ; qy0 = -q sin + r cos
        q_bar = qx0_bar * p.hcos - qy0_bar * p.hsin;
        r_bar = qx0_bar * p.hsin + qy0_bar * p.hcos;
    }
    (void)q_h;
    (void)r_h;
    if (p.friction != 0) {
        if (fr_wet) {
            // qq = (ul cos - vl sin) h ; rr = (ul sin + vl cos) h ; ul = ul0 f1 ; vl = vl0 f2
            const double ul = ul0 * f1, vl = vl0 * f2;
            h_bar += q_bar * (ul * p.fcos - vl * p.fsin) + r_bar * (ul * p.fsin + vl * p.fcos);
            const double ul_bar = (q_bar * p.fcos + r_bar * p.fsin) * h_f;
            const double vl_bar = (-q_bar * p.fsin + r_bar * p.fcos) * h_f;
            double ul0_bar = ul_bar * f1, vl0_bar = vl_bar * f2;
            const double f1_bar = ul_bar * ul0, f2_bar = vl_bar * vl0;
            double un_bar = 0.0;
            // the derivative terms multiply by the reciprocals of h and |u|, taken once
            const double rh = 1.0 / h_f;
            friction_factor_rev(p.friction, p.k1, h_f, un, p.dt, P, f1, f1_bar, k1b, h_bar, un_bar, rh);
            friction_factor_rev(p.friction, p.k2, h_f, un, p.dt, P, f2, f2_bar, k2b, h_bar, un_bar, rh);
            double u_bar = ul0_bar * p.fcos - vl0_bar * p.fsin;
            double v_bar = ul0_bar * p.fsin + vl0_bar * p.fcos;
            if (un > 0.0) {
                const double run = 1.0 / un;
                u_bar += un_bar * u * run;
                v_bar += un_bar * v * run;
            }
            // u = q / h, v = r / h
            q_bar = u_bar * rh;
            r_bar = v_bar * rh;
            h_bar += -u_bar * u * rh - v_bar * v * rh;
        } else {
            q_bar = 0.0;
            r_bar = 0.0;
        }
    }
    (void)q_f;
    (void)r_f;
    if (neg) { h_bar = 0.; q_bar = 0.; r_bar = 0.; }
    // The flush moves a value by less than 1e-16.  Differentiating the branch taken gives 0 (what
    // line-by-line AD of the reference's balance gives); a state at rest sits exactly there, so
    // by default the flush is differentiated as the identity, which central differences see.
    if (p.flush_branch) {
        if (fh) h_bar = 0.;
        if (fq) q_bar = 0.;
        if (fr_) r_bar = 0.;
    }
    hb = h_bar;
    qb = q_bar;
    rb = r_bar;
}

// ---- MUSCL slopes of one cell (swSpHypMusclEvr.cpp:11-115), up to kMaxNbr neighbours.
constexpr int kMaxNbr = 8;

struct SlopeNbr {
    double zj, dx, dy, ax, ay;  // neighbour z, centroid offset (j - c), midpoint offset (m - c)
    bool c_is_r;                // the cell is the R side of the shared edge
};

// The slope functions loop over a compile-time capacity N (with n <= N used entries); for
// N <= 4 the loops are unrolled so that a kernel instantiated for triangles (N = 3) keeps every
// per-neighbour value in registers, larger capacities keep plain loops (local memory).
#if defined(__CUDACC__)
#define SW2D_UNROLL_KU _Pragma("unroll kU")
#else
#define SW2D_UNROLL_KU
#endif

// Forward with the intermediate slopes before each limiter test (for the reverse).
template <int N>
SW2D_HD void slopes_fwd_t(double zc, int n, const SlopeNbr* nb, double& sx, double& sy, double* sxk, double* syk)
{
    constexpr int kU = N <= 4 ? N : 1;
    sx = 0.0;
    sy = 0.0;
    double wsum = 0.0;
    if (n > 1) {
        SW2D_UNROLL_KU
        for (int k = 0; k < N; k++) {
            if (k < n) {
                const double dist = sqrt(nb[k].dx * nb[k].dx + nb[k].dy * nb[k].dy);
                const double w = 1.0 / dist;
                sx += (nb[k].zj - zc) * nb[k].dx / dist / dist * w;
                sy += (nb[k].zj - zc) * nb[k].dy / dist / dist * w;
                wsum += w;
            }
        }
        sx /= wsum;
        sy /= wsum;
    }
    SW2D_UNROLL_KU
    for (int k = 0; k < N; k++) {
        if (k < n) {
            sxk[k] = sx;
            syk[k] = sy;
            const double zL = nb[k].c_is_r ? nb[k].zj : zc;
            const double zR = nb[k].c_is_r ? zc : nb[k].zj;
            const double fmx = smax(zL, zR), fmn = smin(zL, zR);
            const double rec = zc + nb[k].ax * sx + nb[k].ay * sy;
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
    }
}

// (sxb, syb) = bars of the final slopes -> zc_bar and zj_bar[k], k < n <= N
template <int N>
SW2D_HD void slopes_rev_t(double zc, int n, const SlopeNbr* nb, double sxb, double syb, double& zc_bar, double* zj_bar)
{
    constexpr int kU = N <= 4 ? N : 1;
    double sx, sy, sxk[N], syk[N];
    slopes_fwd_t<N>(zc, n, nb, sx, sy, sxk, syk);
    SW2D_UNROLL_KU
    for (int k = 0; k < N; k++) zj_bar[k] = 0.0;
    SW2D_UNROLL_KU
    for (int k = N - 1; k >= 0; k--) {
        if (k >= n) continue;
        const double sx0 = sxk[k], sy0 = syk[k];
        const double zL = nb[k].c_is_r ? nb[k].zj : zc;
        const double zR = nb[k].c_is_r ? zc : nb[k].zj;
        const bool mx_left = !(zL < zR);     // smax(zL, zR) == zL
        const bool mn_left = !(zR < zL);     // smin(zL, zR) == zL
        const double fmx = mx_left ? zL : zR, fmn = mn_left ? zL : zR;
        const double rec = zc + nb[k].ax * sx0 + nb[k].ay * sy0;
        const bool under = rec < fmn, over = rec > fmx;
        if (!under && !over) continue;
        const bool sel_left = under ? mn_left : mx_left;
        const double f = under ? fmn : fmx;
        const double den = rec - zc;
        const double fac = (f - zc) / den;
        const double fac_bar = sxb * sx0 + syb * sy0;
        double sx0_bar = sxb * fac, sy0_bar = syb * fac;
        const double num_bar = fac_bar / den;
        const double den_bar = -fac_bar * fac / den;
        // f = zL or zR ; num = f - zc ; den = rec - zc ; rec = zc + ax sx0 + ay sy0
        const bool f_is_c = sel_left ? !nb[k].c_is_r : nb[k].c_is_r;
        if (f_is_c) zc_bar += num_bar;
        else zj_bar[k] += num_bar;
        zc_bar -= num_bar;  // den = rec - zc does not depend on zc (rec = zc + ax sx0 + ay sy0)
        sx0_bar += den_bar * nb[k].ax;
        sy0_bar += den_bar * nb[k].ay;
        sxb = sx0_bar;
        syb = sy0_bar;
    }
    if (n > 1) {
        double wsum = 0.0;
        SW2D_UNROLL_KU
        for (int k = 0; k < N; k++)
            if (k < n) wsum += 1.0 / sqrt(nb[k].dx * nb[k].dx + nb[k].dy * nb[k].dy);
        const double Sx_bar = sxb / wsum, Sy_bar = syb / wsum;
        SW2D_UNROLL_KU
        for (int k = 0; k < N; k++) {
            if (k < n) {
                const double dist = sqrt(nb[k].dx * nb[k].dx + nb[k].dy * nb[k].dy);
                const double w = 1.0 / dist;
                const double t_bar = Sx_bar * (nb[k].dx / dist / dist * w) + Sy_bar * (nb[k].dy / dist / dist * w);
                zj_bar[k] += t_bar;
                zc_bar -= t_bar;
            }
        }
    }
}

SW2D_HD void slopes_fwd(double zc, int n, const SlopeNbr* nb, double& sx, double& sy, double* sxk, double* syk)
{
    slopes_fwd_t<kMaxNbr>(zc, n, nb, sx, sy, sxk, syk);
}

SW2D_HD void slopes_rev(double zc, int n, const SlopeNbr* nb, double sxb, double syb, double& zc_bar, double* zj_bar)
{
    slopes_rev_t<kMaxNbr>(zc, n, nb, sxb, syb, zc_bar, zj_bar);
}

}  // namespace sw2d
