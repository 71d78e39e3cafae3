// dip_math.cuh — device arithmetic of SW2D's dual integral porosity (DIP) step: the routines that
// differ from the single-porosity step (sp_math.cuh).  The storage porosity phiW is per cell,
// the connectivity porosity phiG per edge, and x = phiW / max(phiG, 1e-16) enters the wave
// speeds and the specific force.  Every function restates one routine of the reference
// (src/sw2dSolver/models/dip/) with the same operand order, for bit-identical results under
// -fmad=false.  The edge factors, CFL step, slopes, friction, singular head loss and velocity
// cap are the SP routines (the reference's DIP versions are the same code over phiW).
#pragma once

#include "sp_math.cuh"

namespace sw2d {

constexpr unsigned kStatusPhiG = 64u;  // specific force with phiG < 1e-16: swDip.cpp:1524-1528 stops

SW2D_HD double dip_x(double phiW, double phiG) { return phiW / smax(phiG, kSmallReal); }

// swDip::lambdaMinus / lambdaPlus (dip/swDip.cpp:1035-1066), with x precomputed (same value)
SW2D_HD double lam_minus_dip(double b, double x, double c, double u)
{
    return b * x * u - sqrt((b * x - 1) * b * x * u * u + c * c / smax(x, kSmallReal));
}
SW2D_HD double lam_plus_dip(double b, double x, double c, double u)
{
    return b * x * u + sqrt((b * x - 1) * b * x * u * u + c * c / smax(x, kSmallReal));
}

// swDip::specificForce (dip/swDip.cpp:1522-1531); the caller flags phiG < 1e-16
SW2D_HD double spec_force_dip(double b, double phiG, double x, double h, double u)
{
    return (b * h * x * x * u * u + 0.5 * kGravity * h * h) * phiG;
}

// swDip::hypGodunovComputeLRStates, one side (dip/swDipHypGodunov.cpp:17-78)
SW2D_HD SideState godunov_side_dip(double h, double q, double r, double zb, double b, double x, double nx, double ny)
{
    SideState s;
    s.z = h + zb;
    s.q = q * nx + r * ny;
    s.r = -q * ny + r * nx;
    const double u = s.q / smax(h, kSmallReal);
    const double c = sqrt(kGravity * h);
    s.lm = lam_minus_dip(b, x, c, u);
    s.lp = lam_plus_dip(b, x, c, u);
    return s;
}

// One side of swDip::hypMusclEvrComputeLRStates (dip/swDipHypMusclEvr.cpp:170-272): the SP
// reconstruction (evr_side) with the DIP wave speeds
SW2D_HD SideState evr_side_dip(bool left, double h, double q, double r, double zb, double b, double x, double zc,
                               double sx, double sy, double dmx, double dmy, double nx, double ny,
                               double dt)
{
    const double ql = q * nx + r * ny;
    const double rl = r * nx - q * ny;
    const double hd = smax(kSmallReal, h);
    const double cl = sqrt(kGravity * hd);
    const double ul = ql / hd;
    const double vl = rl / hd;
    const double lmv = lam_minus_dip(b, x, cl, ul);
    const double lpv = lam_plus_dip(b, x, cl, ul);
    double l1 = left ? smax(0.0, lmv) : smin(0.0, lmv);
    double dx1 = dmx - 0.5 * l1 * dt * nx;
    double dy1 = dmy - 0.5 * l1 * dt * ny;
    double z1 = zc + dx1 * sx + dy1 * sy;
    double h1 = smax(0.0, z1 - zb);
    double l2 = left ? smax(0.0, lpv) : smin(0.0, lpv);
    double dx2 = dmx - 0.5 * l2 * dt * nx;
    double dy2 = dmy - 0.5 * l2 * dt * ny;
    double z2 = zc + dx2 * sx + dy2 * sy;
    double h2 = smax(0.0, z2 - zb);
    SideState s;
    double hr = 0.5 * (h1 + h2);
    s.z = hr + zb;
    s.q = hr * ul;
    s.r = hr * vl;
    const double u = s.q / smax(hr, kSmallReal);
    const double c = sqrt(kGravity * hr);
    s.lm = lam_minus_dip(b, x, c, u);
    s.lp = lam_plus_dip(b, x, c, u);
    return s;
}

// The "both sides" flux of swDip::hypHllc / hypHllcBlending (dip/swDipHyp.cpp:799-870, 953-1030)
SW2D_HD void hllc_dip_both(bool blending, double bL, double bR, double phiG, double phiL, double phiR, double zbL,
                           double zbR, const SideState& L, const SideState& R, double hL, double hR, EdgeFlux& f)
{
    const double x1L = phiL / smax(phiG, kSmallReal);
    const double x1R = phiR / smax(phiG, kSmallReal);
    const double uL = L.q / smax(hL, kSmallReal);
    const double uR = R.q / smax(hR, kSmallReal);
    const double L1 = smin(L.lm, smin(R.lm, 0.));
    const double L2 = smax(L.lp, smax(R.lp, 0.));
    const double den = smax(L2 - L1, kSmallReal);
    double s2L_b, s2R_b;
    if (blending) {
        double alpha_h = 0.0;
        if (fabs(zbL - zbR) > kSmallReal) alpha_h = smax(0.0, smin(1.0, (L.z - R.z) / (zbL - zbR)));
        const double F1h = L2 * phiL * L.q - L1 * phiR * R.q + L1 * L2 * phiG * (hR - hL);
        const double F1z = L2 * phiL * L.q - L1 * phiR * R.q + L1 * L2 * phiG * (R.z - L.z);
        f.f1 = alpha_h * F1h + (1.0 - alpha_h) * F1z;
        f.f1 = f.f1 / den;
        double deltah = smax(0., smin(L.z, zbR) - zbL);
        double h1 = smax(L.z - zbR, 0.);
        double s2L_b_z = -kGravity * deltah * 0.5 * (h1 + hL);
        s2L_b_z = phiG * s2L_b_z;
        const double s2L_b_h = phiG * hL * smin(0.0, zbL - zbR);
        s2L_b = alpha_h * s2L_b_h + (1.0 - alpha_h) * s2L_b_z;
        deltah = smax(0., smin(R.z, zbL) - zbR);
        h1 = smax(R.z - zbL, 0.);
        double s2R_b_z = kGravity * deltah * 0.5 * (h1 + hR);
        s2R_b_z = phiG * s2R_b_z;
        const double s2R_b_h = phiG * hR * smax(0.0, zbL - zbR);
        s2R_b = alpha_h * s2R_b_h + (1.0 - alpha_h) * s2R_b_z;
    } else {
        f.f1 = L2 * phiL * L.q - L1 * phiR * R.q + L1 * L2 * phiG * (R.z - L.z);
        f.f1 = f.f1 / den;
        double deltah = smax(0., smin(L.z, zbR) - zbL);
        double h1 = smax(L.z - zbR, 0.);
        s2L_b = -kGravity * deltah * 0.5 * (h1 + hL);
        s2L_b = phiG * s2L_b;
        deltah = smax(0., smin(R.z, zbL) - zbR);
        h1 = smax(R.z - zbL, 0.);
        s2R_b = kGravity * deltah * 0.5 * (h1 + hR);
        s2R_b = phiG * s2R_b;
    }
    const double s2L_phi = .5 * kGravity * hL * hL * (smin(0., phiG - phiL));
    const double s2R_phi = .5 * kGravity * hR * hR * (smax(0., phiR - phiG));
    const double s2 = s2L_b + s2R_b;
    f.sl = -L1 * s2 / den + s2L_phi;
    f.sr = L2 * s2 / den + s2R_phi;
    if (phiG < kSmallReal) f.bad |= kStatusPhiG;
    const double FL = spec_force_dip(bL, phiG, phiL / smax(phiG, kSmallReal), hL, uL);
    const double FR = spec_force_dip(bR, phiG, phiR / smax(phiG, kSmallReal), hR, uR);
    f.f2 = L2 * FL - L1 * FR + L1 * L2 * (phiR * R.q - phiL * L.q);
    f.f2 = f.f2 / den;
    const double vL = x1L * L.r / smax(hL, kSmallReal);
    const double vR = x1R * R.r / smax(hR, kSmallReal);
    f.f3 = (f.f1 >= 0) ? f.f1 * vL : f.f1 * vR;
}

// swDip::hypHllc (dip/swDipHyp.cpp:759-905) and swDip::hypHllcBlending (:908-1083).  Flags
// kStatusHllcConfig where the reference stops (:787-797, :1071-1082).
SW2D_HD EdgeFlux hllc_dip(bool blending, double bL, double bR, double phiG, double phiL, double phiR, double zbL,
                          double zbR, const SideState& L, const SideState& R, double h_min, double phi_min)
{
    const double hL = L.z - zbL;
    const double hR = R.z - zbR;
    EdgeFlux f;
    f.bad = 0;
    f.f1 = f.f2 = f.f3 = f.sl = f.sr = 0.0;
    if (blending) {
        if ((hL > kSmallReal && hR > kSmallReal) || (hL < kSmallReal && R.z >= zbL) ||
            (hR < kSmallReal && L.z >= zbR)) {
            hllc_dip_both(true, bL, bR, phiG, phiL, phiR, zbL, zbR, L, R, hL, hR, f);
        } else if ((hL <= kSmallReal) && (R.z <= zbL + kSmallReal)) {
            f.sr = phiR * 0.5 * kGravity * hR * hR;
        } else if ((hR <= kSmallReal) && (L.z <= zbR + kSmallReal)) {
            f.sl = -phiL * 0.5 * kGravity * hL * hL;
        } else {
            f.bad = kStatusHllcConfig;
        }
        return f;
    }
    bool both = false, lhs = false, rhs = false, none = false;
    if (((hL <= h_min) && (hR <= h_min)) || ((phiL <= phi_min) && (phiR <= phi_min))) {
        none = true;
    } else {
        both = true;
        if ((phiR <= phi_min) || ((phiR > phi_min) && (hR <= h_min) && (L.z <= zbR + h_min))) {
            lhs = true;
            both = false;
        }
        if ((phiL <= phi_min) || ((phiL > phi_min) && (hL <= h_min) && (R.z <= zbL + h_min))) {
            rhs = true;
            both = false;
        }
    }
    if ((int)both + (int)lhs + (int)rhs + (int)none != 1) {
        f.bad = kStatusHllcConfig;
        return f;
    }
    if (both) {
        hllc_dip_both(false, bL, bR, phiG, phiL, phiR, zbL, zbR, L, R, hL, hR, f);
    } else if (rhs) {
        f.sr = phiR * 0.5 * kGravity * hR * hR;
    } else if (lhs) {
        f.sl = -phiL * 0.5 * kGravity * hL * hL;
    }
    return f;
}

// swDip::hypHCriticalPhiq / hypHCriticalPhiWq (dip/swDipHyp.cpp:717-757)
SW2D_HD double h_critical_phiq(double q, double phiG, double phiW)
{
    double h = q * phiW / smax(phiG, kSmallReal);
    h = h * h / kGravity;
    return sw2d_exp((1. / 3.) * sw2d_log(h));
}
SW2D_HD double h_critical_phiwq(double phiwq, double phiG)
{
    double h = phiwq / smax(phiG, kSmallReal);
    h = h * h / kGravity;
    return sw2d_exp((1. / 3.) * sw2d_log(h));
}

// swDip::hypBoundaryFlux (dip/swDipHyp.cpp:13-155): types 0 'q' (phi q), 1 'h', 2 'z', 3 'fr',
// 4 'phiWq'; the boundary geometric source stays 0.
SW2D_HD unsigned boundary_flux_dip(double bR, double phiG, double phiR, double zbR, const SideState& S, int type,
                                   double bcv, double h_min, double* f1o, double* f2o, double* f3o)
{
    unsigned bad = 0;
    double hR = S.z - zbR;
    double q1 = S.q, r1 = S.r;
    if (hR < h_min) {
        q1 = 0.;
        r1 = 0.;
        hR = 0.;
    }
    const double cR = sqrt(kGravity * smax(hR, kSmallReal));
    const double uR = q1 / smax(hR, kSmallReal);
    const double L1 = smax(0.0, S.lp);
    if (phiG < kSmallReal) bad |= kStatusPhiG;
    const double flux2R = spec_force_dip(bR, phiG, phiR / smax(phiG, kSmallReal), hR, uR);
    double flux1 = 0.0, flux2 = 0.0;
    if (type == 3) {  // fr
        double c = (uR - 2. * cR) / (-bcv - 2.);
        c = smax(c, 0.);
        const double u = -bcv * c;
        const double h = c * c / kGravity;
        flux1 = phiR * u * h;
        flux2 = flux2R + (flux1 - q1 * phiR) * L1;
    } else if (type == 1 || type == 2) {  // h, z
        const double h = (type == 1) ? smax(bcv, 0.) : smax(bcv - zbR, 0.);
        flux1 = phiR * (q1 + L1 * (h - hR));
        flux2 = flux2R + (flux1 - q1 * phiR) * L1;
    } else if (type == 4) {  // phiWq
        const double hc = h_critical_phiwq(bcv, phiG);
        flux1 = (hc >= hR) ? phiG * 1.5 * sqrt(kGravity * hc) * hc : bcv;
        flux2 = flux2R + (flux1 - phiR * q1) * L1;
    } else if (type == 0) {  // q
        const double hc = h_critical_phiq(bcv, phiG, phiR);
        flux1 = (hc >= hR) ? phiG * 1.5 * sqrt(kGravity * hc) * hc : phiR * bcv;
        flux2 = flux2R + (flux1 - phiR * q1) * L1;
    } else {
        bad |= kStatusBcType;
    }
    double flux3;
    if (flux1 > 0) {
        flux3 = 0;
    } else {
        const double vR = r1 / smax(hR, kSmallReal);
        flux3 = flux1 * vR;
    }
    flux2 += smax(phiR - phiG, 0.) * 0.5 * kGravity * hR * hR;  // reaction of the solid boundary
    *f1o = flux1;
    *f2o = flux2;
    *f3o = flux3;
    return bad;
}

// Momentum dissipation of swDip::hypComputeBalance (dip/swDipHyp.cpp:295-324): where the depth
// increased during the balance, the discharge increment is reduced by R(a) diag(mu1, mu2) R(a)^T.
// mu = {mu1, mu2, cos a, sin a}; (h0, q0, r0) is the state before the balance.
SW2D_HD void momentum_dissipation(double mu1, double mu2, double ca, double sa, double h0, double q0, double r0,
                                  double h, double& q, double& r)
{
    if (h > h0 + kSmallReal) {
        const double delta_q = q - q0;
        const double delta_r = r - r0;
        const double local_delta_q = ca * delta_q + sa * delta_r;
        const double local_delta_r = -sa * delta_q + ca * delta_r;
        const double local_delta_q_reduction = mu1 * local_delta_q;
        const double local_delta_r_reduction = mu2 * local_delta_r;
        const double delta_q_reduction = ca * local_delta_q_reduction - sa * local_delta_r_reduction;
        const double delta_r_reduction = sa * local_delta_q_reduction + ca * local_delta_r_reduction;
        q -= delta_q_reduction;
        r -= delta_r_reduction;
    }
}

}  // namespace sw2d
