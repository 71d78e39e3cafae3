// spe_math.cuh — arithmetic of the reference's differentiated step (the "_E" step of its
// assimilation layer, assim/swSpE_*.cpp), forward and reverse.
//
// The forward functions restate the reference with the same operand order, so that with
// -fmad=false (device) or -ffp-contract=off (host) they give the reference's bits (exp, log and
// cbrt are the portable versions of portable_math.h).  Each reverse function takes the inputs
// of its forward function and the adjoints of its outputs, recomputes what it needs, and ADDS
// the adjoints of the inputs.  Branches are differentiated as taken (the derivative of
// (a < b ? a : b) follows the selected operand; a flush to 0 or a clamp has derivative 0);
// a square root whose argument is 0 passes no derivative.
//
// Differences of the _E step from the native one (sp_math.cuh), all from the reference:
//   - MUSCL-EVR velocities through desingVelocity (assim/swSpDesingVelocity.h:27-34);
//   - Godunov velocity q/h only where h > h_min (assim/swSpE_hyp.cpp:507-576);
//   - HLLC with a smooth min of the porosities, phi_LR = (phiL + phiR - sqrt(dphi^2 + 1e-6))/2,
//     and no error on an impossible configuration (swSpE_hyp.cpp:725-832);
//   - every internal edge computes its flux each step (no stale flux; swSpE_hyp.cpp:453-480);
//   - boundary fluxes with guarded divisions, a clamped 'fr' and zero flux for unknown types
//     (swSpE_hyp.cpp:143-240);
//   - the balance adds factor * (F1 * dt) on internal edges (swSpE_hyp.cpp:360-366);
//   - semi-implicit Strickler friction (swSpE_friction.cpp:19-76), guarded head loss
//     (swSpE_friction.cpp:79-126), no velocity correction.
#pragma once

#include "sp_math.cuh"

namespace sw2d {
namespace spe {

constexpr double kHDesing = 5e-3;        // assim/swSpDesingVelocity.h:39
constexpr double kPhiSmoothEps = 1e-3;   // assim/swSpE_hyp.cpp:789
constexpr double kFricG = 9.81;          // assim/swSpE_friction.cpp:23
constexpr double kFricEps = 1e-10;       // assim/swSpE_friction.cpp:24
constexpr double kFricDefaultK = 20.0;   // assim/swSpE_friction.cpp:49-50
constexpr double kDtFloor = 1e-6;        // assim/swSpE_hyp.cpp:634

// Adjoint of sqrt(x) given the adjoint sb of its value s = sqrt(x).  At x == 0: 0 (subgradient
// 0), or with `ieee` the literal sb / (2 sqrt(0)), non-finite unless sb == 0 (what a
// source-transformation AD tool produces; the reference's gradient then zeroes non-finite entries).
SW2D_HD double dsqrt(double s, double sb, bool ieee = false)
{
    if (s > 0.0) return sb * 0.5 / s;
    return (ieee && sb != 0.0) ? sb * 0.5 / s : 0.0;
}

// ---- desingVelocity (assim/swSpDesingVelocity.h:27-34) --------------------------------------
SW2D_HD double desing(double q, double h)
{
    const double h2 = h * h;
    const double h4 = h2 * h2;
    const double e4 = kHDesing * kHDesing * kHDesing * kHDesing;
    const double den = sqrt(h4 + smax(h4, e4));
    return 1.4142135623730951 * h * q / den;
}

SW2D_HD void desing_rev(double q, double h, double yb, double& qb, double& hb)
{
    if (yb == 0.0) return;
    const double h2 = h * h;
    const double h4 = h2 * h2;
    const double e4 = kHDesing * kHDesing * kHDesing * kHDesing;
    const double den = sqrt(h4 + smax(h4, e4));
    const double s = 1.4142135623730951;
    const double num = s * h * q;
    qb += yb * (s * h) / den;
    const double dh4 = 4.0 * h2 * h;
    const double dS = dh4 + ((h4 < e4) ? 0.0 : dh4);  // d(h4 + max(h4, e4))/dh
    const double denb = -yb * num / (den * den);
    hb += yb * (s * q) / den + denb * dS * 0.5 / den;
}

// ---- wave speeds lambda-/+ = b u -/+ sqrt((b-1) b u^2 + c^2) (swSp.cpp:972-995) -----------
// adds the adjoints of u and c given those of lambda- and lambda+
SW2D_HD void lam_rev(double b, double c, double u, double lmb, double lpb, double& ub, double& cb, bool ieee = false)
{
    const double R = sqrt((b - 1.0) * b * u * u + c * c);
    ub += b * (lmb + lpb);
    const double Rb = lpb - lmb;
    if (R > 0.0) {
        ub += Rb * (b - 1.0) * b * u / R;
        cb += Rb * c / R;
    } else if (ieee && Rb != 0.0) {
        const double xb = Rb * 0.5 / R;  // adjoint of the radicand: +-inf
        ub += xb * (2.0 * (b - 1.0) * b * u);
        cb += xb * (2.0 * c);
    }
}

struct ESide {
    double z, q, r, lm, lp;
};
struct ESideBar {
    double z, q, r, lm, lp;
};

// ---- Godunov side (assim/swSpE_hyp.cpp:507-576) --------------------------------------------
SW2D_HD ESide god_side(double h, double q, double r, double zb, double b, double nx, double ny, double h_min)
{
    ESide s;
    s.z = h + zb;
    s.q = q * nx + r * ny;
    s.r = -q * ny + r * nx;
    const double u = (h > h_min) ? s.q / h : 0.0;
    const double c = sqrt(kGravity * h);
    s.lm = lam_minus(b, c, u);
    s.lp = lam_plus(b, c, u);
    return s;
}

// adds the adjoints of the cell's (h, q, r)
SW2D_HD void god_side_rev(double h, double q, double r, double b, double nx, double ny, double h_min,
                          const ESideBar& sb, double& hb, double& qb, double& rb, bool ieee = false)
{
    const double qn = q * nx + r * ny;
    const double u = (h > h_min) ? qn / h : 0.0;
    const double c = sqrt(kGravity * h);
    double ub = 0.0, cb = 0.0;
    lam_rev(b, c, u, sb.lm, sb.lp, ub, cb, ieee);
    hb += sb.z;
    hb += dsqrt(c, cb, ieee) * kGravity;
    double qnb = sb.q;
    if (h > h_min) {
        qnb += ub / h;
        hb -= ub * u / h;
    }
    qb += qnb * nx - sb.r * ny;
    rb += qnb * ny + sb.r * nx;
}

// ---- MUSCL-EVR boundary side (assim/swSpE_muscl.cpp:47-63) ---------------------------------
SW2D_HD ESide evr_bnd_side(double h, double q, double r, double zb, double b, double nx, double ny)
{
    ESide s;
    s.z = h + zb;
    s.q = q * nx + r * ny;
    s.r = -q * ny + r * nx;
    const double u = desing(s.q, h);
    const double c = sqrt(kGravity * h);
    s.lm = lam_minus(b, c, u);
    s.lp = lam_plus(b, c, u);
    return s;
}

SW2D_HD void evr_bnd_side_rev(double h, double q, double r, double b, double nx, double ny, const ESideBar& sb,
                              double& hb, double& qb, double& rb, bool ieee = false)
{
    const double qn = q * nx + r * ny;
    const double u = desing(qn, h);
    const double c = sqrt(kGravity * h);
    double ub = 0.0, cb = 0.0;
    lam_rev(b, c, u, sb.lm, sb.lp, ub, cb, ieee);
    hb += sb.z;
    hb += dsqrt(c, cb, ieee) * kGravity;
    double qnb = sb.q;
    desing_rev(qn, h, ub, qnb, hb);
    qb += qnb * nx - sb.r * ny;
    rb += qnb * ny + sb.r * nx;
}

// ---- MUSCL-EVR internal side (assim/swSpE_muscl.cpp:66-164) ---------------------------------
// zc = h + zb of the cell, (sx, sy) its limited free-surface slope, (dmx, dmy) = edge midpoint -
// cell centroid, dt the time step the reconstruction uses.
SW2D_HD ESide evr_side(bool left, double h, double q, double r, double zb, double b, double zc, double sx, double sy,
                       double dmx, double dmy, double nx, double ny, double dt)
{
    const double ql = q * nx + r * ny;
    const double rl = r * nx - q * ny;
    const double cl = sqrt(kGravity * smax(kSmallReal, h));
    const double ul = desing(ql, h);
    const double vl = desing(rl, h);
    const double lmv = lam_minus(b, cl, ul);
    const double lpv = lam_plus(b, cl, ul);
    const double l1 = left ? smax(0.0, lmv) : smin(0.0, lmv);
    const double dx1 = dmx - 0.5 * l1 * dt * nx;
    const double dy1 = dmy - 0.5 * l1 * dt * ny;
    const double z1 = zc + dx1 * sx + dy1 * sy;
    const double h1 = smax(0.0, z1 - zb);
    const double l2 = left ? smax(0.0, lpv) : smin(0.0, lpv);
    const double dx2 = dmx - 0.5 * l2 * dt * nx;
    const double dy2 = dmy - 0.5 * l2 * dt * ny;
    const double z2 = zc + dx2 * sx + dy2 * sy;
    const double h2 = smax(0.0, z2 - zb);
    ESide s;
    const double hr = 0.5 * (h1 + h2);
    s.z = 0.5 * (h1 + h2) + zb;
    s.q = 0.5 * (h1 + h2) * ul;
    s.r = 0.5 * (h1 + h2) * vl;
    const double u = desing(s.q, hr);
    const double c = sqrt(kGravity * hr);
    s.lm = lam_minus(b, c, u);
    s.lp = lam_plus(b, c, u);
    return s;
}

// Adds the adjoints of the cell's (h, q, r), of zc and of the slope (sx, sy).
SW2D_HD void evr_side_rev(bool left, double h, double q, double r, double zb, double b, double zc, double sx, double sy,
                          double dmx, double dmy, double nx, double ny, double dt, const ESideBar& sb, double& hb,
                          double& qb, double& rb, double& zcb, double& sxb, double& syb, bool ieee = false)
{
    // forward values
    const double ql = q * nx + r * ny;
    const double rl = r * nx - q * ny;
    const double cl = sqrt(kGravity * smax(kSmallReal, h));
    const double ul = desing(ql, h);
    const double vl = desing(rl, h);
    const double lmv = lam_minus(b, cl, ul);
    const double lpv = lam_plus(b, cl, ul);
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
    const double qr = hr * ul;
    const double u = desing(qr, hr);
    const double c = sqrt(kGravity * hr);
    // Riemann state's wave speeds
    double ub = 0.0, cb = 0.0;
    lam_rev(b, c, u, sb.lm, sb.lp, ub, cb, ieee);
    double hrb = sb.z + dsqrt(c, cb, ieee) * kGravity;
    double qrb = sb.q;
    desing_rev(qr, hr, ub, qrb, hrb);
    hrb += qrb * ul + sb.r * vl;
    double ulb = qrb * hr, vlb = sb.r * hr;
    // hr = (h1 + h2) / 2
    const double z1b = (0.0 < z1 - zb) ? 0.5 * hrb : 0.0;
    const double z2b = (0.0 < z2 - zb) ? 0.5 * hrb : 0.0;
    zcb += z1b + z2b;
    sxb += z1b * dx1 + z2b * dx2;
    syb += z1b * dy1 + z2b * dy2;
    const double l1b = -(z1b * sx * nx + z1b * sy * ny) * 0.5 * dt;
    const double l2b = -(z2b * sx * nx + z2b * sy * ny) * 0.5 * dt;
    double lmvb, lpvb;
    if (left) {
        lmvb = (0.0 < lmv) ? l1b : 0.0;
        lpvb = (0.0 < lpv) ? l2b : 0.0;
    } else {
        lmvb = (lmv < 0.0) ? l1b : 0.0;
        lpvb = (lpv < 0.0) ? l2b : 0.0;
    }
    double clb = 0.0;
    lam_rev(b, cl, ul, lmvb, lpvb, ulb, clb, ieee);
    if (kSmallReal < h) hb += dsqrt(cl, clb) * kGravity;
    double qlb = 0.0, rlb = 0.0;
    desing_rev(ql, h, ulb, qlb, hb);
    desing_rev(rl, h, vlb, rlb, hb);
    qb += qlb * nx - rlb * ny;
    rb += qlb * ny + rlb * nx;
}

// ---- HLLC (assim/swSpE_hyp.cpp:725-832) -----------------------------------------------------
struct EFlux {
    double f1, f2, f3, sl, sr;
};

enum : int { kRegNone = 0, kRegBoth = 1, kRegLhs = 2, kRegRhs = 3 };

SW2D_HD int hllc_regime(double phiL, double phiR, double zbL, double zbR, double zL, double zR, double hL, double hR,
                        double h_min, double phi_min)
{
    bool both = false, lhs = false, rhs = false;
    if (((hL <= h_min) && (hR <= h_min)) || ((phiL <= phi_min) && (phiR <= phi_min))) return kRegNone;
    both = true;
    if ((phiR <= phi_min) || ((phiR > phi_min) && (hR <= h_min) && (zL <= zbR + h_min))) {
        lhs = true;
        both = false;
    }
    if ((phiL <= phi_min) || ((phiL > phi_min) && (hL <= h_min) && (zR <= zbL + h_min))) {
        rhs = true;
        both = false;
    }
    if (both) return kRegBoth;
    if (rhs) return kRegRhs;  // the reference tests rhs before lhs (swSpE_hyp.cpp:812-826)
    if (lhs) return kRegLhs;
    return kRegNone;
}

SW2D_HD EFlux hllc(double bL, double bR, double phiL, double phiR, double zbL, double zbR, const ESide& L,
                   const ESide& R, double h_min, double phi_min)
{
    const double hL = (L.z - zbL > 0.0) ? (L.z - zbL) : 0.0;
    const double hR = (R.z - zbR > 0.0) ? (R.z - zbR) : 0.0;
    const int reg = hllc_regime(phiL, phiR, zbL, zbR, L.z, R.z, hL, hR, h_min, phi_min);
    EFlux f;
    f.f1 = f.f2 = f.f3 = f.sl = f.sr = 0.0;
    if (reg == kRegBoth) {
        const double hLs = (hL > kSmallReal) ? hL : kSmallReal;
        const double hRs = (hR > kSmallReal) ? hR : kSmallReal;
        const double uL = L.q / hLs;
        const double uR = R.q / hRs;
        double L1 = (L.lm < R.lm) ? L.lm : R.lm;
        if (L1 > 0.0) L1 = 0.0;
        double L2 = (L.lp > R.lp) ? L.lp : R.lp;
        if (L2 < 0.0) L2 = 0.0;
        double den = L2 - L1;
        if (den < kSmallReal) den = kSmallReal;
        const double dphi = phiL - phiR;
        const double phiLR = 0.5 * (phiL + phiR - sqrt(dphi * dphi + kPhiSmoothEps * kPhiSmoothEps));
        f.f1 = phiLR * (L2 * L.q - L1 * R.q + L1 * L2 * (R.z - L.z)) / den;
        const double fact = 0.5 * phiLR * (hL + hR);
        double s2 = (phiR * hR * hR - phiL * hL * hL) * 0.5 + fact * (L.z - R.z);
        s2 = s2 * kGravity / den;
        f.sl = -L1 * s2;
        f.sr = L2 * s2;
        const double FL = spec_force(bL, phiL, hL, uL);
        const double FR = spec_force(bR, phiR, hR, uR);
        f.f2 = (L2 * (FL + f.sl) - L1 * (FR - f.sr) + L1 * L2 * (phiR * R.q - phiL * L.q)) / den;
        const double vL = L.r / hLs;
        const double vR = R.r / hRs;
        f.f3 = (f.f1 >= 0.0) ? (bL * f.f1 * vL) : (bR * f.f1 * vR);
    } else if (reg == kRegRhs) {
        f.sr = phiR * 0.5 * kGravity * hR * hR;
    } else if (reg == kRegLhs) {
        f.sl = -phiL * 0.5 * kGravity * hL * hL;
    }
    return f;
}

// Adds the adjoints of phiL, phiR and of both Riemann states given the flux adjoints fb.
SW2D_HD void hllc_rev(double bL, double bR, double phiL, double phiR, double zbL, double zbR, const ESide& L,
                      const ESide& R, double h_min, double phi_min, const EFlux& fb, double& phiLb, double& phiRb,
                      ESideBar& Lb, ESideBar& Rb)
{
    const double dzL = L.z - zbL, dzR = R.z - zbR;
    const double hL = (dzL > 0.0) ? dzL : 0.0;
    const double hR = (dzR > 0.0) ? dzR : 0.0;
    const int reg = hllc_regime(phiL, phiR, zbL, zbR, L.z, R.z, hL, hR, h_min, phi_min);
    double hLb = 0.0, hRb = 0.0;
    if (reg == kRegBoth) {
        const double hLs = (hL > kSmallReal) ? hL : kSmallReal;
        const double hRs = (hR > kSmallReal) ? hR : kSmallReal;
        const double uL = L.q / hLs;
        const double uR = R.q / hRs;
        const bool l1_left = (L.lm < R.lm);
        double L1 = l1_left ? L.lm : R.lm;
        const bool l1_clamped = (L1 > 0.0);
        if (l1_clamped) L1 = 0.0;
        const bool l2_left = (L.lp > R.lp);
        double L2 = l2_left ? L.lp : R.lp;
        const bool l2_clamped = (L2 < 0.0);
        if (l2_clamped) L2 = 0.0;
        double den = L2 - L1;
        const bool den_floor = (den < kSmallReal);
        if (den_floor) den = kSmallReal;
        const double dphi = phiL - phiR;
        const double sq = sqrt(dphi * dphi + kPhiSmoothEps * kPhiSmoothEps);
        const double phiLR = 0.5 * (phiL + phiR - sq);
        const double A = L2 * L.q - L1 * R.q + L1 * L2 * (R.z - L.z);
        const double f1 = phiLR * A / den;
        const double fact = 0.5 * phiLR * (hL + hR);
        const double s2a = (phiR * hR * hR - phiL * hL * hL) * 0.5 + fact * (L.z - R.z);
        const double s2 = s2a * kGravity / den;
        const double sl = -L1 * s2, sr = L2 * s2;
        const double FL = spec_force(bL, phiL, hL, uL);
        const double FR = spec_force(bR, phiR, hR, uR);
        const double B = L2 * (FL + sl) - L1 * (FR - sr) + L1 * L2 * (phiR * R.q - phiL * L.q);
        const double f2 = B / den;
        const double vL = L.r / hLs, vR = R.r / hRs;
        double f1b = fb.f1, slb = fb.sl, srb = fb.sr;
        double hLsb = 0.0, hRsb = 0.0, uLb = 0.0, uRb = 0.0, L1b = 0.0, L2b = 0.0, denb = 0.0, phiLRb = 0.0;
        // f3
        if (f1 >= 0.0) {
            f1b += fb.f3 * bL * vL;
            const double vLb = fb.f3 * bL * f1;
            Lb.r += vLb / hLs;
            hLsb -= vLb * vL / hLs;
        } else {
            f1b += fb.f3 * bR * vR;
            const double vRb = fb.f3 * bR * f1;
            Rb.r += vRb / hRs;
            hRsb -= vRb * vR / hRs;
        }
        // f2 = B / den
        const double Bb = fb.f2 / den;
        denb -= fb.f2 * f2 / den;
        const double P = phiR * R.q - phiL * L.q;
        L2b += Bb * (FL + sl) + Bb * L1 * P;
        const double FLb = Bb * L2;
        slb += Bb * L2;
        L1b += -Bb * (FR - sr) + Bb * L2 * P;
        const double FRb = -Bb * L1;
        srb += Bb * L1;
        phiRb += Bb * L1 * L2 * R.q;
        Rb.q += Bb * L1 * L2 * phiR;
        phiLb -= Bb * L1 * L2 * L.q;
        Lb.q -= Bb * L1 * L2 * phiL;
        // specific forces phi (b h u^2 + g h^2 / 2)
        phiLb += FLb * (bL * hL * uL * uL + 0.5 * kGravity * hL * hL);
        hLb += FLb * phiL * (bL * uL * uL + kGravity * hL);
        uLb += FLb * phiL * 2.0 * bL * hL * uL;
        phiRb += FRb * (bR * hR * uR * uR + 0.5 * kGravity * hR * hR);
        hRb += FRb * phiR * (bR * uR * uR + kGravity * hR);
        uRb += FRb * phiR * 2.0 * bR * hR * uR;
        // sources sl = -L1 s2, sr = L2 s2
        double s2b = -slb * L1 + srb * L2;
        L1b -= slb * s2;
        L2b += srb * s2;
        // s2 = s2a g / den
        const double s2ab = s2b * kGravity / den;
        denb -= s2b * s2 / den;
        phiRb += s2ab * 0.5 * hR * hR;
        hRb += s2ab * phiR * hR;
        phiLb -= s2ab * 0.5 * hL * hL;
        hLb -= s2ab * phiL * hL;
        const double factb = s2ab * (L.z - R.z);
        Lb.z += s2ab * fact;
        Rb.z -= s2ab * fact;
        phiLRb += factb * 0.5 * (hL + hR);
        hLb += factb * 0.5 * phiLR;
        hRb += factb * 0.5 * phiLR;
        // f1 = phiLR A / den
        phiLRb += f1b * A / den;
        const double Ab = f1b * phiLR / den;
        denb -= f1b * f1 / den;
        L2b += Ab * (L.q + L1 * (R.z - L.z));
        Lb.q += Ab * L2;
        L1b += Ab * (-R.q + L2 * (R.z - L.z));
        Rb.q -= Ab * L1;
        Rb.z += Ab * L1 * L2;
        Lb.z -= Ab * L1 * L2;
        // smooth min of the porosities
        phiLb += phiLRb * 0.5 * (1.0 - dphi / sq);
        phiRb += phiLRb * 0.5 * (1.0 + dphi / sq);
        // den = max(L2 - L1, small)
        if (!den_floor) {
            L2b += denb;
            L1b -= denb;
        }
        if (!l1_clamped) {
            if (l1_left) Lb.lm += L1b;
            else Rb.lm += L1b;
        }
        if (!l2_clamped) {
            if (l2_left) Lb.lp += L2b;
            else Rb.lp += L2b;
        }
        // velocities u = q / max(h, small)
        Lb.q += uLb / hLs;
        hLsb -= uLb * uL / hLs;
        Rb.q += uRb / hRs;
        hRsb -= uRb * uR / hRs;
        if (hL > kSmallReal) hLb += hLsb;
        if (hR > kSmallReal) hRb += hRsb;
    } else if (reg == kRegRhs) {
        phiRb += fb.sr * 0.5 * kGravity * hR * hR;
        hRb += fb.sr * phiR * kGravity * hR;
    } else if (reg == kRegLhs) {
        phiLb -= fb.sl * 0.5 * kGravity * hL * hL;
        hLb -= fb.sl * phiL * kGravity * hL;
    }
    if (dzL > 0.0) Lb.z += hLb;
    if (dzR > 0.0) Rb.z += hRb;
}

// ---- boundary flux (assim/swSpE_hyp.cpp:143-240); type 0 q, 1 h, 2 z, 3 fr, other: no flux -
struct EBndFlux {
    double f1, f2, f3;
};

SW2D_HD EBndFlux boundary_flux(double bR, double phiR, double zbR, const ESide& S, int type, double bcv, double h_min,
                               double phi_min)
{
    const double hR = S.z - zbR;
    const bool dry = (hR < h_min);
    const double q1 = dry ? 0.0 : S.q;
    const double r1 = dry ? 0.0 : S.r;
    const double hRe = dry ? 0.0 : hR;
    const double hden = (hRe > kSmallReal) ? hRe : kSmallReal;
    const double cR = sqrt(kGravity * hden);
    const double uR = q1 / hden;
    const double L1 = (S.lp > 0.0) ? S.lp : 0.0;
    const double flux2R = spec_force(bR, phiR, hRe, uR);
    EBndFlux f;
    f.f1 = 0.0;
    f.f2 = flux2R;
    if (type == 0) {
        f.f1 = bcv;
        if (bcv > kSmallReal) {
            const double phi_safe = (phiR > phi_min) ? phiR : phi_min;
            const double hc = sw2d_exp((1.0 / 3.0) * sw2d_log((bcv / phi_safe) / kGravity));
            if (hc >= hRe) {
                const double hcs = (hc > kSmallReal) ? hc : kSmallReal;
                f.f1 = phiR * 1.5 * sqrt(kGravity * hcs) * hc;
            }
        }
        f.f2 = flux2R + (f.f1 - q1 * phiR) * L1;
    } else if (type == 3) {
        const double fr = (bcv < 0.0) ? 0.0 : ((bcv > 1.0) ? 1.0 : bcv);
        double c = (uR - 2.0 * cR) / (-fr - 2.0);
        c = (c > 0.0) ? c : 0.0;
        const double u = -fr * c;
        const double h = c * c / kGravity;
        f.f1 = phiR * u * h;
        f.f2 = flux2R + (f.f1 - q1 * phiR) * L1;
    } else if (type == 1 || type == 2) {
        const double h_bc = (type == 2) ? smax(bcv - zbR, 0.0) : smax(bcv, 0.0);
        if (hRe > h_min) {
            f.f1 = phiR * (q1 + L1 * (h_bc - hRe));
            f.f2 = flux2R + (f.f1 - q1 * phiR) * L1;
        } else {
            const double c = sqrt(kGravity * ((h_bc > kSmallReal) ? h_bc : kSmallReal));
            f.f1 = phiR * h_bc * c;
            f.f2 = spec_force(bR, phiR, h_bc, c);
        }
    }
    if (f.f1 > 0.0) {
        f.f3 = 0.0;
    } else {
        const double vR = r1 / ((hRe > kSmallReal) ? hRe : kSmallReal);
        f.f3 = f.f1 * vR;
    }
    return f;
}

// Adds the adjoints of phiR and of the boundary Riemann state given (f1b, f2b, f3b).
SW2D_HD void boundary_flux_rev(double bR, double phiR, double zbR, const ESide& S, int type, double bcv, double h_min,
                               double phi_min, double f1b, double f2b, double f3b, double& phiRb, ESideBar& Sb)
{
    const double hR = S.z - zbR;
    const bool dry = (hR < h_min);
    const double q1 = dry ? 0.0 : S.q;
    const double r1 = dry ? 0.0 : S.r;
    const double hRe = dry ? 0.0 : hR;
    const double hden = (hRe > kSmallReal) ? hRe : kSmallReal;
    const double cR = sqrt(kGravity * hden);
    const double uR = q1 / hden;
    const double L1 = (S.lp > 0.0) ? S.lp : 0.0;
    const EBndFlux f = boundary_flux(bR, phiR, zbR, S, type, bcv, h_min, phi_min);
    double q1b = 0.0, r1b = 0.0, hReb = 0.0, hdenb = 0.0, uRb = 0.0, cRb = 0.0, L1b = 0.0, F2Rb = 0.0;
    // f3
    if (!(f.f1 > 0.0)) {
        f1b += f3b * (r1 / hden);
        r1b += f3b * f.f1 / hden;
        hdenb -= f3b * f.f1 * r1 / (hden * hden);
    }
    bool f2_from_F2R = true;
    if (type == 0 || type == 3 || ((type == 1 || type == 2) && hRe > h_min)) {
        // f2 = flux2R + (f1 - q1 phiR) L1
        F2Rb += f2b;
        f1b += f2b * L1;
        q1b -= f2b * L1 * phiR;
        phiRb -= f2b * L1 * q1;
        L1b += f2b * (f.f1 - q1 * phiR);
    } else if (type == 1 || type == 2) {
        f2_from_F2R = false;
    } else {
        F2Rb += f2b;
    }
    if (type == 0) {
        if (bcv > kSmallReal) {
            const double phi_safe = (phiR > phi_min) ? phiR : phi_min;
            const double hc = sw2d_exp((1.0 / 3.0) * sw2d_log((bcv / phi_safe) / kGravity));
            if (hc >= hRe) {
                const double hcs = (hc > kSmallReal) ? hc : kSmallReal;
                const double sc = sqrt(kGravity * hcs);
                phiRb += f1b * 1.5 * sc * hc;
                double hcb = f1b * phiR * 1.5 * sc;
                if (hc > kSmallReal) hcb += dsqrt(sc, f1b * phiR * 1.5 * hc) * kGravity;
                // hc = (bcv / phi_safe / g)^(1/3): d hc / d phi_safe = -hc / (3 phi_safe)
                if (phiR > phi_min) phiRb -= hcb * hc / (3.0 * phi_safe);
            }
        }
    } else if (type == 3) {
        const double fr = (bcv < 0.0) ? 0.0 : ((bcv > 1.0) ? 1.0 : bcv);
        const double c0 = (uR - 2.0 * cR) / (-fr - 2.0);
        const double c = (c0 > 0.0) ? c0 : 0.0;
        const double u = -fr * c;
        const double h = c * c / kGravity;
        phiRb += f1b * u * h;
        const double ub = f1b * phiR * h;
        const double hb = f1b * phiR * u;
        double cb = hb * 2.0 * c / kGravity - fr * ub;
        if (c0 > 0.0) {
            uRb += cb / (-fr - 2.0);
            cRb -= 2.0 * cb / (-fr - 2.0);
        }
    } else if (type == 1 || type == 2) {
        const double h_bc = (type == 2) ? smax(bcv - zbR, 0.0) : smax(bcv, 0.0);
        if (hRe > h_min) {
            phiRb += f1b * (q1 + L1 * (h_bc - hRe));
            q1b += f1b * phiR;
            L1b += f1b * phiR * (h_bc - hRe);
            hReb -= f1b * phiR * L1;
        } else {
            const double c = sqrt(kGravity * ((h_bc > kSmallReal) ? h_bc : kSmallReal));
            phiRb += f1b * h_bc * c;
            phiRb += f2b * (bR * h_bc * c * c + 0.5 * kGravity * h_bc * h_bc);
        }
    }
    if (f2_from_F2R) {
        phiRb += F2Rb * (bR * hRe * uR * uR + 0.5 * kGravity * hRe * hRe);
        hReb += F2Rb * phiR * (bR * uR * uR + kGravity * hRe);
        uRb += F2Rb * phiR * 2.0 * bR * hRe * uR;
    }
    if (S.lp > 0.0) Sb.lp += L1b;
    q1b += uRb / hden;
    hdenb -= uRb * uR / hden;
    hdenb += dsqrt(cR, cRb) * kGravity;
    if (hRe > kSmallReal) hReb += hdenb;
    if (!dry) {
        Sb.q += q1b;
        Sb.r += r1b;
        Sb.z += hReb;
    }
}

// ---- per-cell update after the balance (assim/swSpE_checkpoint.cpp:675-702) -----------------
// flush |x| < 1e-16 -> 0 (swSpE_hyp.cpp:384-391), h < 0 -> (0, 0, 0), friction, head loss.
struct ECellParams {
    int friction;     // apply sourceFrictionStrickler_E
    int head_loss;    // apply sourceSingularHeadLoss_E
    double k1, k2, ca, sa;           // friction coefficients and axes
    double hs, hk1, hk2, hca, hsa;   // head-loss threshold, coefficients and axes
    double h_min;
};

SW2D_HD double h_threshold(double h_min) { return (h_min > kSmallReal) ? h_min : kSmallReal; }

// sourceFrictionStrickler_E on one cell (swSpE_friction.cpp:19-76)
SW2D_HD void strickler_e(double h, double& q, double& r, double k1, double k2, double ca, double sa, double dt,
                         double h_min)
{
    if (h > h_threshold(h_min)) {
        const double hs = h + kSmallReal;
        const double u = q / hs;
        const double v = r / hs;
        double ul = u * ca + v * sa;
        double vl = -u * sa + v * ca;
        const double un = sqrt(u * u + v * v + 1e-16);
        const double K1 = (k1 > kFricEps) ? k1 : kFricDefaultK;
        const double K2 = (k2 > kFricEps) ? k2 : kFricDefaultK;
        const double h43 = h * sw2d_cbrt(h + 1e-16);
        const double d1 = 1.0 + (dt * kFricG * un) / (K1 * K1 * h43 + kFricEps);
        const double d2 = 1.0 + (dt * kFricG * un) / (K2 * K2 * h43 + kFricEps);
        ul /= d1;
        vl /= d2;
        q = (ul * ca - vl * sa) * h;
        r = (ul * sa + vl * ca) * h;
    } else {
        q = 0.0;
        r = 0.0;
    }
}

// reverse: (qb, rb) = adjoints of the outputs, replaced by those of the inputs; hb, k1b, k2b added
SW2D_HD void strickler_e_rev(double h, double q, double r, double k1, double k2, double ca, double sa, double dt,
                             double h_min, double& hb, double& qb, double& rb, double& k1b, double& k2b)
{
    if (!(h > h_threshold(h_min))) {
        qb = 0.0;
        rb = 0.0;
        return;
    }
    const double hs = h + kSmallReal;
    const double u = q / hs;
    const double v = r / hs;
    const double ul = u * ca + v * sa;
    const double vl = -u * sa + v * ca;
    const double un = sqrt(u * u + v * v + 1e-16);
    const double K1 = (k1 > kFricEps) ? k1 : kFricDefaultK;
    const double K2 = (k2 > kFricEps) ? k2 : kFricDefaultK;
    const double cb3 = sw2d_cbrt(h + 1e-16);
    const double h43 = h * cb3;
    const double E1 = K1 * K1 * h43 + kFricEps, E2 = K2 * K2 * h43 + kFricEps;
    const double N = dt * kFricG * un;
    const double d1 = 1.0 + N / E1, d2 = 1.0 + N / E2;
    const double ul2 = ul / d1, vl2 = vl / d2;
    const double A = ul2 * ca - vl2 * sa, B = ul2 * sa + vl2 * ca;
    hb += qb * A + rb * B;
    const double Ab = qb * h, Bb = rb * h;
    const double ul2b = Ab * ca + Bb * sa;
    const double vl2b = -Ab * sa + Bb * ca;
    const double ulb = ul2b / d1, vlb = vl2b / d2;
    const double d1b = -ul2b * ul2 / d1, d2b = -vl2b * vl2 / d2;
    const double Nb = d1b / E1 + d2b / E2;
    const double E1b = -d1b * N / (E1 * E1), E2b = -d2b * N / (E2 * E2);
    if (k1 > kFricEps) k1b += E1b * 2.0 * K1 * h43;
    if (k2 > kFricEps) k2b += E2b * 2.0 * K2 * h43;
    const double h43b = E1b * K1 * K1 + E2b * K2 * K2;
    hb += h43b * cb3 + h43b * h * cb3 / (3.0 * (h + 1e-16));
    const double unb = Nb * dt * kFricG;
    double ub = unb * u / un + ulb * ca - vlb * sa;
    double vb = unb * v / un + ulb * sa + vlb * ca;
    qb = ub / hs;
    rb = vb / hs;
    hb -= (ub * u + vb * v) / hs;
}

// sourceSingularHeadLoss_E on one cell (swSpE_friction.cpp:79-126); the axes' cos and sin
// are evaluated on the host
SW2D_HD void head_loss_e(double h, double& q, double& r, double hsg, double k1, double k2, double ca, double sa,
                         double dt, double h_min)
{
    double qx = q * ca + r * sa;
    double qy = -q * sa + r * ca;
    if (h > h_threshold(h_min)) {
        double AAx = 0.0, AAy = 0.0;
        if (h > hsg) {
            const double hs = h + kSmallReal;
            const double qn = sqrt(qx * qx + qy * qy + 1e-16);
            AAx = qn * k1 / hs;
            AAy = qn * k2 / hs;
        }
        qx = qx * sw2d_exp(-AAx * dt);
        qy = qy * sw2d_exp(-AAy * dt);
    } else {
        qx = 0.0;
        qy = 0.0;
    }
    q = qx * ca - qy * sa;
    r = qx * sa + qy * ca;
}

SW2D_HD void head_loss_e_rev(double h, double q, double r, double hsg, double k1, double k2, double ca, double sa,
                             double dt, double h_min, double& hb, double& qb, double& rb)
{
    const double qx = q * ca + r * sa;
    const double qy = -q * sa + r * ca;
    const double qx2b = qb * ca + rb * sa;
    const double qy2b = -qb * sa + rb * ca;
    double qxb = 0.0, qyb = 0.0;
    if (h > h_threshold(h_min)) {
        double AAx = 0.0, AAy = 0.0, qn = 0.0, hs = 0.0;
        if (h > hsg) {
            hs = h + kSmallReal;
            qn = sqrt(qx * qx + qy * qy + 1e-16);
            AAx = qn * k1 / hs;
            AAy = qn * k2 / hs;
        }
        const double ex = sw2d_exp(-AAx * dt), ey = sw2d_exp(-AAy * dt);
        qxb = qx2b * ex;
        qyb = qy2b * ey;
        if (h > hsg) {
            const double AAxb = -qx2b * qx * ex * dt;
            const double AAyb = -qy2b * qy * ey * dt;
            const double qnb = AAxb * k1 / hs + AAyb * k2 / hs;
            hb -= (AAxb * AAx + AAyb * AAy) / hs;
            qxb += qnb * qx / qn;
            qyb += qnb * qy / qn;
        }
    }
    qb = qxb * ca - qyb * sa;
    rb = qxb * sa + qyb * ca;
}

// The update of one cell from its raw post-balance state (h, q, r); returns the final state.
SW2D_HD void cell_update(double& h, double& q, double& r, const ECellParams& p, double dt)
{
    if (fabs(h) < kSmallReal) h = 0.0;
    if (fabs(q) < kSmallReal) q = 0.0;
    if (fabs(r) < kSmallReal) r = 0.0;
    if (h < 0.) {
        h = 0.;
        q = 0.;
        r = 0.;
    }
    if (p.friction) strickler_e(h, q, r, p.k1, p.k2, p.ca, p.sa, dt, p.h_min);
    if (p.head_loss) head_loss_e(h, q, r, p.hs, p.hk1, p.hk2, p.hca, p.hsa, dt, p.h_min);
}

// Reverse of cell_update: (hb, qb, rb) = adjoints of the final state, replaced by those of the
// raw post-balance state; friction-coefficient adjoints added.
SW2D_HD void cell_update_rev(double h, double q, double r, const ECellParams& p, double dt, double& hb, double& qb,
                             double& rb, double& k1b, double& k2b)
{
    const bool fh = fabs(h) < kSmallReal, fq = fabs(q) < kSmallReal, fr = fabs(r) < kSmallReal;
    double h1 = fh ? 0.0 : h, q1 = fq ? 0.0 : q, r1 = fr ? 0.0 : r;
    const bool clamp = h1 < 0.;
    if (clamp) {
        h1 = 0.;
        q1 = 0.;
        r1 = 0.;
    }
    double q2 = q1, r2 = r1;
    if (p.friction) strickler_e(h1, q2, r2, p.k1, p.k2, p.ca, p.sa, dt, p.h_min);
    if (p.head_loss) head_loss_e_rev(h1, q2, r2, p.hs, p.hk1, p.hk2, p.hca, p.hsa, dt, p.h_min, hb, qb, rb);
    if (p.friction) strickler_e_rev(h1, q1, r1, p.k1, p.k2, p.ca, p.sa, dt, p.h_min, hb, qb, rb, k1b, k2b);
    if (clamp) {
        hb = 0.0;
        qb = 0.0;
        rb = 0.0;
    }
    if (fh) hb = 0.0;
    if (fq) qb = 0.0;
    if (fr) rb = 0.0;
}

// ---- boundary values: interpolateTimeSeries_E (assim/swSpE.h:138-155) ------------------------
SW2D_HD double bc_value_e(const double* tv, const double* vv, int64_t n, double t)
{
    if (n == 0) return 0.0;
    if (n == 1 || t <= tv[0] - 1.0e-12) return vv[0];
    if (t >= tv[n - 1]) return vv[n - 1];
    int64_t it = 0;
    while (it < n - 1 && t > tv[it + 1]) it++;
    const double t1 = tv[it], t2 = tv[it + 1];
    const double v1 = vv[it], v2 = vv[it + 1];
    const double den = t2 - t1;
    if (den < 1e-12) return v1;
    return v1 + (v2 - v1) * (t - t1) / den;
}

// ---- porosity control transform (assim/swSpE.h:59-107) --------------------------------------
enum : int { kPhiNone = 0, kPhiClamp = 1, kPhiTanh = 2, kPhiNormalize = 3 };

SW2D_HD double phi_correct(int kind, double m, double lambda, double lo, double scale)
{
    switch (kind) {
        case kPhiClamp: return (m < 0.0) ? 0.0 : ((m > 1.05) ? 1.05 : m);
        case kPhiTanh: return 1.0 / (1.0 + sw2d_exp(-lambda * m));
        case kPhiNormalize: return (m - lo) * scale;
        default: return m;
    }
}

SW2D_HD double dphi_dm(int kind, double m, double lambda, double scale)
{
    switch (kind) {
        case kPhiClamp: return (m < 0.0 || m > 1.05) ? 0.0 : 1.0;
        case kPhiTanh: {
            const double s = 1.0 / (1.0 + sw2d_exp(-lambda * m));
            return lambda * s * (1.0 - s);
        }
        case kPhiNormalize: return scale;
        default: return 1.0;
    }
}

}  // namespace spe
}  // namespace sw2d
