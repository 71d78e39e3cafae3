// sp_math.cuh — device arithmetic of SW2D's native single-porosity (SP) step.
//
// Every function restates one routine of the reference (paths relative to the reference
// project) with the same operand order.  The library is compiled with -fmad=false so that no
// multiply-add is contracted: +, -, *, / and sqrt are then IEEE binary64 round-to-nearest on
// both sides and the results match the reference bit for bit.  exp and log are the portable
// versions of portable_math.h, which give the same bits on the host.
//
// std::max(a,b) is (a < b ? b : a) and std::min(a,b) is (b < a ? b : a); smax/smin keep that
// literal form, including what happens with NaN.
#pragma once

#include <cmath>
#include <cstdint>

#include "portable_math.h"

// The same functions compile for the device (the product) and for the host (the adjoint's
// finite-difference tests build them with g++ -ffp-contract=off).
#if defined(__CUDACC__)
#define SW2D_HD __host__ __device__ __forceinline__
#else
#define SW2D_HD inline
#endif

namespace sw2d {

using std::fabs;
using std::sqrt;

constexpr double kSmallReal = 1e-16;  // src/common/param.h:2
constexpr double kGravity = 9.81;     // src/common/param.h:3

// status bits (host maps them to SW2D_E_* codes)
constexpr unsigned kStatusNanFlux = 1u;
constexpr unsigned kStatusHllcConfig = 2u;
constexpr unsigned kStatusNegDepth = 4u;
constexpr unsigned kStatusBcType = 8u;
constexpr unsigned kStatusBcFr = 16u;
constexpr unsigned kStatusUnsupported = 32u;  // a case the reverse kernels do not handle

SW2D_HD double smax(double a, double b) { return (a < b) ? b : a; }
SW2D_HD double smin(double a, double b) { return (b < a) ? b : a; }

// swSp::lambdaMinus / lambdaPlus (src/sw2dSolver/models/sp/swSp.cpp:972-995)
SW2D_HD double lam_minus(double b, double c, double u) { return b * u - sqrt((b - 1.0) * b * u * u + c * c); }
SW2D_HD double lam_plus(double b, double c, double u) { return b * u + sqrt((b - 1.0) * b * u * u + c * c); }

// swSp::specificForce (swSp.cpp:1388-1399)
SW2D_HD double spec_force(double b, double phi, double h, double u)
{
    return phi * (b * h * u * u + 0.5 * kGravity * h * h);
}

// std::max({a,b,c,d}): the first largest under operator<
SW2D_HD double max4(double a, double b, double c, double d)
{
    double m = a;
    if (m < b) m = b;
    if (m < c) m = c;
    if (m < d) m = d;
    return m;
}

struct SideState {
    double z, q, r, lm, lp;
};

// Exact shortcuts for dry cells.  Each replaces an operation by its IEEE result under a
// condition where that result is known exactly, so the bits never change:
//   sqrt(x) == x                         when x == +-0;
//   x / d   == x                         when x == +-0 and d > 0;
//   sqrt(g * max(1e-16, h)) == kC0       when !(1e-16 < h), kC0 = sqrt(g * 1e-16) (host value);
//   sqrt((b-1) b u u + kC0 kC0) == kR0   when u == +-0 and 1 <= b finite (the first term is
//                                        then +0), kR0 = sqrt(kC0 * kC0).
// The shortcut is taken only when every active lane of the warp qualifies (a warp-uniform
// branch); otherwise all lanes run the full operation, whose result is the same.
struct DryConsts {
    double c0, r0;
};

SW2D_HD bool warp_all(bool p)
{
#if defined(__CUDA_ARCH__)
    return __all_sync(__activemask(), p);
#else
    return p;
#endif
}

SW2D_HD double sqrt_z(double x) { return warp_all(x == 0.0) ? x : sqrt(x); }

SW2D_HD double div_z(double x, double d) { return warp_all(x == 0.0) ? x : x / d; }  // d > 0

// First-order rotated state of a cell on an edge (swSpHypGodunov.cpp:17-35 and 44-76; the
// boundary loop of swSpHypMusclEvr.cpp:142-159 is the same expression).
SW2D_HD SideState godunov_side(double h, double q, double r, double zb, double b, double nx, double ny)
{
    SideState s;
    s.z = h + zb;
    s.q = q * nx + r * ny;
    s.r = -q * ny + r * nx;
    const double d = smax(h, kSmallReal);
    double u, c;
    if (warp_all(h == 0.0 && s.q == 0.0)) {  // d == 1e-16 > 0; sqrt(g * +-0) == g * +-0
        u = s.q;
        c = kGravity * h;
    } else {
        u = s.q / d;
        c = sqrt(kGravity * h);
    }
    const double root = sqrt_z((b - 1.0) * b * u * u + c * c);
    s.lm = b * u - root;
    s.lp = b * u + root;
    return s;
}

// One side of swSp::hypMusclEvrComputeLRStates (swSpHypMusclEvr.cpp:176-272): EVR half-step
// reconstruction at the edge midpoint with the limited free-surface slope (sx, sy) of the
// cell.  `left` selects max(0,.) (L side) or min(0,.) (R side) for the wave speeds; dt is the
// previous step's time step; (dmx, dmy) = edge midpoint - cell centroid, the first difference the
// reference evaluates in `mx - cx - 0.5 * l * dt * nx` (a static of the mesh).
SW2D_HD SideState evr_side(bool left, double h, double q, double r, double zb, double b, double zc,
                                              double sx, double sy, double dmx, double dmy,
                                              double nx, double ny, double dt, const DryConsts& k)
{
    const double ql = q * nx + r * ny;
    const double rl = r * nx - q * ny;
    double cl, ul, vl, root1;
    if (warp_all(!(kSmallReal < h) && ql == 0.0 && rl == 0.0 && b < 1.0e308)) {  // b >= 1 and finite
        cl = k.c0;
        ul = ql;
        vl = rl;
        root1 = k.r0;
    } else {
        const double hd = smax(kSmallReal, h);
        cl = sqrt(kGravity * hd);
        ul = ql / hd;
        vl = rl / hd;
        root1 = sqrt((b - 1.0) * b * ul * ul + cl * cl);
    }
    const double lmv = b * ul - root1;
    const double lpv = b * ul + root1;
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
    const double u = div_z(s.q, smax(hr, kSmallReal));
    const double c = sqrt_z(kGravity * hr);
    const double root = sqrt_z((b - 1.0) * b * u * u + c * c);
    s.lm = b * u - root;
    s.lp = b * u + root;
    return s;
}

struct EdgeFlux {
    double f1, f2, f3, sl, sr;
    unsigned bad;  // kStatusHllcConfig for the configuration the reference rejects
};

// swSp::hypHllc (swSpHyp.cpp:664-821) and swSp::hypHllcBlending (swSpHyp.cpp:824-998).
// Flags kStatusHllcConfig for the configuration the reference rejects (:728-739).
SW2D_HD EdgeFlux hllc(bool blending, double bL, double bR, double phiL, double phiR, double zbL,
                                         double zbR, const SideState& L, const SideState& R, double h_min,
                                         double phi_min)
{
    double hL, hR;
    if (blending) {
        hL = L.z - zbL;
        hR = R.z - zbR;
    } else {
        hL = smax(0.0, L.z - zbL);
        hR = smax(0.0, R.z - zbR);
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
    EdgeFlux f;
    f.bad = 0;
    if ((int)both + (int)lhs + (int)rhs + (int)none != 1) {
        f.bad = kStatusHllcConfig;
        f.f1 = f.f2 = f.f3 = f.sl = f.sr = 0.0;
        return f;
    }
    if (both) {
        double uL, uR;
        if (blending) {
            uL = L.q / smax(hL, kSmallReal);
            uR = R.q / smax(hR, kSmallReal);
        } else {
            uL = L.q / smax(kSmallReal, hL);
            uR = R.q / smax(kSmallReal, hR);
        }
        double L1 = smin(L.lm, smin(R.lm, 0.));
        double L2 = smax(L.lp, smax(R.lp, 0.));
        double den = smax(L2 - L1, kSmallReal);
        double phiLR = smin(phiL, phiR);
        double s2;
        if (blending) {
            double alpha_h = 0.0;
            if (fabs(zbL - zbR) > kSmallReal) alpha_h = smax(0.0, smin(1.0, (L.z - R.z) / (zbL - zbR)));
            double F1h = phiLR * (L2 * L.q - L1 * R.q + L1 * L2 * (hR - hL)) / den;
            double F1z = phiLR * (L2 * L.q - L1 * R.q + L1 * L2 * (R.z - L.z)) / den;
            f.f1 = alpha_h * F1h + (1.0 - alpha_h) * F1z;
            double fact = 0.5 * smin(phiL, phiR) * (hL + hR);
            double s2z = (phiR * hR * hR - phiL * hL * hL) * 0.5 + fact * (L.z - R.z);
            double s2h = (zbL > zbR) ? phiR * hR * (zbL - zbR) : phiL * hL * (zbL - zbR);
            s2 = alpha_h * s2h + (1.0 - alpha_h) * s2z;
        } else {
            f.f1 = phiLR * (L2 * L.q - L1 * R.q + L1 * L2 * (R.z - L.z)) / den;
            double fact = 0.5 * smin(phiL, phiR) * (hL + hR);
            s2 = (phiR * hR * hR - phiL * hL * hL) * 0.5 + fact * (L.z - R.z);
        }
        s2 = s2 * kGravity / den;
        f.sl = -L1 * s2;
        f.sr = L2 * s2;
        double FL = spec_force(bL, phiL, hL, uL);
        double FR = spec_force(bR, phiR, hR, uR);
        f.f2 = (L2 * (FL + f.sl) - L1 * (FR - f.sr) + L1 * L2 * (phiR * R.q - phiL * L.q)) / den;
        double vL = L.r / smax(hL, kSmallReal);
        double vR = R.r / smax(hR, kSmallReal);
        f.f3 = (f.f1 >= 0) ? bL * f.f1 * vL : bR * f.f1 * vR;
    } else if (rhs) {
        f.f1 = 0.;
        f.f2 = 0.;
        f.sl = 0.;
        f.sr = phiR * 0.5 * kGravity * hR * hR;
        f.f3 = 0.;
    } else if (lhs) {
        f.f1 = 0.;
        f.f2 = 0.;
        f.sl = -phiL * 0.5 * kGravity * hL * hL;
        f.sr = 0.;
        f.f3 = 0.;
    } else {
        f.f1 = f.f2 = f.f3 = f.sl = f.sr = 0.;
    }
    return f;
}

// swBoundaryConditionTimeSeries::initialise + computeValBC
// (models/common/swBoundaryConditionTimeSeries.cpp:17-96), walked from the initial cursor.
// Simulation time never decreases, so this equals the reference's incremental cursor.
SW2D_HD double bc_value(const double* tv, const double* vv, int64_t n, double time)
{
    double v_inf = vv[0], t_inf = tv[0], v_sup, t_sup;
    bool at_end = false;
    if (n > 1) {
        v_sup = vv[1];
        t_sup = tv[1];
    } else {
        v_sup = v_inf;
        t_sup = t_inf;
        at_end = true;
    }
    int64_t rank = 1;
    while ((time > t_sup) && !at_end) {
        v_inf = v_sup;
        t_inf = t_sup;
        t_sup = tv[rank];
        v_sup = vv[rank];
        ++rank;
        if (rank == n) at_end = true;
    }
    if (time > t_sup) return v_sup;
    if (time < t_inf) return v_inf;
    double d = (time - t_inf) / (t_sup - t_inf);
    return v_inf + (v_sup - v_inf) * d;
}

// swSp::hypHCritical (swSpHyp.cpp:651-661)
SW2D_HD double h_critical(double phi, double q)
{
    return sw2d_exp((1. / 3.) * sw2d_log((q / smax(phi, kSmallReal)) / kGravity));
}

// swSp::hypBoundaryFlux (swSpHyp.cpp:13-135); the boundary geometric source stays 0.  Returns
// kStatusBcFr / kStatusBcType where the reference stops, else 0.
SW2D_HD unsigned boundary_flux(double bR, double phiR, double zbR, const SideState& S, int type,
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
    double cR = sqrt(kGravity * smax(hR, kSmallReal));
    double uR = q1 / smax(hR, kSmallReal);
    double L1 = smax(0.0, S.lp);
    double flux2R = spec_force(bR, phiR, hR, uR);
    double flux1 = 0.0, flux2 = 0.0;
    if (type == 3) {  // fr
        if ((bcv < 0.) | (bcv > 1.)) bad |= kStatusBcFr;
        double c = (uR - 2. * cR) / (-bcv - 2.);
        c = smax(c, 0.);
        double u = -bcv * c;
        double h = c * c / kGravity;
        flux1 = phiR * u * h;
        flux2 = flux2R + (flux1 - q1 * phiR) * L1;
    } else if (type == 1 || type == 2) {  // h, z
        double h_bc = (type == 1) ? smax(bcv, 0.) : smax(bcv - zbR, 0.);
        if (hR > h_min) {
            flux1 = phiR * (q1 + L1 * (h_bc - hR));
            flux2 = flux2R + (flux1 - q1 * phiR) * L1;
        } else {
            double c = sqrt(kGravity * h_bc);
            flux1 = phiR * h_bc * c;
            flux2 = spec_force(bR, phiR, h_bc, c);
        }
    } else if (type == 0) {  // q
        flux1 = bcv;
        double hc = h_critical(phiR, bcv);
        if (hc >= hR) flux1 = phiR * 1.5 * sqrt(kGravity * hc) * hc;
        flux2 = flux2R + (flux1 - q1 * phiR) * L1;
    } else {
        bad |= kStatusBcType;
    }
    double flux3;
    if (flux1 > 0) {
        flux3 = 0;
    } else {
        double vR = r1 / smax(hR, kSmallReal);
        flux3 = flux1 * vR;
    }
    *f1o = flux1;
    *f2o = flux2;
    *f3o = flux3;
    return bad;
}

// h^(-4/3) of the Manning and Strickler factors, as the reference evaluates it: exp(-4/3 log h)
SW2D_HD double friction_power(double h) { return sw2d_exp(-4.0 / 3.0 * sw2d_log(h)); }

// swSource::frictionChezy1D / frictionManning1D / frictionStrickler1D
// (models/common/swSourceFriction.cpp:7-79); model 1 chezy, 2 manning, 3 strickler.
// friction_factor_p takes P = friction_power(h) (unused by Chezy), which the two directions of a
// cell share: the same operations in the same order as the reference's expression.
SW2D_HD double friction_factor_p(int model, double k, double h, double un, double dt, double P)
{
    double factor = 1.0;
    if (model == 1) {
        if ((h > kSmallReal) && (k > kSmallReal)) factor = sw2d_exp(-kGravity * un / k / k / h * dt);
        else factor = 0.0;
    } else if (model == 2) {
        if (h > kSmallReal) factor = sw2d_exp(-kGravity * un * k * k * P * dt);
        else factor = 0.0;
    } else {
        if ((h > kSmallReal) && (k > kSmallReal)) factor = sw2d_exp(-kGravity * un / k / k * P * dt);
        else factor = 0.0;
    }
    return factor;
}

SW2D_HD double friction_factor(int model, double k, double h, double un, double dt)
{
    const double P = (model != 1 && h > kSmallReal) ? friction_power(h) : 0.0;
    return friction_factor_p(model, k, h, un, dt, P);
}

}  // namespace sw2d
