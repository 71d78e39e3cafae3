// ddp_math.cuh — device arithmetic of SW2D's depth-dependent porosity (DDP) step.
//
// The DDP model (src/sw2dSolver/models/ddp/) carries the stored volume per unit area
// thetaW = integral of phiW(z) dz and its momentum thetaW * u, and describes each cell and each
// internal edge by a porosity table: levels z_k with a porosity phi_k constant on
// [z_k, z_k+1) and the cumulated volume theta_k = sum_(j<k) (z_(j+1) - z_j) phi_j.  Every
// function below restates one routine of swDdp with the same operand order; the library is
// compiled with -fmad=false, so the results are the reference's bit for bit (exp and log are
// the portable versions of portable_math.h).
//
// Table lookups reproduce the reference's linear scans, ties included (phiWOfZ / thetaWOfZ
// advance while z > z_k, the pressure-force integrals while z >= z_(k+1)).  Where the reference
// would index level -1 (a NaN elevation or volume) these return NaN and raise kStatusTable.
#pragma once

#include "sp_math.cuh"

namespace sw2d {

constexpr unsigned kStatusTable = 128u;  // NaN elevation or volume in a porosity-table lookup

namespace ddp {

// one level of a porosity table as it is stored: {z_k, phi_k}.  The cumulated volume
// theta_k = theta_(k-1) + (z_k - z_(k-1)) phi_(k-1), theta_0 = 0, is rebuilt while a lookup walks
// the levels, by the recurrence that builds the reference's thetaW_tab (swDdp.cpp:1921-1929),
// so it has the same bits and the table keeps 16 bytes per level.
struct alignas(16) Lvl {
    double z, phi;
};

// a level with its cumulated volume
struct LvlT {
    double z, phi, theta;
};

struct PhiTheta {
    double phi, theta;
};

SW2D_HD double quiet_nan() { return __builtin_nan(""); }

SW2D_HD Lvl load_level(const Lvl* p)
{
#if defined(__CUDA_ARCH__)
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    return Lvl{a.x, a.y};
#else
    return *p;
#endif
}

// Visits the n levels of a table in order with their cumulated volumes.  Every level is
// visited (no early exit, so the loads do not wait on the comparisons): the reference's scans
// stop at the first failing comparison, which the visitors below reproduce with a flag.
template <class F>
SW2D_HD void for_levels(const Lvl* t, int n, F&& f)
{
    double theta = 0.0;
    Lvl prev{0.0, 0.0};
    for (int k = 0; k < n; k++) {
        const Lvl lv = load_level(t + k);
        if (k > 0) theta += (lv.z - prev.z) * prev.phi;
        f(k, LvlT{lv.z, lv.phi, theta});
        prev = lv;
    }
}

// One pass over a table answering phiWOfZ / thetaWOfZ (equally phiGIntOfZ / thetaGIntOfZ;
// swDdp.cpp:1049-1097, 2678-2736) at the NQ elevations zq and the pressure-force integral
// pressureForceOmegaOfZ / pressureForceGammaOfZ (swDdp.cpp:1214-1273) at the NP elevations zp,
// each with the reference's own scan semantics and summation order:
//   phi, theta at z: 0 at or below z_0; else level l - 1 where l counts the leading levels with
//     z > z_k (the scan stops at the first that fails), theta = theta_(l-1) + (z - z_(l-1)) phi_(l-1);
//   force at z: when z > z_0, sum over the leading levels k >= 1 with z >= z_k of
//     phi_(k-1) (z - (z_(k-1) + z_k) / 2) (z_k - z_(k-1)), then phi_l max(0, z - z_l)^2 / 2 at
//     the last such level l; times g.
template <int NQ, int NP>
SW2D_HD void table_pass(const Lvl* t, int n, const double* zq, PhiTheta* pq, const double* zp, double* pp,
                        unsigned& bad)
{
    const double z0 = load_level(t).z;
    bool run[NQ > 0 ? NQ : 1];
    bool hit[NQ > 0 ? NQ : 1];
    LvlT a[NQ > 0 ? NQ : 1];
    bool prun[NP > 0 ? NP : 1];
    bool started[NP > 0 ? NP : 1];
    double acc[NP > 0 ? NP : 1];
    LvlT cur[NP > 0 ? NP : 1];
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        run[q] = true;
        hit[q] = false;
        a[q] = LvlT{0, 0, 0};
    }
#pragma unroll
    for (int p = 0; p < NP; p++) {
        started[p] = zp[p] > z0;
        prun[p] = started[p];
        acc[p] = 0;
        cur[p] = LvlT{0, 0, 0};
    }
    LvlT prev{0, 0, 0};
    for_levels(t, n, [&](int k, const LvlT& lv) {
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            if (run[q]) {
                if (zq[q] > lv.z) {
                    hit[q] = true;
                    a[q] = lv;
                } else {
                    run[q] = false;
                }
            }
        }
#pragma unroll
        for (int p = 0; p < NP; p++) {
            if (k == 0) {
                cur[p] = lv;
            } else if (prun[p] && zp[p] >= lv.z) {
                const double dz1 = zp[p] - (prev.z + lv.z) / 2.;
                const double dz2 = lv.z - prev.z;
                acc[p] += prev.phi * dz1 * dz2;
                cur[p] = lv;
            } else {
                prun[p] = false;
            }
        }
        prev = lv;
    });
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        if (zq[q] <= z0) {
            pq[q] = PhiTheta{0.0, 0.0};
        } else if (!hit[q]) {
            bad |= kStatusTable;
            pq[q] = PhiTheta{quiet_nan(), quiet_nan()};
        } else {
            double theta = a[q].theta;
            if (zq[q] > a[q].z) theta += (zq[q] - a[q].z) * a[q].phi;
            pq[q] = PhiTheta{a[q].phi, theta};
        }
    }
#pragma unroll
    for (int p = 0; p < NP; p++) {
        double v = 0;
        if (started[p]) {
            v = acc[p];
            const double dz1 = smax(0., zp[p] - cur[p].z);
            v += cur[p].phi * dz1 * dz1 / 2.;
        }
        v *= kGravity;
        pp[p] = v;
    }
}

// phiWOfZ and thetaWOfZ at one elevation
SW2D_HD PhiTheta phi_theta(const Lvl* t, int n, double z, unsigned& bad)
{
    const double zq[1] = {z};
    PhiTheta pq[1];
    const double zp[1] = {0.0};
    double pp[1];
    table_pass<1, 0>(t, n, zq, pq, zp, pp, bad);
    return pq[0];
}

// pressureForceOmegaOfZ / pressureForceGammaOfZ at one elevation
SW2D_HD double pressure_force(const Lvl* t, int n, double z)
{
    unsigned bad = 0;
    const double zq[1] = {0.0};
    PhiTheta pq[1];
    const double zp[1] = {z};
    double pp[1];
    table_pass<0, 1>(t, n, zq, pq, zp, pp, bad);
    return pp[0];
}

// swDdp::zOfThetaW (swDdp.cpp:3368-3388): theta_0 ... scanned while theta > theta_k
SW2D_HD double z_of_theta(const Lvl* t, int n, double theta, unsigned& bad)
{
    bool run = true, hit = false;
    LvlT a{0, 0, 0};
    double z0 = 0;
    for_levels(t, n, [&](int k, const LvlT& lv) {
        if (k == 0) z0 = lv.z;
        if (run) {
            if (theta > lv.theta) {
                hit = true;
                a = lv;
            } else {
                run = false;
            }
        }
    });
    if (theta <= 0) return z0;
    if (!hit) {
        bad |= kStatusTable;
        return quiet_nan();
    }
    double z = a.z;
    z += (theta - a.theta) / a.phi;
    return z;
}

// swDdp::pressureWaveCelerity (swDdp.cpp:1276-1286)
SW2D_HD double celerity(double theta, double phi) { return sqrt(kGravity * theta / smax(phi, kSmallReal)); }

// swDdp::lambdaMinus / lambdaPlus (swDdp.cpp:994-1021)
SW2D_HD double lam_minus(double u, double c, double x_phi, double x_theta, double b)
{
    return b * x_theta * u -
           sqrt(x_theta * x_theta * (b - 1. / smax(x_phi, kSmallReal)) * b * u * u + c * c / smax(x_theta, kSmallReal));
}
SW2D_HD double lam_plus(double u, double c, double x_phi, double x_theta, double b)
{
    return b * x_theta * u +
           sqrt(x_theta * x_theta * (b - 1. / smax(x_phi, kSmallReal)) * b * u * u + c * c / smax(x_theta, kSmallReal));
}

// swDdp::specificForce (swDdp.cpp:2426-2437)
SW2D_HD double spec_force(double theta_velocity, double velocity, double pressure)
{
    return theta_velocity * velocity + pressure;
}

// One side of an internal edge in swDdp::hypGodunovComputeLRStates (swDdpHypGodunov.cpp:59-149):
// the rotated momentum (zeroed on a shallow side that has an interface) and the wave speeds
// lambda-/+ with x_phi = phiW/phiG and x_theta = thetaW/thetaG.  `omega` and `gamma` are the
// cell's and the edge's tables at the side's elevation; `shallow(omega_min, gamma_min)` gives
// them at the reference's shallow-side elevation (cell_z_tab[L][0] + h_min on the left,
// cell_z_tab[R][1] + h_min on the right, as swDdpHypGodunov.cpp:84,130 write them), asked for
// only on a shallow side that has an interface.
struct Side {
    double tu, tv, lm, lp;
};

template <class MinF>
SW2D_HD Side lr_side(double theta, double thu, double thv, double z, double z_tab0, double b, double nx, double ny,
                     PhiTheta omega, PhiTheta gamma, MinF&& shallow, double h_min)
{
    const double h = smax(z - z_tab0, 0.);
    Side s;
    s.tu = thu * nx + thv * ny;
    s.tv = -thu * ny + thv * nx;
    double phi_omega = omega.phi, phi_gamma = gamma.phi;
    double theta_omega = omega.theta, theta_gamma = gamma.theta;
    double x_phi = 1.0, x_theta = 1.0;
    if (theta_gamma * theta_omega > kSmallReal) {
        if (h < h_min) {
            s.tu = 0.;
            s.tv = 0.;
            PhiTheta omega_min, gamma_min;
            shallow(omega_min, gamma_min);  // the tables at the shallow-side level
            phi_omega = omega_min.phi;
            phi_gamma = gamma_min.phi;
            theta_omega = omega_min.theta;
            theta_gamma = gamma_min.theta;
        }
        x_phi = phi_omega / smax(phi_gamma, kSmallReal);
        x_theta = theta_omega / smax(theta_gamma, kSmallReal);
    }
    const double u = s.tu / smax(theta, kSmallReal);
    const double c = celerity(theta, phi_omega);
    s.lp = lam_plus(u, c, x_phi, x_theta, b);
    s.lm = lam_minus(u, c, x_phi, x_theta, b);
    return s;
}

// Fluxes and geometric sources of an internal edge.
struct Flux {
    double f1, f2, f3, sl, sr;
    unsigned bad;
};

// Inputs of swDdp::hypHllc (swDdpHyp.cpp:821-1007) for one internal edge, each table
// quantity evaluated once: the cells' own tables at their elevations (omega_*), the edge's
// table at both elevations (gamma_*), each cell's table at the other side's elevation
// (theta_RL = thetaW(R, zL), theta_LR = thetaW(L, zR)), the pressure forces against the cells
// (force_omega_*) and against the edge (force_gamma_*).
struct HllcIn {
    double bL, bR, zL, uL, vL, zR, uR, vR;
    PhiTheta omega_L, omega_R, gamma_L, gamma_R;
    double theta_RL, theta_LR;
    double force_omega_L, force_omega_R, force_gamma_L, force_gamma_R;
    double theta_gamma_hmin, z_gamma_min;
};

// swDdp::hypHllc (swDdpHyp.cpp:821-1007), branch for branch.  Flags kStatusHllcConfig where
// the reference stops with "Impossible case".
SW2D_HD Flux hllc(const HllcIn& in, double h_min, double chi_phi_max)
{
    Flux f{0.0, 0.0, 0.0, 0.0, 0.0, 0u};
    const double phi_omega_L = in.omega_L.phi, phi_omega_R = in.omega_R.phi;
    const double theta_omega_L = in.omega_L.theta, theta_omega_R = in.omega_R.theta;
    const double uL = in.uL, uR = in.uR;
    const double theta_velocity_omega_L = uL * theta_omega_L;
    const double theta_velocity_omega_R = uR * theta_omega_R;

    const double theta_gamma_L = in.gamma_L.theta;
    const double theta_gamma_R = in.gamma_R.theta;
    const double theta_gamma_hmin = in.theta_gamma_hmin;
    double theta_velocity_gamma_L = theta_velocity_omega_L * smin(theta_gamma_L / theta_gamma_hmin, 1.0);
    double theta_velocity_gamma_R = theta_velocity_omega_R * smin(theta_gamma_R / theta_gamma_hmin, 1.0);
    double velocity_gamma_L = theta_velocity_gamma_L / smax(theta_gamma_L, kSmallReal);
    double velocity_gamma_R = theta_velocity_gamma_R / smax(theta_gamma_R, kSmallReal);

    const double z_gamma_min = in.z_gamma_min;
    if (in.zL - z_gamma_min < h_min) {
        const double umax = sqrt(uL * uL + 2. * kGravity * smax(in.zL - z_gamma_min, kSmallReal));
        velocity_gamma_L = smin(umax, smax(velocity_gamma_L, -umax));
        theta_velocity_gamma_L = velocity_gamma_L * theta_gamma_L;
    }
    if (in.zR - z_gamma_min < h_min) {
        const double umax = sqrt(uR * uR + 2. * kGravity * smax(in.zR - z_gamma_min, kSmallReal));
        velocity_gamma_R = smin(umax, smax(velocity_gamma_R, -umax));
        theta_velocity_gamma_R = velocity_gamma_R * theta_gamma_R;
    }

    // swDdp::computePressureForceOmegaOntoGammaOfZ (swDdp.cpp:492-524)
    const double Fp_L = in.force_gamma_L;
    const double Fb_L = smax(0., in.force_omega_L - Fp_L);
    const double Fp_R = in.force_gamma_R;
    const double Fb_R = smax(0., in.force_omega_R - Fp_R);

    const double M_L = spec_force(theta_velocity_gamma_L, velocity_gamma_L, Fp_L);
    const double M_R = spec_force(theta_velocity_gamma_R, velocity_gamma_R, Fp_R);
    const double zzL = smax(in.zL, z_gamma_min);
    const double zzR = smax(in.zR, z_gamma_min);

    const double min_theta = smax(smin(in.theta_RL, theta_gamma_L), smin(in.theta_LR, theta_gamma_R));
    if (((theta_omega_L > kSmallReal) && (theta_omega_R > kSmallReal)) || (min_theta >= kSmallReal)) {
        const double cL = celerity(theta_omega_L, phi_omega_L);
        const double cR = celerity(theta_omega_R, phi_omega_R);
        const double phi_gamma_L = in.gamma_L.phi;
        const double phi_gamma_R = in.gamma_R.phi;
        const double chi_theta_L = theta_omega_L / smax(theta_gamma_L, theta_gamma_hmin);
        const double chi_theta_R = theta_omega_R / smax(theta_gamma_R, theta_gamma_hmin);
        double chi_phi_L = phi_omega_L / smax(phi_gamma_L, kSmallReal);
        double chi_phi_R = phi_omega_R / smax(phi_gamma_R, kSmallReal);
        chi_phi_L = smin(chi_phi_max, chi_phi_L);
        chi_phi_R = smin(chi_phi_max, chi_phi_R);

        const double L1L = lam_minus(uL, cL, chi_phi_L, chi_theta_L, in.bL);
        const double L2L = lam_plus(uL, cL, chi_phi_L, chi_theta_L, in.bL);
        const double L1R = lam_minus(uR, cR, chi_phi_R, chi_theta_R, in.bR);
        const double L2R = lam_plus(uR, cR, chi_phi_R, chi_theta_R, in.bR);
        // std::min({L1L, L1R, 0.}) and std::max({L2L, L2R, 0.}): first extreme under operator<
        double L1 = L1L;
        if (L1R < L1) L1 = L1R;
        if (0. < L1) L1 = 0.;
        double L2 = L2L;
        if (L2 < L2R) L2 = L2R;
        if (L2 < 0.) L2 = 0.;

        f.f1 = (L2 * phi_omega_R * theta_velocity_gamma_L - L1 * phi_omega_L * theta_velocity_gamma_R +
                L1 * L2 * smin(phi_omega_L, phi_omega_R) * smin(phi_gamma_L, phi_gamma_R) * (zzR - zzL)) /
               smax(phi_omega_R * L2 - phi_omega_L * L1, kSmallReal);
        f.f2 = (L2 * M_L - L1 * M_R + L1 * L2 * (theta_omega_R * uR - theta_omega_L * uL)) / smax(L2 - L1, kSmallReal);
        if (f.f1 < 0)
            f.f3 = f.f1 * in.vR;
        else
            f.f3 = f.f1 * in.vL;
        f.sl = -Fb_L;
        f.sr = Fb_R;
        if ((theta_gamma_L < kSmallReal) && (theta_gamma_R < kSmallReal)) {
            f.f1 = 0.;
            f.f2 = 0.;
            f.f3 = 0.;
        }
    } else if ((theta_omega_L < kSmallReal) && (min_theta < kSmallReal)) {
        f.sl = 0.;
        f.sr = Fb_R;
    } else if ((theta_omega_R < kSmallReal) && (min_theta < kSmallReal)) {
        f.sl = -Fb_L;
        f.sr = 0.;
    } else {
        f.bad = kStatusHllcConfig;
    }
    return f;
}

// swDdp::hypBoundaryFlux (swDdpHyp.cpp:13-135), domain on the right of the edge.  `omega` is
// the cell's table at zR, `force_omega` the pressure force there, theta_bc the cell's volume at
// the prescribed level (types h and z).  Types: SW2D_BC_Q, _H, _Z, _FR; any other one flags
// kStatusBcType, where the reference stops.
SW2D_HD unsigned boundary_flux(double bR, double uR, double vR, PhiTheta omega, double force_omega, int type,
                               double bc_val, double theta_bc, double* flux1, double* flux2, double* flux3)
{
    const double phi_omega = omega.phi;
    const double phi_gamma = phi_omega;
    const double x_phi = phi_omega / smax(phi_gamma, kSmallReal);
    const double theta_omega = omega.theta;
    const double theta_gamma = theta_omega;
    const double x_theta = theta_omega / smax(theta_gamma, kSmallReal);
    const double theta_velocity_omega = theta_omega * uR;
    const double cR = celerity(theta_omega, phi_omega);
    const double lambda_in = smax(lam_plus(uR, cR, x_phi, x_theta, bR), kSmallReal);
    double f1 = 0, f2 = 0;
    unsigned bad = 0;
    if (type == 3) {  // fr: critical section
        f1 = -bc_val * cR * theta_omega;
        f2 = spec_force(theta_velocity_omega, uR, force_omega) + lambda_in * (f1 - theta_velocity_omega);
    } else if (type == 1 || type == 2) {  // h or z prescribed
        if (lambda_in < kSmallReal) {
            f1 = theta_velocity_omega;
            f2 = spec_force(theta_velocity_omega, uR, force_omega);
        } else {
            f1 = theta_velocity_omega + lambda_in * (theta_bc - theta_omega);
            f2 = spec_force(theta_velocity_omega, uR, force_omega) + lambda_in * (f1 - theta_velocity_omega);
        }
    } else if (type == 0) {  // q prescribed
        const double lambda_critic = sw2d_exp((1. / 3.) * sw2d_log(kGravity * smax(bc_val, 0.)));
        const double lambda = smax(lambda_in, lambda_critic);
        f1 = bc_val;
        f2 = spec_force(theta_velocity_omega, uR, force_omega) + lambda * (f1 - theta_velocity_omega);
    } else {
        bad |= kStatusBcType;
    }
    *flux1 = f1;
    *flux2 = f2;
    *flux3 = (f1 > 0) ? 0 : f1 * vR;
    return bad;
}

// Level prescribed by a boundary of type h (depth above the cell's lowest level) or z
// (swDdpHyp.cpp:69-72,86-87).
SW2D_HD double boundary_level(int type, double bc_val, double z_tab0)
{
    return (type == 1) ? smax(bc_val, 0.) + z_tab0 : bc_val;
}

}  // namespace ddp
}  // namespace sw2d
