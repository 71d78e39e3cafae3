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

// one level of a porosity table: {z_k, phi_k, theta_k}
struct alignas(32) Lvl {
    double z, phi, theta, pad;
};

struct PhiTheta {
    double phi, theta;
};

SW2D_HD double quiet_nan() { return __builtin_nan(""); }

// phiWOfZ / phiGIntOfZ (swDdp.cpp:1049-1097) and thetaWOfZ / thetaGIntOfZ (swDdp.cpp:2678-2736)
// at the same elevation: both run the same scan, so one scan gives both.
SW2D_HD PhiTheta phi_theta(const Lvl* t, int n, double z, unsigned& bad)
{
    if (z <= t[0].z) return {0.0, 0.0};
    int l = 0;
    while ((l < n) && (z > t[l].z)) ++l;
    if (l == 0) {
        bad |= kStatusTable;
        return {quiet_nan(), quiet_nan()};
    }
    const Lvl a = t[l - 1];
    double theta = a.theta;
    if (z > a.z) theta += (z - a.z) * a.phi;
    return {a.phi, theta};
}

// swDdp::zOfThetaW (swDdp.cpp:3368-3388)
SW2D_HD double z_of_theta(const Lvl* t, int n, double theta, unsigned& bad)
{
    if (theta <= 0) return t[0].z;
    int l = 0;
    while ((l < n) && (theta > t[l].theta)) ++l;
    if (l == 0) {
        bad |= kStatusTable;
        return quiet_nan();
    }
    const Lvl a = t[l - 1];
    double z = a.z;
    z += (theta - a.theta) / a.phi;
    return z;
}

// swDdp::pressureForceOmegaOfZ / pressureForceGammaOfZ (swDdp.cpp:1214-1273): g times the
// integral of phi(zeta) (z - zeta) over the wetted levels.
SW2D_HD double pressure_force(const Lvl* t, int n, double z)
{
    double p = 0;
    if (z > t[0].z) {
        int l = 0;
        while ((l < n - 1) && (z >= t[l + 1].z)) {
            const double z1 = t[l].z;
            const double z2 = t[l + 1].z;
            const double dz1 = z - (z1 + z2) / 2.;
            const double dz2 = z2 - z1;
            p += t[l].phi * dz1 * dz2;
            ++l;
        }
        const double dz1 = smax(0., z - t[l].z);
        p += t[l].phi * dz1 * dz1 / 2.;
    }
    p *= kGravity;
    return p;
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
// cell's and the edge's tables at the side's elevation, `omega_min` and `gamma_min` at the
// reference's shallow-side elevation (cell_z_tab[L][0] + h_min on the left, cell_z_tab[R][1] +
// h_min on the right, as swDdpHypGodunov.cpp:84,130 write them).
struct Side {
    double tu, tv, lm, lp;
};

SW2D_HD Side lr_side(double theta, double thu, double thv, double z, double z_tab0, double b, double nx, double ny,
                     PhiTheta omega, PhiTheta gamma, PhiTheta omega_min, PhiTheta gamma_min, double h_min)
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
