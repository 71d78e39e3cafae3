// Host composition of the DDP step from the device functions of ddp_math.cuh, in the reference's
// serial order (swDdp::execute's loop body, src/sw2dSolver/models/ddp/swDdp.cpp:595-690), built
// with g++ -ffp-contract=off into a shared library that tests/test_ddp_host.py drives against
// the reference's own swDdp.  It checks the arithmetic and the branch structure of the DDP
// kernels on the CPU; the kernels' parallel decomposition (balance slots, derived per-cell
// values, ordered dry-cell lists) is checked against the reference on the GPU.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "ddp_math.cuh"
#include "dip_math.cuh"

using namespace sw2d;
using ddp::Lvl;
using ddp::PhiTheta;

extern "C" {

struct HostCase {
    int64_t nc, ni, nb;
    const double *area, *zb, *bous;
    const int64_t *L, *R;
    const double *nx, *ny, *len;
    const int64_t* bcell;
    const double *bnx, *bny, *blen;
    const int32_t* bbc;
    const int64_t* ctoff;  // cell tables, levels [ctoff[c], ctoff[c+1])
    const double *cz, *cphi, *ctheta;
    const int64_t* etoff;  // internal-edge tables
    const double *ez, *ephi, *etheta;
    const int32_t* bctype;
    const int64_t* bcoff;
    const double *bct, *bcv;
    double h_min, cfl_max, dt_max, dt_map, t_max, v_max, fr_max, chi_phi_max, h_min_ddp;
    int32_t friction, head_loss, dissipation, div_corr, n_it_div_max, neg_detect;
    const double *f1, *f2, *fa;         // friction coefficients, angle (degrees)
    const double *hs, *hk1, *hk2, *ha;  // singular head loss
    const double *mu1, *mu2, *mua;      // momentum dissipation
};

struct HostState {
    double *theta, *tu, *tv;
    double *t, *dt;
    // persistent fluxes (the reference keeps an edge's previous ones when it is dry)
    double *F1i, *F2i, *F3i, *s2Li, *s2Ri, *F1b, *F2b, *F3b, *s2Rb;
    double *lmi, *lmb;  // lambda_max of the last step
    int32_t* status;
};

}  // extern "C"

namespace {

struct Tabs {
    std::vector<std::vector<Lvl>> cell, eint;
};

Tabs make_tabs(const HostCase& c)
{
    Tabs t;
    t.cell.resize(c.nc);
    for (int64_t i = 0; i < c.nc; i++)
        for (int64_t k = c.ctoff[i]; k < c.ctoff[i + 1]; k++) t.cell[i].push_back(Lvl{c.cz[k], c.cphi[k]});
    t.eint.resize(c.ni);
    for (int64_t i = 0; i < c.ni; i++)
        for (int64_t k = c.etoff[i]; k < c.etoff[i + 1]; k++) t.eint[i].push_back(Lvl{c.ez[k], c.ephi[k]});
    return t;
}

PhiTheta pt(const std::vector<Lvl>& t, double z, unsigned& bad) { return ddp::phi_theta(t.data(), (int)t.size(), z, bad); }
double zt(const std::vector<Lvl>& t, double th, unsigned& bad) { return ddp::z_of_theta(t.data(), (int)t.size(), th, bad); }
double pf(const std::vector<Lvl>& t, double z) { return ddp::pressure_force(t.data(), (int)t.size(), z); }

int one_step(const HostCase& c, const Tabs& T, HostState& s)
{
    unsigned bad = 0;
    const int64_t nc = c.nc, ni = c.ni, nb = c.nb;
    const double t = *s.t;
    if (!(t < c.t_max)) return 0;
    std::vector<double> z(nc);
    for (int64_t i = 0; i < nc; i++) z[i] = zt(T.cell[i], s.theta[i], bad);
    // ---- Riemann states (swDdpHypGodunov.cpp)
    std::vector<double> bh(nb), btu(nb), btv(nb), blp(nb);
    for (int64_t e = 0; e < nb; e++) {
        const int64_t k = c.bcell[e];
        const double h_in = smax(z[k] - T.cell[k][0].z, 0.);
        bh[e] = h_in;
        double tu = s.tu[k] * c.bnx[e] + s.tv[k] * c.bny[e];
        double tv = -s.tu[k] * c.bny[e] + s.tv[k] * c.bnx[e];
        if (h_in < c.h_min) {
            tu = 0.;
            tv = 0.;
        }
        btu[e] = tu;
        btv[e] = tv;
        const double phi_omega = pt(T.cell[k], z[k], bad).phi;
        const double c_in = ddp::celerity(s.theta[k], phi_omega);
        const double u_in = tu / smax(s.theta[k], kSmallReal);
        const double lp = ddp::lam_plus(u_in, c_in, 1.0, 1.0, c.bous[k]);
        const double lm = ddp::lam_minus(u_in, c_in, 1.0, 1.0, c.bous[k]);
        blp[e] = lp;
        s.lmb[e] = smax(std::fabs(lp), std::fabs(lm));
    }
    std::vector<ddp::Side> SL(ni), SR(ni);
    for (int64_t e = 0; e < ni; e++) {
        const int64_t a = c.L[e], b = c.R[e];
        const auto& ta = T.cell[a];
        const auto& tb = T.cell[b];
        const auto& te = T.eint[e];
        SL[e] = ddp::lr_side(s.theta[a], s.tu[a], s.tv[a], z[a], ta[0].z, c.bous[a], c.nx[e], c.ny[e], pt(ta, z[a], bad),
                             pt(te, z[a], bad),
                             [&](PhiTheta& om, PhiTheta& gm) {
                                 om = pt(ta, ta[0].z + c.h_min, bad);
                                 gm = pt(te, ta[0].z + c.h_min, bad);
                             },
                             c.h_min);
        SR[e] = ddp::lr_side(s.theta[b], s.tu[b], s.tv[b], z[b], tb[0].z, c.bous[b], c.nx[e], c.ny[e], pt(tb, z[b], bad),
                             pt(te, z[b], bad),
                             [&](PhiTheta& om, PhiTheta& gm) {
                                 om = pt(tb, tb[1].z + c.h_min, bad);
                                 gm = pt(te, tb[1].z + c.h_min, bad);
                             },
                             c.h_min);
        s.lmi[e] = max4(std::fabs(SL[e].lm), std::fabs(SL[e].lp), std::fabs(SR[e].lm), std::fabs(SR[e].lp));
    }
    // ---- time step (swDdpHyp.cpp:522-636)
    double dt = c.dt_max;
    std::vector<double> swept(nc, 0.);
    for (int64_t e = 0; e < nb; e++) {
        const int64_t k = c.bcell[e];
        if (z[k] - T.cell[k][0].z > c.h_min) swept[k] += s.lmb[e] * c.blen[e];
    }
    for (int64_t e = 0; e < ni; e++) {
        double lambda = 0.;
        const int64_t a = c.L[e], b = c.R[e];
        if (z[a] - T.cell[a][0].z > c.h_min) lambda = s.lmi[e];
        swept[a] += lambda * c.len[e];
        if (z[b] - T.cell[b][0].z > c.h_min) lambda = s.lmi[e];
        swept[b] += lambda * c.len[e];
    }
    for (int64_t i = 0; i < nc; i++) {
        const double x = c.cfl_max * (c.area[i] / smax(swept[i], kSmallReal));
        if (x < dt) dt = x;
    }
    if (c.dt_map > kSmallReal) {
        int now = (int)((double)(int)t / c.dt_map);
        int later = (int)((double)(int)(t + dt) / c.dt_map);
        if (later > now) dt = later * c.dt_map - t;
    }
    if ((t + dt) > c.t_max) dt = c.t_max - t;
    // ---- fluxes (swDdpHyp.cpp:356-488)
    for (int64_t e = 0; e < nb; e++) {
        const int64_t k = c.bcell[e];
        double uR = 0.0, vR = 0.0;
        if (bh[e] > kSmallReal) {
            uR = btu[e] / bh[e];
            vR = btv[e] / bh[e];
        }
        const int bi = c.bbc[e];
        const double val = bc_value(c.bct + c.bcoff[bi], c.bcv + c.bcoff[bi], c.bcoff[bi + 1] - c.bcoff[bi], t);
        const int type = c.bctype[bi];
        double theta_bc = 0.0;
        if (type == 1 || type == 2)
            theta_bc = pt(T.cell[k], ddp::boundary_level(type, val, T.cell[k][0].z), bad).theta;
        const PhiTheta om = pt(T.cell[k], z[k], bad);
        bad |= ddp::boundary_flux(c.bous[k], uR, vR, om, pf(T.cell[k], z[k]), type, val, theta_bc, &s.F1b[e], &s.F2b[e],
                                  &s.F3b[e]);
        s.s2Rb[e] = 0.0;
    }
    for (int64_t e = 0; e < ni; e++) {
        const int64_t a = c.L[e], b = c.R[e];
        const double hL = z[a] - c.zb[a], hR = z[b] - c.zb[b];
        if (!((hL > c.h_min) || (hR > c.h_min))) continue;
        const auto& te = T.eint[e];
        ddp::HllcIn in;
        in.bL = c.bous[a];
        in.bR = c.bous[b];
        in.zL = z[a];
        in.zR = z[b];
        in.uL = in.vL = in.uR = in.vR = 0.0;
        if (s.theta[a] > kSmallReal) {
            in.uL = SL[e].tu / s.theta[a];
            in.vL = SL[e].tv / s.theta[a];
        }
        if (s.theta[b] > kSmallReal) {
            in.uR = SR[e].tu / s.theta[b];
            in.vR = SR[e].tv / s.theta[b];
        }
        in.omega_L = pt(T.cell[a], z[a], bad);
        in.omega_R = pt(T.cell[b], z[b], bad);
        in.gamma_L = pt(te, z[a], bad);
        in.gamma_R = pt(te, z[b], bad);
        in.theta_RL = pt(T.cell[b], z[a], bad).theta;
        in.theta_LR = pt(T.cell[a], z[b], bad).theta;
        in.force_omega_L = pf(T.cell[a], z[a]);
        in.force_omega_R = pf(T.cell[b], z[b]);
        in.force_gamma_L = pf(te, z[a]);
        in.force_gamma_R = pf(te, z[b]);
        in.theta_gamma_hmin = pt(te, te[0].z + c.h_min_ddp, bad).theta;
        in.z_gamma_min = te[0].z;
        const ddp::Flux f = ddp::hllc(in, c.h_min, c.chi_phi_max);
        bad |= f.bad;
        if (std::isnan(f.f1)) bad |= kStatusNanFlux;
        s.F1i[e] = f.f1;
        s.F2i[e] = f.f2;
        s.F3i[e] = f.f3;
        s.s2Li[e] = f.sl;
        s.s2Ri[e] = f.sr;
    }
    // ---- balance (swDdpHyp.cpp:236-349) with the edge factors of swDdp.cpp:399-489
    std::vector<double> o0(s.theta, s.theta + nc), o1(s.tu, s.tu + nc), o2(s.tv, s.tv + nc);
    auto balance_bnd = [&](int64_t e) {
        const int64_t k = c.bcell[e];
        const double cf = c.blen[e] / c.area[k], nx = c.bnx[e], ny = c.bny[e];
        s.theta[k] += (+cf) * s.F1b[e] * dt;
        s.tu[k] += ((+cf * nx) * s.F2b[e] + (+cf * nx) * s.s2Rb[e] + (-cf * ny) * s.F3b[e]) * dt;
        s.tv[k] += ((+cf * ny) * s.F2b[e] + (+cf * ny) * s.s2Rb[e] + (+cf * nx) * s.F3b[e]) * dt;
    };
    for (int64_t e = 0; e < nb; e++) balance_bnd(e);
    auto int_terms = [&](int64_t e, bool left, double& a1, double& a2, double& a3) {
        const int64_t k = left ? c.L[e] : c.R[e];
        const double cf = c.len[e] / c.area[k], nx = c.nx[e], ny = c.ny[e];
        if (left) {
            a1 = (-cf) * s.F1i[e];
            a2 = (-cf * nx) * s.F2i[e] + (+cf * nx) * s.s2Li[e] + (+cf * ny) * s.F3i[e];
            a3 = (-cf * ny) * s.F2i[e] + (+cf * ny) * s.s2Li[e] + (-cf * nx) * s.F3i[e];
        } else {
            a1 = (+cf) * s.F1i[e];
            a2 = (+cf * nx) * s.F2i[e] + (+cf * nx) * s.s2Ri[e] + (-cf * ny) * s.F3i[e];
            a3 = (+cf * ny) * s.F2i[e] + (+cf * ny) * s.s2Ri[e] + (+cf * nx) * s.F3i[e];
        }
    };
    for (int64_t e = 0; e < ni; e++) {
        double a1, a2, a3;
        int_terms(e, true, a1, a2, a3);
        s.theta[c.L[e]] += a1 * dt;
        int_terms(e, false, a1, a2, a3);
        s.theta[c.R[e]] += a1 * dt;
        int_terms(e, true, a1, a2, a3);
        s.tu[c.L[e]] += a2 * dt;
        int_terms(e, false, a1, a2, a3);
        s.tu[c.R[e]] += a2 * dt;
        int_terms(e, true, a1, a2, a3);
        s.tv[c.L[e]] += a3 * dt;
        int_terms(e, false, a1, a2, a3);
        s.tv[c.R[e]] += a3 * dt;
    }
    if (c.dissipation) {
        for (int64_t i = 0; i < nc; i++) {
            const double al = c.mua[i] * atan(1.0) / 45.0;
            momentum_dissipation(c.mu1[i], c.mu2[i], cos(al), sin(al), o0[i], o1[i], o2[i], s.theta[i], s.tu[i], s.tv[i]);
        }
    }
    // ---- divergence correction (swDdpHyp.cpp:640-768)
    if (c.div_corr == 2) {
        const double dt_initial = dt;
        double dt_avoid = dt;
        bool some = false;
        for (int64_t i = 0; i < nc; i++)
            if (s.theta[i] <= 0.0) {
                const double cell = dt * (o0[i] - s.theta[i]) / s.theta[i];
                dt_avoid = (dt_avoid < cell) ? dt_avoid : cell;  // std::min(cell, dt_avoid)
                some = true;
            }
        dt = smin(dt, dt_avoid);
        if (some) {
            const double r = dt / dt_initial;
            for (int64_t i = 0; i < nc; i++) {
                s.theta[i] = o0[i] * (1.0 - r) + s.theta[i] * r;
                s.tu[i] = o1[i] * (1.0 - r) + s.tu[i] * r;
                s.tv[i] = o2[i] * (1.0 - r) + s.tv[i] * r;
            }
        }
    } else if (c.div_corr == 1) {
        std::vector<int64_t> nbo(nc, 0), nio(nc, 0);
        for (int64_t e = 0; e < nb; e++) nbo[c.bcell[e]]++;
        for (int64_t e = 0; e < ni; e++) {
            nio[c.L[e]]++;
            nio[c.R[e]]++;
        }
        int nbiter = 0;
        for (;;) {
            int64_t ndry = 0;
            for (int64_t i = 0; i < nc; i++) {
                if (s.theta[i] < 0.0) {
                    ndry++;
                    const double r = o0[i] / (o0[i] - s.theta[i]);
                    for (int64_t j = 0; j < nbo[i]; j++) {
                        s.F1b[j] *= r;
                        s.F2b[j] *= r;
                        s.F3b[j] *= r;
                        s.s2Rb[j] *= r;
                    }
                    for (int64_t j = 0; j < nio[i]; j++) {
                        s.F1i[j] *= r;
                        s.F2i[j] *= r;
                        s.F3i[j] *= r;
                        s.s2Li[j] *= r;
                        s.s2Ri[j] *= r;
                    }
                }
            }
            ++nbiter;
            for (int64_t e = 0; e < ni; e++) {
                double a1, a2, a3;
                const int64_t a = c.L[e], b = c.R[e];
                int_terms(e, true, a1, a2, a3);
                s.theta[a] = o0[a] + a1 * dt;
                s.tu[a] = o1[a] + a2 * dt;
                s.tv[a] = o2[a] + a3 * dt;
                int_terms(e, false, a1, a2, a3);
                s.theta[b] = o0[b] + a1 * dt;
                s.tu[b] = o1[b] + a2 * dt;
                s.tv[b] = o2[b] + a3 * dt;
            }
            if ((ndry == 0) || (nbiter > c.n_it_div_max)) break;
        }
    }
    // ---- negative volume (swDdpHyp.cpp:203-229)
    for (int64_t i = 0; i < nc; i++) {
        if (c.neg_detect) {
            if (s.theta[i] < 0) bad |= kStatusNegDepth;
        } else if (s.theta[i] < 0.) {
            s.theta[i] = 0.;
            s.tu[i] = 0.;
            s.tv[i] = 0.;
        }
    }
    // ---- friction, singular head loss (swDdpSourceFriction.cpp), velocity cap (swDdp.cpp:527-561)
    const double hthr = smax(c.h_min, kSmallReal);
    for (int64_t i = 0; i < nc; i++) {
        const double th = s.theta[i];
        double qq = s.tu[i], rr = s.tv[i];
        if (c.friction) {
            if (th > hthr) {
                const double al = c.fa[i] * atan(1.0) / 45.0;
                const double ca = cos(al), sa = sin(al);
                double u = qq / th, v = rr / th;
                double ul = u * ca + v * sa;
                double vl = -u * sa + v * ca;
                double un = std::sqrt(u * u + v * v);
                ul *= friction_factor(c.friction, c.f1[i], th, un, dt);
                vl *= friction_factor(c.friction, c.f2[i], th, un, dt);
                qq = (ul * ca - vl * sa) * th;
                rr = (ul * sa + vl * ca) * th;
            } else {
                qq = 0.;
                rr = 0.;
            }
        }
        if (c.head_loss) {
            const double al = c.ha[i] * atan(1.0) / 45.0;
            const double ca = cos(al), sa = sin(al);
            double qx = qq * ca + rr * sa;
            double qy = -qq * sa + rr * ca;
            if (th > hthr) {
                double ax = 0, ay = 0;
                if (th > c.hs[i]) {
                    ax = std::sqrt(qx * qx + qy * qy) * c.hk1[i] / th;
                    ay = std::sqrt(qx * qx + qy * qy) * c.hk2[i] / th;
                }
                qx = qx * sw2d_exp(-ax * dt);
                qy = qy * sw2d_exp(-ay * dt);
            } else {
                qx = 0.;
                qy = 0.;
            }
            qq = qx * ca - qy * sa;
            rr = qx * sa + qy * ca;
        }
        if (th > c.h_min) {
            double qn = std::sqrt(qq * qq + rr * rr);
            double cc = std::sqrt(kGravity * th);
            double Fr = qn / cc / th;
            double fact = smax(qn / (th * c.v_max), Fr / c.fr_max);
            if (fact > 1.0) {
                qq = qq / fact;
                rr = rr / fact;
            }
        }
        s.tu[i] = qq;
        s.tv[i] = rr;
    }
    *s.t = t + dt;
    *s.dt = dt;
    *s.status |= (int32_t)bad;
    return 1;
}

}  // namespace

extern "C" int ddp_host_steps(const HostCase* c, HostState* s, int n)
{
    const Tabs T = make_tabs(*c);
    int done = 0;
    for (int i = 0; i < n; i++) {
        if (!one_step(*c, T, *s)) break;
        done++;
        if (*s->status) break;
    }
    return done;
}

// the device functions on single inputs, for direct checks
extern "C" double ddp_host_z_of_theta(const double* z, const double* phi, const double* theta, int n, double th)
{
    std::vector<Lvl> t(n);
    for (int i = 0; i < n; i++) t[i] = Lvl{z[i], phi[i]};
    unsigned bad = 0;
    return ddp::z_of_theta(t.data(), n, th, bad);
}
