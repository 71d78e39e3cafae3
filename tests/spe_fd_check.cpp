// Finite-difference check of the reverse functions of the differentiated step (csrc/spe_math.cuh),
// on the host: the same source the GPU kernels compile, built here with g++.  For each function
// f: R^n -> R^m and random (x, v, w), the reverse gives xbar = J(x)^T w; the check compares
// xbar . v with the central difference w . (f(x + e v) - f(x - e v)) / (2 e).
//
// Output: one line per function, "name samples failures max_rel_err".
#include <cmath>
#include <cstdio>
#include <functional>
#include <random>
#include <vector>

#include "spe_math.cuh"

using namespace sw2d;
using namespace sw2d::spe;
using Vec = std::vector<double>;

static std::mt19937_64 rng(4242);
static double U(double a, double b) { return std::uniform_real_distribution<double>(a, b)(rng); }

struct Stats {
    int n = 0, fail = 0;
    double worst = 0.0;
};

static void check(Stats& st, const Vec& x, const Vec& v_in, const std::function<Vec(const Vec&)>& f,
                  const std::function<Vec(const Vec&, const Vec&)>& rev, double tol = 1e-5)
{
    Vec v = v_in;
    for (size_t i = 0; i < x.size(); i++) v[i] *= std::max(1.0, std::fabs(x[i]));
    const Vec y0 = f(x);
    Vec w(y0.size());
    for (double& e : w) e = U(-1.0, 1.0);
    const Vec xb = rev(x, w);
    double ad = 0.0, scale = 0.0;
    for (size_t i = 0; i < x.size(); i++) {
        ad += xb[i] * v[i];
        scale += std::fabs(xb[i] * v[i]);
    }
    const double eps = 1e-7;
    Vec xp = x, xm = x;
    for (size_t i = 0; i < x.size(); i++) {
        xp[i] += eps * v[i];
        xm[i] -= eps * v[i];
    }
    const Vec yp = f(xp), ym = f(xm);
    double fd = 0.0, fs = 0.0;
    for (size_t i = 0; i < w.size(); i++) {
        fd += w[i] * (yp[i] - ym[i]) / (2.0 * eps);
        fs += std::fabs(w[i] * (yp[i] - ym[i]) / (2.0 * eps));
    }
    double ysc = 0.0;
    for (double e : y0) ysc = std::max(ysc, std::fabs(e));
    const double denom = std::max({scale, fs, 1e-8 * std::max(1.0, ysc)});
    const double err = std::fabs(fd - ad) / denom;
    st.n++;
    if (!(err <= tol)) st.fail++;
    if (err > st.worst || std::isnan(err)) st.worst = std::isnan(err) ? 1e300 : err;
}

static Vec rand_dir(size_t n)
{
    Vec v(n);
    for (double& e : v) e = U(-1.0, 1.0);
    return v;
}

static void report(const char* name, const Stats& s) { std::printf("%s %d %d %.3e\n", name, s.n, s.fail, s.worst); }

static ESide side_of(const Vec& x, int o) { return ESide{x[o], x[o + 1], x[o + 2], x[o + 3], x[o + 4]}; }

int main()
{
    const int N = 2000;
    const double h_min = 1e-5, phi_min = 1e-16;

    {  // desing: x = (q, h)
        Stats s;
        for (int it = 0; it < N; it++) {
            Vec x{U(-2, 2), (it % 3 == 0) ? U(1e-4, 8e-3) : U(8e-3, 2.0)};
            auto f = [&](const Vec& x) { return Vec{desing(x[0], x[1])}; };
            auto r = [&](const Vec& x, const Vec& w) {
                double qb = 0, hb = 0;
                desing_rev(x[0], x[1], w[0], qb, hb);
                return Vec{qb, hb};
            };
            check(s, x, rand_dir(2), f, r);
        }
        report("desing", s);
    }

    for (int kind = 0; kind < 2; kind++) {  // god_side / evr_bnd_side: x = (h, q, r)
        Stats s;
        for (int it = 0; it < N; it++) {
            const double b = U(1.0, 1.3), a = U(0, 6.283), nx = std::cos(a), ny = std::sin(a), zb = U(-1, 1);
            Vec x{(it % 4 == 0) ? U(1e-3, 2e-2) : U(0.02, 3.0), U(-3, 3), U(-3, 3)};
            auto f = [&](const Vec& x) {
                ESide S = kind ? evr_bnd_side(x[0], x[1], x[2], zb, b, nx, ny) : god_side(x[0], x[1], x[2], zb, b, nx, ny, h_min);
                return Vec{S.z, S.q, S.r, S.lm, S.lp};
            };
            auto r = [&](const Vec& x, const Vec& w) {
                double hb = 0, qb = 0, rb = 0;
                ESideBar sb{w[0], w[1], w[2], w[3], w[4]};
                if (kind) evr_bnd_side_rev(x[0], x[1], x[2], b, nx, ny, sb, hb, qb, rb);
                else god_side_rev(x[0], x[1], x[2], b, nx, ny, h_min, sb, hb, qb, rb);
                return Vec{hb, qb, rb};
            };
            check(s, x, rand_dir(3), f, r);
        }
        report(kind ? "evr_bnd_side" : "god_side", s);
    }

    for (int left = 0; left < 2; left++) {  // evr_side: x = (h, q, r, zc, sx, sy)
        Stats s;
        for (int it = 0; it < N; it++) {
            const double b = U(1.0, 1.3), a = U(0, 6.283), nx = std::cos(a), ny = std::sin(a);
            const double dmx = U(-0.5, 0.5), dmy = U(-0.5, 0.5), dt = U(0.0, 0.2), zb = U(-0.5, 0.5);
            const double h = (it % 5 == 0) ? U(0.001, 0.05) : U(0.05, 2.0);
            Vec x{h, U(-2, 2), U(-2, 2), h + zb + U(-0.05, 0.05), U(-0.5, 0.5), U(-0.5, 0.5)};
            auto f = [&](const Vec& x) {
                ESide S = evr_side(left, x[0], x[1], x[2], zb, b, x[3], x[4], x[5], dmx, dmy, nx, ny, dt);
                return Vec{S.z, S.q, S.r, S.lm, S.lp};
            };
            auto r = [&](const Vec& x, const Vec& w) {
                double hb = 0, qb = 0, rb = 0, zcb = 0, sxb = 0, syb = 0;
                evr_side_rev(left, x[0], x[1], x[2], zb, b, x[3], x[4], x[5], dmx, dmy, nx, ny, dt,
                             ESideBar{w[0], w[1], w[2], w[3], w[4]}, hb, qb, rb, zcb, sxb, syb);
                return Vec{hb, qb, rb, zcb, sxb, syb};
            };
            check(s, x, rand_dir(6), f, r);
        }
        report(left ? "evr_side_left" : "evr_side_right", s);
    }

    for (int reg = 0; reg < 3; reg++) {  // hllc: x = (phiL, phiR, zL, qL, rL, lmL, lpL, zR, qR, rR, lmR, lpR)
        Stats s;
        for (int it = 0; it < N; it++) {
            const double bL = U(1.0, 1.2), bR = U(1.0, 1.2), zbL = U(-0.5, 0.5), zbR = U(-0.5, 0.5);
            double hL = U(0.05, 2.0), hR = U(0.05, 2.0);
            if (reg == 1) {  // left dry, right's level below the left bed: rhs alone
                hL = -U(0.01, 0.2);
                hR = std::max(0.05, zbL - zbR - 0.05 - U(0.0, 0.3));
                if (zbR + hR >= zbL) hR = 0.05, hL = -0.1;
            }
            if (reg == 2) {
                hR = -U(0.01, 0.2);
                hL = std::max(0.05, zbR - zbL - 0.05 - U(0.0, 0.3));
            }
            const double phiL = U(0.2, 1.0), phiR = (it % 4 == 0) ? phiL + U(-1e-3, 1e-3) : U(0.2, 1.0);
            Vec x{phiL, phiR, zbL + hL, U(-2, 2), U(-2, 2), U(-6, 1), U(-1, 6), zbR + hR, U(-2, 2), U(-2, 2), U(-6, 1),
                  U(-1, 6)};
            if (reg == 1 && !(x[7] <= zbL + h_min)) continue;
            if (reg == 2 && !(x[2] <= zbR + h_min)) continue;
            auto f = [&](const Vec& x) {
                EFlux F = hllc(bL, bR, x[0], x[1], zbL, zbR, side_of(x, 2), side_of(x, 7), h_min, phi_min);
                return Vec{F.f1, F.f2, F.f3, F.sl, F.sr};
            };
            auto r = [&](const Vec& x, const Vec& w) {
                double pLb = 0, pRb = 0;
                ESideBar Lb{0, 0, 0, 0, 0}, Rb{0, 0, 0, 0, 0};
                hllc_rev(bL, bR, x[0], x[1], zbL, zbR, side_of(x, 2), side_of(x, 7), h_min, phi_min,
                         EFlux{w[0], w[1], w[2], w[3], w[4]}, pLb, pRb, Lb, Rb);
                return Vec{pLb, pRb, Lb.z, Lb.q, Lb.r, Lb.lm, Lb.lp, Rb.z, Rb.q, Rb.r, Rb.lm, Rb.lp};
            };
            check(s, x, rand_dir(12), f, r);
        }
        report(reg == 0 ? "hllc_wet" : reg == 1 ? "hllc_left_dry" : "hllc_right_dry", s);
    }

    const char* tn[] = {"q", "h", "z", "fr"};
    for (int type = 0; type < 4; type++) {
        for (int wet = 0; wet < 2; wet++) {  // boundary_flux: x = (phiR, z, q, r, lp)
            Stats s;
            for (int it = 0; it < N; it++) {
                const double bR = U(1.0, 1.2), zbR = U(-0.5, 0.5);
                const double h = wet ? U(0.05, 2.0) : U(-0.2, 0.5 * h_min);
                double bcv = type == 0 ? U(0.05, 3.0) : type == 3 ? U(0.05, 0.95) : U(0.0, 2.0) + (type == 2 ? zbR : 0.0);
                if (type == 0 && it % 7 == 0) bcv = 0.0;  // walls
                Vec x{U(0.2, 1.0), zbR + h, U(-2, 2), U(-2, 2), U(-3, 5)};
                auto f = [&](const Vec& x) {
                    EBndFlux F = boundary_flux(bR, x[0], zbR, ESide{x[1], x[2], x[3], 0.0, x[4]}, type, bcv, h_min, phi_min);
                    return Vec{F.f1, F.f2, F.f3};
                };
                auto r = [&](const Vec& x, const Vec& w) {
                    double pb = 0;
                    ESideBar Sb{0, 0, 0, 0, 0};
                    boundary_flux_rev(bR, x[0], zbR, ESide{x[1], x[2], x[3], 0.0, x[4]}, type, bcv, h_min, phi_min, w[0], w[1], w[2],
                                      pb, Sb);
                    return Vec{pb, Sb.z, Sb.q, Sb.r, Sb.lp};
                };
                check(s, x, rand_dir(5), f, r);
            }
            char name[64];
            std::snprintf(name, sizeof name, "boundary_flux_%s_%s", tn[type], wet ? "wet" : "dry");
            report(name, s);
        }
    }

    for (int fr = 0; fr < 2; fr++) {
        for (int hl = 0; hl < 2; hl++) {  // cell_update: x = (h, q, r, k1, k2)
            Stats s;
            for (int it = 0; it < N; it++) {
                ECellParams p;
                p.friction = fr;
                p.head_loss = hl;
                p.ca = std::cos(U(0, 6.283));
                p.sa = std::sin(std::acos(p.ca)) * (U(0, 1) < 0.5 ? -1.0 : 1.0);
                p.hs = U(0.0, 0.5);
                p.hk1 = U(0.0, 2.0);
                p.hk2 = U(0.0, 2.0);
                const double ah = U(0, 6.283);
                p.hca = std::cos(ah);
                p.hsa = std::sin(ah);
                p.h_min = h_min;
                const double dt = U(0.001, 0.3);
                Vec x{(it % 6 == 0) ? U(1e-3, 2e-2) : U(0.02, 3.0), U(-3, 3), U(-3, 3), U(5, 80), U(5, 80)};
                auto f = [&](const Vec& x) {
                    ECellParams q = p;
                    q.k1 = x[3];
                    q.k2 = x[4];
                    double h = x[0], qq = x[1], rr = x[2];
                    cell_update(h, qq, rr, q, dt);
                    return Vec{h, qq, rr};
                };
                auto r = [&](const Vec& x, const Vec& w) {
                    ECellParams q = p;
                    q.k1 = x[3];
                    q.k2 = x[4];
                    double hb = w[0], qb = w[1], rb = w[2], k1b = 0, k2b = 0;
                    cell_update_rev(x[0], x[1], x[2], q, dt, hb, qb, rb, k1b, k2b);
                    return Vec{hb, qb, rb, k1b, k2b};
                };
                check(s, x, rand_dir(5), f, r);
            }
            char name[64];
            std::snprintf(name, sizeof name, "cell_update_friction%d_headloss%d", fr, hl);
            report(name, s);
        }
    }

    for (int kind = 0; kind < 4; kind++) {  // the porosity transform: x = (m)
        Stats s;
        for (int it = 0; it < N; it++) {
            const double lambda = U(0.5, 4.0), lo = U(-0.5, 0.5), scale = U(0.5, 2.0);
            Vec x{U(-1.0, 2.0)};
            if (kind == kPhiClamp && (std::fabs(x[0]) < 1e-3 || std::fabs(x[0] - 1.05) < 1e-3)) continue;
            auto f = [&](const Vec& x) { return Vec{phi_correct(kind, x[0], lambda, lo, scale)}; };
            auto r = [&](const Vec& x, const Vec& w) { return Vec{w[0] * dphi_dm(kind, x[0], lambda, scale)}; };
            check(s, x, rand_dir(1), f, r);
        }
        const char* kn[] = {"transform_none", "transform_clamp", "transform_tanh", "transform_normalize"};
        report(kn[kind], s);
    }
    return 0;
}
