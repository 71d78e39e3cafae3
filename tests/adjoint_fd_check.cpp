// Finite-difference check of the hand-written reverse functions of sp_adjoint.cuh, on the host.
//
// The forward functions (sp_math.cuh) and their reverses (sp_adjoint.cuh) are the same source
// the GPU kernels compile; here g++ builds them for the CPU.  For each function f: R^n -> R^m
// and random (x, v, w), the reverse gives xbar = J(x)^T w and the check compares xbar . v with
// the central difference w . (f(x + e v) - f(x - e v)) / (2 e).  Samples whose branches change
// between x - e v and x + e v are rare (the inputs are continuous random numbers); the test
// that runs this program allows a small fraction of them.
//
// Output: one line per function, "name samples failures max_rel_err".
#include <cmath>
#include <cstdio>
#include <functional>
#include <random>
#include <vector>

#include "sp_adjoint.cuh"

using namespace sw2d;
using Vec = std::vector<double>;

static std::mt19937_64 rng(12345);
static double U(double a, double b) { return std::uniform_real_distribution<double>(a, b)(rng); }

struct Stats {
    int n = 0, fail = 0;
    double worst = 0.0;
};

// f(x) -> y; rev(x, w) -> xbar
static void check(Stats& st, const Vec& x, const Vec& v_in, const std::function<Vec(const Vec&)>& f,
                  const std::function<Vec(const Vec&, const Vec&)>& rev, double tol = 1e-5)
{
    Vec v = v_in;  // step relative to each input's magnitude
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
    const double eps = 1e-6;
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

int main()
{
    const int N = 2000;
    const DryConsts dry{std::sqrt(kGravity * kSmallReal), std::sqrt(std::sqrt(kGravity * kSmallReal) * std::sqrt(kGravity * kSmallReal))};

    {  // godunov_side: x = (h, q, r, zb)
        Stats s;
        for (int it = 0; it < N; it++) {
            const double b = U(1.0, 1.3), a = U(0, 6.283), nx = std::cos(a), ny = std::sin(a);
            Vec x{U(0.01, 3.0), U(-3, 3), U(-3, 3), U(-1, 1)};
            auto f = [&](const Vec& x) {
                SideState S = godunov_side(x[0], x[1], x[2], x[3], b, nx, ny);
                return Vec{S.z, S.q, S.r, S.lm, S.lp};
            };
            auto r = [&](const Vec& x, const Vec& w) {
                CellBar cb{0, 0, 0, 0, 0, 0, 0};
                godunov_side_rev(x[0], x[1], x[2], b, nx, ny, SideBar{w[0], w[1], w[2], w[3], w[4]}, cb);
                return Vec{cb.h, cb.q, cb.r, cb.zb};
            };
            check(s, x, rand_dir(4), f, r);
        }
        report("godunov_side", s);
    }

    for (int left = 0; left < 2; left++) {  // evr_side: x = (h, q, r, zb, zc, sx, sy)
        Stats s;
        for (int it = 0; it < N; it++) {
            const double b = U(1.0, 1.3), a = U(0, 6.283), nx = std::cos(a), ny = std::sin(a);
            const double cx = U(-1, 1), cy = U(-1, 1), mx = cx + U(-0.5, 0.5), my = cy + U(-0.5, 0.5);
            const double dt = U(0.0, 0.2);
            const double zb = U(-0.5, 0.5), h = (it % 5 == 0) ? U(0.001, 0.05) : U(0.05, 2.0);
            Vec x{h, U(-2, 2), U(-2, 2), zb, h + zb + U(-0.05, 0.05), U(-0.5, 0.5), U(-0.5, 0.5)};
            auto f = [&](const Vec& x) {
                SideState S = evr_side(left, x[0], x[1], x[2], x[3], b, x[4], x[5], x[6], mx - cx, my - cy, nx, ny, dt, dry);
                return Vec{S.z, S.q, S.r, S.lm, S.lp};
            };
            auto r = [&](const Vec& x, const Vec& w) {
                CellBar cb{0, 0, 0, 0, 0, 0, 0};
                evr_side_rev(left, x[0], x[1], x[2], x[3], b, x[4], x[5], x[6], mx - cx, my - cy, nx, ny, dt,
                             SideBar{w[0], w[1], w[2], w[3], w[4]}, cb);
                return Vec{cb.h, cb.q, cb.r, cb.zb, cb.zc, cb.sx, cb.sy};
            };
            check(s, x, rand_dir(7), f, r);
        }
        report(left ? "evr_side_left" : "evr_side_right", s);
    }

    for (int blend = 0; blend < 2; blend++) {
        for (int regime = 0; regime < 3; regime++) {  // 0: both wet, 1: L dry, 2: R dry
            Stats s;
            for (int it = 0; it < N; it++) {
                const double bL = U(1.0, 1.2), bR = U(1.0, 1.2), phiL = U(0.3, 1.0), phiR = U(0.3, 1.0);
                const double zbL = U(-0.5, 0.5), zbR = (it % 4 == 0) ? zbL : U(-0.5, 0.5);
                const double hmin = 1e-5;
                auto side = [&](double zb, bool dry) {
                    if (dry) return Vec{zb, 0.0, 0.0, 0.0, 0.0};  // h = 0: godunov_side's state
                    const double h = U(0.05, 2.0), u = U(-2, 2), v = U(-2, 2), c = std::sqrt(kGravity * h);
                    return Vec{h + zb, h * u, h * v, u - c, u + c};
                };
                Vec Ls = side(zbL, regime == 1), Rs = side(zbR, regime == 2);
                if (regime == 1 && !(Ls[0] <= zbR + hmin)) continue;  // a dry side the wet side floods
                if (regime == 2 && !(Rs[0] <= zbL + hmin)) continue;
                Vec x(12);
                for (int i = 0; i < 5; i++) {
                    x[i] = Ls[i];
                    x[5 + i] = Rs[i];
                }
                x[10] = zbL;
                x[11] = zbR;
                Vec v = rand_dir(12);
                // equal beds: the blending weight is 0 there and jumps for any bed difference
                // (a discontinuity of the forward), so such beds move together
                if (zbL == zbR) v[11] = v[10];
                // the dry side stays dry and at rest (its depth sits on the kink of max(0, .))
                if (regime == 1) v[0] = v[1] = v[2] = v[3] = v[4] = v[10] = v[11] = 0.0;
                if (regime == 2) v[5] = v[6] = v[7] = v[8] = v[9] = v[10] = v[11] = 0.0;
                auto f = [&](const Vec& x) {
                    SideState L{x[0], x[1], x[2], x[3], x[4]}, R{x[5], x[6], x[7], x[8], x[9]};
                    EdgeFlux F = hllc(blend, bL, bR, phiL, phiR, x[10], x[11], L, R, hmin, 1e-16);
                    return Vec{F.f1, F.f2, F.f3, F.sl, F.sr};
                };
                auto r = [&](const Vec& x, const Vec& w) {
                    SideState L{x[0], x[1], x[2], x[3], x[4]}, R{x[5], x[6], x[7], x[8], x[9]};
                    EdgeFlux fb{w[0], w[1], w[2], w[3], w[4], 0};
                    SideBar Lb{0, 0, 0, 0, 0}, Rb{0, 0, 0, 0, 0};
                    double zl = 0, zr = 0;
                    hllc_rev(blend, bL, bR, phiL, phiR, x[10], x[11], L, R, hmin, 1e-16, fb, Lb, Rb, zl, zr);
                    return Vec{Lb.z, Lb.q, Lb.r, Lb.lm, Lb.lp, Rb.z, Rb.q, Rb.r, Rb.lm, Rb.lp, zl, zr};
                };
                check(s, x, v, f, r);
            }
            char name[64];
            std::snprintf(name, sizeof name, "hllc_%s_%s", blend ? "blending" : "discontinuous",
                          regime == 0 ? "wet" : regime == 1 ? "left_dry" : "right_dry");
            report(name, s);
        }
    }

    for (int type = 0; type < 4; type++) {  // boundary_flux: x = (z, q, r, lm, lp, zbR)
        for (int wet = 0; wet < 2; wet++) {
            Stats s;
            for (int it = 0; it < N; it++) {
                const double bR = U(1.0, 1.2), phiR = U(0.3, 1.0), zb = U(-0.5, 0.5);
                const double h = wet ? U(0.05, 2.0) : U(0.0, 1e-6);
                const double u = U(-1.5, 1.5), c = std::sqrt(kGravity * h);
                double bcv;
                if (type == 0) bcv = U(-2.0, 2.0);
                else if (type == 1) bcv = U(0.1, 2.0);
                else if (type == 2) bcv = zb + U(0.1, 2.0);
                else bcv = U(0.05, 0.95);
                Vec x{h + zb, h * u, h * U(-1, 1), u - c, u + c, zb};
                Vec v = rand_dir(6);
                if (!wet) v[0] = v[5] = 0.0;
                auto f = [&](const Vec& x) {
                    SideState S{x[0], x[1], x[2], x[3], x[4]};
                    double f1, f2, f3;
                    boundary_flux(bR, phiR, x[5], S, type, bcv, 1e-5, &f1, &f2, &f3);
                    return Vec{f1, f2, f3};
                };
                auto r = [&](const Vec& x, const Vec& w) {
                    SideState S{x[0], x[1], x[2], x[3], x[4]};
                    SideBar sb{0, 0, 0, 0, 0};
                    double zbb = 0.0;
                    boundary_flux_rev(bR, phiR, x[5], S, type, bcv, 1e-5, w[0], w[1], w[2], sb, zbb);
                    return Vec{sb.z, sb.q, sb.r, sb.lm, sb.lp, zbb};
                };
                check(s, x, v, f, r);
            }
            char name[64];
            std::snprintf(name, sizeof name, "boundary_flux_%s_%s", type == 0 ? "q" : type == 1 ? "h" : type == 2 ? "z" : "fr",
                          wet ? "wet" : "dry");
            report(name, s);
        }
    }

    for (int fric = 0; fric < 4; fric++) {  // update_cell: x = (hB, qB, rB, k1, k2)
        for (int hl = 0; hl < 2; hl++) {
            for (int cap = 0; cap < 2; cap++) {
                Stats s;
                for (int it = 0; it < N; it++) {
                    UpdateParams p;
                    p.friction = fric;
                    p.head_loss = hl;
                    p.clamp_negative = true;
                    p.flush_branch = false;
                    p.h_min = 1e-5;
                    p.v_max = cap ? 0.5 : 100.0;
                    p.fr_max = cap ? ((it & 1) ? 0.3 : 100.0) : 100.0;
                    p.dt = U(0.01, 0.5);
                    const double a = U(0, 6.283);
                    p.fcos = std::cos(a);
                    p.fsin = std::sin(a);
                    p.hs = U(0.0, 0.5);
                    p.hk1 = U(0.0, 2.0);
                    p.hk2 = U(0.0, 2.0);
                    const double b2 = U(0, 6.283);
                    p.hcos = std::cos(b2);
                    p.hsin = std::sin(b2);
                    const double k = fric == 2 ? U(0.01, 0.08) : fric == 3 ? U(10.0, 80.0) : U(20.0, 80.0);
                    Vec x{U(0.05, 2.0), U(-2, 2), U(-2, 2), k, k * U(0.8, 1.2)};
                    auto f = [&](const Vec& x) {
                        UpdateParams q = p;
                        q.k1 = x[3];
                        q.k2 = x[4];
                        // forward: the same sequence as k_update after the balance
                        double hh = x[0], qq = x[1], rr = x[2];
                        double hb, qb, rb, k1b = 0, k2b = 0;
                        (void)hb;
                        (void)qb;
                        (void)rb;
                        (void)k1b;
                        (void)k2b;
                        if (std::fabs(hh) < kSmallReal) hh = 0.;
                        if (std::fabs(qq) < kSmallReal) qq = 0.;
                        if (std::fabs(rr) < kSmallReal) rr = 0.;
                        if (hh < 0.) hh = qq = rr = 0.;
                        const double hthr = smax(q.h_min, kSmallReal);
                        if (q.friction) {
                            if (hh > hthr) {
                                double u = qq / hh, v = rr / hh;
                                double ul = u * q.fcos + v * q.fsin, vl = -u * q.fsin + v * q.fcos;
                                double un = std::sqrt(u * u + v * v);
                                ul *= friction_factor(q.friction, q.k1, hh, un, q.dt);
                                vl *= friction_factor(q.friction, q.k2, hh, un, q.dt);
                                qq = (ul * q.fcos - vl * q.fsin) * hh;
                                rr = (ul * q.fsin + vl * q.fcos) * hh;
                            } else {
                                qq = rr = 0.;
                            }
                        }
                        if (q.head_loss) {
                            double qx = qq * q.hcos + rr * q.hsin, qy = -qq * q.hsin + rr * q.hcos;
                            if (hh > hthr) {
                                double ax = 0, ay = 0;
                                if (hh > q.hs) {
                                    ax = std::sqrt(qx * qx + qy * qy) * q.hk1 / hh;
                                    ay = std::sqrt(qx * qx + qy * qy) * q.hk2 / hh;
                                }
                                qx = qx * sw2d_exp(-ax * q.dt);
                                qy = qy * sw2d_exp(-ay * q.dt);
                            } else {
                                qx = qy = 0.;
                            }
                            qq = qx * q.hcos - qy * q.hsin;
                            rr = qx * q.hsin + qy * q.hcos;
                        }
                        if (hh > q.h_min) {
                            double qn = std::sqrt(qq * qq + rr * rr), cc = std::sqrt(kGravity * hh);
                            double Fr = qn / cc / hh;
                            double fact = smax(qn / (hh * q.v_max), Fr / q.fr_max);
                            if (fact > 1.0) {
                                qq = qq / fact;
                                rr = rr / fact;
                            }
                        }
                        return Vec{hh, qq, rr};
                    };
                    auto r = [&](const Vec& x, const Vec& w) {
                        UpdateParams q = p;
                        q.k1 = x[3];
                        q.k2 = x[4];
                        double hb, qb, rb, k1b = 0, k2b = 0;
                        update_cell_rev(q, x[0], x[1], x[2], w[0], w[1], w[2], hb, qb, rb, k1b, k2b);
                        return Vec{hb, qb, rb, k1b, k2b};
                    };
                    check(s, x, rand_dir(5), f, r);
                }
                char name[64];
                std::snprintf(name, sizeof name, "update_friction%d_headloss%d_cap%d", fric, hl, cap);
                report(name, s);
            }
        }
    }

    for (int n = 2; n <= 6; n++) {  // slopes: x = (zc, zj...)
        Stats s;
        for (int it = 0; it < N; it++) {
            SlopeNbr nb[kMaxNbr];
            for (int k = 0; k < n; k++) {
                const double a = 6.283 * k / n + U(-0.3, 0.3), d = U(0.5, 1.5);
                nb[k].dx = d * std::cos(a);
                nb[k].dy = d * std::sin(a);
                nb[k].ax = 0.5 * nb[k].dx + U(-0.1, 0.1);
                nb[k].ay = 0.5 * nb[k].dy + U(-0.1, 0.1);
                nb[k].c_is_r = (it >> k) & 1;
            }
            Vec x(n + 1);
            x[0] = U(-1, 1);
            for (int k = 0; k < n; k++) x[k + 1] = x[0] + U(-1, 1);
            auto f = [&](const Vec& x) {
                SlopeNbr loc[kMaxNbr];
                for (int k = 0; k < n; k++) {
                    loc[k] = nb[k];
                    loc[k].zj = x[k + 1];
                }
                double sx, sy, a[kMaxNbr], b[kMaxNbr];
                slopes_fwd(x[0], n, loc, sx, sy, a, b);
                return Vec{sx, sy};
            };
            auto r = [&](const Vec& x, const Vec& w) {
                SlopeNbr loc[kMaxNbr];
                for (int k = 0; k < n; k++) {
                    loc[k] = nb[k];
                    loc[k].zj = x[k + 1];
                }
                double zcb = 0.0, zjb[kMaxNbr];
                slopes_rev(x[0], n, loc, w[0], w[1], zcb, zjb);
                Vec out(n + 1);
                out[0] = zcb;
                for (int k = 0; k < n; k++) out[k + 1] = zjb[k];
                return out;
            };
            check(s, x, rand_dir(n + 1), f, r);
        }
        char name[64];
        std::snprintf(name, sizeof name, "slopes_n%d", n);
        report(name, s);
    }
    return 0;
}
