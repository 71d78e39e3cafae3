// Whole-step check of the differentiated step's reverse sweep, on the host: a small triangulated
// channel, N steps of the _E step (the device functions of spe_math.cuh and the slope functions of
// sp_adjoint.cuh, composed in plain loops in the same order as the CUDA kernels of sw2d_assim.cu),
// and the reverse of those steps composed the same way as the reverse kernels.  The gradient of a
// misfit J(phi, h0) is compared with central differences in random directions.
//
// Output: "name samples failures max_rel_err" per scheme.
#include <cmath>
#include <cstdio>
#include <map>
#include <random>
#include <vector>

#include "spe_math.cuh"
#include "sp_adjoint.cuh"

using namespace sw2d;
using Vec = std::vector<double>;

struct double4 {
    double x, y, z, w;
};

struct Mesh {
    int nc = 0, ni = 0, nb = 0;
    Vec area, cx, cy, zb;
    std::vector<int> L, R, bc;
    Vec nx, ny, len, mx, my, bnx, bny, blen;
    std::vector<std::vector<int>> bnd_of, int_of;   // per cell, edge indices in increasing order
};

// nx * ny squares of side 1, each cut into two triangles; bed sloping in x with a bump
static Mesh make_mesh(int nx, int ny)
{
    Mesh m;
    auto node = [&](int i, int j) { return j * (nx + 1) + i; };
    std::vector<double> X((nx + 1) * (ny + 1)), Y(X.size());
    for (int j = 0; j <= ny; j++)
        for (int i = 0; i <= nx; i++) {
            X[node(i, j)] = i + 0.13 * std::sin(1.7 * i + 2.3 * j) * (i > 0 && i < nx);
            Y[node(i, j)] = j + 0.11 * std::cos(2.1 * i + 1.3 * j) * (j > 0 && j < ny);
        }
    std::vector<std::vector<int>> tri;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            tri.push_back({node(i, j), node(i + 1, j), node(i + 1, j + 1)});
            tri.push_back({node(i, j), node(i + 1, j + 1), node(i, j + 1)});
        }
    m.nc = (int)tri.size();
    std::map<std::pair<int, int>, std::vector<int>> edges;
    for (int c = 0; c < m.nc; c++) {
        const auto& t = tri[c];
        const double a = 0.5 * ((X[t[1]] - X[t[0]]) * (Y[t[2]] - Y[t[0]]) - (X[t[2]] - X[t[0]]) * (Y[t[1]] - Y[t[0]]));
        m.area.push_back(std::fabs(a));
        const double cx = (X[t[0]] + X[t[1]] + X[t[2]]) / 3.0, cy = (Y[t[0]] + Y[t[1]] + Y[t[2]]) / 3.0;
        m.cx.push_back(cx);
        m.cy.push_back(cy);
        m.zb.push_back(0.02 * (nx - cx) + 0.05 * std::exp(-((cx - 0.5 * nx) * (cx - 0.5 * nx) + (cy - 0.5 * ny) * (cy - 0.5 * ny)) / 2.0));
        for (int k = 0; k < 3; k++) {
            int a0 = t[k], a1 = t[(k + 1) % 3];
            edges[{std::min(a0, a1), std::max(a0, a1)}].push_back(c);
        }
    }
    m.bnd_of.resize(m.nc);
    m.int_of.resize(m.nc);
    for (auto& kv : edges) {
        const int a0 = kv.first.first, a1 = kv.first.second;
        const double ex = X[a1] - X[a0], ey = Y[a1] - Y[a0], l = std::sqrt(ex * ex + ey * ey);
        double nxx = ey / l, nyy = -ex / l;
        const double mxx = 0.5 * (X[a0] + X[a1]), myy = 0.5 * (Y[a0] + Y[a1]);
        const int c0 = kv.second[0];
        if ((mxx - m.cx[c0]) * nxx + (myy - m.cy[c0]) * nyy < 0) nxx = -nxx, nyy = -nyy;  // away from c0
        if (kv.second.size() == 2) {
            m.int_of[c0].push_back(m.ni);
            m.int_of[kv.second[1]].push_back(m.ni);
            m.L.push_back(c0);
            m.R.push_back(kv.second[1]);
            m.nx.push_back(nxx);
            m.ny.push_back(nyy);
            m.len.push_back(l);
            m.mx.push_back(mxx);
            m.my.push_back(myy);
            m.ni++;
        } else {
            m.bnd_of[c0].push_back(m.nb);
            m.bc.push_back(c0);
            m.bnx.push_back(-nxx);   // into the domain
            m.bny.push_back(-nyy);
            m.blen.push_back(l);
            m.nb++;
        }
    }
    return m;
}

struct Step {
    int scheme;  // 0 godunov, 1 muscl
    double dt;
};

// state: h, q, r per cell
struct State {
    Vec h, q, r;
};

static void slopes_all(const Mesh& m, const State& s, Vec& sx, Vec& sy)
{
    sx.assign(m.nc, 0.0);
    sy.assign(m.nc, 0.0);
    for (int c = 0; c < m.nc; c++) {
        SlopeNbr nb[kMaxNbr];
        int n = 0;
        for (int e : m.int_of[c]) {
            const bool is_r = m.R[e] == c;
            const int j = is_r ? m.L[e] : m.R[e];
            nb[n].zj = s.h[j] + m.zb[j];
            nb[n].dx = m.cx[j] - m.cx[c];
            nb[n].dy = m.cy[j] - m.cy[c];
            nb[n].ax = m.mx[e] - m.cx[c];
            nb[n].ay = m.my[e] - m.cy[c];
            nb[n].c_is_r = is_r;
            n++;
        }
        double sxk[kMaxNbr], syk[kMaxNbr];
        slopes_fwd(s.h[c] + m.zb[c], n, nb, sx[c], sy[c], sxk, syk);
    }
}

struct EdgeRec {
    spe::ESide SL, SR;
    spe::EFlux f;
};

static void sides(const Mesh& m, const State& s, const Vec& sx, const Vec& sy, int e, int scheme, double dt,
                  spe::ESide& SL, spe::ESide& SR)
{
    const int a = m.L[e], b = m.R[e];
    if (scheme == 0) {
        SL = spe::god_side(s.h[a], s.q[a], s.r[a], m.zb[a], 1.0, m.nx[e], m.ny[e], 1e-5);
        SR = spe::god_side(s.h[b], s.q[b], s.r[b], m.zb[b], 1.0, m.nx[e], m.ny[e], 1e-5);
    } else {
        SL = spe::evr_side(true, s.h[a], s.q[a], s.r[a], m.zb[a], 1.0, s.h[a] + m.zb[a], sx[a], sy[a], m.mx[e] - m.cx[a],
                           m.my[e] - m.cy[a], m.nx[e], m.ny[e], dt);
        SR = spe::evr_side(false, s.h[b], s.q[b], s.r[b], m.zb[b], 1.0, s.h[b] + m.zb[b], sx[b], sy[b], m.mx[e] - m.cx[b],
                           m.my[e] - m.cy[b], m.nx[e], m.ny[e], dt);
    }
}

static double coefv(const Mesh& m, double w, int c, const Vec& phi) { return (phi[c] > 1e-16) ? w / m.area[c] / phi[c] : 0.0; }

// one step; bal = raw post-balance state
static void step_fwd(const Mesh& m, const Vec& phi, State& s, int scheme, double dt, State* bal)
{
    Vec sx, sy;
    if (scheme) slopes_all(m, s, sx, sy);
    std::vector<double4> slot_int(2 * m.ni), slot_bnd(m.nb);
    for (int e = 0; e < m.ni; e++) {
        spe::ESide SL, SR;
        sides(m, s, sx, sy, e, scheme, dt, SL, SR);
        const int a = m.L[e], b = m.R[e];
        const spe::EFlux f = spe::hllc(1.0, 1.0, phi[a], phi[b], m.zb[a], m.zb[b], SL, SR, 1e-5, 1e-16);
        const double nx = m.nx[e], ny = m.ny[e];
        double c = coefv(m, m.len[e], a, phi);
        slot_int[2 * e] = double4{f.f1, (-c * nx) * f.f2 + (c * nx) * f.sl + (c * ny) * f.f3,
                                  (-c * ny) * f.f2 + (c * ny) * f.sl + (-c * nx) * f.f3, -c};
        c = coefv(m, m.len[e], b, phi);
        slot_int[2 * e + 1] = double4{f.f1, (c * nx) * f.f2 + (c * nx) * f.sr + (-c * ny) * f.f3,
                                      (c * ny) * f.f2 + (c * ny) * f.sr + (c * nx) * f.f3, c};
    }
    for (int e = 0; e < m.nb; e++) {
        const int c = m.bc[e];
        const spe::ESide S = scheme ? spe::evr_bnd_side(s.h[c], s.q[c], s.r[c], m.zb[c], 1.0, m.bnx[e], m.bny[e])
                                    : spe::god_side(s.h[c], s.q[c], s.r[c], m.zb[c], 1.0, m.bnx[e], m.bny[e], 1e-5);
        const spe::EBndFlux F = spe::boundary_flux(1.0, phi[c], m.zb[c], S, 0, 0.0, 1e-5, 1e-16);
        const double cf = coefv(m, m.blen[e], c, phi), nx = m.bnx[e], ny = m.bny[e];
        slot_bnd[e] = double4{cf * F.f1, (cf * nx) * F.f2 + (cf * nx) * 0.0 + (-cf * ny) * F.f3,
                              (cf * ny) * F.f2 + (cf * ny) * 0.0 + (cf * nx) * F.f3, 1.0};
    }
    State o = s;
    for (int c = 0; c < m.nc; c++) {
        double hh = s.h[c], qq = s.q[c], rr = s.r[c];
        auto add = [&](const double4& v) {
            hh += v.w * (v.x * dt);
            qq += v.y * dt;
            rr += v.z * dt;
        };
        for (int e : m.bnd_of[c]) add(slot_bnd[e]);
        for (int e : m.int_of[c]) add(slot_int[2 * e + (m.R[e] == c ? 1 : 0)]);
        if (bal) {
            bal->h[c] = hh;
            bal->q[c] = qq;
            bal->r[c] = rr;
        }
        spe::ECellParams p{};
        p.h_min = 1e-5;
        spe::cell_update(hh, qq, rr, p, dt);
        o.h[c] = hh;
        o.q[c] = qq;
        o.r[c] = rr;
    }
    s = o;
}

static double misfit(const State& s, const Vec& w, const Vec& obs)
{
    double J = 0.0;
    for (size_t c = 0; c < s.h.size(); c++) J += w[c] * (s.h[c] - obs[c]) * (s.h[c] - obs[c]);
    return J;
}

static double run(const Mesh& m, const Vec& phi, State s, int scheme, const Vec& dts, const Vec& w, const Vec& obs)
{
    for (double dt : dts) step_fwd(m, phi, s, scheme, dt, nullptr);
    return misfit(s, w, obs);
}

// gradient of run() with respect to phi and h0, composed as the reverse kernels are
static void grad(const Mesh& m, const Vec& phi, const State& s0, int scheme, const Vec& dts, const Vec& w,
                 const Vec& obs, Vec& gphi, Vec& gh0)
{
    const int N = (int)dts.size();
    std::vector<State> st(N + 1), bal(N);
    st[0] = s0;
    for (int j = 0; j < N; j++) {
        st[j + 1] = st[j];
        bal[j] = st[j];
        step_fwd(m, phi, st[j + 1], scheme, dts[j], &bal[j]);
    }
    State lam{Vec(m.nc, 0.0), Vec(m.nc, 0.0), Vec(m.nc, 0.0)};
    for (int c = 0; c < m.nc; c++) lam.h[c] = 2.0 * w[c] * (st[N].h[c] - obs[c]);
    gphi.assign(m.nc, 0.0);
    for (int j = N - 1; j >= 0; j--) {
        const double dt = dts[j];
        const State& s = st[j];
        // k_e_update_rev
        State lb = lam;
        for (int c = 0; c < m.nc; c++) {
            spe::ECellParams p{};
            p.h_min = 1e-5;
            double k1b = 0, k2b = 0;
            spe::cell_update_rev(bal[j].h[c], bal[j].q[c], bal[j].r[c], p, dt, lb.h[c], lb.q[c], lb.r[c], k1b, k2b);
        }
        lam = lb;
        Vec sx, sy, sxb(m.nc, 0.0), syb(m.nc, 0.0);
        if (scheme) slopes_all(m, s, sx, sy);
        // k_e_edges_rev + k_e_cells_rev (accumulated directly)
        for (int e = 0; e < m.ni; e++) {
            spe::ESide SL, SR;
            sides(m, s, sx, sy, e, scheme, dt, SL, SR);
            const int a = m.L[e], b = m.R[e];
            const spe::EFlux f = spe::hllc(1.0, 1.0, phi[a], phi[b], m.zb[a], m.zb[b], SL, SR, 1e-5, 1e-16);
            const double nx = m.nx[e], ny = m.ny[e];
            const double cL = coefv(m, m.len[e], a, phi), cR = coefv(m, m.len[e], b, phi);
            spe::EFlux fb;
            fb.f1 = dt * (-cL * lb.h[a] + cR * lb.h[b]);
            fb.f2 = dt * (cL * (-nx * lb.q[a] - ny * lb.r[a]) + cR * (nx * lb.q[b] + ny * lb.r[b]));
            fb.f3 = dt * (cL * (ny * lb.q[a] - nx * lb.r[a]) + cR * (-ny * lb.q[b] + nx * lb.r[b]));
            fb.sl = dt * cL * (nx * lb.q[a] + ny * lb.r[a]);
            fb.sr = dt * cR * (nx * lb.q[b] + ny * lb.r[b]);
            const double cLb = dt * (-f.f1 * lb.h[a] + (-nx * f.f2 + nx * f.sl + ny * f.f3) * lb.q[a] +
                                     (-ny * f.f2 + ny * f.sl - nx * f.f3) * lb.r[a]);
            const double cRb = dt * (f.f1 * lb.h[b] + (nx * f.f2 + nx * f.sr - ny * f.f3) * lb.q[b] +
                                     (ny * f.f2 + ny * f.sr + nx * f.f3) * lb.r[b]);
            double pLb = (phi[a] > 1e-16) ? -cLb * cL / phi[a] : 0.0;
            double pRb = (phi[b] > 1e-16) ? -cRb * cR / phi[b] : 0.0;
            spe::ESideBar Lb{0, 0, 0, 0, 0}, Rb{0, 0, 0, 0, 0};
            spe::hllc_rev(1.0, 1.0, phi[a], phi[b], m.zb[a], m.zb[b], SL, SR, 1e-5, 1e-16, fb, pLb, pRb, Lb, Rb);
            gphi[a] += pLb;
            gphi[b] += pRb;
            if (scheme == 0) {
                spe::god_side_rev(s.h[a], s.q[a], s.r[a], 1.0, nx, ny, 1e-5, Lb, lam.h[a], lam.q[a], lam.r[a]);
                spe::god_side_rev(s.h[b], s.q[b], s.r[b], 1.0, nx, ny, 1e-5, Rb, lam.h[b], lam.q[b], lam.r[b]);
            } else {
                double zcb = 0;
                spe::evr_side_rev(true, s.h[a], s.q[a], s.r[a], m.zb[a], 1.0, s.h[a] + m.zb[a], sx[a], sy[a],
                                  m.mx[e] - m.cx[a], m.my[e] - m.cy[a], nx, ny, dt, Lb, lam.h[a], lam.q[a], lam.r[a], zcb,
                                  sxb[a], syb[a]);
                lam.h[a] += zcb;
                zcb = 0;
                spe::evr_side_rev(false, s.h[b], s.q[b], s.r[b], m.zb[b], 1.0, s.h[b] + m.zb[b], sx[b], sy[b],
                                  m.mx[e] - m.cx[b], m.my[e] - m.cy[b], nx, ny, dt, Rb, lam.h[b], lam.q[b], lam.r[b], zcb,
                                  sxb[b], syb[b]);
                lam.h[b] += zcb;
            }
        }
        for (int e = 0; e < m.nb; e++) {
            const int c = m.bc[e];
            const spe::ESide S = scheme ? spe::evr_bnd_side(s.h[c], s.q[c], s.r[c], m.zb[c], 1.0, m.bnx[e], m.bny[e])
                                        : spe::god_side(s.h[c], s.q[c], s.r[c], m.zb[c], 1.0, m.bnx[e], m.bny[e], 1e-5);
            const spe::EBndFlux F = spe::boundary_flux(1.0, phi[c], m.zb[c], S, 0, 0.0, 1e-5, 1e-16);
            const double cf = coefv(m, m.blen[e], c, phi), nx = m.bnx[e], ny = m.bny[e];
            const double f1b = cf * dt * lb.h[c], f2b = dt * cf * (nx * lb.q[c] + ny * lb.r[c]);
            const double f3b = dt * cf * (-ny * lb.q[c] + nx * lb.r[c]);
            const double cfb = dt * (F.f1 * lb.h[c] + (nx * F.f2 - ny * F.f3) * lb.q[c] + (ny * F.f2 + nx * F.f3) * lb.r[c]);
            double pb = (phi[c] > 1e-16) ? -cfb * cf / phi[c] : 0.0;
            spe::ESideBar Sb{0, 0, 0, 0, 0};
            spe::boundary_flux_rev(1.0, phi[c], m.zb[c], S, 0, 0.0, 1e-5, 1e-16, f1b, f2b, f3b, pb, Sb);
            gphi[c] += pb;
            if (scheme) spe::evr_bnd_side_rev(s.h[c], s.q[c], s.r[c], 1.0, nx, ny, Sb, lam.h[c], lam.q[c], lam.r[c]);
            else spe::god_side_rev(s.h[c], s.q[c], s.r[c], 1.0, nx, ny, 1e-5, Sb, lam.h[c], lam.q[c], lam.r[c]);
        }
        // k_limiter_rev + k_nbr_rev: the slope of each cell depends on its own z and its neighbours'
        if (scheme) {
            for (int c = 0; c < m.nc; c++) {
                SlopeNbr nb[kMaxNbr];
                int n = 0, js[kMaxNbr];
                for (int e : m.int_of[c]) {
                    const bool is_r = m.R[e] == c;
                    const int j = is_r ? m.L[e] : m.R[e];
                    js[n] = j;
                    nb[n].zj = s.h[j] + m.zb[j];
                    nb[n].dx = m.cx[j] - m.cx[c];
                    nb[n].dy = m.cy[j] - m.cy[c];
                    nb[n].ax = m.mx[e] - m.cx[c];
                    nb[n].ay = m.my[e] - m.cy[c];
                    nb[n].c_is_r = is_r;
                    n++;
                }
                double zcb = 0.0, zjb[kMaxNbr];
                slopes_rev(s.h[c] + m.zb[c], n, nb, sxb[c], syb[c], zcb, zjb);
                lam.h[c] += zcb;
                for (int k = 0; k < n; k++) lam.h[js[k]] += zjb[k];
            }
        }
    }
    gh0 = lam.h;
}

int main()
{
    std::mt19937_64 rng(77);
    std::normal_distribution<double> N01(0.0, 1.0);
    std::uniform_real_distribution<double> U01(0.0, 1.0);
    const Mesh m = make_mesh(8, 5);
    for (int scheme = 0; scheme < 2; scheme++) {
        int samples = 0, fails = 0;
        double worst = 0.0;
        for (int trial = 0; trial < 6; trial++) {
            Vec phi(m.nc), w(m.nc), obs(m.nc);
            State s0{Vec(m.nc), Vec(m.nc), Vec(m.nc)};
            for (int c = 0; c < m.nc; c++) {
                phi[c] = 0.6 + 0.4 * U01(rng);
                s0.h[c] = 0.3 + 0.1 * std::sin(1.3 * m.cx[c] + 0.7 * m.cy[c] + trial) - m.zb[c] + 0.05;
                s0.q[c] = 0.05 * std::cos(0.9 * m.cx[c] - trial);
                s0.r[c] = 0.03 * std::sin(1.1 * m.cy[c] + trial);
                w[c] = 0.5 + U01(rng);
                obs[c] = s0.h[c] + 0.02 * N01(rng);
            }
            Vec dts(12);
            for (double& d : dts) d = 0.02 + 0.02 * U01(rng);
            Vec gphi, gh0;
            grad(m, phi, s0, scheme, dts, w, obs, gphi, gh0);
            for (int dir = 0; dir < 3; dir++) {
                Vec dp(m.nc), dh(m.nc);
                for (int c = 0; c < m.nc; c++) {
                    dp[c] = N01(rng);
                    dh[c] = N01(rng);
                }
                double ad = 0.0;
                for (int c = 0; c < m.nc; c++) ad += gphi[c] * dp[c] + gh0[c] * dh[c];
                double best = 1e300;
                for (double eps : {1e-5, 1e-6, 1e-7}) {
                    Vec pp = phi, pm = phi;
                    State sp = s0, sm = s0;
                    for (int c = 0; c < m.nc; c++) {
                        pp[c] += eps * dp[c];
                        pm[c] -= eps * dp[c];
                        sp.h[c] += eps * dh[c];
                        sm.h[c] -= eps * dh[c];
                    }
                    const double fd = (run(m, pp, sp, scheme, dts, w, obs) - run(m, pm, sm, scheme, dts, w, obs)) / (2 * eps);
                    best = std::min(best, std::fabs(fd - ad) / std::max(std::fabs(fd), 1e-12));
                }
                samples++;
                if (!(best < 1e-6)) fails++;
                worst = std::max(worst, best);
            }
        }
        std::printf("%s %d %d %.3e\n", scheme ? "step_muscl_evr" : "step_godunov", samples, fails, worst);
    }
    return 0;
}
