// sw2d_case.cpp — case-folder loader of the C ABI: reads an SW2D case folder the way
// sw2dSolver's init does and creates the model it names (SP, DIP or DDP).  Host code only.
//
// Files and the reference readers they restate (paths relative to the reference project):
//   input/input.solv                      swSolverParam::readInputFile   src/sw2dSolver/common/swSolverParam.cpp:663-890
//   input/geometry.sw2d (version 2)       swMesh::readGeometryFileV2     src/common/geometry/swMesh.cpp:213-471
//   per-cell / per-edge parameter maps    swIO::readVectorParameterFile  src/common/swIO.cpp:1005-1191
//   input/hydro_boundary_time_series.txt  swIO::readBoundaryTimeSeriesFile src/common/swIO.cpp:687-817
//   DDP porosity-law maps                 swDdp::readPorosityFile        src/sw2dSolver/models/ddp/swDdp.cpp:1289-1481
// and the model set-up they feed: swSp::init / setInitialConditions (sp/swSp.cpp:720-969,
// 1119-1224), swDip::init (dip/swDip.cpp:900-1030), swDdp::init (ddp/swDdp.cpp:780-991).
// Numbers are parsed with strtod, which rounds correctly as the reference's std::stod does.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sw2d_b200.h"

struct sw2d_case {
    std::string folder;
    std::map<std::string, std::string> opts;  // input.solv, keys lower-cased
    int model = 0;                            // 0 sp, 1 dip, 2 ddp
    // mesh
    int64_t nc = 0, ni = 0, nb = 0;
    std::vector<double> area, cx, cy, zb;
    std::vector<int64_t> lr, bcell;
    std::vector<double> ilen, inx, iny, imx, imy, imz, blen, bnx, bny, bmz;
    std::vector<int32_t> bcode, bbc;
    // fields
    std::vector<double> phi, bous, f1, f2, fa, hs, hk1, hk2, ha, mu1, mu2, mua, pgi, pgb;
    std::vector<double> h0, q0, r0;  // SP/DIP: h, q, r; DDP: the initial-condition columns as read
    int32_t ic_columns = 0;
    // boundary series
    std::vector<int32_t> bc_codes, bc_type;
    std::vector<int64_t> bc_off;
    std::vector<double> bc_t, bc_v;
    // DDP laws
    std::vector<int64_t> lc_off, li_off, lb_off;
    std::vector<double> lc_val, li_val, lb_val;
};

namespace {

std::string g_case_error;

struct Fail {
    std::string msg;
};

[[noreturn]] void fail(const std::string& m) { throw Fail{m}; }

std::string read_line(std::ifstream& f)
{
    std::string s;
    std::getline(f, s);
    while (!s.empty() && (s.back() == '\r' || s.back() == '\n')) s.pop_back();
    return s;
}

// tokens of swIO::stringSplit: maximal runs of [a-zA-Z0-9-_.+]
std::vector<std::string> tokens(const std::string& s)
{
    std::vector<std::string> out;
    std::string cur;
    for (char ch : s) {
        const bool in = std::isalnum((unsigned char)ch) || ch == '-' || ch == '_' || ch == '.' || ch == '+';
        if (in) {
            cur += ch;
        } else if (!cur.empty()) {
            out.push_back(cur);
            cur.clear();
        }
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
}

// whitespace split (swString::splitStr with \s+ after trim)
std::vector<std::string> words(const std::string& s)
{
    std::vector<std::string> out;
    std::string cur;
    for (char ch : s) {
        if (std::isspace((unsigned char)ch)) {
            if (!cur.empty()) {
                out.push_back(cur);
                cur.clear();
            }
        } else {
            cur += ch;
        }
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
}

double to_double(const std::string& s, const std::string& where)
{
    char* end = nullptr;
    const double v = std::strtod(s.c_str(), &end);
    if (end == s.c_str() || *end != '\0') fail(where + ": cannot read a number from '" + s + "'");
    return v;
}

long to_int(const std::string& s, const std::string& where)
{
    char* end = nullptr;
    const long v = std::strtol(s.c_str(), &end, 10);
    if (end == s.c_str() || *end != '\0') fail(where + ": cannot read an integer from '" + s + "'");
    return v;
}

std::string lower(std::string s)
{
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

std::string input_path(const sw2d_case& c, const std::string& name) { return c.folder + "/input/" + name; }

// ---- input.solv
void read_solv(sw2d_case& c)
{
    const std::string p = input_path(c, "input.solv");
    std::ifstream f(p);
    if (!f) fail("unable to open " + p);
    while (f) {
        std::string ln = read_line(f);
        if (ln.empty() || ln[0] == '#' || ln[0] == '=') continue;
        // an inline "# comment" after the value: the assimilation keys of a case such as
        // sp_toce carry one; the reference's assimilation driver filters those lines before
        // swSolverParam sees them (assim/assimConfig.cpp, AssimConfig::load_and_filter)
        const size_t hash = ln.find('#');
        if (hash != std::string::npos) ln = ln.substr(0, hash);
        const auto w = words(ln);
        if (w.empty()) continue;
        if (w.size() != 2) fail(p + ": line is misformatted: '" + ln + "'");
        c.opts[lower(w[0])] = w[1];
    }
}

std::string opt(const sw2d_case& c, const std::string& k, const std::string& d)
{
    auto it = c.opts.find(k);
    return it == c.opts.end() ? d : it->second;
}

double optd(const sw2d_case& c, const std::string& k, double d)
{
    auto it = c.opts.find(k);
    return it == c.opts.end() ? d : to_double(it->second, "input.solv " + k);
}

// ---- geometry.sw2d version 2
template <class T>
T take(const std::vector<char>& b, size_t& off)
{
    if (off + sizeof(T) > b.size()) fail("geometry.sw2d is truncated");
    T v;
    std::memcpy(&v, b.data() + off, sizeof(T));
    off += sizeof(T);
    return v;
}

void read_geometry(sw2d_case& c)
{
    const std::string p = input_path(c, "geometry.sw2d");
    std::ifstream f(p, std::ios::binary);
    if (!f) fail("unable to open " + p);
    std::vector<char> b((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    size_t off = 0;
    const uint64_t vlen = take<uint64_t>(b, off);
    if (vlen > 16 || off + vlen > b.size()) fail(p + ": bad version header");
    const std::string version(b.data() + off, b.data() + off + vlen);
    off += vlen;
    if (version != "2") fail(p + ": unsupported geometry version '" + version + "'");
    const uint64_t nc = take<uint64_t>(b, off), nb = take<uint64_t>(b, off), ni = take<uint64_t>(b, off);
    const uint64_t nn = take<uint64_t>(b, off), nbnd = take<uint64_t>(b, off);
    c.nc = (int64_t)nc;
    c.nb = (int64_t)nb;
    c.ni = (int64_t)ni;
    std::vector<uint64_t> per_cell(nc);
    c.area.resize(nc);
    c.cx.resize(nc);
    c.cy.resize(nc);
    c.zb.resize(nc);
    for (uint64_t i = 0; i < nc; i++) {  // 6 counters, area, perimeter, x, y, zb (88 bytes)
        take<uint64_t>(b, off);
        take<uint64_t>(b, off);
        const uint64_t nbn = take<uint64_t>(b, off), nbe = take<uint64_t>(b, off), nie = take<uint64_t>(b, off),
                       nne = take<uint64_t>(b, off);
        per_cell[i] = nbn + nbe + nie + nne;
        c.area[i] = take<double>(b, off);
        take<double>(b, off);
        c.cx[i] = take<double>(b, off);
        c.cy[i] = take<double>(b, off);
        c.zb[i] = take<double>(b, off);
    }
    off += nn * 56;  // nodes: idx, sms id, x, y, z, cell and edge counts
    c.bcell.resize(nb);
    c.blen.resize(nb);
    c.bnx.resize(nb);
    c.bny.resize(nb);
    c.bmz.resize(nb);
    c.bcode.resize(nb);
    for (uint64_t e = 0; e < nb; e++) {  // idx, n1, n2, mx, my, mz, d_norm, length, nx, ny, code, cell (92)
        take<uint64_t>(b, off);
        take<uint64_t>(b, off);
        take<uint64_t>(b, off);
        take<double>(b, off);
        take<double>(b, off);
        c.bmz[e] = take<double>(b, off);
        take<double>(b, off);
        c.blen[e] = take<double>(b, off);
        c.bnx[e] = take<double>(b, off);
        c.bny[e] = take<double>(b, off);
        c.bcode[e] = take<int32_t>(b, off);
        const uint64_t cell = take<uint64_t>(b, off);
        if (cell >= nc) fail(p + ": boundary edge refers to a missing cell");
        c.bcell[e] = (int64_t)cell;
    }
    c.lr.resize(2 * ni);
    c.ilen.resize(ni);
    c.inx.resize(ni);
    c.iny.resize(ni);
    c.imx.resize(ni);
    c.imy.resize(ni);
    c.imz.resize(ni);
    for (uint64_t e = 0; e < ni; e++) {  // idx, n1, n2, mx, my, mz, d_norm, length, nx, ny, c0, c1 (96)
        take<uint64_t>(b, off);
        take<uint64_t>(b, off);
        take<uint64_t>(b, off);
        c.imx[e] = take<double>(b, off);
        c.imy[e] = take<double>(b, off);
        c.imz[e] = take<double>(b, off);
        take<double>(b, off);
        c.ilen[e] = take<double>(b, off);
        c.inx[e] = take<double>(b, off);
        c.iny[e] = take<double>(b, off);
        const uint64_t c0 = take<uint64_t>(b, off), c1 = take<uint64_t>(b, off);
        if (c0 >= nc || c1 >= nc) fail(p + ": internal edge refers to a missing cell");
        c.lr[2 * e] = (int64_t)c0;
        c.lr[2 * e + 1] = (int64_t)c1;
    }
    // the per-code edge lists, the codes, the per-cell links and the node-cell lists follow; the
    // step reads none of them
    (void)nbnd;
}

// ---- per-cell / per-edge maps (swIO::readVectorParameterFile)
std::vector<std::vector<double>> read_map(const sw2d_case& c, const std::string& name, size_t n_params,
                                          size_t n_records, std::vector<std::string>* names = nullptr)
{
    const std::string p = input_path(c, name);
    std::ifstream f(p);
    if (!f) fail("unable to open " + p);
    auto head = tokens(read_line(f));
    if (head.size() != 2 || (head[1] != "0" && head[1] != "1")) fail(p + ": bad 'Unif' line");
    const bool unif = head[1] == "1";
    read_line(f);
    auto hdr = tokens(read_line(f));
    if (hdr.size() != n_params) fail(p + ": expecting " + std::to_string(n_params) + " parameters");
    if (names) *names = hdr;
    std::vector<std::vector<double>> out(n_params, std::vector<double>(n_records));
    if (unif) {
        auto v = tokens(read_line(f));
        if (v.size() != n_params) fail(p + ": misformatted uniform line");
        for (size_t k = 0; k < n_params; k++) {
            const double x = to_double(v[k], p);
            for (size_t r = 0; r < n_records; r++) out[k][r] = x;
        }
        return out;
    }
    read_line(f);
    read_line(f);
    for (size_t r = 0; r < n_records; r++) {
        if (!f) fail(p + ": not enough records");
        auto v = tokens(read_line(f));
        if (v.size() != n_params) fail(p + ": misformatted record " + std::to_string(r));
        for (size_t k = 0; k < n_params; k++) out[k][r] = to_double(v[k], p);
    }
    return out;
}

// ---- DDP porosity-law maps (swDdp::readPorosityFile with swDdp::porosityLineSize)
size_t law_length(double law, double n, const std::string& p)
{
    if (law == -2 || law == -1) return (size_t)(2 * (long)n + 2);
    if (law == 0) return (size_t)((long)n + 2);
    if (law == 1) return 4;
    if (law == 2) return 6;
    if (law == 3) return 7;
    fail(p + ": porosity law type not in {-2, -1, 0, 1, 2, 3}");
}

void read_laws(const sw2d_case& c, const std::string& name, size_t n_records, std::vector<int64_t>& off,
               std::vector<double>& val)
{
    const std::string p = input_path(c, name);
    std::ifstream f(p);
    if (!f) fail("unable to open " + p);
    auto head = tokens(read_line(f));
    if (head.size() != 2 || (head[1] != "0" && head[1] != "1")) fail(p + ": bad 'Unif' line");
    const bool unif = head[1] == "1";
    read_line(f);
    read_line(f);
    auto parse = [&](const std::string& ln) {
        auto t = tokens(ln);
        std::vector<double> v;
        for (auto& s : t) v.push_back(to_double(s, p));
        if (v.size() < 2 || v.size() != law_length(v[0], v[1], p))
            fail(p + ": law type is not compatible with the line's parameter count");
        return v;
    };
    off.assign(1, 0);
    val.clear();
    if (unif) {
        const auto v = parse(read_line(f));
        for (size_t r = 0; r < n_records; r++) {
            val.insert(val.end(), v.begin(), v.end());
            off.push_back((int64_t)val.size());
        }
        return;
    }
    read_line(f);
    read_line(f);
    for (size_t r = 0; r < n_records; r++) {
        if (!f) fail(p + ": not enough records");
        const auto v = parse(read_line(f));
        val.insert(val.end(), v.begin(), v.end());
        off.push_back((int64_t)val.size());
    }
}

// ---- boundary series (swIO::readBoundaryTimeSeriesFile)
void read_bc(sw2d_case& c)
{
    const std::string p = input_path(c, "hydro_boundary_time_series.txt");
    std::ifstream f(p);
    if (!f) fail("unable to open " + p);
    read_line(f);
    read_line(f);
    const auto wn = words(read_line(f));
    if (wn.size() != 1) fail(p + ": line 3 must hold the number of series");
    const long ns = to_int(wn[0], p);
    read_line(f);
    const auto codes = words(read_line(f));
    read_line(f);
    const auto types = words(read_line(f));
    if ((long)codes.size() != ns || (long)types.size() != ns) fail(p + ": incorrect number of boundary conditions");
    read_line(f);
    read_line(f);
    std::vector<double> t;
    std::vector<std::vector<double>> v(ns);
    while (f) {
        const std::string ln = read_line(f);
        if (ln.empty()) continue;
        const auto w = words(ln);
        if ((long)w.size() < ns + 1) fail(p + ": misformatted record '" + ln + "'");
        t.push_back(to_double(w[0], p));
        for (long j = 0; j < ns; j++) v[j].push_back(to_double(w[j + 1], p));
    }
    if (t.empty()) fail(p + ": no boundary condition values");
    c.bc_codes.clear();
    c.bc_type.clear();
    c.bc_off.assign(1, 0);
    c.bc_t.clear();
    c.bc_v.clear();
    for (long j = 0; j < ns; j++) {
        c.bc_codes.push_back((int32_t)to_int(codes[j], p));
        const std::string& ty = types[j];
        // the type strings hypBoundaryFlux compares against (sp/swSpHyp.cpp:40-120); any other
        // one is kept as an unknown type, which the step reports where the reference stops
        c.bc_type.push_back(ty == "q" ? SW2D_BC_Q : ty == "h" ? SW2D_BC_H : ty == "z" ? SW2D_BC_Z
                            : ty == "fr" ? SW2D_BC_FR : ty == "phiWq" ? SW2D_BC_PHIWQ : 99);
        c.bc_t.insert(c.bc_t.end(), t.begin(), t.end());
        c.bc_v.insert(c.bc_v.end(), v[j].begin(), v[j].end());
        c.bc_off.push_back((int64_t)c.bc_t.size());
    }
    c.bbc.resize(c.nb);
    for (int64_t e = 0; e < c.nb; e++) {
        int32_t k = -1;
        for (size_t j = 0; j < c.bc_codes.size(); j++)
            if (c.bc_codes[j] == c.bcode[e]) k = (int32_t)j;
        if (k < 0) fail("boundary code " + std::to_string(c.bcode[e]) + " of the mesh has no time series");
        c.bbc[e] = k;
    }
}

int col(const std::vector<std::string>& names, const char* n)
{
    for (size_t i = 0; i < names.size(); i++)
        if (names[i] == n) return (int)i;
    return -1;
}

const char* kFrictionFiles[] = {"", "friction_chezy_map.txt", "friction_manning_map.txt", "friction_strickler_map.txt"};

void read_case(sw2d_case& c)
{
    read_solv(c);
    const std::string hyp = lower(opt(c, "model_hyperb", "swes"));
    if (hyp == "sp") c.model = 0;
    else if (hyp == "dip") c.model = 1;
    else if (hyp == "ddp") c.model = 2;
    else fail("model_hyperb '" + hyp + "': only sp, dip and ddp are implemented");
    read_geometry(c);
    const size_t n = (size_t)c.nc;
    // initial conditions (swSp::setInitialConditions, sp/swSp.cpp:1119-1224; swDdp's,
    // ddp/swDdp.cpp:1608-1726): h or z, then q or u, then r or v
    std::vector<std::string> names;
    auto ic = read_map(c, "initial_conditions_map.txt", 3, n, &names);
    const int ih = col(names, "h"), iz = col(names, "z"), iq = col(names, "q"), iu = col(names, "u");
    const int ir = col(names, "r"), iv = col(names, "v");
    if (ih < 0 && iz < 0) fail("initial conditions: neither h nor z");
    if (iq < 0 && iu < 0) fail("initial conditions: neither q nor u");
    if (ir < 0 && iv < 0) fail("initial conditions: neither r nor v");
    if (c.model == 2) {
        c.h0 = ic[iz >= 0 ? iz : ih];
        c.q0 = ic[iu >= 0 ? iu : iq];
        c.r0 = ic[iv >= 0 ? iv : ir];
        c.ic_columns = (iz >= 0 ? SW2D_DDP_IC_LEVEL_Z : 0) | (iu >= 0 ? SW2D_DDP_IC_X_VELOCITY : 0) |
                       (iv >= 0 ? SW2D_DDP_IC_Y_VELOCITY : 0);
    } else {
        c.h0.assign(n, 0.0);
        if (ih >= 0) c.h0 = ic[ih];
        if (iz >= 0)
            for (size_t i = 0; i < n; i++) c.h0[i] = std::max(ic[iz][i] - c.zb[i], 0.0);
        c.q0 = iq >= 0 ? ic[iq] : std::vector<double>(n);
        if (iu >= 0)
            for (size_t i = 0; i < n; i++) c.q0[i] = c.h0[i] * ic[iu][i];
        c.r0 = ir >= 0 ? ic[ir] : std::vector<double>(n);
        if (iv >= 0)
            for (size_t i = 0; i < n; i++) c.r0[i] = c.h0[i] * ic[iv][i];
    }
    // porosity
    if (c.model == 0) {
        c.phi = read_map(c, "SP_cell_porosity_map.txt", 1, n)[0];
    } else if (c.model == 1) {
        c.phi = read_map(c, "DIP_cell_porosity_map.txt", 1, n)[0];
        c.pgi = read_map(c, "DIP_edge_int_porosity_map.txt", 1, (size_t)c.ni)[0];
        c.pgb = read_map(c, "DIP_edge_bnd_porosity_map.txt", 1, (size_t)c.nb)[0];
    } else {
        c.phi.assign(n, 1.0);
        read_laws(c, "DDP_cell_porosity_map.txt", n, c.lc_off, c.lc_val);
        read_laws(c, "DDP_edge_int_porosity_map.txt", (size_t)c.ni, c.li_off, c.li_val);
        read_laws(c, "DDP_edge_bnd_porosity_map.txt", (size_t)c.nb, c.lb_off, c.lb_val);
    }
    if (c.model != 0 && lower(opt(c, "model_momentum_dissipation", "none")) != "none") {
        auto mu = read_map(c, "cell_momentum_dissipation_map.txt", 3, n);
        c.mu1 = mu[0];
        c.mu2 = mu[1];
        c.mua = mu[2];
    }
    c.bous = read_map(c, "Boussinesq_map.txt", 1, n)[0];
    const std::string fm = lower(opt(c, "model_friction", "none"));
    const int fk = fm == "chezy" ? 1 : fm == "manning" ? 2 : fm == "strickler" ? 3 : fm == "none" ? 0 : -1;
    if (fk < 0) fail("model_friction '" + fm + "' not handled");
    if (fk > 0) {
        auto fr = read_map(c, kFrictionFiles[fk], 3, n);
        c.f1 = fr[0];
        c.f2 = fr[1];
        c.fa = fr[2];
    }
    if (lower(opt(c, "model_singular_head_loss", "none")) != "none") {
        auto hl = read_map(c, "singular_head_loss_map.txt", 4, n);
        c.hs = hl[0];
        c.hk1 = hl[1];
        c.hk2 = hl[2];
        c.ha = hl[3];
    }
    read_bc(c);
}

const double* dp(const std::vector<double>& v) { return v.empty() ? nullptr : v.data(); }

int create(const sw2d_case& c, int device, sw2d_handle** out)
{
    sw2d_mesh m{c.nc, c.ni, c.nb, dp(c.area), dp(c.cx), dp(c.cy), dp(c.zb), c.lr.data(), dp(c.ilen), dp(c.inx),
                dp(c.iny), dp(c.imx), dp(c.imy), c.bcell.data(), dp(c.blen), dp(c.bnx), dp(c.bny), c.bbc.data()};
    // the input.solv keys of this path, defaults of swSolverParam.h:144-194
    const std::string scheme = lower(opt(c, "num_scheme", "godunov"));
    const std::string topo = lower(opt(c, "topo_discretization", "discontinuous"));
    const std::string fm = lower(opt(c, "model_friction", "none"));
    sw2d_params p{};
    p.scheme = scheme == "muscl_evr" ? SW2D_SCHEME_MUSCL_EVR : scheme == "godunov" ? SW2D_SCHEME_GODUNOV : -1;
    p.topo = topo == "blending" ? SW2D_TOPO_BLENDING : topo == "discontinuous" ? SW2D_TOPO_DISCONTINUOUS : -1;
    p.friction = fm == "chezy" ? 1 : fm == "manning" ? 2 : fm == "strickler" ? 3 : 0;
    p.singular_head_loss = lower(opt(c, "model_singular_head_loss", "none")) != "none";
    p.negative_depth_detection = lower(opt(c, "negative_depth_detection", "none")) == "active";
    p.variant = SW2D_VARIANT_NATIVE;
    p.cfl_max = optd(c, "cfl_max", 1.0);
    p.dt_max = optd(c, "dt_max", 10.0);
    p.dt_map = optd(c, "dt_map", 100.0);
    p.h_min = optd(c, "h_min", 1e-5);
    p.phi_min = optd(c, "phi_min", 1e-16);
    p.v_max = optd(c, "v_max", 100.0);
    p.fr_max = optd(c, "fr_max", 100.0);
    p.t_0 = optd(c, "t_0", 0.0);
    p.t_max = optd(c, "t_max", 100.0);
    if (p.scheme < 0) fail("num_scheme '" + scheme + "' not implemented");
    if (p.topo < 0) fail("topo_discretization '" + topo + "' not recognised");
    sw2d_cell_fields f{dp(c.phi), dp(c.bous), dp(c.f1), dp(c.f2), dp(c.fa), dp(c.hs), dp(c.hk1), dp(c.hk2), dp(c.ha)};
    sw2d_bc_table bc{(int32_t)c.bc_codes.size(), c.bc_type.data(), c.bc_off.data(), dp(c.bc_t), dp(c.bc_v)};
    const bool diss = !c.mu1.empty();
    if (c.model == 1) {
        sw2d_dip_fields d{dp(c.pgi), dp(c.pgb), diss ? 1 : 0, dp(c.mu1), dp(c.mu2), dp(c.mua)};
        return sw2d_create_dip(&m, &p, &f, &d, &bc, c.h0.data(), c.q0.data(), c.r0.data(), device, out);
    }
    if (c.model == 2) {
        const std::string div = lower(opt(c, "div_corr", "none"));
        const int dc = div == "none" ? SW2D_DIV_CORR_NONE : div == "limit_flux" ? SW2D_DIV_CORR_LIMIT_FLUX
                     : div == "limit_timestep" ? SW2D_DIV_CORR_LIMIT_TIMESTEP : -1;
        if (dc < 0) fail("div_corr '" + div + "' not in {none, limit_flux, limit_timestep}");
        sw2d_ddp_fields d{};
        d.cell = sw2d_ddp_records{c.lc_off.data(), dp(c.lc_val)};
        d.edge_int = sw2d_ddp_records{c.li_off.data(), dp(c.li_val)};
        d.edge_bnd = sw2d_ddp_records{c.lb_off.data(), dp(c.lb_val)};
        d.edge_int_mz = dp(c.imz);
        d.edge_bnd_mz = dp(c.bmz);
        d.n_por_tab_max = (int64_t)optd(c, "n_por_tab_max", 5);
        d.h_min_ddp = 1e-3;  // no input.solv key in the reference (swSolverParam.h:171)
        d.chi_phi_max = optd(c, "ddp_chi_phi_max", 20.0);
        d.chi_theta_max = optd(c, "ddp_chi_theta_max", 20.0);
        d.div_corr = dc;
        d.ic_columns = c.ic_columns;
        d.n_it_div_max = (int64_t)optd(c, "n_it_div_max", 10);
        d.momentum_dissipation = diss ? 1 : 0;
        d.mu_1 = dp(c.mu1);
        d.mu_2 = dp(c.mu2);
        d.mu_alpha = dp(c.mua);
        return sw2d_create_ddp(&m, &p, &f, &d, &bc, c.h0.data(), c.q0.data(), c.r0.data(), device, out);
    }
    return sw2d_create(&m, &p, &f, &bc, c.h0.data(), c.q0.data(), c.r0.data(), device, out);
}

}  // namespace

extern "C" {

int sw2d_case_read(const char* folder, sw2d_case** out)
{
    if (!folder || !out) {
        g_case_error = "invalid arguments";
        return SW2D_E_ARG;
    }
    *out = nullptr;
    std::unique_ptr<sw2d_case> c(new sw2d_case());
    c->folder = folder;
    try {
        read_case(*c);
    } catch (const Fail& e) {
        g_case_error = e.msg;
        return SW2D_E_ARG;
    } catch (const std::exception& e) {
        g_case_error = e.what();
        return SW2D_E_ARG;
    }
    *out = c.release();
    return SW2D_OK;
}

int64_t sw2d_case_array(const sw2d_case* c, const char* name, double* out, int64_t capacity)
{
    if (!c || !name || !out) return SW2D_E_ARG;
    const std::string n(name);
    std::vector<double> tmp;
    const std::vector<double>* v = nullptr;
    auto from_i = [&](const std::vector<int64_t>& a) { tmp.assign(a.begin(), a.end()); return &tmp; };
    auto from_i32 = [&](const std::vector<int32_t>& a) { tmp.assign(a.begin(), a.end()); return &tmp; };
    if (n == "cell_area") v = &c->area;
    else if (n == "cell_x") v = &c->cx;
    else if (n == "cell_y") v = &c->cy;
    else if (n == "cell_z_b") v = &c->zb;
    else if (n == "edge_int_cells") v = from_i(c->lr);
    else if (n == "edge_int_length") v = &c->ilen;
    else if (n == "edge_int_nx") v = &c->inx;
    else if (n == "edge_int_ny") v = &c->iny;
    else if (n == "edge_int_mx") v = &c->imx;
    else if (n == "edge_int_my") v = &c->imy;
    else if (n == "edge_int_mz") v = &c->imz;
    else if (n == "edge_bnd_cell") v = from_i(c->bcell);
    else if (n == "edge_bnd_length") v = &c->blen;
    else if (n == "edge_bnd_nx") v = &c->bnx;
    else if (n == "edge_bnd_ny") v = &c->bny;
    else if (n == "edge_bnd_mz") v = &c->bmz;
    else if (n == "edge_bnd_code") v = from_i32(c->bcode);
    else if (n == "edge_bnd_series") v = from_i32(c->bbc);
    else if (n == "h0") v = &c->h0;
    else if (n == "q0") v = &c->q0;
    else if (n == "r0") v = &c->r0;
    else if (n == "phi") v = &c->phi;
    else if (n == "boussinesq") v = &c->bous;
    else if (n == "friction_1") v = &c->f1;
    else if (n == "friction_2") v = &c->f2;
    else if (n == "friction_alpha") v = &c->fa;
    else if (n == "hl_h_sing") v = &c->hs;
    else if (n == "hl_coeff_1") v = &c->hk1;
    else if (n == "hl_coeff_2") v = &c->hk2;
    else if (n == "hl_alpha") v = &c->ha;
    else if (n == "mu_1") v = &c->mu1;
    else if (n == "mu_2") v = &c->mu2;
    else if (n == "mu_alpha") v = &c->mua;
    else if (n == "phi_g_int") v = &c->pgi;
    else if (n == "phi_g_bnd") v = &c->pgb;
    else if (n == "bc_times") v = &c->bc_t;
    else if (n == "bc_values") v = &c->bc_v;
    else if (n == "bc_offset") v = from_i(c->bc_off);
    else if (n == "bc_type") v = from_i32(c->bc_type);
    else if (n == "bc_code") v = from_i32(c->bc_codes);
    else if (n == "ddp_cell_offset") v = from_i(c->lc_off);
    else if (n == "ddp_cell_values") v = &c->lc_val;
    else if (n == "ddp_edge_int_offset") v = from_i(c->li_off);
    else if (n == "ddp_edge_int_values") v = &c->li_val;
    else if (n == "ddp_edge_bnd_offset") v = from_i(c->lb_off);
    else if (n == "ddp_edge_bnd_values") v = &c->lb_val;
    if (!v) return SW2D_E_ARG;
    const int64_t len = (int64_t)v->size();
    if (capacity < len) return SW2D_E_ARG;
    if (len) std::memcpy(out, v->data(), len * sizeof(double));
    return len;
}

int sw2d_case_info(const sw2d_case* c, int64_t* sizes)
{
    if (!c || !sizes) return SW2D_E_ARG;
    sizes[0] = c->nc;
    sizes[1] = c->ni;
    sizes[2] = c->nb;
    sizes[3] = c->model;
    sizes[4] = c->ic_columns;
    return SW2D_OK;
}

const char* sw2d_case_option(const sw2d_case* c, const char* key)
{
    if (!c || !key) return nullptr;
    auto it = c->opts.find(lower(key));
    return it == c->opts.end() ? nullptr : it->second.c_str();
}

int sw2d_case_create(const sw2d_case* c, int device, sw2d_handle** out)
{
    if (!c || !out) return SW2D_E_ARG;
    try {
        return create(*c, device, out);
    } catch (const Fail& e) {
        g_case_error = e.msg;
        return SW2D_E_ARG;
    }
}

void sw2d_case_free(sw2d_case* c) { delete c; }

const char* sw2d_case_last_error(void) { return g_case_error.c_str(); }

int sw2d_load_case(const char* folder, int device, sw2d_handle** out)
{
    sw2d_case* c = nullptr;
    int st = sw2d_case_read(folder, &c);
    if (st != SW2D_OK) return st;
    st = sw2d_case_create(c, device, out);
    sw2d_case_free(c);
    return st;
}

}  // extern "C"
