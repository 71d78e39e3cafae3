// Test harness around the reference's differentiated-step layer (assim/swSpE_*.cpp and
// assim/assimConfig.cpp, compiled from the reference sources by oracle/Makefile).  It is a
// checker, never part of the product.
//
// The layer is written for Enzyme: `get_spatial_gradient_checkpointed` calls
// `__enzyme_autodiff` on `ckpt_segment_E`.  Without the Enzyme compiler plugin the gradient
// cannot run, but everything it differentiates can: the dry run `build_checkpoint_records`
// (assim/swSpE_checkpoint.cpp:97-455), the segment function `ckpt_segment_E` as a plain forward
// (:584-715) and the frozen-trajectory cost `replay_trajectory_cost` (:1311-1427).  This file
// supplies the Enzyme globals (an aborting `__enzyme_autodiff`: nothing here may call it) and
// the four members the layer declares but defines in files that need absent libraries
// (swSpE_minimize.cpp: LBFGSpp/Eigen) or nowhere.
//
// C entry points (ctypes):
//   sw2dref_e_open(folder, quiet)      init exactly as assim/main_enzyme.cpp:55-131 does: the
//                                      assimilation keys of input.solv are read by the
//                                      reference's AssimConfig, the native parser reads the
//                                      filtered copy (written under the system temp directory:
//                                      the case folder may be read-only)
//   sw2dref_e_load_observations        the reference's load_all_observations + the pointer set-up
//                                      of main_enzyme.cpp:206-219
//   sw2dref_e_set_frames / _set_gauges observations given directly
//   sw2dref_e_record(m, stride)        update_phi_norm_bounds + build_checkpoint_records
//   sw2dref_e_segment(k, ...)          one recorded segment: t_start, steps, dt, obs triggers,
//                                      checkpoint state
//   sw2dref_e_set_window(...)          the assimilation window and tiles (restated below from
//                                      get_spatial_gradient_checkpointed, which cannot run)
//   sw2dref_e_replay_cost(m)           replay_trajectory_cost (leaves the replayed end state)
//   sw2dref_e_generate_references(m)   the gen-ref-e mode, generate_references_E
//                                      (assim/swSpE_checkpoint.cpp:470-515), writing its maps
//                                      into the handle's own temporary folder
//                                      (sw2dref_e_folder(h)/reference), never the case's
#include <unistd.h>

#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../src/common/swFile.h"
#include "../src/common/swIO.h"
#include "../src/common/swLog.h"
#include "../src/common/swMessage.h"
#include "../src/common/geometry/swMesh.h"
#include "../src/sw2dSolver/common/swSolverParam.h"
#include "swSpE.h"
#include "assimConfig.h"

// ---- what the Enzyme plugin and the absent translation units would provide -------------------
int enzyme_dup, enzyme_const, enzyme_out, enzyme_dupnoneed;
extern "C" void __enzyme_autodiff(void*, ...)
{
    std::fprintf(stderr, "__enzyme_autodiff called in the oracle harness\n");
    std::abort();
}
bool swSpE::begin_reference_generation() { gen_ref_mode = true; n_ref_written = 0; return true; }
bool swSpE::finalize_reference_generation() { gen_ref_mode = false; return true; }
double swSpE::run_pure_simulation(double) { return 0.0; }
// The reader swSpE_minimize.cpp defines (assim/swSpE_minimize.cpp:130-197), for the two formats
// it accepts: the SW2D map format ("Unif ..." first line) through the reference's own
// swIO::readVectorParameterFile, and "cell_id,value" rows with an optional header.
bool swSpE::load_phi_csv(const std::string& filepath, double* out)
{
    std::ifstream f(filepath);
    if (!f) return false;
    std::string first;
    while (std::getline(f, first)) {
        size_t p = first.find_first_not_of(" \t\r\n");
        if (p != std::string::npos) { first = first.substr(p); break; }
    }
    if (first.rfind("Unif", 0) == 0 || first.rfind("unif", 0) == 0) {
        std::vector<std::string> names;
        std::vector<std::vector<double>> arr;
        swIO::readVectorParameterFile(filepath, 1, cell_nb, names, arr);
        if (arr.empty() || arr[0].size() != cell_nb) return false;
        for (size_t i = 0; i < cell_nb; i++) out[i] = arr[0][i];
        return true;
    }
    f.clear();
    f.seekg(0);
    std::string line;
    std::streampos start = f.tellg();
    if (std::getline(f, line)) {
        const bool numeric = !line.empty() && (std::isdigit((unsigned char)line[0]) || line[0] == '-' || line[0] == '+');
        if (numeric) f.seekg(start);
    }
    size_t count = 0;
    while (std::getline(f, line)) {
        if (line.empty()) continue;
        for (char& c : line) if (c == ',') c = ' ';
        std::stringstream ls(line);
        long id;
        double v;
        if (!(ls >> id >> v)) continue;
        if (id < 0 || (size_t)id >= cell_nb) return false;
        out[id] = v;
        count++;
    }
    return count == cell_nb;
}

namespace {

namespace fs = std::filesystem;

// The native members the harness reads are protected in swSp; this subclass republishes them.
class RefE : public swSpE
{
public:
    using swSpE::cell_nb;
    using swSpE::edge_bnd_nb;
    using swSpE::phi;
    using swSpE::t;
    using swSpE::t_0;
    using swSpE::t_max;
    using swSpE::unit_discharge_x;
    using swSpE::unit_discharge_y;
    using swSpE::water_depth;
};

struct HandleE
{
    swIO* io = nullptr;
    RefE* m = nullptr;
    std::ofstream* log = nullptr;
    AssimConfig cfg;
    std::string tmp;
    std::vector<double> times;
    std::vector<std::vector<double>> frames;
    std::vector<const double*> ptrs;
};

struct QuietOut
{
    std::streambuf* so = nullptr;
    std::streambuf* se = nullptr;
    std::ostringstream sink;
    explicit QuietOut(bool on)
    {
        if (on) {
            so = std::cout.rdbuf(sink.rdbuf());
            se = std::cerr.rdbuf(sink.rdbuf());
        }
    }
    ~QuietOut()
    {
        if (so) std::cout.rdbuf(so);
        if (se) std::cerr.rdbuf(se);
    }
};

void wire_observations(HandleE* hd)
{
    hd->ptrs.clear();
    for (auto& f : hd->frames) hd->ptrs.push_back(f.data());
    hd->m->obs_times_vec = hd->times;
    hd->m->current_obs_times = hd->m->obs_times_vec.data();
    hd->m->current_obs_frames = hd->ptrs.data();
    hd->m->current_n_obs = hd->times.size();
}

}  // namespace

extern "C" {

void* sw2dref_e_open(const char* folder, int quiet)
{
    QuietOut qo(quiet != 0);
    HandleE* hd = new HandleE();
    char tmpl[] = "/tmp/sw2dref_e_XXXXXX";
    if (!mkdtemp(tmpl)) return nullptr;
    hd->tmp = tmpl;
    const fs::path user(folder), tmp(hd->tmp);
    std::error_code ec;
    fs::create_directories(tmp / "input", ec);
    for (const auto& e : fs::directory_iterator(user / "input"))
        fs::create_symlink(fs::absolute(e.path()), tmp / "input" / e.path().filename(), ec);
    if (fs::exists(user / "reference")) fs::create_directory_symlink(fs::absolute(user / "reference"), tmp / "reference", ec);
    fs::remove(tmp / "input" / "input.solv", ec);
    if (!hd->cfg.load_and_filter((user / "input" / "input.solv").string(), (tmp / "input" / "input.solv").string()))
        return nullptr;
    hd->io = new swIO(hd->tmp);
    hd->io->createEmptyFolders(swFile::log_solver_file);
    hd->log = new std::ofstream(hd->io->absolutePath(swFile::log_solver_file));
    swMessage::outfile = hd->log;
    swSolverParam* param = new swSolverParam(hd->io);
    if (param->readParameters() != EXIT_SUCCESS) return nullptr;
    if (param->getModelHyp() != "sp") return nullptr;
    swMesh* mesh = new swMesh(hd->io);
    if (mesh->build() != EXIT_SUCCESS) return nullptr;
    hd->m = new RefE();
    hd->m->setIOPointer(hd->io);
    if (!param->getHotstart()) hd->io->createEmptyOutputFolder(true);
    hd->m->importAttributesFromSolverParam(param);
    hd->cfg.apply_to(hd->m);
    if (hd->m->init(mesh) != EXIT_SUCCESS) return nullptr;
    hd->m->resolve_cost_weight(hd->m->h_weight_spec, hd->m->h_weight_map, "h_weight");
    hd->m->resolve_cost_weight(hd->m->q_weight_spec, hd->m->q_weight_map, "q_weight");
    hd->m->init_primal_memory();
    hd->m->save_initial_state();
    hd->m->set_quiet_logs(true);
    return hd;
}

long sw2dref_e_cell_nb(void* h) { return (long)static_cast<HandleE*>(h)->m->cell_nb; }

// AssimConfig values as the reference read them: [checkpoint_stride, windowed, window_duration,
// window_steps, n_windows, t_state_assimilation, cost_normalize, phi_transform (0 none, 1 clamp,
// 2 tanh, 3 normalize), lambda_tanh, dt_map_ad, mask_wall_gradient, alpha_reg, t_0, t_max]
void sw2dref_e_config(void* h, double* out)
{
    HandleE* hd = static_cast<HandleE*>(h);
    const AssimConfig& c = hd->cfg;
    const std::string pt = c.phi_transform;
    out[0] = (double)c.checkpoint_stride;
    out[1] = c.windowed_assimilation ? 1.0 : 0.0;
    out[2] = c.assimilation_window_duration;
    out[3] = (double)c.assimilation_window_steps;
    out[4] = (double)c.n_assimilation_windows;
    out[5] = c.t_state_assimilation;
    out[6] = c.cost_normalize ? 1.0 : 0.0;
    out[7] = (double)(int)hd->m->phi_transform;
    out[8] = c.lambda_tanh;
    out[9] = c.dt_map_ad;
    out[10] = c.mask_wall_gradient ? 1.0 : 0.0;
    out[11] = c.alpha_reg;
    out[12] = hd->m->t_0;
    out[13] = hd->m->t_max;
}

void sw2dref_e_get_phi(void* h, double* out)
{
    HandleE* hd = static_cast<HandleE*>(h);
    std::memcpy(out, hd->m->phi_data(), hd->m->cell_nb * sizeof(double));
}

int sw2dref_e_load_phi_map(void* h, const char* path, double* out)
{
    return static_cast<HandleE*>(h)->m->load_phi_csv(path, out) ? 0 : 1;
}

void sw2dref_e_set_options(void* h, int cost_normalize, int phi_transform, double lambda_tanh)
{
    RefE* m = static_cast<HandleE*>(h)->m;
    m->cost_normalize = cost_normalize != 0;
    m->phi_transform = (PhiTransform)phi_transform;
    m->lambda_tanh = lambda_tanh;
}

// The window keys of input.solv (AssimConfig::apply_to, assim/assimConfig.cpp:37-66).
void sw2dref_e_set_window_keys(void* h, int windowed, double duration, long steps, long n_windows, double t_state)
{
    swSpE* m = static_cast<HandleE*>(h)->m;
    m->windowed_assimilation = windowed != 0;
    m->assimilation_window_duration = duration;
    m->assimilation_window_steps = steps;
    m->n_assimilation_windows = n_windows;
    m->t_state_assimilation = t_state;
}

void sw2dref_e_set_weights(void* h, const double* wh, const double* wq)
{
    RefE* m = static_cast<HandleE*>(h)->m;
    m->h_weight_map.assign(wh, wh + m->cell_nb);
    m->q_weight_map.assign(wq, wq + m->cell_nb);
}

// The reference's own reader of reference/ResultHydro_p*.txt (assim/swSpE_ad.cpp:47-154), then
// the stable pointers of assim/main_enzyme.cpp:206-219.  Returns the number of frames, or -1.
int sw2dref_e_load_observations(void* h, int quiet)
{
    QuietOut qo(quiet != 0);
    HandleE* hd = static_cast<HandleE*>(h);
    if (!hd->m->load_all_observations()) return -1;
    hd->times.clear();
    hd->frames.clear();
    for (auto const& kv : hd->m->observations_map) {
        hd->times.push_back(kv.first);
        hd->frames.push_back(kv.second);
    }
    hd->m->obs_type = "cells";
    wire_observations(hd);
    return (int)hd->times.size();
}

void sw2dref_e_get_observation(void* h, int k, double* t, double* frame)
{
    HandleE* hd = static_cast<HandleE*>(h);
    *t = hd->times[k];
    std::memcpy(frame, hd->frames[k].data(), hd->frames[k].size() * sizeof(double));
}

// Full-field observations: frames[k] = (h, qx, qy) of every cell at times[k].
void sw2dref_e_set_frames(void* h, int n_obs, const double* times, const double* frames)
{
    HandleE* hd = static_cast<HandleE*>(h);
    const size_t n = hd->m->cell_nb;
    hd->times.assign(times, times + n_obs);
    hd->frames.assign(n_obs, std::vector<double>(3 * n));
    for (int k = 0; k < n_obs; k++) std::memcpy(hd->frames[k].data(), frames + (size_t)k * 3 * n, 3 * n * sizeof(double));
    hd->m->obs_type = "cells";
    wire_observations(hd);
}

// Gauge observations: values[k][g] is the depth observed at cells[g] at times[k].
void sw2dref_e_set_gauges(void* h, int n_obs, const double* times, int n_gauges, const long* cells, const double* w,
                          const double* values)
{
    HandleE* hd = static_cast<HandleE*>(h);
    hd->times.assign(times, times + n_obs);
    hd->frames.assign(n_obs, std::vector<double>(n_gauges));
    for (int k = 0; k < n_obs; k++) std::memcpy(hd->frames[k].data(), values + (size_t)k * n_gauges, n_gauges * sizeof(double));
    RefE* m = hd->m;
    m->obs_type = "gauges";
    m->n_gauges = (size_t)n_gauges;
    m->gauge_cell_idx.assign(cells, cells + n_gauges);
    m->gauge_w.assign(w, w + n_gauges);
    wire_observations(hd);
}

// update_phi_norm_bounds + build_checkpoint_records (what get_spatial_gradient_checkpointed
// runs before its reverse loop, assim/swSpE_checkpoint.cpp:740).  Returns the segment count.
long sw2dref_e_record(void* h, const double* m_map, long stride, int quiet)
{
    QuietOut qo(quiet != 0);
    HandleE* hd = static_cast<HandleE*>(h);
    std::vector<double> m(m_map, m_map + hd->m->cell_nb);
    hd->m->adjoint_truncation_seg_ = -1;
    hd->m->assim_window_tiles_.clear();
    hd->m->update_phi_norm_bounds(m.data());
    hd->m->build_checkpoint_records(m.data(), (size_t)stride);
    return (long)hd->m->segs_record_.size();
}

// Segment k of the record; any output pointer may be null.
long sw2dref_e_segment(void* h, long k, double* t_start, double* dt_seq, int* obs_trig, double* hh, double* q,
                       double* r)
{
    HandleE* hd = static_cast<HandleE*>(h);
    const SegPhysData& s = hd->m->segs_record_[(size_t)k];
    if (t_start) *t_start = s.t_start;
    if (dt_seq) std::memcpy(dt_seq, s.dt_seq.data(), s.n_steps * sizeof(double));
    if (obs_trig) std::memcpy(obs_trig, s.obs_trig.data(), s.n_steps * sizeof(int));
    const size_t n = hd->m->cell_nb;
    if (hh) std::memcpy(hh, s.h_ckpt.data(), n * sizeof(double));
    if (q) std::memcpy(q, s.qx_ckpt.data(), n * sizeof(double));
    if (r) std::memcpy(r, s.qy_ckpt.data(), n * sizeof(double));
    return (long)s.n_steps;
}

// The assimilation window and its tiles as get_spatial_gradient_checkpointed sets them before
// its reverse loop (assim/swSpE_checkpoint.cpp:781-951), restated because that function
// cannot run without Enzyme.  Writes the first segment of the window and the tile starts
// (tiles_out: up to K entries); returns the number of tiles (0: one continuous window).
int sw2dref_e_set_window(void* h, long* first_out, long* tiles_out)
{
    HandleE* hd = static_cast<HandleE*>(h);
    RefE* m = hd->m;
    const size_t K = m->segs_record_.size();
    size_t first = 0;
    m->adjoint_truncation_seg_ = -1;
    m->assim_window_tiles_.clear();
    if (m->windowed_assimilation && K > 0) {
        if (m->assimilation_window_steps > 0) {
            long acc = 0;
            for (long k = (long)K - 1; k >= 0; --k) {
                acc += (long)m->segs_record_[(size_t)k].n_steps;
                if (acc >= m->assimilation_window_steps) {
                    first = (size_t)k;
                    break;
                }
            }
        } else if (m->assimilation_window_duration > 0.) {
            const double t_start_window = m->t_max - m->assimilation_window_duration;
            for (size_t k = 0; k < K; ++k) {
                if (m->segs_record_[k].t_start <= t_start_window + 1e-9) first = k;
                else break;
            }
        } else if (m->t_state_assimilation > m->t_0) {
            for (size_t k = 0; k < K; ++k) {
                if (m->segs_record_[k].t_start <= m->t_state_assimilation + 1e-9) first = k;
                else break;
            }
        }
        if (first > 0) m->adjoint_truncation_seg_ = (int)first - 1;
    }
    const bool tiled = (m->n_assimilation_windows > 1) && (first < K);
    if (tiled) {
        const size_t M = K - first;
        size_t n = (size_t)m->n_assimilation_windows;
        if (n > M) n = M;
        for (size_t t = 0; t < n; ++t) m->assim_window_tiles_.push_back(first + (t * M) / n);
    }
    *first_out = (long)first;
    for (size_t t = 0; t < m->assim_window_tiles_.size(); t++) tiles_out[t] = (long)m->assim_window_tiles_[t];
    return (int)m->assim_window_tiles_.size();
}

// Replays from segment `truncation + 1` (or the tiles) as replay_trajectory_cost does.
void sw2dref_e_set_truncation(void* h, long seg)
{
    static_cast<HandleE*>(h)->m->adjoint_truncation_seg_ = (int)seg;
}

double sw2dref_e_replay_cost(void* h, const double* m_map, int quiet)
{
    QuietOut qo(quiet != 0);
    HandleE* hd = static_cast<HandleE*>(h);
    std::vector<double> m(m_map, m_map + hd->m->cell_nb);
    return hd->m->replay_trajectory_cost(m.data());
}

// One call of ckpt_segment_E (assim/swSpE_checkpoint.cpp:584-715) on segment k of the record
// from the given state; returns its cost and leaves the end state in the model.
double sw2dref_e_run_segment(void* h, long k, const double* m_map, const double* hh, const double* q, const double* r)
{
    HandleE* hd = static_cast<HandleE*>(h);
    RefE* m = hd->m;
    const SegPhysData& s = m->segs_record_[(size_t)k];
    std::vector<double> mm(m_map, m_map + m->cell_nb);
    std::vector<double> h0(hh, hh + m->cell_nb), q0(q, q + m->cell_nb), r0(r, r + m->cell_nb);
    m->phi_ptr = m->phi.data();
    return swSpE::ckpt_segment_E(m, mm.data(), h0.data(), q0.data(), r0.data(), s.dt_seq.data(), s.bc_flat.data(),
                                 s.obs_trig.data(), s.n_steps, m->edge_bnd_nb, m->current_obs_times,
                                 m->current_obs_frames, m->current_n_obs, s.t_start);
}

void sw2dref_e_get_state(void* h, double* hh, double* q, double* r)
{
    RefE* m = static_cast<HandleE*>(h)->m;
    std::memcpy(hh, m->water_depth.data(), m->cell_nb * sizeof(double));
    std::memcpy(q, m->unit_discharge_x.data(), m->cell_nb * sizeof(double));
    std::memcpy(r, m->unit_discharge_y.data(), m->cell_nb * sizeof(double));
}

double sw2dref_e_time(void* h) { return static_cast<HandleE*>(h)->m->t; }

const char* sw2dref_e_folder(void* h) { return static_cast<HandleE*>(h)->tmp.c_str(); }

// The reference's gen-ref-e mode on phi_map.  Its begin_reference_generation empties and
// recreates <case>/reference: the temporary folder's `reference` entry, a link to the case's own
// folder for load_observations, is first replaced by an empty directory of its own.  Returns the
// number of maps written, or -1.
long sw2dref_e_generate_references(void* h, const double* phi_map, long stride, int quiet)
{
    QuietOut qo(quiet != 0);
    HandleE* hd = static_cast<HandleE*>(h);
    const fs::path ref = fs::path(hd->tmp) / "reference";
    std::error_code ec;
    if (fs::is_symlink(fs::symlink_status(ref, ec))) fs::remove(ref, ec);
    if (fs::exists(fs::symlink_status(ref, ec)) && fs::is_symlink(fs::symlink_status(ref, ec))) return -1;
    fs::create_directories(ref, ec);
    std::vector<double> mm(phi_map, phi_map + hd->m->cell_nb);
    if (!hd->m->generate_references_E(mm.data(), (size_t)stride)) return -1;
    return (long)hd->m->n_ref_written;
}

void sw2dref_e_close(void* h)
{
    HandleE* hd = static_cast<HandleE*>(h);
    std::error_code ec;
    if (!hd->tmp.empty()) fs::remove_all(hd->tmp, ec);
}

}  // extern "C"
