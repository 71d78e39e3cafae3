// sw2d_internal.cuh — definitions shared by the forward step (sw2d_sp.cu) and its adjoint
// (sw2d_adjoint.cu): the device-resident loop control, the device view of the mesh and state,
// the handle behind the C ABI, and the host helpers both translation units use.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/sw2d_b200.h"
#include "dip_math.cuh"
#include "ddp_math.cuh"

namespace sw2d {

constexpr int kBlock = 256;

// porosity model of a handle
constexpr int kModelSp = 0;
constexpr int kModelDip = 1;
constexpr int kModelDdp = 2;

// divergence correction of the DDP step (div_corr: none | limit_flux | limit_timestep)
constexpr int kDivCorrNone = 0;
constexpr int kDivCorrFlux = 1;
constexpr int kDivCorrTimestep = 2;

// Device-resident loop control.  t and t_max decide whether a step runs; `go` and `dt` are
// written by the CFL kernel's last block (or by the frozen-dt kernel of a replay) and read by
// the update kernel.
struct Ctrl {
    double t;
    double dt;
    double t_max;
    long long steps;
    unsigned int status;
    unsigned int blocks_done;
    int go;
    int store_map;  // DDP: the step ends on a storage time (swDdpHyp.cpp:590-609)
    // the fused step's running minimum of the CFL bounds, as an order-preserving integer key of
    // the double (kDminEmpty between steps)
    unsigned long long dmin;
};

constexpr unsigned long long kDminEmpty = ~0ull;

// Order-preserving map of a non-NaN double onto unsigned 64-bit integers (and back): a < b as
// doubles iff key(a) < key(b) as integers, so an integer atomicMin takes the double minimum.
__host__ __device__ __forceinline__ unsigned long long dmin_key(unsigned long long bits)
{
    return (bits >> 63) ? ~bits : (bits | 0x8000000000000000ull);
}
__host__ __device__ __forceinline__ unsigned long long dmin_bits(unsigned long long key)
{
    return (key >> 63) ? (key & 0x7fffffffffffffffull) : ~key;
}

// One balance slot: the dt-free contributions {a, b, c} of one edge to one cell's h, q and r
// (hypComputeBalance, swSpHyp.cpp:221-263: h += a dt, q += b dt, r += c dt).
struct Slot {
    double a, b, c;
};

__host__ __device__ __forceinline__ Slot make_slot(double a, double b, double c)
{
    Slot s;
    s.a = a;
    s.b = b;
    s.c = c;
    return s;
}

// One tile of the fused step (sw2d_tile.cu): cells [c0, c0 + nt) of the internal numbering,
// nh1 cells one edge away and nh2 two edges away (halo[hoff ..]); internal edges with a cell in
// the tile: the owned range [e0, e0 + ne_own) (lower cell in the tile) and nx_flux incoming edges,
// then nx_slope edges that only the ring-1 slopes need (xe[xoff ..]); per tile edge the local
// {L, R} indices (eloc[loff ..]); the neighbour lists of the tile and ring-1 cells (scsr[soff ..],
// offsets soffs[so_off ..], nent entries); boundary edges [b0, b1); first balance slot s0.
struct TileInfo {
    int c0, nt, nh1, nh2, hoff, e0, ne_own, xoff, nx_flux, nx_slope, loff, soff, so_off, b0, b1, s0, nent;
};

struct TileMesh {
    int ntiles = 0, tile_cells = 0;
    int slopes_in = 1;  // MUSCL-EVR: 1 slopes computed by k_flux (ring 2 staged); 0 read from k_slopes' output
    // the largest tile: staged cells, tile + ring-1 cells, tile cells, slot range, flux edges, all
    // tile edges, neighbour-list entries
    int nl_max = 0, nf_max = 0, nt_max = 0, ns_max = 0, ne_max = 0, na_max = 0, nent_max = 0;
    // byte offsets of the stage's sections in shared memory and its size (sw2d_tile.cu)
    int o_st = 0, o_cst = 0, o_xy = 0, o_sl = 0, o_coff = 0, o_lam = 0, o_en = 0, o_ecf = 0, o_elen = 0, o_esl = 0,
        o_epg = 0, o_em = 0, o_ell = 0, o_ent = 0, o_so = 0, smem = 0;
    const TileInfo* info = nullptr;
    const int* halo = nullptr;
    const int* xe = nullptr;
    const ushort2* eloc = nullptr;
    const unsigned* scsr = nullptr;        // local neighbour | tile edge << 16 | side << 31
    const unsigned* soffs = nullptr;
};

struct DdpCtrl;       // sw2d_ddp.cu
struct ResultWriter;  // sw2d_result.cu

struct DevMesh {
    int nc, ni, nb;
    // cells
    double4* st;             // {h, q, r, z}
    double4* st_out;         // optional: where the cell update writes the new state (else st, in
                             // place; the adjoint's recompute writes each step into its segment)
    const double4* cst;      // {z_b, boussinesq, phi, area}
    const double2* cxy;      // centroid
    double2* slope;          // MUSCL slopes
    const double4* fric;     // {k1, k2, cos a, sin a} (friction)
    const double4* hla;      // {h_sing, k1, k2, -} (singular head loss)
    const double2* hlb;      // {cos a, sin a}
    const double* zbv;       // z_b
    const double* area;
    const int2* coff;        // [nc+1] {first internal-neighbour entry, first balance slot}
    const int2* cint;        // {edge*2 + side, neighbour} (MUSCL slopes)
    Slot* slot;              // balance slots {a, b, c}
    double4* slot4;          // balance slots of the differentiated step {f1 F1, b, c, f1} (sw2d_assim.cu)
    double* slot_w;          // CFL contribution of the slot (null: not written, for steps whose
                             // dt is frozen)
    double4* bal;            // post-balance state {h, q, r, ±P} with P = h^(-4/3) of the friction
                             // stage, negative where the velocity cap acted (written only by the
                             // recording update)
    // internal edges
    const int2* lr;
    const int2* eslot;       // {slot of (L, e), slot of (R, e)}
    const double2* nxy;
    const double2* mxy;
    const double4* emc;      // {mx - cx_L, my - cy_L, mx - cx_R, my - cy_R}
    const double* len;
    const double2* coef;     // {coefL, coefR}
    double2* flux;           // optional copy: 3 x double2 per edge {F1,F2},{F3,S2L},{S2R,-} (tests)
    double2* rstate;         // optional: the two Riemann states per edge, 5 planes of ni double2
                             // (the adjoint's segment recompute keeps them for k_edges_rev)
    double* lmax;            // optional copy of lambda_max (tests)
    // boundary edges
    const int* bcell;
    const int* bbc;
    const int* bslot;
    const double4* bgeo;     // {nx, ny, length, coef}
    double4* bflux;          // optional copy {F1, F2, F3, -} (tests)
    double* lmaxb;           // optional copy of lambda_max (tests)
    // boundary series
    const int* bctype;
    const long long* bcoff;
    const double *bctimes, *bcvals;
    // DIP: connectivity porosity of internal and boundary edges, momentum dissipation
    // {mu1, mu2, cos a, sin a} per cell (the cell statics' phi holds the storage porosity)
    const double* phig;
    const double* phigb;
    const double4* mu;
    // DDP: porosity tables (levels {z, phi, theta}) of the cells and of the internal edges in
    // the internal numbering, record k holding levels [off[k], off[k+1]); the per-cell values
    // derived from the current state {phiW(z), thetaW(z), pressure force Omega(z), -} (z in
    // st.w); per-cell statics {phiW, thetaW at z_tab[0] + h_min; phiW, thetaW at z_tab[1] +
    // h_min}; per internal edge two records {thetaG_hmin, z_tab[0], phiG, thetaG at the L cell's
    // shallow level}, {phiG, thetaG at the R cell's shallow level, -, -}; the pre-balance state
    // (divergence correction) and the loop control of the divergence correction
    const ddp::Lvl* ctab;
    const int* ctoff;
    const ddp::Lvl* etab;
    const int* etoff;
    double4* dv;
    const double4* dcs;
    const double4* des;
    double4* old;
    DdpCtrl* dctl;
    double chi_phi_max;
    int div_corr;
    int n_it_div_max;
    // parameters
    double h_min, phi_min, cfl_max, dt_max, dt_map, v_max, fr_max;
    DryConsts dry;
    int neg_detect;
    int rev_update;  // the cell update walks its blocks from the last cells to the first
    // dt reduction scratch
    double* part;
    Ctrl* ctrl;
};

// read-only loads through the non-coherent path (data not written by the same kernel)
template <class T>
__device__ __forceinline__ T ld(const T* p) { return __ldg(p); }

__device__ __forceinline__ double4 ld(const double4* p)
{
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = __ldg(q), b = __ldg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// Loads issued where they stand: a volatile asm is neither sunk below a later branch nor
// reordered against the other volatile asms, so a kernel can have all of an element's loads in
// flight before it uses the first one.  For data no kernel writes meanwhile (non-coherent path).
__device__ __forceinline__ double2 ld_now(const double2* p)
{
    double2 v;
    asm volatile("ld.global.nc.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}
__device__ __forceinline__ int2 ld_now(const int2* p)
{
    int2 v;
    asm volatile("ld.global.nc.v2.s32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p));
    return v;
}

__device__ __forceinline__ int ld_now(const int* p)
{
    int v;
    asm volatile("ld.global.nc.s32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ double ld_now(const double* p)
{
    double v;
    asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ bool step_active(const Ctrl* c) { return c->t < c->t_max; }

inline unsigned grid_for(long long n) { return (unsigned)((n + kBlock - 1) / kBlock); }

struct AdjointState;  // sw2d_adjoint.cu
struct AssimState;    // sw2d_assim.cu
struct DdpState;      // sw2d_ddp.cu
struct ClosureState;  // sw2d_mlp.cu

}  // namespace sw2d

struct sw2d_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    int64_t nc = 0, ni = 0, nb = 0;
    sw2d_params p{};
    int model = 0;             // kModelSp, kModelDip or kModelDdp
    int sms = 0;               // the device's SM count (0 until first needed)
    int dissipation = 0;       // DIP momentum dissipation active
    std::vector<int> cell_perm, int_perm, bnd_perm;  // [new] = caller index
    std::vector<void*> allocs;
    sw2d::DevMesh m{};
    sw2d::Ctrl* ctrl = nullptr;
    sw2d::Ctrl* ctrl_host = nullptr;  // pinned
    int* d_cell_perm = nullptr;
    int* d_int_perm = nullptr;
    int* d_bnd_perm = nullptr;
    double* stage = nullptr;    // 3 * nc doubles
    double* lmax_buf = nullptr;   // allocated by the option record_wave_speeds
    double* lmaxb_buf = nullptr;
    double2* flux_buf = nullptr;  // allocated by the option record_fluxes
    double4* bflux_buf = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    int edge_variant = 0;   // index into kVariants (sw2d_autotune)
    int slope_variant = 2;
    sw2d::AdjointState* adj = nullptr;  // recorded trajectory, checkpoints and adjoint buffers
    int adj_flush_branch = 0;           // option "adjoint_flush_branch"
    int adj_keep_nonfinite = 0;         // option "adjoint_keep_nonfinite"
    int adj_trace = 0;                  // option "adjoint_trace"
    int adj_store_states = 1;           // option "adjoint_store_states"
    void* saved_point = nullptr;        // sw2d_save_point: state, balance slots, control block
    int adj_edge_variant = 0;           // option "adjoint_edge_variant"
    sw2d::AssimState* assim = nullptr;  // porosity assimilation with the differentiated step
    int assim_sqrt_zero = 0;            // option "assim_sqrt_zero"
    int assim_chained = 0;              // option "assim_chained_recompute"
    sw2d::DdpState* ddp = nullptr;      // DDP model: tables, divergence-correction scratch
    sw2d::ResultWriter* result = nullptr;   // binary map file (sw2d_result_open)
    sw2d::ClosureState* closure = nullptr;  // learned momentum-exchange closure (sw2d_set_closure)
    sw2d::TileMesh tiles{};             // tiles of the fused step (SP and DIP models)
    std::vector<void*> tile_allocs;     // device arrays of the tiles
    std::vector<int2> h_coff, h_cint, h_lr;  // host tables the tiles are built from
    int tile_default = 384;                  // tile size of the first build (SW2D_TILE_CELLS)
    std::vector<int> h_bcell;
    int fused = 0;                      // step as the two kernels k_flux + k_update (option "fused_step")
    int fused_slopes = 0;               // MUSCL-EVR: slopes inside k_flux (1) or by k_slopes first (0)
    int flux_variant = 0;               // launch variant of k_flux (sw2d_autotune)
    std::string err;
};

namespace sw2d {

// Records `msg` as the handle's last error (or the creation error) and returns `code`.
int fail(sw2d_handle* h, int code, const std::string& msg);
// Maps the device status word to an SW2D_E_* code (and its message).
int status_to_code(sw2d_handle* h, unsigned st);

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return ::sw2d::fail(h, SW2D_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <class T>
int dev_upload(sw2d_handle* h, const std::vector<T>& v, T** out)
{
    size_t bytes = std::max<size_t>(1, v.size()) * sizeof(T);
    void* p = nullptr;
    CK(cudaMalloc(&p, bytes));
    h->allocs.push_back(p);
    if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, h->stream));
    *out = static_cast<T*>(p);
    return SW2D_OK;
}

template <class T>
int dev_alloc(sw2d_handle* h, size_t n, T** out)
{
    void* p = nullptr;
    CK(cudaMalloc(&p, std::max<size_t>(1, n) * sizeof(T)));
    h->allocs.push_back(p);
    CK(cudaMemsetAsync(p, 0, std::max<size_t>(1, n) * sizeof(T), h->stream));
    *out = static_cast<T*>(p);
    return SW2D_OK;
}

// Forward kernels on an explicit device view `m` (the handle's own, or one whose state points
// into a replay buffer), on the handle's stream, with the handle's launch variants.
void launch_slopes_on(sw2d_handle* h, const DevMesh& m);
void launch_edges_on(sw2d_handle* h, const DevMesh& m);
void launch_cfl_on(sw2d_handle* h, const DevMesh& m);
// The update kernel; with store_balance it also writes the post-balance state to m.bal.
void launch_update_on(sw2d_handle* h, const DevMesh& m, bool store_balance);
// One whole time step of the handle (its four kernels, its launch variants) on its stream.
void launch_step_on(sw2d_handle* h);

// ensemble work queue (sw2d_queue.cu): one persistent kernel over (step, phase, member, tile)
struct QueueState;
int queue_eligible(sw2d_handle* const* members, int n, std::string& why);
int queue_build(QueueState*& q, sw2d_handle* const* members, int n, int variant, int cells_per_tile, int edges_per_tile,
                std::string& why);
int queue_launch(QueueState* q, int steps, cudaStream_t stream);
unsigned queue_read_status(QueueState* q);
void queue_clear_status(QueueState* q);
void queue_release(QueueState* q);
int queue_variants();
std::string queue_variant_label(int v);
void queue_set_polls(QueueState* q, long long polls);
int queue_grid(const QueueState* q);

// The fused step's flux kernel (sw2d_tile.cu) on the handle's stream with launch variant v; with
// attr_only only its shared-memory attribute is set (before a graph capture).  The tiles are
// built by tiles_build from the internal-numbering tables.
cudaError_t launch_flux(sw2d_handle* h, const DevMesh& m, int v, bool attr_only);
int flux_variants();
std::string flux_variant_label(int v);
int tiles_build(sw2d_handle* h, const std::vector<int2>& coff, const std::vector<int2>& cint,
                const std::vector<int2>& lr, const std::vector<int>& bcell, int tile_cells, std::string& why);

// The CFL kernel with the DDP model's map-storage snap (swDdpHyp.cpp:588-600).
void launch_cfl_ddp_on(sw2d_handle* h, const DevMesh& m);
// Friction, singular head loss and the velocity cap of one cell (swSpSourceFriction.cpp,
// swSp.cpp:447-479; the DDP model applies the same formulas to thetaW and its momentum,
// swDdpSourceFriction.cpp, swDdp.cpp:527-561).
template <int kFriction, bool kHeadLoss>
__device__ __forceinline__ void cell_sources(const DevMesh& m, int c, double dt, double hh, double& qq, double& rr,
                                             double* P_out = nullptr, const double4* fr_pre = nullptr,
                                             bool* capped_out = nullptr)
{
    const double hthr = smax(m.h_min, kSmallReal);
    // friction (swSpSourceFriction.cpp:39-171); fr_pre: the cell's coefficients, when the caller
    // loaded them already
    if (kFriction != SW2D_FRICTION_NONE) {
        if (hh > hthr) {
            const double4 fr = fr_pre ? *fr_pre : ld(&m.fric[c]);
            double u = qq / hh;
            double v = rr / hh;
            double ca = fr.z, sa = fr.w;
            double ul = u * ca + v * sa;
            double vl = -u * sa + v * ca;
            double un = sqrt(u * u + v * v);
            // h^(-4/3) once per cell; isotropic friction (equal coefficients): the same factor,
            // computed once
            const double P = (kFriction != SW2D_FRICTION_CHEZY && hh > kSmallReal) ? friction_power(hh) : 0.0;
            if (P_out) *P_out = P;
            double f1 = friction_factor_p(kFriction, fr.x, hh, un, dt, P);
            double f2 = (fr.y == fr.x) ? f1 : friction_factor_p(kFriction, fr.y, hh, un, dt, P);
            ul *= f1;
            vl *= f2;
            qq = (ul * ca - vl * sa) * hh;
            rr = (ul * sa + vl * ca) * hh;
        } else {
            qq = 0.;
            rr = 0.;
        }
    }
    // singular head loss (swSpSourceFriction.cpp:174-219)
    if (kHeadLoss) {
        const double2 cs = ld(&m.hlb[c]);
        double ca = cs.x, sa = cs.y;
        double qx = qq * ca + rr * sa;
        double qy = -qq * sa + rr * ca;
        if (hh > hthr) {
            const double4 hl = ld(&m.hla[c]);
            double ax = 0, ay = 0;
            if (hh > hl.x) {
                ax = sqrt(qx * qx + qy * qy) * hl.y / hh;
                ay = sqrt(qx * qx + qy * qy) * hl.z / hh;
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
    // swSp::correctVelocity (swSp.cpp:447-479)
    if (hh > m.h_min) {
        double qn = sqrt(qq * qq + rr * rr);
        double cc = sqrt(kGravity * hh);
        double Fr = qn / cc / hh;
        double fact = smax(qn / (hh * m.v_max), Fr / m.fr_max);
        if (fact > 1.0) {
            if (capped_out) *capped_out = true;
            qq = qq / fact;
            rr = rr / fact;
        }
    }
}

// DDP model (sw2d_ddp.cu): one step on the handle's stream; the per-cell values derived from
// the state, recomputed after the state was set from outside; the DDP setup of sw2d_create_ddp.
void launch_ddp_step(sw2d_handle* h);
// phase i of a DDP step (0 none, 1 edges, 2 cfl, 3 the cell update and any divergence correction)
void launch_ddp_phase(sw2d_handle* h, int i);
void launch_ddp_edges(sw2d_handle* h, const DevMesh& m, int variant);
// {threads per block, minimum resident blocks} of the DDP edge kernel's launch variant v
void ddp_variant(int v, int* block, int* minb);
int ddp_kernels_per_step(sw2d_handle* h);
int64_t ddp_get_array(sw2d_handle* h, const char* name, double* out, int64_t capacity, bool* handled);
int64_t ddp_get_array_staged(sw2d_handle* h, const char* name, double* out, int64_t capacity, double* stage,
                             int64_t stage_cap, bool* handled);
// Looks up the device address of the no-allocation staging array on the handle's device (done
// by the create functions, so that sw2d_get_array_noalloc itself never needs to).
int noalloc_prepare(sw2d_handle* h);
int64_t ddp_get_table(sw2d_handle* h, int which, int64_t record, double* z, double* phi, double* theta,
                      int64_t capacity);
int ddp_derive(sw2d_handle* h);
int ddp_setup(sw2d_handle* h, const sw2d_mesh* mesh, const sw2d_cell_fields* fields, const sw2d_ddp_fields* ddp,
              const double* ic_level, const double* ic_x, const double* ic_y);
void ddp_release(sw2d_handle* h);
// Validates the DDP arguments before anything is allocated.
int ddp_check(const sw2d_mesh* mesh, const sw2d_ddp_fields* ddp, std::string& why);

// The binary map file (sw2d_result.cu): the frame kernels after a step, the steps per chunk
// while a file is attached, the wait for frames in flight, the hand-over of stored frames to
// the writer thread (stream synchronised), a frame of the current state, whether the run's
// first frame is stored, the release.
void result_after_step(sw2d_handle* h);
int result_chunk(const sw2d_handle* h);
int result_wait(sw2d_handle* h, long long in_flight);
int result_drain(sw2d_handle* h);
int result_force(sw2d_handle* h);
bool result_started(const sw2d_handle* h);
void result_release(sw2d_handle* h);

// The learned closure (sw2d_mlp.cu): the DIP cell update with the network at the closure site,
// the release, and the feature record switch.
void closure_update(sw2d_handle* h, const DevMesh& m);
void closure_release(sw2d_handle* h);
int closure_record(sw2d_handle* h, int on);
int closure_set_ctas(sw2d_handle* h, int per_sm);  // resident CTAs per SM of the update (0: all that fit)

// Releases the adjoint buffers of the handle (sw2d_adjoint.cu).
void adjoint_release(sw2d_handle* h);
// Releases the assimilation buffers of the handle (sw2d_assim.cu).
void assim_release(sw2d_handle* h);
// Called when the physical parameters or the state change under a recorded trajectory.
void adjoint_invalidate(sw2d_handle* h);

}  // namespace sw2d
