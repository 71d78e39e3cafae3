// Test harness around the reference's own native SP, DIP and DDP solvers (compiled from the
// reference sources by oracle/Makefile).  It is a checker, never part of the product.
//
// The reference only runs a whole simulation (`swSp::execute`, src/sw2dSolver/models/sp/swSp.cpp:482-670;
// `swDip::execute`, models/dip/swDip.cpp, the same loop).  This subclass template reaches the
// protected members the same way the reference's own assimilation layer does (assim/swSpE.h:50
// subclasses swSp) and re-states the body of the time loop (swSp.cpp:522-589) without the
// result storage, so that a test can advance the reference N steps and read its state, fluxes
// and Riemann states at full precision.
//
// C entry points (ctypes):
//   sw2dref_open(folder, quiet)        init exactly as src/sw2dSolver/main.cpp:99-163 does
//   sw2dref_step(handle, n)            n passes of the loop body; stops when t >= t_max
//   sw2dref_run(handle)                the reference's own execute() (whole loop, with storage)
//   sw2dref_get/set_state, sw2dref_get_array, sw2dref_time, sw2dref_dt, sizes

#include <algorithm>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../common/param.h"
#include "../common/swFile.h"
#include "../common/swIO.h"
#include "../common/swLog.h"
#include "../common/swMessage.h"
#include "../common/geometry/swMesh.h"
#include "common/swSolverParam.h"
#include "models/ddp/swDdp.h"
#include "models/dip/swDip.h"
#include "models/sp/swSp.h"

#include <type_traits>

namespace {

// The operations a test needs, whichever model runs.
class RefModel
{
public:
    virtual ~RefModel() {}
    virtual swParent* parent() = 0;
    virtual bool stepOnce() = 0;
    virtual void beginTime() = 0;
    virtual void slopes(double* sx, double* sy) = 0;
    virtual int getArray(const std::string& name, double* out) = 0;
    virtual void setState(const double* h, const double* q, const double* r) = 0;
    virtual size_t nCells() const = 0;
    virtual size_t nInt() const = 0;
    virtual size_t nBnd() const = 0;
    virtual double time() const = 0;
    virtual double timeStep() const = 0;
    virtual double tMax() const = 0;
    virtual bool run() = 0;
    virtual long table(int which, long record, double* z, double* phi, double* theta, long cap) = 0;
    bool failed = false;  // the reference's execute() would have stopped with EXIT_FAILURE
};

template <class M>
class Ref : public M, public RefModel
{
public:
    swParent* parent() override { return this; }
    bool run() override { return this->execute(); }

    // One pass of the body of swSp::execute's time loop (sp/swSp.cpp:522-589), storage left out.
    // Where execute() returns EXIT_FAILURE (a failing hypCompute: NaN flux, impossible HLLC
    // configuration, negative depth with detection) the pass stops there and `failed` is set.
    bool stepOnce() override
    {
        if (failed || !(this->t < this->t_max)) return false;
        this->computeBC(this->t);
        auto hyp = [&]() { return this->hypCompute(this->div_corr_option, this->n_it_div_max, this->num_scheme, this->dt); };
        if constexpr (std::is_void<decltype(hyp())>::value) {
            hyp();  // SP and DIP report their failures through the result of the step itself
        } else if (hyp() != EXIT_SUCCESS) {
            failed = true;
            return false;
        }
        if (this->model_momentum_diffusion != "none") this->parabComputeExplicit();
        if (this->model_friction != "none") this->sourceFriction(this->model_friction, this->dt);
        if (this->model_singular_head_loss != "none") this->sourceSingularHeadLoss(this->dt);
        if (this->model_runoff != "none")
        {
            if (this->model_porosity_rainfall == "everywhere") this->sourceRunoffEverywhere();
            else if (this->model_porosity_rainfall == "water_only") this->sourceRunoffWateronly();
        }
        if (this->model_infiltration != "none") this->sourceInfiltration();
        if (this->model_wind != "none") this->sourceWind();
        this->correctVelocity();
        this->t += this->dt;
        return true;
    }

    void beginTime() override { this->t = this->t_0; }

    static constexpr bool kDdp = std::is_same<M, swDdp>::value;

    // Limited free-surface slopes exactly as the MUSCL-EVR reconstruction computes them
    // (sp/swSpHypMusclEvr.cpp:126-139), for kernel-level checks (SP and DIP).
    void slopes(double* sx, double* sy) override
    {
        if constexpr (kDdp) {
            (void)sx;
            (void)sy;
            return;
        } else {
        std::vector<double> z_cell(this->cell_nb), dzx(this->cell_nb), dzy(this->cell_nb);
        for (size_t i = 0; i < this->cell_nb; i++) z_cell[i] = this->water_depth[i] + this->cell_z_b[i];
        this->computeMusclSlopes(this->cell_centre_x, this->cell_centre_y, this->cell_neigh_cell_idx,
                           this->edge_int_midpoint_x, this->edge_int_midpoint_y,
                           this->edge_int_celL_idx, this->edge_int_celR_idx, z_cell, dzx, dzy);
        std::memcpy(sx, dzx.data(), this->cell_nb * sizeof(double));
        std::memcpy(sy, dzy.data(), this->cell_nb * sizeof(double));
        }
    }

    // DDP porosity tables (swDdp.h:243-281): which 0 cells, 1 internal edges, 2 boundary edges
    long table(int which, long record, double* z, double* phi, double* theta, long cap) override
    {
        if constexpr (kDdp) {
            const std::vector<std::vector<double>>* tz = which == 0 ? &this->cell_z_tab : which == 1 ? &this->edge_int_z_tab : &this->edge_bnd_z_tab;
            const std::vector<std::vector<double>>* tp = which == 0 ? &this->phiW_tab : which == 1 ? &this->phiG_int_tab : &this->phiG_bnd_tab;
            const std::vector<std::vector<double>>* tt = which == 0 ? &this->thetaW_tab : which == 1 ? &this->thetaG_int_tab : &this->thetaG_bnd_tab;
            if (record < 0 || (size_t)record >= tz->size()) return -1;
            const long n = (long)(*tz)[record].size();
            for (long l = 0; l < n && l < cap; l++) {
                z[l] = (*tz)[record][l];
                phi[l] = (*tp)[record][l];
                theta[l] = (*tt)[record][l];
            }
            return n;
        } else {
            (void)which; (void)record; (void)z; (void)phi; (void)theta; (void)cap;
            return -1;
        }
    }

    int getArray(const std::string& name, double* out) override
    {
        auto put = [&](const std::vector<double>& v) { std::memcpy(out, v.data(), v.size() * sizeof(double)); return (int)v.size(); };
        auto put2 = [&](const std::vector<std::array<double, 2>>& v, int side) {
            for (size_t i = 0; i < v.size(); i++) out[i] = v[i][side];
            return (int)v.size();
        };
        if constexpr (kDdp) {
            // state (swDdp.h:199-201), Riemann states, tables' derived values
            if (name == "h" || name == "theta") return put(this->thetaW);
            if (name == "q" || name == "theta_u") return put(this->thetaW_velocity_x);
            if (name == "r" || name == "theta_v") return put(this->thetaW_velocity_y);
            if (name == "theta_riemann_L") return put2(this->theta_riemann_int, 0);
            if (name == "theta_riemann_R") return put2(this->theta_riemann_int, 1);
            if (name == "theta_u_riemann_L") return put2(this->theta_u_riemann_int, 0);
            if (name == "theta_u_riemann_R") return put2(this->theta_u_riemann_int, 1);
            if (name == "theta_v_riemann_L") return put2(this->theta_v_riemann_int, 0);
            if (name == "theta_v_riemann_R") return put2(this->theta_v_riemann_int, 1);
            if (name == "thetaG_int_hmin") return put(this->thetaG_int_hmin);
            if (name == "z_riemann_bnd") return put(this->z_riemann_bnd);
            if (name == "surface_elevation" || name == "water_depth" || name == "unit_discharge_x" ||
                name == "unit_discharge_y") {
                // swDdp::storeResultMaps (swDdp.cpp:2489-2513)
                for (size_t n = 0; n < this->cell_nb; n++) {
                    double theta = this->thetaW[n];
                    double z = this->zOfThetaW(n, theta);
                    double h = std::max(0.0, z - this->cell_z_tab[n][0]);
                    double u = 0.0, v = 0.0;
                    if (theta > small_real) {
                        u = this->thetaW_velocity_x[n] / theta;
                        v = this->thetaW_velocity_y[n] / theta;
                    }
                    out[n] = name == "surface_elevation" ? z : name == "water_depth" ? h : name == "unit_discharge_x" ? u * h : v * h;
                }
                return (int)this->cell_nb;
            }
        } else {
            if (name == "h") return put(this->water_depth);
            if (name == "q") return put(this->unit_discharge_x);
            if (name == "r") return put(this->unit_discharge_y);
            if (name == "q_riemann_L") return put2(this->q_riemann_int, 0);
            if (name == "q_riemann_R") return put2(this->q_riemann_int, 1);
            if (name == "r_riemann_L") return put2(this->r_riemann_int, 0);
            if (name == "r_riemann_R") return put2(this->r_riemann_int, 1);
            if (name == "phi") {
                if constexpr (std::is_same<M, swDip>::value) return put(this->phiW);
                else return put(this->phi);
            }
        }
        if (name == "F1_int") return put(this->F1_int);
        if (name == "F2_int") return put(this->F2_int);
        if (name == "F3_int") return put(this->F3_int);
        if (name == "s2L_int") return put(this->s2L_int);
        if (name == "s2R_int") return put(this->s2R_int);
        if (name == "F1_bnd") return put(this->F1_bnd);
        if (name == "F2_bnd") return put(this->F2_bnd);
        if (name == "F3_bnd") return put(this->F3_bnd);
        if (name == "s2R_bnd") return put(this->s2R_bnd);
        if (name == "lambda_max_int") return put(this->lambda_max_int);
        if (name == "lambda_max_bnd") return put(this->lambda_max_bnd);
        if (name == "z_riemann_L") return put2(this->z_riemann_int, 0);
        if (name == "z_riemann_R") return put2(this->z_riemann_int, 1);
        if (name == "lambda_minus_L") return put2(this->lambda_minus_int, 0);
        if (name == "lambda_minus_R") return put2(this->lambda_minus_int, 1);
        if (name == "lambda_plus_L") return put2(this->lambda_plus_int, 0);
        if (name == "lambda_plus_R") return put2(this->lambda_plus_int, 1);
        if constexpr (std::is_same<M, swDip>::value) {
            if (name == "phiG_int") return put(this->phiG_int);
            if (name == "phiG_bnd") return put(this->phiG_bnd);
        }
        if (name == "area") return put(this->cell_area);
        if (name == "z_b") return put(this->cell_z_b);
        if (name == "cx") return put(this->cell_centre_x);
        if (name == "cy") return put(this->cell_centre_y);
        return -1;
    }

    void setState(const double* h, const double* q, const double* r) override
    {
        if constexpr (kDdp) {
            std::memcpy(this->thetaW.data(), h, this->cell_nb * sizeof(double));
            std::memcpy(this->thetaW_velocity_x.data(), q, this->cell_nb * sizeof(double));
            std::memcpy(this->thetaW_velocity_y.data(), r, this->cell_nb * sizeof(double));
        } else {
            std::memcpy(this->water_depth.data(), h, this->cell_nb * sizeof(double));
            std::memcpy(this->unit_discharge_x.data(), q, this->cell_nb * sizeof(double));
            std::memcpy(this->unit_discharge_y.data(), r, this->cell_nb * sizeof(double));
        }
    }

    size_t nCells() const override { return this->cell_nb; }
    size_t nInt() const override { return this->edge_int_nb; }
    size_t nBnd() const override { return this->edge_bnd_nb; }
    double time() const override { return this->t; }
    double timeStep() const override { return this->dt; }
    double tMax() const override { return this->t_max; }
};

struct Handle
{
    swIO* io = nullptr;
    RefModel* model = nullptr;
    std::ofstream* log = nullptr;
};

struct QuietErr
{
    std::streambuf* saved = nullptr;
    std::ostringstream sink;
    explicit QuietErr(bool on) { if (on) saved = std::cerr.rdbuf(sink.rdbuf()); }
    ~QuietErr() { if (saved) std::cerr.rdbuf(saved); }
};

}  // namespace

extern "C" {

// Mirrors src/sw2dSolver/main.cpp:76-163 for an SP, DIP or DDP case (model_hyperb sp | dip | ddp).
void* sw2dref_open(const char* folder, int quiet)
{
    QuietErr q(quiet != 0);
    Handle* hd = new Handle();
    hd->io = new swIO(folder);
    hd->io->createEmptyFolders(swFile::log_solver_file);
    hd->log = new std::ofstream(hd->io->absolutePath(swFile::log_solver_file));
    swMessage::outfile = hd->log;
    swSolverParam* param = new swSolverParam(hd->io);
    if (param->readParameters() != EXIT_SUCCESS) return nullptr;
    const std::string hyp = param->getModelHyp();
    if (hyp != "sp" && hyp != "dip" && hyp != "ddp") return nullptr;
    swMesh* mesh = new swMesh(hd->io);
    if (mesh->build() != EXIT_SUCCESS) return nullptr;
    if (param->getHotstart() == false) hd->io->createEmptyOutputFolder(true);
    if (hyp == "ddp") hd->model = new Ref<swDdp>();
    else if (hyp == "dip") hd->model = new Ref<swDip>();
    else hd->model = new Ref<swSp>();
    swParent* p = hd->model->parent();
    p->setIOPointer(hd->io);
    p->importAttributesFromSolverParam(param);
    if (p->init(mesh) != EXIT_SUCCESS) return nullptr;
    delete param;
    delete mesh;
    hd->model->beginTime();
    return hd;
}

int sw2dref_step(void* h, int n)
{
    QuietErr q(true);
    Handle* hd = static_cast<Handle*>(h);
    int done = 0;
    for (int i = 0; i < n; i++)
    {
        if (!hd->model->stepOnce()) break;
        done++;
    }
    return done;
}

int sw2dref_run(void* h)
{
    QuietErr q(true);
    Handle* hd = static_cast<Handle*>(h);
    return hd->model->run() == EXIT_SUCCESS ? 0 : 1;
}

int sw2dref_failed(void* h) { return static_cast<Handle*>(h)->model->failed ? 1 : 0; }

double sw2dref_time(void* h) { return static_cast<Handle*>(h)->model->time(); }
double sw2dref_dt(void* h) { return static_cast<Handle*>(h)->model->timeStep(); }
double sw2dref_t_max(void* h) { return static_cast<Handle*>(h)->model->tMax(); }
long sw2dref_cell_nb(void* h) { return (long)static_cast<Handle*>(h)->model->nCells(); }
long sw2dref_edge_int_nb(void* h) { return (long)static_cast<Handle*>(h)->model->nInt(); }
long sw2dref_edge_bnd_nb(void* h) { return (long)static_cast<Handle*>(h)->model->nBnd(); }

void sw2dref_get_state(void* h, double* hh, double* q, double* r)
{
    RefModel* m = static_cast<Handle*>(h)->model;
    m->getArray("h", hh);
    m->getArray("q", q);
    m->getArray("r", r);
}

void sw2dref_set_state(void* h, const double* hh, const double* q, const double* r)
{
    static_cast<Handle*>(h)->model->setState(hh, q, r);
}

int sw2dref_get_array(void* h, const char* name, double* out)
{
    return static_cast<Handle*>(h)->model->getArray(name, out);
}

long sw2dref_ddp_table(void* h, int which, long record, double* z, double* phi, double* theta, long cap)
{
    return static_cast<Handle*>(h)->model->table(which, record, z, phi, theta, cap);
}

void sw2dref_slopes(void* h, double* sx, double* sy)
{
    static_cast<Handle*>(h)->model->slopes(sx, sy);
}

}  // extern "C"
