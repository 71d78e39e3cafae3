// The reference-side binding of INTEGRATION.md, compiled against the reference's own headers and
// objects (oracle/Makefile, into oracle/_ref/libsw2d_b200_binding.so): a model class that the
// reference's factory swParent::create (src/sw2dSolver/models/swParent.cpp:125-173) can return
// for model_hyperb sp, which reads the case with the reference's own swSp and runs the time loop
// on the GPU through the C ABI of include/sw2d_b200.h.  The tests drive it through the C entry
// points below, the way src/sw2dSolver/main.cpp:76-173 drives a model, and compare its result
// with the reference's own solver on the same case folder.
//
// swSp::init and swSp::execute are final (src/sw2dSolver/models/sp/swSp.h:20-22), so the class
// derives from swParent and holds the swSp that reads the files; a subclass of swSp with a friend
// gives it read access to the tables swSp::init builds (protected members).
//
//   b200_open(folder, device)     main.cpp:99-163 with swSpB200 in place of swSp
//   b200_execute(handle, steps)   swSpB200::execute (the whole run, no result storage)
//   b200_state(handle, h, q, r)   the state execute() leaves in the swSp vectors
//   b200_error(handle), b200_close(handle)

#include <cmath>
#include <cstdint>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../common/swFile.h"
#include "../common/swIO.h"
#include "../common/swMessage.h"
#include "../common/geometry/swMesh.h"
#include "common/swSolverParam.h"
#include "models/common/swBoundaryConditionTimeSeries.h"
#include "models/sp/swSp.h"
#include "sw2d_b200.h"

class swSpB200;

// swSp with read access for swSpB200 (a friend of a derived class reaches the protected members
// of the base through objects of the derived class)
class swSpTables : public swSp
{
    friend class swSpB200;
};

class swSpB200 : public swParent
{
public:
    ~swSpB200() { if (gpu) sw2d_destroy(gpu); }

    void importAttributesFromSolverParam(swSolverParam* p) override
    {
        sp.setIOPointer(m_io);
        sp.importAttributesFromSolverParam(p);
    }

    // swSp::init reads every input file, checks the parameters and builds the tables; they go to
    // the GPU unchanged, with the angles in the map files' degrees read again by the reference's
    // own reader (swSp keeps radians, and converting them back would not give the same bits)
    bool init(swMesh* mesh) override
    {
        if (sp.init(mesh) != EXIT_SUCCESS) return EXIT_FAILURE;
        const size_t nc = sp.cell_nb, ni = sp.edge_int_nb, nb = sp.edge_bnd_nb;
        std::vector<int64_t> lr(2 * ni), bcell(nb);
        for (size_t e = 0; e < ni; e++) {
            lr[2 * e] = (int64_t)sp.edge_int_celL_idx[e];
            lr[2 * e + 1] = (int64_t)sp.edge_int_celR_idx[e];
        }
        for (size_t e = 0; e < nb; e++) bcell[e] = (int64_t)sp.edge_bnd_cell_idx[e];
        std::vector<int32_t> bnd_bc(nb, -1), type;
        std::vector<int64_t> off{0};
        std::vector<double> times, vals;
        for (swBoundaryConditionTimeSeries* s : sp.bc_timeseries_list) {
            const std::string ty = s->getBCType();
            if (ty == "q") type.push_back(SW2D_BC_Q);
            else if (ty == "h") type.push_back(SW2D_BC_H);
            else if (ty == "z") type.push_back(SW2D_BC_Z);
            else if (ty == "fr") type.push_back(SW2D_BC_FR);
            else return fail("boundary condition type not handled by the GPU step: " + ty);
            times.insert(times.end(), s->time_values.begin(), s->time_values.end());
            vals.insert(vals.end(), s->bc_values.begin(), s->bc_values.end());
            off.push_back((int64_t)times.size());
        }
        for (size_t e = 0; e < nb; e++) {
            for (size_t k = 0; k < sp.bc_timeseries_list.size(); k++)
                if (sp.edge_bnd_bc_pointer[e] == sp.bc_timeseries_list[k]) bnd_bc[e] = (int32_t)k;
            if (bnd_bc[e] < 0) return fail("a boundary edge has no time-series condition (rating curves are not handled)");
        }
        sw2d_mesh m{(int64_t)nc, (int64_t)ni, (int64_t)nb, sp.cell_area.data(), sp.cell_centre_x.data(),
                    sp.cell_centre_y.data(), sp.cell_z_b.data(), lr.data(), sp.edge_int_length.data(),
                    sp.edge_int_norm_x.data(), sp.edge_int_norm_y.data(), sp.edge_int_midpoint_x.data(),
                    sp.edge_int_midpoint_y.data(), bcell.data(), sp.edge_bnd_length.data(), sp.edge_bnd_norm_x.data(),
                    sp.edge_bnd_norm_y.data(), bnd_bc.data()};
        const std::string& fr = sp.model_friction;
        if (sp.num_scheme != "muscl_evr" && sp.num_scheme != "godunov") return fail("scheme not handled: " + sp.num_scheme);
        sw2d_params p{sp.num_scheme == "muscl_evr" ? SW2D_SCHEME_MUSCL_EVR : SW2D_SCHEME_GODUNOV,
                      sp.topo_discretization == "blending" ? SW2D_TOPO_BLENDING : SW2D_TOPO_DISCONTINUOUS,
                      fr == "chezy" ? SW2D_FRICTION_CHEZY : fr == "manning" ? SW2D_FRICTION_MANNING
                                                            : fr == "strickler" ? SW2D_FRICTION_STRICKLER
                                                                                 : SW2D_FRICTION_NONE,
                      sp.model_singular_head_loss != "none" ? 1 : 0,
                      sp.negative_depth_detection == "active" ? 1 : 0, SW2D_VARIANT_NATIVE, sp.cfl_max, sp.dt_max,
                      sp.dt_map, sp.h_min, sp.phi_min, sp.v_max, sp.fr_max, sp.t_0, sp.t_max};
        std::vector<double> fr_deg(nc, 0.0), hl_deg(nc, 0.0);
        if (fr != "none") {
            const std::string file = fr == "chezy" ? swFile::input_friction_chezy_map
                                     : fr == "manning" ? swFile::input_friction_manning_map
                                                       : swFile::input_friction_strickler_map;
            std::vector<std::string> names;
            std::vector<std::vector<double>> arr;
            swIO::readVectorParameterFile(m_io->absolutePath(file), 3, nc, names, arr);
            fr_deg = arr[2];
        }
        if (sp.model_singular_head_loss != "none") {
            std::vector<std::string> names;
            std::vector<std::vector<double>> arr;
            swIO::readVectorParameterFile(m_io->absolutePath(swFile::input_singular_head_loss_map), 4, nc, names, arr);
            hl_deg = arr[3];
        }
        auto ptr = [](std::vector<double>& v) { return v.empty() ? nullptr : v.data(); };
        sw2d_cell_fields f{sp.phi.data(), sp.boussinesq.data(), ptr(sp.friction_coeff_direction_1),
                           ptr(sp.friction_coeff_direction_2), fr_deg.data(), ptr(sp.singular_head_loss_h_sing),
                           ptr(sp.singular_head_loss_coeff_direction_1), ptr(sp.singular_head_loss_coeff_direction_2),
                           hl_deg.data()};
        sw2d_bc_table bc{(int32_t)type.size(), type.data(), off.data(), times.data(), vals.data()};
        if (sw2d_create(&m, &p, &f, &bc, sp.water_depth.data(), sp.unit_discharge_x.data(), sp.unit_discharge_y.data(),
                        device, &gpu) != SW2D_OK)
            return fail(std::string("sw2d_create: ") + sw2d_last_error(nullptr));
        return EXIT_SUCCESS;
    }

    // swSp::execute's time loop on the GPU, to t_max, without result storage; the final state
    // comes back into the swSp vectors
    bool execute() override
    {
        int64_t n = 0;
        const int st = sw2d_execute(gpu, &n);
        steps = n;
        sw2d_get_state(gpu, sp.water_depth.data(), sp.unit_discharge_x.data(), sp.unit_discharge_y.data());
        if (st != SW2D_OK) return fail(sw2d_last_error(gpu));
        return EXIT_SUCCESS;
    }

    size_t cells() const { return sp.cell_nb; }

    void state(double* hh, double* q, double* r) const
    {
        for (size_t i = 0; i < sp.cell_nb; i++) {
            hh[i] = sp.water_depth[i];
            q[i] = sp.unit_discharge_x[i];
            r[i] = sp.unit_discharge_y[i];
        }
    }

    bool fail(const std::string& msg)
    {
        error = msg;
        return EXIT_FAILURE;
    }

    swSpTables sp;
    sw2d_handle* gpu = nullptr;
    int device = 0;
    int64_t steps = 0;
    std::string error;
};

namespace {

struct Binding {
    swIO* io = nullptr;
    swSpB200* model = nullptr;
    std::ofstream* log = nullptr;
    std::string error;
};

}  // namespace

extern "C" {

void* b200_open(const char* folder, int device)
{
    Binding* b = new Binding();
    b->io = new swIO(folder);
    b->io->createEmptyFolders(swFile::log_solver_file);
    b->log = new std::ofstream(b->io->absolutePath(swFile::log_solver_file));
    swMessage::outfile = b->log;
    swSolverParam* param = new swSolverParam(b->io);
    if (param->readParameters() != EXIT_SUCCESS || param->getModelHyp() != "sp") return nullptr;
    swMesh* mesh = new swMesh(b->io);
    if (mesh->build() != EXIT_SUCCESS) return nullptr;
    if (param->getHotstart() == false) b->io->createEmptyOutputFolder(true);
    b->model = new swSpB200();
    b->model->device = device;
    b->model->setIOPointer(b->io);
    b->model->importAttributesFromSolverParam(param);
    if (b->model->init(mesh) != EXIT_SUCCESS) {
        b->error = b->model->error.empty() ? "swSp::init failed" : b->model->error;
        return b;
    }
    delete param;
    delete mesh;
    return b;
}

int b200_execute(void* h, int64_t* steps)
{
    Binding* b = static_cast<Binding*>(h);
    if (!b->model || !b->model->gpu) return 1;
    const bool rc = b->model->execute();
    if (steps) *steps = b->model->steps;
    return rc == EXIT_SUCCESS ? 0 : 1;
}

long b200_cell_nb(void* h) { return (long)static_cast<Binding*>(h)->model->cells(); }

void b200_state(void* h, double* hh, double* q, double* r) { static_cast<Binding*>(h)->model->state(hh, q, r); }

const char* b200_error(void* h)
{
    Binding* b = static_cast<Binding*>(h);
    if (!b->error.empty() || !b->model) return b->error.c_str();
    return b->model->error.c_str();
}

void b200_close(void* h)
{
    Binding* b = static_cast<Binding*>(h);
    delete b->model;
    delete b;
}

}  // extern "C"
