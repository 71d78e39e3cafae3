/*
 * sw2d_b200.h — C ABI of the B200 implementation of SW2D's single-porosity (SP) explicit
 * finite-volume step.
 *
 * The reference exposes this path through C++ class seams, not a C ABI:
 *   - the model interface swParent::init(swMesh*) / importAttributesFromSolverParam() /
 *     execute()  (src/sw2dSolver/models/swParent.h:25-27), implemented for SP by
 *     swSp::init (src/sw2dSolver/models/sp/swSp.cpp:720-969), importAttributesFromSolverParam
 *     (swSp.cpp:685-717) and execute (swSp.cpp:482-670);
 *   - the driver that builds and runs it, sw2dSolver's main (src/sw2dSolver/main.cpp:99-173).
 * Each entry point below names the reference routine it replaces.  A binding for another
 * host language sees plain pointers, sizes and int status codes only.
 *
 * Conventions (the reference's, restated):
 *   - mesh arrays are in the reference numbering (cells, internal edges, boundary edges as
 *     read from geometry.sw2d, src/common/geometry/swMesh.cpp:213-471); the library
 *     renumbers internally and always returns per-cell data in the caller's numbering;
 *   - per-cell contributions are summed in the reference's order (boundary edges by
 *     increasing index, then internal edges by increasing index), so results do not
 *     depend on the internal numbering;
 *   - all arithmetic is IEEE binary64;
 *   - status: 0 = success, < 0 = error (SW2D_E_*); the reference calls exit(1) instead
 *     (src/common/swMessage.cpp:74-84).  sw2d_last_error() returns the message text;
 *   - one CUDA stream per handle; calls on one handle are not thread-safe, calls on
 *     different handles are.
 */
#ifndef SW2D_B200_H
#define SW2D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SW2D_ABI_VERSION 3

/* status codes */
#define SW2D_OK 0
#define SW2D_E_ARG (-1)          /* invalid argument / inconsistent sizes                   */
#define SW2D_E_CUDA (-2)         /* CUDA runtime error (message in sw2d_last_error)         */
#define SW2D_E_NAN_FLUX (-3)     /* NaN mass flux: src/sw2dSolver/models/sp/swSpHyp.cpp:374-392 */
#define SW2D_E_HLLC_CONFIG (-4)  /* impossible wet/dry configuration: swSpHyp.cpp:728-739     */
#define SW2D_E_NEG_DEPTH (-5)    /* negative depth with detection active: swSpHyp.cpp:184-196 */
#define SW2D_E_BC_TYPE (-6)      /* unknown boundary type: swSpHyp.cpp:116-120               */
#define SW2D_E_BC_FR (-7)        /* 'fr' boundary value outside [0,1]: swSpHyp.cpp:57-62     */
#define SW2D_E_UNSUPPORTED (-8)  /* option outside the implemented path                     */
#define SW2D_E_NO_DEVICE (-9)    /* no usable CUDA device                                    */
#define SW2D_E_PHIG (-10)        /* DIP connectivity porosity < 1e-16 in a specific force:
                                    src/sw2dSolver/models/dip/swDip.cpp:1524-1528            */
#define SW2D_E_DDP_TABLE (-11)   /* DDP: NaN elevation or volume in a porosity-table lookup, where
                                    the reference indexes level -1 (swDdp.cpp:1090-1096, 3382-3386) */
#define SW2D_E_IO (-12)          /* writing the result file failed (the reference: logFatal)     */

/* enumerations of the input.solv string keys (src/sw2dSolver/common/swSolverParam.h:130-153) */
enum sw2d_scheme { SW2D_SCHEME_GODUNOV = 0, SW2D_SCHEME_MUSCL_EVR = 1 };
enum sw2d_topo { SW2D_TOPO_DISCONTINUOUS = 0, SW2D_TOPO_BLENDING = 1 };
enum sw2d_friction { SW2D_FRICTION_NONE = 0, SW2D_FRICTION_CHEZY = 1, SW2D_FRICTION_MANNING = 2,
                     SW2D_FRICTION_STRICKLER = 3 };
enum sw2d_bc_type { SW2D_BC_Q = 0, SW2D_BC_H = 1, SW2D_BC_Z = 2, SW2D_BC_FR = 3,
                    SW2D_BC_PHIWQ = 4 /* DIP only */ };
enum sw2d_variant { SW2D_VARIANT_NATIVE = 0, SW2D_VARIANT_ENZYME_E = 1 };

/* Mesh tables, as swParent::setMeshTables builds them (src/sw2dSolver/models/swParent.cpp:391-501).
 * Normals of internal edges point from the L cell to the R cell; normals of boundary edges
 * point into the domain (swEdgeIntern.cpp:97-112, swEdgeBoundary.cpp:98-112). */
typedef struct sw2d_mesh {
    int64_t cell_nb;
    int64_t edge_int_nb;
    int64_t edge_bnd_nb;
    const double* cell_area;       /* [cell_nb] */
    const double* cell_x;          /* [cell_nb] centroid */
    const double* cell_y;          /* [cell_nb] */
    const double* cell_z_b;        /* [cell_nb] bottom level */
    const int64_t* edge_int_cells; /* [2*edge_int_nb] (L, R) pairs */
    const double* edge_int_length; /* [edge_int_nb] */
    const double* edge_int_nx;
    const double* edge_int_ny;
    const double* edge_int_mx;     /* midpoint */
    const double* edge_int_my;
    const int64_t* edge_bnd_cell;  /* [edge_bnd_nb] */
    const double* edge_bnd_length;
    const double* edge_bnd_nx;
    const double* edge_bnd_ny;
    const int32_t* edge_bnd_bc;    /* [edge_bnd_nb] index into the boundary table (0..bc_nb-1) */
} sw2d_mesh;

/* The input.solv keys this path reads (swSp::importAttributesFromSolverParam, swSp.cpp:685-717;
 * defaults in src/sw2dSolver/common/swSolverParam.h:144-194). */
typedef struct sw2d_params {
    int32_t scheme;                   /* enum sw2d_scheme   (num_scheme)                 */
    int32_t topo;                     /* enum sw2d_topo     (topo_discretization)        */
    int32_t friction;                 /* enum sw2d_friction (model_friction)             */
    int32_t singular_head_loss;       /* 0 none, 1 active   (model_singular_head_loss)   */
    int32_t negative_depth_detection; /* 0 none, 1 active                                 */
    int32_t variant;                  /* enum sw2d_variant; only NATIVE is implemented    */
    double cfl_max;
    double dt_max;
    double dt_map;
    double h_min;
    double phi_min;
    double v_max;
    double fr_max;
    double t_0;
    double t_max;
} sw2d_params;

/* Per-cell model parameters (swSp::setPorosityParameter, setBoussinesqParameter,
 * setFrictionParameters, setSingularHeadLossParameters: swSp.cpp:997-1072,1250-1273,1330-1360).
 * Angles are in degrees, as in the map files.  Arrays not needed by the chosen options may be NULL. */
typedef struct sw2d_cell_fields {
    const double* phi;            /* [cell_nb] porosity                                   */
    const double* boussinesq;     /* [cell_nb]                                            */
    const double* friction_1;     /* [cell_nb] coefficient, 1st principal direction       */
    const double* friction_2;     /* [cell_nb] coefficient, 2nd principal direction       */
    const double* friction_alpha; /* [cell_nb] degrees                                    */
    const double* hl_h_sing;      /* [cell_nb] singular head loss threshold depth         */
    const double* hl_coeff_1;
    const double* hl_coeff_2;
    const double* hl_alpha;       /* degrees */
} sw2d_cell_fields;

/* Boundary time series (swBoundaryConditionTimeSeries, models/common/swBoundaryConditionTimeSeries.cpp:17-96).
 * Series k has type[k] and records times[offset[k] .. offset[k+1]), values[...] alike. */
typedef struct sw2d_bc_table {
    int32_t bc_nb;
    const int32_t* type;     /* [bc_nb] enum sw2d_bc_type */
    const int64_t* offset;   /* [bc_nb+1] */
    const double* times;
    const double* values;
} sw2d_bc_table;

typedef struct sw2d_handle sw2d_handle;

/* Replaces swParent::create + importAttributesFromSolverParam + swSp::init
 * (swParent.cpp:125-173, swSp.cpp:685-969): validates, renumbers, uploads, computes the
 * edge factors (swSp::computeEdgeFactors, swSp.cpp:338-444) and sets t = t_0.
 * `device` is the CUDA ordinal. */
int sw2d_create(const sw2d_mesh* mesh, const sw2d_params* params, const sw2d_cell_fields* fields,
                const sw2d_bc_table* bc, const double* h0, const double* q0, const double* r0,
                int device, sw2d_handle** out);

/* The dual integral porosity (DIP) model: fields beyond the SP ones.  fields->phi of
 * sw2d_create_dip is the cell (storage) porosity phiW (DIP_cell_porosity_map.txt). */
typedef struct sw2d_dip_fields {
    const double* phi_g_int;       /* [edge_int_nb] connectivity porosity (DIP_edge_int_porosity_map.txt) */
    const double* phi_g_bnd;       /* [edge_bnd_nb] (DIP_edge_bnd_porosity_map.txt)                     */
    int32_t momentum_dissipation;  /* 0 none, 1 active (model_momentum_dissipation)                     */
    const double* mu_1;            /* [cell_nb] dissipation coefficients and direction (degrees)        */
    const double* mu_2;            /* (cell_momentum_dissipation_map.txt); NULL when inactive           */
    const double* mu_alpha;
} sw2d_dip_fields;

/* Replaces swParent::create + swDip::init (swParent.cpp:125-173, dip/swDip.cpp:900-1030) for
 * model_hyperb dip: the SP arguments plus the DIP fields, checked as
 * swDip::checkParameterConsistency does (phiG in [0,1] and not above the adjacent cells' phiW).
 * The step is swDip's (dip/swDipHyp.cpp): DIP wave speeds and specific force, DIP HLLC and
 * boundary fluxes (boundary types q, h, z, fr, phiWq), momentum dissipation. */
int sw2d_create_dip(const sw2d_mesh* mesh, const sw2d_params* params, const sw2d_cell_fields* fields,
                    const sw2d_dip_fields* dip, const sw2d_bc_table* bc, const double* h0, const double* q0,
                    const double* r0, int device, sw2d_handle** out);

/* The depth-dependent porosity (DDP) model (model_hyperb ddp, src/sw2dSolver/models/ddp/).
 *
 * A porosity-law record is one line of a DDP map file as swDdp::readPorosityFile reads it
 * (swDdp.cpp:1289-1481): {law type, n, parameters...}.  Law types (swDdp.cpp:1787-1935):
 *   -2  n couples (z_k, phi_k) used as they are;   -1  n couples re-tabulated on n_por_tab_max levels;
 *    0  n levels z_k, phi rising linearly 0 -> 1;   1  {z_0, phi}: uniform phi from z_0;
 *    2  {z_0, phi_0, z_1, phi_1} linear;            3  the same plus phi_2 above z_1.
 * Elevations are relative to the cell's bottom z_b or to the edge's midpoint elevation.
 * Record k is values[offset[k] .. offset[k+1]). */
typedef struct sw2d_ddp_records {
    const int64_t* offset;  /* [records + 1] */
    const double* values;
} sw2d_ddp_records;

enum sw2d_div_corr { SW2D_DIV_CORR_NONE = 0, SW2D_DIV_CORR_LIMIT_FLUX = 1, SW2D_DIV_CORR_LIMIT_TIMESTEP = 2 };

/* initial-condition columns (swDdp::setInitialConditions, swDdp.cpp:1608-1726): the level array
 * holds "h" (depth above the cell's lowest tabulated level) unless LEVEL_Z ("z"); the x and y
 * arrays hold unit discharges "q", "r" unless X_VELOCITY / Y_VELOCITY ("u", "v") */
#define SW2D_DDP_IC_LEVEL_Z 1
#define SW2D_DDP_IC_X_VELOCITY 2
#define SW2D_DDP_IC_Y_VELOCITY 4

typedef struct sw2d_ddp_fields {
    sw2d_ddp_records cell;          /* DDP_cell_porosity_map.txt      [cell_nb records]     */
    sw2d_ddp_records edge_int;      /* DDP_edge_int_porosity_map.txt  [edge_int_nb records] */
    sw2d_ddp_records edge_bnd;      /* DDP_edge_bnd_porosity_map.txt  [edge_bnd_nb records] */
    const double* edge_int_mz;      /* [edge_int_nb] edge midpoint elevation (swEdgeIntern::getZM) */
    const double* edge_bnd_mz;      /* [edge_bnd_nb] (swEdgeBoundary::getZM)                      */
    int64_t n_por_tab_max;          /* n_por_tab_max (default 5)                                  */
    double h_min_ddp;               /* h_min_ddp (default 1e-3)                                   */
    double chi_phi_max;             /* ddp_chi_phi_max (default 20)                               */
    double chi_theta_max;           /* ddp_chi_theta_max: read by the reference, unused in its step */
    int32_t div_corr;               /* enum sw2d_div_corr (div_corr)                              */
    int32_t ic_columns;             /* SW2D_DDP_IC_* bits                                         */
    int64_t n_it_div_max;           /* n_it_div_max (default 10)                                  */
    int32_t momentum_dissipation;   /* 0 none, 1 active (model_momentum_dissipation)              */
    int32_t pad;
    const double* mu_1;             /* [cell_nb] cell_momentum_dissipation_map.txt; NULL when inactive */
    const double* mu_2;
    const double* mu_alpha;         /* degrees */
} sw2d_ddp_fields;

/* Replaces swParent::create + swDdp::init (swParent.cpp:125-173, ddp/swDdp.cpp:780-991) for
 * model_hyperb ddp: tabulates the porosity laws as swDdp::setPorosityParameters does, checks them
 * as swDdp::checkParameterConsistency does (phi in [0,1], an edge's phi not above its cells' at
 * the same level), converts the initial conditions to the model's state (thetaW, thetaW*u,
 * thetaW*v) and sets t = t_0.  fields->phi is not read; boussinesq, friction and head-loss maps
 * are as for SP.  The step (ddp/swDdpHyp.cpp) is Godunov with the discontinuous topography only,
 * as in the reference (scheme and topo must say so); boundary types q, h, z, fr.
 * On a DDP handle sw2d_get_state / sw2d_set_state carry (thetaW, thetaW_velocity_x,
 * thetaW_velocity_y), the members of swDdp (swDdp.h:199-201); sw2d_get_array adds
 * "water_depth", "unit_discharge_x", "unit_discharge_y", "surface_elevation" (the map outputs of
 * swDdp::storeResultMaps, swDdp.cpp:2489-2513) and "thetaG_int_hmin". */
int sw2d_create_ddp(const sw2d_mesh* mesh, const sw2d_params* params, const sw2d_cell_fields* fields,
                    const sw2d_ddp_fields* ddp, const sw2d_bc_table* bc, const double* ic_level, const double* ic_x,
                    const double* ic_y, int device, sw2d_handle** out);

/* The tabulated porosity law of one record, as swDdp keeps it (cell_z_tab / phiW_tab /
 * thetaW_tab, edge_int_z_tab / phiG_int_tab / thetaG_int_tab, edge_bnd_*; swDdp.h:243-281):
 * which = 0 cells, 1 internal edges, 2 boundary edges; record in the caller's numbering.
 * Writes min(levels, capacity) values to each non-NULL array; returns the level count, < 0 on error. */
int64_t sw2d_ddp_get_table(sw2d_handle* h, int which, int64_t record, double* z, double* phi, double* theta,
                           int64_t capacity);

/* Case folders.  sw2d_load_case replaces sw2dSolver's main up to init (src/sw2dSolver/main.cpp:
 * 99-163): it reads input/input.solv (swSolverParam::readInputFile), input/geometry.sw2d version 2
 * (swMesh::readGeometryFileV2), the initial conditions, the porosity maps of the model that
 * model_hyperb names (sp, dip or ddp), the Boussinesq, friction, singular head loss and
 * momentum dissipation maps and the boundary time series, with the reference's readers' formats
 * and checks, and creates that model on `device`.  The two-step form reads first
 * (sw2d_case_read, no GPU needed), lets the caller inspect what was read (sw2d_case_array: the
 * mesh tables and fields by their sw2d_mesh / sw2d_cell_fields names, "h0"/"q0"/"r0", "bc_*",
 * "ddp_*_offset"/"_values"; sw2d_case_info: {cells, internal edges, boundary edges, model 0 sp /
 * 1 dip / 2 ddp, DDP initial-condition columns}; sw2d_case_option: an input.solv value), then
 * creates.  Errors of the reading return SW2D_E_ARG with the text in sw2d_case_last_error(). */
typedef struct sw2d_case sw2d_case;
int sw2d_load_case(const char* folder, int device, sw2d_handle** out);
int sw2d_case_read(const char* folder, sw2d_case** out);
int64_t sw2d_case_array(const sw2d_case* c, const char* name, double* out, int64_t capacity);
int sw2d_case_info(const sw2d_case* c, int64_t* sizes /* [5] */);
const char* sw2d_case_option(const sw2d_case* c, const char* key);
int sw2d_case_create(const sw2d_case* c, int device, sw2d_handle** out);
void sw2d_case_free(sw2d_case* c);
const char* sw2d_case_last_error(void);

/* Learned momentum-exchange closure (the DIP/DDP dissipation site): an MLP of 10 features ->
 * 64 -> 64 -> 2 outputs with GELU, BF16 operands and FP32 accumulation on the tensor cores
 * (tcgen05).  params: sw2d_mlp_param_count() floats, W1 [64 x 10], b1 [64], W2 [64 x 64], b2 [64],
 * W3 [2 x 64], b3 [2] (row-major, out x in).  norm: feature means [10], feature standard
 * deviations [10], output means [2], output standard deviations [2]: the network sees
 * (x - mean) / std and its outputs are scaled back by y * std + mean.  Host buffers throughout. */
typedef struct sw2d_mlp sw2d_mlp;
int sw2d_mlp_param_count(void);
int sw2d_mlp_create(int device, const float* params, const float* norm, sw2d_mlp** out);
int sw2d_mlp_destroy(sw2d_mlp* m);
const char* sw2d_mlp_last_error(sw2d_mlp* m);
int sw2d_mlp_get_params(sw2d_mlp* m, float* params);
/* outputs [n x 2] of raw features [n x 10]; `layers` (may be NULL) receives Z1, H1, Z2, H2
 * ([n x 64] each: pre-activations and activations of the two hidden layers) */
int sw2d_mlp_infer(sw2d_mlp* m, const float* features, int64_t n, float* outputs, float* layers);
/* mean squared error of the normalised outputs against targets [n x 2] and its gradient with
 * respect to the parameters ([sw2d_mlp_param_count()] floats, may be NULL) */
int sw2d_mlp_loss_grad(sw2d_mlp* m, const float* features, const float* targets, int64_t n, double* loss,
                       float* grad);
/* one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) with the gradient of the last sw2d_mlp_loss_grad */
int sw2d_mlp_adam_step(sw2d_mlp* m, float lr);
/* Poll limit of the first wait on each tensor-core chunk in this network's GEMMs (no counterpart
 * in the reference): a wait that runs out sets the status, waits once more with the full limit
 * for the MMA in flight, frees the kernel's TMEM and returns; the call then fails with
 * SW2D_E_CUDA ("tensor-core wait ran out") and the network stays usable.  polls < 0 restores the
 * default (2^26 polls, seconds); 0 makes every first wait give up at once (tests of that path). */
int sw2d_mlp_set_wait_polls(sw2d_mlp* m, int64_t polls);

/* Attaches a closure network to a DIP model (net NULL detaches).  The network then stands in
 * for the momentum-dissipation closure of the DIP balance (dip/swDipHyp.cpp:295-324): in every
 * step, after the flux balance and before the round-off flush and the sources, the cells whose
 * ten features lie within [hull_lo, hull_hi] (per feature) get the network's momentum
 * correction, and the others the plain closure (the model's mu map, when
 * model_momentum_dissipation is active), exactly as without a network.  Features, from the
 * state at the start of the step (h0, q0, r0) and after the flux balance (h, q, r): h0, q0, r0,
 * h - h0, q - q0, r - r0, phiW, the smallest phiG of the cell's internal edges, dt,
 * sqrt(q0^2 + r0^2) / max(h0, 1e-3).  Outputs: the corrections of q and r, added times `scale`.
 * The network runs inside the cell-update kernel (tensor cores): the step has no more launches.
 * The network must live on the model's device and outlive the attachment.  Option
 * "closure_record" (sw2d_set_option) keeps each step's features and outputs for
 * sw2d_closure_record. */
int sw2d_set_closure(sw2d_handle* h, sw2d_mlp* net, const float* hull_lo, const float* hull_hi, float scale);
/* The features and network outputs of every cell in the last step taken with "closure_record"
 * on, in the caller's cell order: [n_cells x 12] floats (the ten features, then the two outputs
 * in physical units before `scale` and the hull test).  Returns the number of floats written or
 * a negative status.  No counterpart in the reference (training-data capture). */
int64_t sw2d_closure_record(sw2d_handle* h, float* out, int64_t capacity);

/* Replaces the end time t_max of the run (swSp member t_max): the time step is clipped to it,
 * so a run can be brought exactly to any time. */
int sw2d_set_t_max(sw2d_handle* h, double t_max);

/* ---- binary map file (ResultHydro.bin) -------------------------------------------------------
 * The reference's output_format bin: swIO::initBinFileMapDecimal (src/common/swIO.cpp:311-645)
 * writes the header, swIO::fillBinFileMapDecimal (:285-309) one frame per stored map, with the
 * values of storeResultMaps (sp/swSp.cpp:1514-1605, dip/swDip.cpp:1657-1750,
 * ddp/swDdp.cpp:2440-2555) at the times of swParent::checkStore (swParent.cpp:46-69).
 * Header: the geometry file's part from its start to the node-to-cell lists, the variable count
 * (u64), "bottom_elevation" and the names of map_storage_mode (u64 length + bytes), t_0, t_max,
 * dt_map.  Frame: t, then per cell (caller's numbering) z_b and the mode's values (f64).
 * mode: map_storage_mode default (h, qx, qy, |q|), all (15 values) or none. */
/* ---- porosity mapper (sw2dPorosityMapper, footprint input) -------------------------------------
 * The geometry of swPorosityMapperPipeline::cellPorosity / edgePorosity
 * (src/sw2dPorosityMapper/swPorosityMapperPipeline.cpp:31-90, 256-388) and of the swGeometry
 * polygon routines they call (src/common/swGeometry.cpp), on the GPU: for every cell
 * 1 - (area inside building footprints) / area, for every edge 1 - (length inside them) / length,
 * at each level h of `levels` (a building counts at h when its height exceeds h; with
 * `height` NULL every building counts at every level, as for SP and DIP).  Outputs are
 * [element x n_levels].  Cells of up to 8 nodes, buildings of up to 64 vertices. */
typedef struct sw2d_map_mesh {
    int64_t cell_nb, node_nb, edge_int_nb, edge_bnd_nb;
    const double* node_x;
    const double* node_y;
    const int64_t* cell_node_offsets; /* [cell_nb + 1] */
    const int64_t* cell_nodes;        /* node indices of each cell */
    const double* cell_area;
    const int64_t* edge_int_nodes;    /* [edge_int_nb x 2] (node_beg, node_end) */
    const double* edge_int_length;
    const int64_t* edge_bnd_nodes;    /* [edge_bnd_nb x 2] */
    const double* edge_bnd_length;
} sw2d_map_mesh;
typedef struct sw2d_buildings {
    int64_t n;
    const int64_t* offsets; /* [n + 1] into x, y */
    const double* x;
    const double* y;
    const double* height;   /* [n] or NULL */
} sw2d_buildings;
/* edge_int_phi / edge_bnd_phi may be NULL (cells only).  Errors: SW2D_E_ARG with the text in
 * sw2d_map_last_error(). */
int sw2d_map_porosity(int device, const sw2d_map_mesh* mesh, const sw2d_buildings* buildings, const double* levels,
                      int n_levels, double* cell_phi, double* edge_int_phi, double* edge_bnd_phi);
/* The raster input (swRasterBuildings, src/sw2dPorosityMapper/swRasterBuildings.cpp): building
 * heights on a grid of pixel centres x [nx] and y [ny], both ascending, height [ny x nx] (row j at
 * y[j]); a pixel counts at level h when its height exceeds h.  A cell or an edge outside the
 * raster is an error, as in the reference. */
typedef struct sw2d_raster {
    int64_t nx, ny;
    const double* x;
    const double* y;
    const double* height;
} sw2d_raster;
int sw2d_map_porosity_raster(int device, const sw2d_map_mesh* mesh, const sw2d_raster* raster, const double* levels,
                             int n_levels, double* cell_phi, double* edge_int_phi, double* edge_bnd_phi);
const char* sw2d_map_last_error(void);

enum sw2d_result_mode { SW2D_RESULT_DEFAULT = 0, SW2D_RESULT_ALL = 1, SW2D_RESULT_NONE = 2 };
/* Writes the header alone (host only; model 0 SP, 1 DIP, 2 DDP). */
int sw2d_result_header(const char* path, const char* geometry_path, int model, int mode, double t_0, double t_max,
                       double dt_map);
/* Creates `path` with the header (t_0 and dt_map of the model, its current t_max) and attaches
 * it: sw2d_execute then appends the run's first frame (once), a frame after every step that
 * ends on a storage time, and a frame at its end, as swSp::execute does (swSp.cpp:501-632);
 * sw2d_step_n appends the frames of its steps.  Frames are copied from the device while the
 * next steps run and written by a thread of the library; sw2d_execute returns once its frames
 * are on file. */
int sw2d_result_open(sw2d_handle* h, const char* path, const char* geometry_path, int mode);
/* Waits for every frame to reach the file, closes and detaches it. */
int sw2d_result_close(sw2d_handle* h);

/* Advances at most n_steps passes of the body of swSp::execute's time loop
 * (swSp.cpp:522-589: hypCompute, friction, singular head loss, correctVelocity, t += dt),
 * stopping once t >= t_max.  The loop runs on the device (CUDA graph); the host does not
 * synchronise between steps.  *steps_done receives the number of steps taken (may be NULL). */
int sw2d_step_n(sw2d_handle* h, int64_t n_steps, int64_t* steps_done);
/* Saves the run's point on the device (state, the balance slots that carry the fluxes of edges
 * left dry from step to step, time, dt and step count); sw2d_restore_point returns the run to
 * it, so that the steps that follow give the same bits as from the saved point.  One point per
 * handle (saving again replaces it).  SP and DIP models.  No counterpart in the reference. */
int sw2d_save_point(sw2d_handle* h);
int sw2d_restore_point(sw2d_handle* h);
/* Captures and instantiates the CUDA graph sw2d_step_n launches (32 steps, or the result file's
 * chunk), without taking a step, so that a timed run does not include the capture; the graph is
 * captured again after an option or launch configuration changes.  No counterpart in the
 * reference. */
int sw2d_prepare_steps(sw2d_handle* h);

/* Replaces swSp::execute (swSp.cpp:482-670) without result storage: runs until t >= t_max. */
int sw2d_execute(sw2d_handle* h, int64_t* steps_done);

/* State access (swSp members water_depth, unit_discharge_x/_y, swSp.h:170-180), host buffers
 * of cell_nb doubles in the caller's numbering.  The copies are synchronous. */
int sw2d_get_state(sw2d_handle* h, double* water_depth, double* unit_discharge_x, double* unit_discharge_y);
int sw2d_set_state(sw2d_handle* h, const double* water_depth, const double* unit_discharge_x,
                   const double* unit_discharge_y);

/* Same, on device buffers (caller's numbering) already on the handle's device, ordered on
 * the handle's stream. */
int sw2d_get_state_device(sw2d_handle* h, double* d_water_depth, double* d_unit_discharge_x,
                          double* d_unit_discharge_y);
int sw2d_set_state_device(sw2d_handle* h, const double* d_water_depth, const double* d_unit_discharge_x,
                          const double* d_unit_discharge_y);

/* Simulation time t and the last time step dt (swSp members t, dt, swSp.h:154-156). */
int sw2d_get_time(sw2d_handle* h, double* t, double* dt);
int sw2d_set_time(sw2d_handle* h, double t, double dt);

/* Per-edge intermediate arrays of the last step, in the caller's edge numbering, for
 * kernel-level checks: name is one of "F1_int","F2_int","F3_int","s2L_int","s2R_int",
 * "F1_bnd","F2_bnd","F3_bnd","s2R_bnd","lambda_max_int","lambda_max_bnd",
 * "slope_x","slope_y" (per cell).  The fused step keeps the slopes only while the option
 * "record_fluxes" or "record_wave_speeds" is on (SW2D_E_ARG otherwise).  Returns the element
 * count written, or < 0. */
int64_t sw2d_get_array(sw2d_handle* h, const char* name, double* out, int64_t capacity);

/* Device time of each phase of the step, averaged over n_steps steps that this call runs
 * (they advance the simulation).  The analogue of the reference's per-phase clock() totals
 * (LRStates / TimeStep / Fluxes / Balance + sources, swSp.cpp:491-501,645-667): the phases are
 * the step's kernels, named by sw2d_phase_label: "k_flux", "k_update" for the fused step of the
 * SP and DIP models (LRStates + TimeStep + Fluxes, then Balance + sources), "k_slopes",
 * "k_edges", "k_cfl", "k_update" for the four-kernel step (option "fused_step" 0) and the DDP
 * model.  Launches each kernel separately with CUDA events on the handle's stream.  Returns the
 * number of phases written to ms (milliseconds), or < 0. */
int sw2d_phase_times(sw2d_handle* h, int64_t n_steps, double* ms, int capacity);
/* Name of phase i of this handle's step (sw2d_phase_times). */
const char* sw2d_phase_label(sw2d_handle* h, int i);
/* Phase names of the four-kernel step ("k_slopes", "k_edges", "k_cfl", "k_update"). */
const char* sw2d_phase_name(int i);

/* Run-time options.  "fused_step" (0/1): 1 runs each time step as k_flux (per tile of
 * consecutive cells staged with their neighbours in shared memory: Riemann states, fluxes,
 * balance terms, CFL bound and the grid's dt) and k_update, with k_slopes first for MUSCL-EVR
 * unless "fused_slopes" is 1 (then k_flux also stages the second ring of neighbours and computes
 * the slopes itself); 0 runs the four-kernel step (k_slopes, k_edges, k_cfl, k_update).  Every
 * form gives the same bits.  Default 0, the faster form on B200 for both schemes
 * (sw2d_autotune_step measures them on the caller's mesh and state).  "fused_slopes" (0/1, default 0): see above; the
 * tiles are rebuilt.  "tile_cells" (32..8192): cells per tile of the fused step (384 by
 * default, or the environment variable SW2D_TILE_CELLS read when the handle is created); the
 * tiles are rebuilt.  "flux_variant": the launch variant of k_flux (sw2d_autotune picks it).
 * "update_reverse" (0/1): k_update takes its blocks from the last cells to the first.
 * "record_wave_speeds" (0/1): also keep lambda_max per edge for
 * sw2d_get_array("lambda_max_int"/"lambda_max_bnd") (the reference's lambda_max_int/_bnd
 * members, swSp.h:201-203); off by default since the step itself only needs lambda_max * length.
 * "record_fluxes" (0/1): keep F1, F2, F3, s2L, s2R per edge for sw2d_get_array.
 * "adjoint_flush_branch" (0/1): how sw2d_adjoint differentiates the round-off flush
 * |x| < 1e-16 -> 0 after the balance (swSpHyp.cpp:197-199, assim/swSpE_hyp.cpp:390-392).  0 (the
 * default): as the identity, which is what finite differences see (a state at rest sits exactly
 * on the flush).  1: as the branch taken (zero derivative for flushed values), which is what
 * differentiating the reference's code line by line gives.
 * "adjoint_keep_nonfinite" (0/1): 1 hands back sw2d_adjoint's non-finite gradient entries as
 * they are (still counted by sw2d_adjoint_nonfinite) instead of zeroing them, to locate them.
 * "adjoint_store_states" (0/1, default 1): the segment recompute keeps each step's slopes and
 * Riemann states for the reverse steps when they fit in half of the free device memory.
 * "adjoint_trace" (0/1): record the state adjoint's magnitude per reverse step
 * (sw2d_adjoint_trace). */
int sw2d_set_option(sw2d_handle* h, const char* name, int64_t value);
/* Current value of "fused_step", "flux_variant", "tile_cells" (0 without tiles),
 * "record_fluxes" or "record_wave_speeds".  No counterpart in the reference. */
int sw2d_get_option(sw2d_handle* h, const char* name, int64_t* value);

/* Launch-configuration autotuner (no counterpart in the reference): times every
 * {threads per block, register cap} variant of the kernels of the handle's current step form
 * (k_slopes and k_edges, or k_flux) `iters` times on the current state, keeps the fastest and
 * writes a one-line report.  Those kernels recompute the same outputs from the same state; the
 * control block (time, dt, pending dt) is saved before and put back after, so the run continues
 * with the same bits as without the call.  The chosen variants can be read back and set again
 * (sw2d_get/set_launch_config, the "flux_variant" option) so that a caller can persist them. */
int sw2d_autotune(sw2d_handle* h, int iters, char* report, int capacity);
/* Step-form autotuner (no counterpart in the reference): times, on the current state, the
 * four-kernel step and the fused step at each of the n_tile_sizes tile sizes (192, 256, 320, 384,
 * 512 cells when n_tile_sizes is 0), for MUSCL-EVR with the slopes inside k_flux and with
 * k_slopes first, each at its fastest launch variant (k_update, the same in every form, is left
 * out of the sums); then sets the fastest form ("fused_step", "fused_slopes", "tile_cells",
 * "flux_variant" and the launch config can be read back to persist it).  The run continues with
 * the same bits, as for sw2d_autotune.  DDP handles: sw2d_autotune. */
int sw2d_autotune_step(sw2d_handle* h, int iters, const int* tile_sizes, int n_tile_sizes, char* report,
                       int capacity);
int sw2d_get_launch_config(sw2d_handle* h, int* slopes_variant, int* edges_variant);
int sw2d_set_launch_config(sw2d_handle* h, int slopes_variant, int edges_variant);

/* Evaluates, on device `device`, fn = 0: the portable exp, 1: the portable log used by the step
 * (no counterpart in the reference, which calls the host libm's exp/log), 2: CUDA's exp,
 * 3: CUDA's log, on n host values; for the tests of the elementary functions. */
int sw2d_eval_math(int device, int fn, const double* x, double* y, int64_t n);

/* sw2d_get_array without any allocation.  No counterpart in the reference (which keeps these
 * arrays in host memory).  For callers that must not allocate device memory once their run has
 * started: it stages the array in a fixed buffer compiled into the library (2^20 doubles =
 * 8 MiB, held by every GPU that loads the library until the process exits) instead of a
 * buffer allocated per call.  It serves the same names as sw2d_get_array, the DDP model's map
 * outputs ("water_depth", "unit_discharge_x", "unit_discharge_y", "surface_elevation",
 * "thetaG_int_hmin") included.  Arrays longer than 2^20 values are rejected with SW2D_E_ARG and
 * a message naming the limit (use sw2d_get_array for them).  The buffer's device address is
 * looked up (cudaGetSymbolAddress) once per device, by sw2d_create, sw2d_create_dip and
 * sw2d_create_ddp when they make a handle on that device, so this call itself does no set-up
 * for a handle made by them; the address stays cached for the life of the process, so after
 * cudaDeviceReset (or anything else that destroys the device's primary context) this entry
 * point must not be used again in that process.  All calls share the one buffer: calls that
 * overlap on the GPU (from several threads or handles on the same device) race; this call
 * returns only after its copy has completed. */
int64_t sw2d_get_array_noalloc(sw2d_handle* h, const char* name, double* out, int64_t capacity);

/* ---- Adjoint: gradient of an observation misfit along a recorded trajectory ----------------
 *
 * The reference differentiates its AD variant of the step with Enzyme along a frozen dt
 * sequence: swSpE::get_spatial_gradient_checkpointed (assim/swSpE_checkpoint.cpp:722-1281) over
 * ckpt_segment_E (assim/swSpE_checkpoint.cpp:584-715, assim/swSpE.h:237-251), with
 * replay_trajectory_cost as the matching cost (`func()`), gauge or frame costs
 * (assim/swSpE_gauges.cpp:166-179, assim/swSpE_ad.cpp:273-308).  Here the native step is
 * differentiated by hand-written reverse kernels, with respect to the per-cell friction
 * coefficients (Manning n for the Manning law), the initial state and the bed elevation, along
 * a trajectory whose dt sequence and boundary values are recorded once and then frozen.
 *
 * J = scale * sum over observation k, observed cell p of
 *        w_h[p] (h - h_obs[k][p])^2 + w_q[p] ((q - q_obs[k][p])^2 + (r - r_obs[k][p])^2)
 * with h, q, r the replayed state after steps[k] steps of the trajectory, scale = 1 / n_times
 * when normalize is set (the reference's cost_normalize), else 1. */
typedef struct sw2d_obs {
    int64_t n_points;       /* observed cells (gauges, or every cell for a full frame) */
    const int64_t* cells;   /* [n_points] cell indices (caller numbering), all distinct */
    const double* w_h;      /* [n_points] weights of the depth misfit */
    const double* w_q;      /* [n_points] weights of the discharge misfit, or NULL for none */
    int64_t n_times;        /* observations */
    const int64_t* steps;   /* [n_times] step index after the trajectory's start (0 = initial
                               state), strictly increasing */
    const double* h_obs;    /* [n_times * n_points], observation-major */
    const double* q_obs;    /* [n_times * n_points] or NULL when w_q is NULL */
    const double* r_obs;
    int normalize;
} sw2d_obs;

/* Gradient outputs of sw2d_adjoint: host arrays of cell_nb doubles (caller numbering); any may
 * be NULL.  friction_1 / friction_2 are the coefficients along the two friction directions
 * (swSp members friction_coeff_direction_1/_2): Manning n, Strickler K or Chezy C. */
typedef struct sw2d_gradient {
    double* h0;
    double* q0;
    double* r0;
    double* z_b;
    double* friction_1;
    double* friction_2;
} sw2d_gradient;

/* Runs n_steps CFL-driven steps from the current state (as sw2d_step_n) and records them as
 * the trajectory: the dt sequence, and checkpoints (state, balance terms, time) every
 * checkpoint_every steps.  Stops early at t_max (*steps_done tells).  The analogue of the
 * reference's dry run before its reverse loop (build_checkpoint_records,
 * assim/swSpE_checkpoint.cpp:210-425). */
int sw2d_record(sw2d_handle* h, int64_t n_steps, int64_t checkpoint_every, int64_t* steps_done);

/* Records the trajectory again from its initial state with the current parameters (new CFL dt
 * sequence, same requested length and checkpoint interval).  The reference re-runs its dry run
 * at each gradient evaluation of the minimisation (swSpE_minimize.cpp:404-410); the
 * observations stay attached to step indices. */
int sw2d_rerecord(sw2d_handle* h, int64_t* steps_done);

/* Recorded length, checkpoint interval, start time and end time of the trajectory. */
int sw2d_trajectory_info(sw2d_handle* h, int64_t* n_steps, int64_t* checkpoint_every, double* t_start,
                         double* t_end);

/* The recorded dt sequence (capacity >= n_steps). */
int sw2d_get_trajectory_dt(sw2d_handle* h, double* dt, int64_t capacity);

/* Replaces the trajectory's initial state (a control of the adjoint). */
int sw2d_set_trajectory_start(sw2d_handle* h, const double* h0, const double* q0, const double* r0);

/* Per-cell parameters (caller numbering): "friction_1", "friction_2", "friction" (both
 * directions; set only) and "z_b".  The analogue of the reference's control transform
 * (assim/swSpE.h:59-107), which writes the control into the solver before each replay.
 * Changing z_b keeps h and moves z = h + z_b, for the current state and the trajectory's
 * initial state. */
int sw2d_set_param(sw2d_handle* h, const char* name, const double* values);
int sw2d_get_param(sw2d_handle* h, const char* name, double* values);

/* Observation set of the cost (copied). */
int sw2d_set_observations(sw2d_handle* h, const sw2d_obs* obs);

/* Replays the trajectory from its initial state with the recorded dt and the current
 * parameters and returns J (replay_trajectory_cost, assim/swSpE_checkpoint.cpp:1380-1453).
 * Leaves the model at the end of the trajectory. */
int sw2d_replay_cost(sw2d_handle* h, double* J);

/* Replays the trajectory and returns h (and q, r when non-NULL) at the given cells after each
 * of the given steps: [n_times * n_points], observation-major.  For twin experiments. */
int sw2d_replay_sample(sw2d_handle* h, int64_t n_points, const int64_t* cells, int64_t n_times, const int64_t* steps,
                       double* h_out, double* q_out, double* r_out);

/* J and its gradient (get_spatial_gradient_checkpointed, assim/swSpE_checkpoint.cpp:722-1281):
 * one reverse sweep over the checkpointed segments, each recomputed forward once.  The same J
 * as sw2d_replay_cost, bit for bit.  Leaves the model at the end of the trajectory. */
int sw2d_adjoint(sw2d_handle* h, double* J, const sw2d_gradient* grad);

/* Gradient entries that came out NaN or infinite in the last sw2d_adjoint and were set to 0,
 * per control: counts[6] = {h0, q0, r0, z_b, friction_1, friction_2}.  The reference cleans its
 * gradient the same way (assim/swSpE_checkpoint.cpp:1196-1207): near-dry cells carry the
 * 1/max(h, 1e-16) factors of the wave speeds and velocities, and over long windows their
 * adjoint can overflow. */
int sw2d_adjoint_nonfinite(sw2d_handle* h, int64_t* counts);
/* With the option "adjoint_trace" on, the last sw2d_adjoint's state adjoint after each reverse
 * step j (trajectory order): entries with a non-finite component, the largest finite |adjoint of
 * h| and of q or r, and the first cell (caller numbering; -1 for none) holding a non-finite one.
 * Arrays of `capacity` values, any may be NULL; returns the trajectory's step count.  No
 * counterpart in the reference. */
int sw2d_adjoint_trace(sw2d_handle* h, int64_t* nonfinite, double* max_h, double* max_qr, int64_t* first_cell,
                       int64_t capacity);

/* ---- Ensembles ---------------------------------------------------------------------------------
 * The reference runs one simulation per process; its assimilation evaluates line-search trial
 * points and perturbed members one after another (assim/swSpE_minimize.cpp:749-840).  A batch
 * advances M independent member handles (created as usual, any sizes, models and options, on one
 * device) together: one CUDA graph holds every member's step kernels on its own stream branch,
 * so one launch advances the whole ensemble and small members run side by side.  Each member
 * keeps its own CFL time steps, t_max and status; its results are bit for bit those of the
 * member run alone.  The batch captures the members' options and launch variants when it first
 * steps; change them before that.
 *
 * When every member is an SP model of one scheme and topography discretisation (without a
 * learned closure), the batch runs by default as ONE persistent kernel over a work queue of
 * (step, phase, member, tile) items: CTAs take items in order from an atomic ticket counter;
 * an item waits (bounded) for the phase it depends on to be complete for its member; each member
 * keeps its own last-tile-done dt reduction.  The same bits as the member run alone. */
typedef struct sw2d_batch sw2d_batch;

int sw2d_batch_create(sw2d_handle* const* members, int n_members, sw2d_batch** out);

/* At most n_steps steps of every member (each stops at its own t_max); steps_done[i] (may be
 * NULL) receives member i's count.  Returns the first member error, if any
 * (sw2d_batch_last_error names the member). */
int sw2d_batch_step_n(sw2d_batch* b, int64_t n_steps, int64_t* steps_done);

/* sw2d_adjoint of every member (each with its recorded trajectory and observations), run
 * concurrently from n_threads host threads (<= 0: 16): J[i] and grads[i] (grads may be NULL). */
int sw2d_batch_adjoint(sw2d_batch* b, double* J, const sw2d_gradient* grads, int n_threads);

/* Form of the batch's step: mode 0 the graph of per-member stream branches, 1 the work queue
 * (SW2D_E_UNSUPPORTED when the members do not qualify).  For mode 1: the launch variant
 * (threads per CTA x CTAs per SM, see sw2d_batch_autotune's report) and the cells (edges) per
 * tile of an item; values < 0 (variant) or <= 0 (tiles) keep the current ones.  No counterpart
 * in the reference. */
int sw2d_batch_configure(sw2d_batch* b, int mode, int variant, int cells_per_tile, int edges_per_tile);
int sw2d_batch_get_config(sw2d_batch* b, int* mode, int* variant, int* cells_per_tile, int* edges_per_tile);
/* Times the work queue for `steps` steps at every launch variant and each of the n_tile_sizes
 * tile sizes (1024 to 16384 cells when 0), with CUDA events on the batch's stream, on the
 * members' current states (saved before and put back after every trial, so the run continues
 * with the same bits), then sets the fastest and writes a one-line report. */
int sw2d_batch_autotune(sw2d_batch* b, int steps, const int* tile_sizes, int n_tile_sizes, char* report, int capacity);
/* Poll limit of the work queue's waits (< 0: the default, about a second).  A wait that runs out
 * ends the launch with SW2D_E_CUDA ("a wait ... ran out"); the members' states are then partial. */
int sw2d_batch_set_wait_polls(sw2d_batch* b, int64_t polls);
/* The batch's stream (a cudaStream_t): the work queue runs on it. */
void* sw2d_batch_stream(sw2d_batch* b);
int sw2d_batch_size(sw2d_batch* b);
int sw2d_batch_destroy(sw2d_batch* b);   /* the member handles stay valid */
const char* sw2d_batch_last_error(sw2d_batch* b);

/* ---- Porosity assimilation: the reference's differentiated step and its gradient ---------------
 * The reference's assimilation engine (class swSpE, assim/swSpE*.cpp) runs its own variant of
 * the SP step, the "_E" step (assim/swSpE_hyp.cpp, swSpE_muscl.cpp, swSpE_friction.cpp):
 * desingularised MUSCL velocities, an HLLC with a smooth min of the porosities, every edge's
 * flux computed each step, semi-implicit Strickler friction.  These calls are its seam
 * (assim/main_enzyme.cpp:113-264), on any SP handle:
 *   sw2d_assim_record       swSpE::build_checkpoint_records  (swSpE_checkpoint.cpp:97-455)
 *   sw2d_assim_replay_cost  swSpE::replay_trajectory_cost    (swSpE_checkpoint.cpp:1311-1427)
 *   sw2d_assim_gradient     swSpE::get_spatial_gradient_checkpointed (swSpE_checkpoint.cpp:722-1281),
 *                           which the reference differentiates with Enzyme; here a hand-written
 *                           reverse sweep.
 * The control is the per-cell map m, with porosity phi = T(m) (phi_transform, swSpE.h:59-107).
 * The trajectory starts from the state and time the handle has when sw2d_assim_configure is
 * called (swSpE::save_initial_state after init) and runs to t_max.  These calls overwrite the
 * handle's state buffer (it holds the end of the last record or replay). */
#define SW2D_PHI_NONE 0
#define SW2D_PHI_CLAMP 1
#define SW2D_PHI_TANH 2
#define SW2D_PHI_NORMALIZE 3

#define SW2D_OBS_FRAMES 0   /* full-field (h, qx, qy) maps: compute_cost_frame_ptr (swSpE_ad.cpp:273-308) */
#define SW2D_OBS_GAUGES 1   /* depths at gauge cells: compute_cost_gauges_ptr (swSpE_gauges.cpp:166-179) */

/* The assimilation keys of input.solv (assim/assimConfig.h:17-55) this path reads. */
typedef struct sw2d_assim_params {
    int32_t phi_transform;           /* SW2D_PHI_*                                                */
    double lambda_tanh;              /* slope of the tanh transform                               */
    int32_t windowed;                /* windowed_assimilation                                     */
    double window_duration;          /* assimilation_window_duration (s); <= 0: unused            */
    int64_t window_steps;            /* assimilation_window_steps; <= 0: unused                   */
    int64_t n_windows;               /* n_assimilation_windows: tiles of the window (>= 1)        */
    double t_state_assimilation;     /* fallback start of the window                              */
    int32_t cost_normalize;          /* divide each observation's cost by the number of frames    */
    int32_t mask_wall_gradient;      /* zero the gradient where phi <= phi_min                    */
    int64_t forced_first_segment;    /* forced_first_seg_ of the L-BFGS-B driver; -1: none        */
} sw2d_assim_params;

typedef struct sw2d_assim_obs {
    int32_t kind;                    /* SW2D_OBS_FRAMES or SW2D_OBS_GAUGES                        */
    int32_t n_obs;
    const double* times;             /* [n_obs], increasing (s)                                   */
    const double* frames;            /* FRAMES: [n_obs][3][n_cells] h, qx, qy, caller order       */
    const double* h_weight;          /* FRAMES: [n_cells] weight of dh^2 (NULL: 1)                */
    const double* q_weight;          /* FRAMES: [n_cells] weight of dqx^2 + dqy^2 (NULL: 1)       */
    int32_t n_gauges;                /* GAUGES                                                    */
    const int64_t* gauge_cells;      /* [n_gauges] cell of each gauge (repeats allowed)           */
    const double* gauge_weight;      /* [n_gauges]                                                */
    const double* gauge_h;           /* [n_obs][n_gauges] observed depths                         */
} sw2d_assim_obs;

/* What get_spatial_gradient_checkpointed reports (its diagnostics, swSpE_checkpoint.cpp:1214-1234). */
typedef struct sw2d_assim_info {
    double J;                        /* replay cost at m (the cost the gradient belongs to)       */
    double grad_l2;                  /* ||dJ/dm||_2                                               */
    double grad_max;                 /* the entry of largest magnitude (signed)                   */
    int64_t grad_argmax;             /* its cell (caller numbering)                               */
    double dh_peak;                  /* largest ||adjoint of h||_2 at a segment start             */
    int64_t n_steps, n_segments;     /* of the recorded trajectory                                */
    int64_t first_segment;           /* first segment of the window                               */
    int64_t truncation_segment;      /* the replay starts after it (-1: from the first segment)   */
    int64_t n_tiles;                 /* tiles of the window (0: one continuous window)            */
    int64_t exploded_segment;        /* segment where the adjoint blew up (-1: none)              */
    int64_t n_nonfinite;             /* gradient entries set to 0 because not finite              */
    int64_t n_masked;                /* entries set to 0 in all (non-finite + walls)              */
} sw2d_assim_info;

int sw2d_assim_configure(sw2d_handle* h, const sw2d_assim_params* params);
int sw2d_assim_set_observations(sw2d_handle* h, const sw2d_assim_obs* obs);

/* The dry run at control m (caller numbering): the CFL time steps, snapped onto the observation
 * times, the boundary values, the observation triggers and a checkpoint every `stride` steps;
 * then the window and tiles of the gradient.  n_steps / n_segments may be NULL. */
int sw2d_assim_record(sw2d_handle* h, const double* m, int64_t stride, int64_t* n_steps, int64_t* n_segments);

/* J(m) on the recorded trajectory (frozen time steps, boundary values and triggers), from the
 * window's first checkpoint, or per tile from each tile's checkpoint. */
int sw2d_assim_replay_cost(sw2d_handle* h, const double* m, double* J);

/* record at m, then the reverse sweep: dJ/dm (required), and optionally dJ/dK1, dJ/dK2 (the
 * Strickler coefficients the _E friction reads) and dJ/d(h, qx, qy) at the start of the window
 * ([3][n_cells]); all in the caller's numbering.  info may be NULL. */
int sw2d_assim_gradient(sw2d_handle* h, const double* m, int64_t stride, double* dJ_dm, double* dJ_dk1,
                        double* dJ_dk2, double* dJ_dstate, sw2d_assim_info* info);

/* The recorded trajectory: per segment its start time and step count; per step its dt and
 * observation trigger (-1 or the observation index).  Capacities in entries. */
int sw2d_assim_segments(sw2d_handle* h, double* t_start, int64_t* n_steps, int64_t capacity);
int sw2d_assim_steps(sw2d_handle* h, double* dt, int32_t* obs_trig, int64_t capacity);
/* Replaces the start state of the trajectory (swSpE::save_initial_state); with a recorded
 * trajectory, its first checkpoint too (time steps, boundary values and triggers stay frozen). */
int sw2d_assim_set_start(sw2d_handle* h, const double* water_depth, const double* unit_discharge_x,
                         const double* unit_discharge_y);
/* The states the reference's gen-ref-e mode writes (swSpE::generate_references_E,
 * assim/swSpE_checkpoint.cpp:470-515, with storeReferenceMap at each observation trigger,
 * :360-375): the recorded trajectory replayed at control m from its start state, and for each
 * observation k that a step lands on, the state after that step, caller numbering, at
 * [k * n_cells].  n_written receives the number of observations a step landed on; the rows of
 * the others are left as they were.  Needs a recorded trajectory (sw2d_assim_record). */
int sw2d_assim_trigger_states(sw2d_handle* h, const double* m, double* water_depth, double* unit_discharge_x,
                              double* unit_discharge_y, int64_t n_obs_capacity, int64_t* n_written);
/* Checkpoint k (the state at the start of segment k), caller numbering. */
int sw2d_assim_checkpoint(sw2d_handle* h, int64_t k, double* water_depth, double* unit_discharge_x,
                          double* unit_discharge_y);

/* Internal numbering (for tests and tools): perm[new] = caller index, for cells. */
int sw2d_get_cell_permutation(sw2d_handle* h, int64_t* perm);

/* CUDA stream of the handle (cudaStream_t), for callers that order their own work on it. */
void* sw2d_get_stream(sw2d_handle* h);

/* Launches of this library's kernels per time step (for the bench's launch count). */
int sw2d_kernels_per_step(sw2d_handle* h);

int sw2d_destroy(sw2d_handle* h);

/* Text of the last error on this handle (or of the last failed sw2d_create when h is NULL). */
const char* sw2d_last_error(sw2d_handle* h);

int sw2d_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SW2D_B200_H */
