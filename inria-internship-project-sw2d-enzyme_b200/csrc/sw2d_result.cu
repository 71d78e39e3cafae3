// sw2d_result.cu — the run's binary map file (ResultHydro.bin) as the reference writes it:
// swIO::initBinFileMapDecimal (src/common/swIO.cpp:311-645) for the header, then one frame per
// stored map, swIO::fillBinFileMapDecimal (:285-309), with the values of storeResultMaps
// (sp/swSp.cpp:1514-1605, dip/swDip.cpp:1657-1750, ddp/swDdp.cpp:2440-2555) and the storage
// times of swParent::checkStore (swParent.cpp:46-69) inside swSp::execute (swSp.cpp:501-632);
// DDP decides them with the time step instead (ddp/swDdpHyp.cpp:590-609, swDdp.cpp:676-682).
//
// File layout (host byte order, as the reference's std::ofstream::write):
//   header  the geometry file's bytes from its start to the end of the node-to-cell lists (the
//           reference reads and writes them field by field, in file order), the variable count
//           (u64: the names + 1), "bottom_elevation" and each name (u64 length + bytes), then
//           t_0, t_max, dt_map (f64)
//   frame   t (f64), then per cell in the caller's numbering: z_b and the mode's variables (f64)
//
// Frames come from the device.  With a file attached, every step ends with k_frame: where the
// step ran and stores a map (checkStore's test on the new time, or DDP's flag), it writes
// the frame into a ring of device slots in the file's layout, and k_frame_commit counts it.
// The host drains the ring after each chunk of steps: a copy into pinned memory on a side
// stream, then a writer thread appends it to the file while the next chunk computes.  A chunk
// has at most as many steps as half the ring, and the host waits before a chunk until the
// frames of the chunk before last are on file: no slot is written while it is being read.
#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <fstream>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/sw2d_b200.h"
#include "sw2d_internal.cuh"

namespace sw2d {

constexpr int kMaxRing = 16;

struct FrameCtl {
    long long count;  // frames written into the ring so far
    double time[kMaxRing];
};

struct ResultWriter {
    int mode = SW2D_RESULT_DEFAULT;
    int nv = 0;             // values per cell in a frame (z_b included)
    int ring = 2, half = 1;  // device slots; steps per chunk
    int64_t frame_vals = 0;  // nc * nv
    double* d_ring = nullptr;
    FrameCtl* d_fc = nullptr;
    std::vector<double*> host;  // pinned, one per slot
    cudaStream_t cs = nullptr;
    std::vector<cudaEvent_t> ev;
    long long issued = 0;  // frames handed to the writer thread
    bool any = false;      // a frame has been stored (the run's first)
    // the writer thread
    std::FILE* f = nullptr;
    std::thread th;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<std::pair<int, double>> q;
    long long written = 0;
    bool stop = false;
    std::string io_err;
    int device = 0;
};

namespace {

// storeResultMaps's values of one cell, z_b first (the file skips x and y)
template <int kModel>
__device__ __forceinline__ void frame_values(const DevMesh& m, int c, int mode, double* v)
{
    const double4 s = m.st[c];
    const double4 cs = m.cst[c];
    if (kModel == kModelDdp) {
        // swDdp.cpp:2476-2497: h from the free surface, u = thetaW u / thetaW where wet
        const double h = smax(0.0, s.w - cs.z);
        double u = 0.0, w = 0.0;
        if (s.x > kSmallReal) {
            u = s.y / s.x;
            w = s.z / s.x;
        }
        v[0] = cs.z;
        v[1] = h;
        v[2] = u * h;
        v[3] = w * h;
        v[4] = h * sqrt(u * u + w * w);
        if (mode == SW2D_RESULT_ALL) {  // swDdp.cpp:2500-2530
            const double z = s.w;
            const double vn = sqrt(u * u + w * w);
            unsigned bad = 0;
            const int o = m.ctoff[c], n = m.ctoff[c + 1] - o;
            const double phi = ddp::phi_theta(m.ctab + o, n, z, bad).phi;  // phiWOfZ
            v[5] = z;
            v[6] = u;
            v[7] = w;
            v[8] = vn;
            v[9] = vn / ddp::celerity(s.x, phi);
            v[10] = h + 0.5 * vn * vn / kGravity;
            v[11] = z + 0.5 * vn * vn / kGravity;
            v[12] = s.x;
            v[13] = u * s.x;
            v[14] = w * s.x;
            v[15] = vn * s.x;
        }
        return;
    }
    const double h = s.x, qx = s.y, qy = s.z, zb = cs.x;
    const double qn = sqrt(qx * qx + qy * qy);  // swSp.cpp:1555-1556
    v[0] = zb;
    v[1] = h;
    v[2] = qx;
    v[3] = qy;
    v[4] = qn;
    if (mode == SW2D_RESULT_ALL) {  // swSp.cpp:1565-1585 (phiW for DIP, dip/swDip.cpp:1708-1728)
        const double phi = cs.z;
        v[5] = h + zb;
        v[6] = qx / smax(h, kSmallReal);
        v[7] = qy / smax(h, kSmallReal);
        const double vn = sqrt(qx * qx + qy * qy) / smax(kSmallReal, h);
        v[8] = vn;
        v[9] = vn / smax(sqrt(kGravity * h), kSmallReal);
        v[10] = h + 0.5 * vn * vn / kGravity;
        v[11] = v[10] + zb;
        v[12] = h * phi;
        v[13] = qx * phi;
        v[14] = qy * phi;
        v[15] = qn;
    }
}

// swParent::checkStore (swParent.cpp:58-69) on the time at the end of the step
__device__ __forceinline__ bool store_due(double t, double dt_map)
{
    if (dt_map <= -kSmallReal) return true;
    if (dt_map > kSmallReal) return (t / dt_map) == (double)(int)(t / dt_map);
    return false;
}

// whether the step just taken stores a map: SP and DIP test the new time (checkStore), DDP
// decided it with the time step (swDdpHyp.cpp:590-609, k_cfl's store_map)
template <int kModel>
__device__ __forceinline__ bool stored(const DevMesh& m)
{
    if (!m.ctrl->go) return false;
    if (kModel == kModelDdp) return m.ctrl->store_map != 0;
    return store_due(m.ctrl->t, m.dt_map);
}

template <int kModel>
__global__ void k_frame(DevMesh m, const int* __restrict__ perm, double* ring, const FrameCtl* fc, int nslots,
                        int nv, int mode, int forced)
{
    if (!forced && !stored<kModel>(m)) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    double v[16];
    frame_values<kModel>(m, c, mode, v);
    double* dst = ring + (size_t)(fc->count % nslots) * (size_t)m.nc * nv + (size_t)perm[c] * nv;
    for (int k = 0; k < nv; k++) dst[k] = v[k];
}

template <int kModel>
__global__ void k_frame_commit(DevMesh m, FrameCtl* fc, int nslots, int forced)
{
    if (!forced && !stored<kModel>(m)) return;
    fc->time[fc->count % nslots] = m.ctrl->t;
    fc->count += 1;
}

void writer_loop(ResultWriter* w)
{
    cudaSetDevice(w->device);
    for (;;) {
        std::pair<int, double> job;
        {
            std::unique_lock<std::mutex> lk(w->mu);
            w->cv.wait(lk, [&] { return w->stop || !w->q.empty(); });
            if (w->q.empty()) return;  // stop requested and nothing left
            job = w->q.front();
        }
        bool ok = cudaEventSynchronize(w->ev[job.first]) == cudaSuccess;
        if (ok && w->io_err.empty()) {
            ok = std::fwrite(&job.second, sizeof(double), 1, w->f) == 1 &&
                 std::fwrite(w->host[job.first], sizeof(double), (size_t)w->frame_vals, w->f) == (size_t)w->frame_vals;
        }
        std::lock_guard<std::mutex> lk(w->mu);
        if (!ok && w->io_err.empty()) w->io_err = "writing a frame of the result file failed";
        w->q.pop_front();
        w->written += 1;
        w->cv.notify_all();
    }
}

const std::vector<std::string>& var_names(int model, int mode)
{
    // the names of swSp::init / swDip::init / swDdp::init (swSp.cpp:733-744, swDip.cpp:789-800,
    // swDdp.cpp:794-805)
    static const std::vector<std::string> none;
    static const std::vector<std::string> def = {"water_depth", "unit_discharge_x", "unit_discharge_y",
                                                 "unit_discharge_norm"};
    static const std::vector<std::string> all = {"water_depth", "unit_discharge_x", "unit_discharge_y",
                                                 "unit_discharge_norm", "surface_elevation", "velocity_x",
                                                 "velocity_y", "velocity_norm", "froude", "specific_head",
                                                 "total_head", "phi_by_water_depth", "phi_by_unit_discharge_x",
                                                 "phi_by_unit_discharge_y", "phi_by_unit_discharge_norm"};
    static const std::vector<std::string> ddp_def = {"water_depth", "unit_discharge_x", "unit_discharge_y",
                                                     "unit_disch_norm"};
    static const std::vector<std::string> ddp_all = {"water_depth", "unit_discharge_x", "unit_discharge_y",
                                                     "unit_disc_norm", "surface_elevation", "velocity_x",
                                                     "velocity_y", "velocity_norm", "froude", "specific_head",
                                                     "total_head", "phi_by_wat_depth", "phi_by_disc_x",
                                                     "phi_by_disc_y", "phi_by_disc_norm"};
    if (mode == SW2D_RESULT_NONE) return none;
    if (model == kModelDdp) return mode == SW2D_RESULT_ALL ? ddp_all : ddp_def;
    return mode == SW2D_RESULT_ALL ? all : def;
}

// length of the geometry file's part that the header repeats: version, counts, cells, nodes,
// boundary and internal edges, the per-code edge lists and codes, the per-cell links and the
// node-to-cell lists (the node-to-edge lists that may follow are not repeated)
bool geometry_prefix(const std::vector<char>& b, size_t& len, std::string& why)
{
    size_t off = 0;
    auto take = [&](size_t n, void* dst) {
        if (off + n > b.size()) return false;
        if (dst) std::memcpy(dst, b.data() + off, n);
        off += n;
        return true;
    };
    uint64_t vlen = 0, nc = 0, nb = 0, ni = 0, nn = 0, nbnd = 0;
    if (!take(8, &vlen) || vlen > 64 || !take(vlen, nullptr) || !take(8, &nc) || !take(8, &nb) || !take(8, &ni) ||
        !take(8, &nn) || !take(8, &nbnd)) {
        why = "geometry file truncated in its counts";
        return false;
    }
    std::vector<uint64_t> links(nc);
    for (uint64_t i = 0; i < nc; i++) {  // idx, sms, nodes, bnd edges, int edges, neighbours, 5 f64
        uint64_t cnt[6];
        if (!take(48, cnt) || !take(40, nullptr)) {
            why = "geometry file truncated in its cells";
            return false;
        }
        links[i] = cnt[2] + cnt[3] + cnt[4] + cnt[5];
    }
    std::vector<uint64_t> node_cells(nn);
    for (uint64_t p = 0; p < nn; p++) {  // idx, sms, x, y, z, cells, edges
        uint64_t rec[7];
        if (!take(56, rec)) {
            why = "geometry file truncated in its nodes";
            return false;
        }
        node_cells[p] = rec[5];
    }
    if (!take(nb * 92, nullptr) || !take(ni * 96, nullptr)) {
        why = "geometry file truncated in its edges";
        return false;
    }
    for (uint64_t k = 0; k < nbnd; k++) {
        uint64_t n = 0;
        if (!take(8, &n) || n > b.size() || !take(n * 8, nullptr)) {
            why = "geometry file truncated in its boundary lists";
            return false;
        }
    }
    if (!take(nbnd * 4, nullptr)) {
        why = "geometry file truncated in its boundary codes";
        return false;
    }
    for (uint64_t i = 0; i < nc; i++)
        if (links[i] > b.size() || !take(links[i] * 8, nullptr)) {
            why = "geometry file truncated in its cell links";
            return false;
        }
    for (uint64_t p = 0; p < nn; p++)
        if (node_cells[p] > b.size() || !take(node_cells[p] * 8, nullptr)) {
            why = "geometry file truncated in its node links";
            return false;
        }
    len = off;
    return true;
}

int write_header(const char* path, const char* geometry_path, int model, int mode, double t_0, double t_max,
                 double dt_map, std::string& why, int64_t* cells)
{
    std::ifstream g(geometry_path, std::ios::binary);
    if (!g) {
        why = std::string("cannot open ") + geometry_path;
        return SW2D_E_ARG;
    }
    std::vector<char> b((std::istreambuf_iterator<char>(g)), std::istreambuf_iterator<char>());
    size_t len = 0;
    if (!geometry_prefix(b, len, why)) return SW2D_E_ARG;
    uint64_t nc = 0;
    std::memcpy(&nc, b.data() + 8 + *reinterpret_cast<const uint64_t*>(b.data()), 8);
    if (cells) *cells = (int64_t)nc;
    std::FILE* f = std::fopen(path, "wb");
    if (!f) {
        why = std::string("cannot create ") + path;
        return SW2D_E_IO;
    }
    bool ok = std::fwrite(b.data(), 1, len, f) == len;
    const auto& names = var_names(model, mode);
    const uint64_t nvar = names.size() + 1;
    ok = ok && std::fwrite(&nvar, 8, 1, f) == 1;
    auto put = [&](const std::string& s) {
        const uint64_t n = s.size();
        ok = ok && std::fwrite(&n, 8, 1, f) == 1 && std::fwrite(s.data(), 1, n, f) == n;
    };
    put("bottom_elevation");
    for (const auto& s : names) put(s);
    ok = ok && std::fwrite(&t_0, 8, 1, f) == 1 && std::fwrite(&t_max, 8, 1, f) == 1 &&
         std::fwrite(&dt_map, 8, 1, f) == 1;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) {
        why = std::string("writing ") + path + " failed";
        return SW2D_E_IO;
    }
    return SW2D_OK;
}

template <int kModel>
void launch_frame_m(sw2d_handle* h, int forced)
{
    ResultWriter* w = h->result;
    k_frame<kModel><<<grid_for(h->nc), kBlock, 0, h->stream>>>(h->m, h->d_cell_perm, w->d_ring, w->d_fc, w->ring,
                                                              w->nv, w->mode, forced);
}

void launch_frame(sw2d_handle* h, int forced)
{
    ResultWriter* w = h->result;
    if (w->mode == SW2D_RESULT_NONE) return;
    if (h->model == kModelDdp) {
        launch_frame_m<kModelDdp>(h, forced);
        k_frame_commit<kModelDdp><<<1, 1, 0, h->stream>>>(h->m, w->d_fc, w->ring, forced);
    } else {
        launch_frame_m<kModelSp>(h, forced);
        k_frame_commit<kModelSp><<<1, 1, 0, h->stream>>>(h->m, w->d_fc, w->ring, forced);
    }
}

void writer_free(ResultWriter* w)
{
    if (!w) return;
    if (w->th.joinable()) {
        {
            std::lock_guard<std::mutex> lk(w->mu);
            w->stop = true;
        }
        w->cv.notify_all();
        w->th.join();
    }
    if (w->f) std::fclose(w->f);
    for (double* p : w->host)
        if (p) cudaFreeHost(p);
    for (cudaEvent_t e : w->ev)
        if (e) cudaEventDestroy(e);
    if (w->cs) cudaStreamDestroy(w->cs);
    if (w->d_ring) cudaFree(w->d_ring);
    if (w->d_fc) cudaFree(w->d_fc);
    delete w;
}

}  // namespace

void result_after_step(sw2d_handle* h) { launch_frame(h, 0); }

int result_chunk(const sw2d_handle* h) { return h->result->half; }

// Waits until at most `in_flight` frames are not yet on file.
int result_wait(sw2d_handle* h, long long in_flight)
{
    ResultWriter* w = h->result;
    std::unique_lock<std::mutex> lk(w->mu);
    w->cv.wait(lk, [&] { return w->issued - w->written <= in_flight; });
    if (!w->io_err.empty()) return fail(h, SW2D_E_IO, w->io_err);
    return SW2D_OK;
}

// Hands the frames the device stored since the last call to the writer thread; the caller has
// synchronised the handle's stream.
int result_drain(sw2d_handle* h)
{
    ResultWriter* w = h->result;
    if (w->mode == SW2D_RESULT_NONE) return SW2D_OK;
    FrameCtl fc;
    CK(cudaMemcpy(&fc, w->d_fc, sizeof(FrameCtl), cudaMemcpyDeviceToHost));
    if (fc.count - w->issued > w->ring) return fail(h, SW2D_E_IO, "result frames overran the device ring");
    for (long long k = w->issued; k < fc.count; k++) {
        const int slot = (int)(k % w->ring);
        CK(cudaMemcpyAsync(w->host[slot], w->d_ring + (size_t)slot * (size_t)w->frame_vals,
                           (size_t)w->frame_vals * sizeof(double), cudaMemcpyDeviceToHost, w->cs));
        CK(cudaEventRecord(w->ev[slot], w->cs));
        std::lock_guard<std::mutex> lk(w->mu);
        w->q.emplace_back(slot, fc.time[slot]);
        w->issued += 1;
        w->any = true;
        w->cv.notify_all();
    }
    return SW2D_OK;
}

// A frame of the current state, whatever the time (the run's first and last maps).
int result_force(sw2d_handle* h)
{
    ResultWriter* w = h->result;
    if (w->mode == SW2D_RESULT_NONE) {
        w->any = true;
        return SW2D_OK;
    }
    int rc = result_wait(h, w->ring - 1);
    if (rc) return rc;
    launch_frame(h, 1);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    return result_drain(h);
}

bool result_started(const sw2d_handle* h) { return h->result->any; }

void result_release(sw2d_handle* h)
{
    writer_free(h->result);
    h->result = nullptr;
}

}  // namespace sw2d

using namespace sw2d;

extern "C" {

int sw2d_result_header(const char* path, const char* geometry_path, int model, int mode, double t_0, double t_max,
                       double dt_map)
{
    if (!path || !geometry_path || model < 0 || model > 2 || mode < 0 || mode > 2) return SW2D_E_ARG;
    std::string why;
    return write_header(path, geometry_path, model, mode, t_0, t_max, dt_map, why, nullptr);
}

int sw2d_result_open(sw2d_handle* h, const char* path, const char* geometry_path, int mode)
{
    if (!h) return SW2D_E_ARG;
    if (!path || !geometry_path || mode < 0 || mode > 2) return fail(h, SW2D_E_ARG, "invalid arguments");
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    result_release(h);
    CK(cudaMemcpy(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    std::string why;
    int64_t cells = 0;
    int rc = write_header(path, geometry_path, h->model, mode, h->p.t_0, h->ctrl_host->t_max, h->p.dt_map, why, &cells);
    if (rc) return fail(h, rc, why);
    if (cells != h->nc) return fail(h, SW2D_E_ARG, "the geometry file's cell count differs from the model's");
    ResultWriter* w = new ResultWriter();
    w->device = h->device;
    w->mode = mode;
    w->nv = mode == SW2D_RESULT_ALL ? 16 : 5;
    w->frame_vals = h->nc * w->nv;
    // ring slots: up to 16, within about 1 GiB of frames
    const double frame_bytes = (double)w->frame_vals * sizeof(double);
    w->ring = (int)std::max(2.0, std::min((double)kMaxRing, std::floor((1024.0 * 1024.0 * 1024.0) / frame_bytes)));
    w->ring -= w->ring % 2;
    w->half = w->ring / 2;
    bool ok = (w->f = std::fopen(path, "ab")) != nullptr;
    if (!ok) {
        writer_free(w);
        return fail(h, SW2D_E_IO, std::string("cannot append to ") + path);
    }
    cudaError_t e = cudaSuccess;
    if (mode != SW2D_RESULT_NONE) {
        e = cudaMalloc(&w->d_ring, (size_t)w->ring * (size_t)frame_bytes);
        if (e == cudaSuccess) e = cudaMalloc(&w->d_fc, sizeof(FrameCtl));
        if (e == cudaSuccess) e = cudaMemset(w->d_fc, 0, sizeof(FrameCtl));
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&w->cs, cudaStreamNonBlocking);
        w->host.assign(w->ring, nullptr);
        w->ev.assign(w->ring, nullptr);
        for (int s = 0; s < w->ring && e == cudaSuccess; s++) {
            e = cudaMallocHost(&w->host[s], (size_t)frame_bytes);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w->ev[s], cudaEventDisableTiming);
        }
    }
    if (e != cudaSuccess) {
        writer_free(w);
        return fail(h, SW2D_E_CUDA, std::string("result buffers: ") + cudaGetErrorString(e));
    }
    w->th = std::thread(writer_loop, w);
    h->result = w;
    if (h->graph) {  // the captured steps lack the frame kernels
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    return SW2D_OK;
}

int sw2d_result_close(sw2d_handle* h)
{
    if (!h) return SW2D_E_ARG;
    if (!h->result) return SW2D_OK;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    int rc = result_wait(h, 0);
    std::FILE* f = h->result->f;
    h->result->f = nullptr;
    const bool closed = f ? std::fclose(f) == 0 : true;
    result_release(h);
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    if (rc) return rc;
    if (!closed) return fail(h, SW2D_E_IO, "closing the result file failed");
    return SW2D_OK;
}

}  // extern "C"
