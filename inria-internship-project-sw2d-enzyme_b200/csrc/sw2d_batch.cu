// sw2d_batch.cu — ensembles of independent simulations (4D-Var line-search trial points,
// perturbed-friction members, meshes of uneven sizes) advanced together on one GPU.
//
// A batch holds M member handles created as usual (any mesh, model, options).  Its step is one
// CUDA graph holding every member's step kernels, one stream branch per member: the branches
// fork from the batch's stream, run concurrently on the device, and join again.  One graph
// launch therefore advances the whole ensemble by a chunk of steps, and the small members,
// whose kernels alone cannot fill the GPU, run side by side instead of one after another.
// Each member keeps its own device-side control block, so each takes its own CFL time steps and
// stops at its own t_max; its results are bit for bit those of the same member run alone.
//
// When every member is an SP model of one scheme and topography discretisation (no learned
// closure), the batch runs instead as one persistent kernel over a work queue of
// (step, phase, member, tile) items (sw2d_queue.cu): no per-member launches, no per-member grid
// reductions between kernels, and the same bits.  sw2d_batch_configure picks the form, the tile
// sizes and the launch variant; sw2d_batch_autotune times them on the members' current states
// (saved and restored around each trial).
//
// The gradients of an ensemble come from the members' adjoints run concurrently from a pool of
// host threads (one handle per thread at a time; handles are independent).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "sw2d_internal.cuh"

using namespace sw2d;

struct sw2d_batch {
    int device = 0;
    std::vector<sw2d_handle*> members;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> joins;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    // work-queue form
    sw2d::QueueState* queue = nullptr;
    int mode = 0;  // SW2D_BATCH_BRANCHES or SW2D_BATCH_QUEUE
    int q_variant = 3, q_cells = 4096, q_edges = 4096;  // 128 threads x 6 CTAs per SM, the C4 ensemble's best
    cudaGraphExec_t qgraph = nullptr;
    int qgraph_steps = 0;
    std::string err;
};

namespace {

std::string g_batch_create_error;

int bfail(sw2d_batch* b, int code, const std::string& msg)
{
    if (b) b->err = msg;
    else g_batch_create_error = msg;
    return code;
}

#define BCK(call)                                                                                     \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) return bfail(b, SW2D_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// graph of `steps` steps of every member: fork from the batch's stream, one branch per member
// on the member's own stream, join back
int ensure_graph(sw2d_batch* b, int steps)
{
    if (b->graph && b->graph_steps == steps) return SW2D_OK;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaGraph_t g;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaEventRecord(b->fork, b->stream);
    for (size_t i = 0; i < b->members.size() && e == cudaSuccess; i++) {
        sw2d_handle* h = b->members[i];
        e = cudaStreamWaitEvent(h->stream, b->fork, 0);
        for (int s = 0; s < steps && e == cudaSuccess; s++) launch_step_on(h);
        if (e == cudaSuccess) e = cudaEventRecord(b->joins[i], h->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->joins[i], 0);
    }
    const cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
    if (e != cudaSuccess || e2 != cudaSuccess)
        return bfail(b, SW2D_E_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
    const cudaError_t e3 = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e3 != cudaSuccess) return bfail(b, SW2D_E_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(e3));
    b->graph_steps = steps;
    return SW2D_OK;
}

// graph of `steps` steps of the work-queue form: counters zeroed, then the persistent kernel
int ensure_qgraph(sw2d_batch* b, int steps)
{
    if (b->qgraph && b->qgraph_steps == steps) return SW2D_OK;
    if (b->qgraph) {
        cudaGraphExecDestroy(b->qgraph);
        b->qgraph = nullptr;
    }
    cudaGraph_t g;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = queue_launch(b->queue, steps, b->stream);
    const cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
    if (rc != SW2D_OK || e2 != cudaSuccess) return bfail(b, SW2D_E_CUDA, "work-queue graph capture failed");
    const cudaError_t e3 = cudaGraphInstantiate(&b->qgraph, g, 0);
    cudaGraphDestroy(g);
    if (e3 != cudaSuccess) return bfail(b, SW2D_E_CUDA, std::string("work-queue graph instantiate: ") + cudaGetErrorString(e3));
    b->qgraph_steps = steps;
    return SW2D_OK;
}

// the work-queue form: n_steps steps of every member on the batch's stream
int queue_steps(sw2d_batch* b, int64_t n_steps)
{
    // work queued on the members' own streams comes first
    for (sw2d_handle* h : b->members) BCK(cudaStreamSynchronize(h->stream));
    const int chunk = 32;
    const int64_t full = n_steps / chunk, rem = n_steps % chunk;
    int rc;
    if (full > 0) {
        if ((rc = ensure_qgraph(b, chunk))) return rc;
        for (int64_t k = 0; k < full; k++) BCK(cudaGraphLaunch(b->qgraph, b->stream));
    }
    if (rem > 0 && queue_launch(b->queue, (int)rem, b->stream) != SW2D_OK)
        return bfail(b, SW2D_E_CUDA, "work-queue launch failed");
    BCK(cudaGetLastError());
    BCK(cudaStreamSynchronize(b->stream));
    if (queue_read_status(b->queue)) {
        queue_clear_status(b->queue);
        return bfail(b, SW2D_E_CUDA, "work queue: a wait for a member's phase ran out (members' states are partial)");
    }
    return SW2D_OK;
}

// members' step counters (and status words) into their pinned control copies
int read_controls(sw2d_batch* b)
{
    for (sw2d_handle* h : b->members)
        BCK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
    for (sw2d_handle* h : b->members) BCK(cudaStreamSynchronize(h->stream));
    return SW2D_OK;
}

}  // namespace

extern "C" {

int sw2d_batch_create(sw2d_handle* const* members, int n_members, sw2d_batch** out)
{
    sw2d_batch* b = nullptr;
    if (!out || !members || n_members <= 0) return bfail(b, SW2D_E_ARG, "invalid arguments");
    *out = nullptr;
    for (int i = 0; i < n_members; i++) {
        if (!members[i]) return bfail(b, SW2D_E_ARG, "NULL member handle");
        if (members[i]->result) return bfail(b, SW2D_E_ARG, "a member has a result file attached");
        if (members[i]->device != members[0]->device)
            return bfail(b, SW2D_E_ARG, "batch members must share one device");
        for (int j = 0; j < i; j++)
            if (members[j] == members[i]) return bfail(b, SW2D_E_ARG, "a handle appears twice in the batch");
    }
    b = new sw2d_batch();
    b->device = members[0]->device;
    b->members.assign(members, members + n_members);
    auto bail = [&](int code) {
        g_batch_create_error = b->err;
        sw2d_batch_destroy(b);
        return code;
    };
    if (cudaSetDevice(b->device) != cudaSuccess) return bail(bfail(b, SW2D_E_NO_DEVICE, "cudaSetDevice failed"));
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
        return bail(bfail(b, SW2D_E_CUDA, "stream or event creation failed"));
    b->joins.assign(n_members, nullptr);
    for (auto& e : b->joins)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            return bail(bfail(b, SW2D_E_CUDA, "event creation failed"));
    // work already queued on the members' streams (uploads, earlier steps) comes first
    for (sw2d_handle* h : b->members)
        if (cudaStreamSynchronize(h->stream) != cudaSuccess)
            return bail(bfail(b, SW2D_E_CUDA, "member stream synchronisation failed"));
    std::string why;
    if (queue_eligible(members, n_members, why)) {
        if (queue_build(b->queue, members, n_members, b->q_variant, b->q_cells, b->q_edges, why) == SW2D_OK) b->mode = 1;
        else return bail(bfail(b, SW2D_E_CUDA, why));
    }
    *out = b;
    return SW2D_OK;
}

int sw2d_batch_step_n(sw2d_batch* b, int64_t n_steps, int64_t* steps_done)
{
    if (!b || n_steps < 0) return bfail(b, SW2D_E_ARG, "invalid arguments");
    BCK(cudaSetDevice(b->device));
    const size_t M = b->members.size();
    int rc = read_controls(b);
    if (rc) return rc;
    std::vector<long long> before(M);
    for (size_t i = 0; i < M; i++) before[i] = b->members[i]->ctrl_host->steps;
    const int chunk = 32;
    const int64_t full = n_steps / chunk, rem = n_steps % chunk;
    if (b->mode == 1) {
        if ((rc = queue_steps(b, n_steps))) return rc;
    } else if (full > 0) {
        if ((rc = ensure_graph(b, chunk))) return rc;
        for (int64_t k = 0; k < full; k++) BCK(cudaGraphLaunch(b->graph, b->stream));
    }
    if (b->mode == 0 && rem > 0) {
        // the remainder, eagerly, on each member's stream after the graph's work
        BCK(cudaEventRecord(b->fork, b->stream));
        for (size_t i = 0; i < M; i++) {
            sw2d_handle* h = b->members[i];
            BCK(cudaStreamWaitEvent(h->stream, b->fork, 0));
            for (int64_t s = 0; s < rem; s++) launch_step_on(h);
        }
    }
    BCK(cudaGetLastError());
    BCK(cudaStreamSynchronize(b->stream));
    if ((rc = read_controls(b))) return rc;
    int first = SW2D_OK;
    for (size_t i = 0; i < M; i++) {
        sw2d_handle* h = b->members[i];
        if (steps_done) steps_done[i] = h->ctrl_host->steps - before[i];
        const int st = status_to_code(h, h->ctrl_host->status);
        if (st && first == SW2D_OK) {
            first = st;
            b->err = "member " + std::to_string(i) + ": " + h->err;
        }
    }
    return first;
}

int sw2d_batch_adjoint(sw2d_batch* b, double* J, const sw2d_gradient* grads, int n_threads)
{
    if (!b || !J) return bfail(b, SW2D_E_ARG, "invalid arguments");
    const int M = (int)b->members.size();
    const int T = std::max(1, std::min(n_threads > 0 ? n_threads : 16, M));
    std::vector<int> codes(M, SW2D_OK);
    std::atomic<int> next{0};
    auto work = [&] {
        for (int i = next++; i < M; i = next++)
            codes[i] = sw2d_adjoint(b->members[i], &J[i], grads ? &grads[i] : nullptr);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < T; t++) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    for (int i = 0; i < M; i++)
        if (codes[i] != SW2D_OK) {
            b->err = "member " + std::to_string(i) + ": " + b->members[i]->err;
            return codes[i];
        }
    return SW2D_OK;
}

int sw2d_batch_configure(sw2d_batch* b, int mode, int variant, int cells_per_tile, int edges_per_tile)
{
    if (!b || (mode != 0 && mode != 1)) return bfail(b, SW2D_E_ARG, "invalid arguments");
    BCK(cudaSetDevice(b->device));
    if (mode == 1) {
        std::string why;
        if (!queue_eligible(b->members.data(), (int)b->members.size(), why))
            return bfail(b, SW2D_E_UNSUPPORTED, "work queue: " + why);
        const int v = variant >= 0 ? variant : b->q_variant;
        const int ct = cells_per_tile > 0 ? cells_per_tile : b->q_cells;
        const int et = edges_per_tile > 0 ? edges_per_tile : b->q_edges;
        BCK(cudaStreamSynchronize(b->stream));
        const int rc = queue_build(b->queue, b->members.data(), (int)b->members.size(), v, ct, et, why);
        if (rc) return bfail(b, rc, why);
        b->q_variant = v;
        b->q_cells = ct;
        b->q_edges = et;
        if (b->qgraph) {
            cudaGraphExecDestroy(b->qgraph);
            b->qgraph = nullptr;
        }
    }
    b->mode = mode;
    return SW2D_OK;
}

int sw2d_batch_get_config(sw2d_batch* b, int* mode, int* variant, int* cells_per_tile, int* edges_per_tile)
{
    if (!b) return bfail(b, SW2D_E_ARG, "invalid arguments");
    if (mode) *mode = b->mode;
    if (variant) *variant = b->q_variant;
    if (cells_per_tile) *cells_per_tile = b->q_cells;
    if (edges_per_tile) *edges_per_tile = b->q_edges;
    return SW2D_OK;
}

int sw2d_batch_set_wait_polls(sw2d_batch* b, int64_t polls)
{
    if (!b || !b->queue) return bfail(b, SW2D_E_ARG, "no work queue");
    queue_set_polls(b->queue, polls >= 0 ? (long long)polls : (1ll << 25));
    if (b->qgraph) {  // the graph holds the previous limit
        cudaGraphExecDestroy(b->qgraph);
        b->qgraph = nullptr;
    }
    return SW2D_OK;
}

int sw2d_batch_autotune(sw2d_batch* b, int steps, const int* tile_sizes, int n_tile_sizes, char* report, int capacity)
{
    if (!b || steps <= 0 || n_tile_sizes < 0 || (n_tile_sizes && !tile_sizes)) return bfail(b, SW2D_E_ARG, "invalid arguments");
    std::string why;
    if (!queue_eligible(b->members.data(), (int)b->members.size(), why)) return bfail(b, SW2D_E_UNSUPPORTED, "work queue: " + why);
    BCK(cudaSetDevice(b->device));
    static const int kTiles[] = {1024, 2048, 4096, 8192, 16384};
    if (!n_tile_sizes) {
        tile_sizes = kTiles;
        n_tile_sizes = (int)(sizeof(kTiles) / sizeof(int));
    }
    const size_t M = b->members.size();
    // the members' states, balance slots (which carry the fluxes of edges left dry) and control
    // blocks are saved, and put back after each trial
    std::vector<void*> saved(M, nullptr);
    std::vector<size_t> st_bytes(M), sl_bytes(M);
    auto release = [&] {
        for (void* p : saved) cudaFree(p);
    };
    for (size_t i = 0; i < M; i++) {
        sw2d_handle* h = b->members[i];
        BCK(cudaStreamSynchronize(h->stream));
        st_bytes[i] = (size_t)h->nc * sizeof(double4);
        sl_bytes[i] = (size_t)h->h_coff.back().y * sizeof(Slot);
        if (cudaMalloc(&saved[i], st_bytes[i] + sl_bytes[i] + sizeof(Ctrl)) != cudaSuccess) {
            release();
            return bfail(b, SW2D_E_CUDA, "autotune: no memory for the members' saved states");
        }
        char* d = static_cast<char*>(saved[i]);
        cudaMemcpyAsync(d, h->m.st, st_bytes[i], cudaMemcpyDeviceToDevice, b->stream);
        cudaMemcpyAsync(d + st_bytes[i], h->m.slot, sl_bytes[i], cudaMemcpyDeviceToDevice, b->stream);
        cudaMemcpyAsync(d + st_bytes[i] + sl_bytes[i], h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToDevice, b->stream);
    }
    auto restore = [&] {
        for (size_t i = 0; i < M; i++) {
            sw2d_handle* h = b->members[i];
            const char* d = static_cast<const char*>(saved[i]);
            cudaMemcpyAsync(h->m.st, d, st_bytes[i], cudaMemcpyDeviceToDevice, b->stream);
            cudaMemcpyAsync(h->m.slot, d + st_bytes[i], sl_bytes[i], cudaMemcpyDeviceToDevice, b->stream);
            cudaMemcpyAsync(h->ctrl, d + st_bytes[i] + sl_bytes[i], sizeof(Ctrl), cudaMemcpyDeviceToDevice, b->stream);
        }
    };
    cudaEvent_t e0, e1;
    BCK(cudaEventCreate(&e0));
    BCK(cudaEventCreate(&e1));
    std::string rep;
    double best = 1e300;
    int bv = b->q_variant, bc = b->q_cells, be = b->q_edges;
    for (int v = 0; v < queue_variants(); v++)
        for (int k = 0; k < n_tile_sizes; k++) {
            const int tile = tile_sizes[k];
            if (queue_build(b->queue, b->members.data(), (int)M, v, tile, tile, why) != SW2D_OK) continue;
            queue_launch(b->queue, 1, b->stream);  // warm
            restore();
            cudaEventRecord(e0, b->stream);
            const int rc = queue_launch(b->queue, steps, b->stream);
            cudaEventRecord(e1, b->stream);
            cudaEventSynchronize(e1);
            restore();
            cudaStreamSynchronize(b->stream);
            if (rc != SW2D_OK || queue_read_status(b->queue)) {
                queue_clear_status(b->queue);
                continue;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            const double per = (double)ms / steps;
            rep += queue_variant_label(v) + "/tile" + std::to_string(tile) + "=" + std::to_string(per) + "ms ";
            if (per < best) {
                best = per;
                bv = v;
                bc = tile;
                be = tile;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    BCK(cudaStreamSynchronize(b->stream));
    release();
    const int rc = queue_build(b->queue, b->members.data(), (int)M, bv, bc, be, why);
    if (rc) return bfail(b, rc, why);
    b->q_variant = bv;
    b->q_cells = bc;
    b->q_edges = be;
    b->mode = 1;
    if (b->qgraph) {
        cudaGraphExecDestroy(b->qgraph);
        b->qgraph = nullptr;
    }
    rep += "chosen " + queue_variant_label(bv) + "/tile" + std::to_string(bc) + " (" + std::to_string(queue_grid(b->queue)) +
           " CTAs)";
    if (report && capacity > 0) {
        std::strncpy(report, rep.c_str(), (size_t)capacity - 1);
        report[capacity - 1] = '\0';
    }
    return SW2D_OK;
}

void* sw2d_batch_stream(sw2d_batch* b) { return b ? (void*)b->stream : nullptr; }

int sw2d_batch_size(sw2d_batch* b) { return b ? (int)b->members.size() : 0; }

int sw2d_batch_destroy(sw2d_batch* b)
{
    if (!b) return SW2D_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->qgraph) cudaGraphExecDestroy(b->qgraph);
    queue_release(b->queue);
    for (auto e : b->joins)
        if (e) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return SW2D_OK;
}

const char* sw2d_batch_last_error(sw2d_batch* b) { return b ? b->err.c_str() : g_batch_create_error.c_str(); }

}  // extern "C"
