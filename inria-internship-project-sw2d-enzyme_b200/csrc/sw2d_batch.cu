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
// The gradients of an ensemble come from the members' adjoints run concurrently from a pool of
// host threads (one handle per thread at a time; handles are independent).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
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
    if (full > 0) {
        if ((rc = ensure_graph(b, chunk))) return rc;
        for (int64_t k = 0; k < full; k++) BCK(cudaGraphLaunch(b->graph, b->stream));
    }
    if (rem > 0) {
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

int sw2d_batch_size(sw2d_batch* b) { return b ? (int)b->members.size() : 0; }

int sw2d_batch_destroy(sw2d_batch* b)
{
    if (!b) return SW2D_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (auto e : b->joins)
        if (e) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return SW2D_OK;
}

const char* sw2d_batch_last_error(sw2d_batch* b) { return b ? b->err.c_str() : g_batch_create_error.c_str(); }

}  // extern "C"
