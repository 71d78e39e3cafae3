// sw2d_queue.cu — the ensemble step as one persistent kernel over a work queue of mesh tiles.
//
// An ensemble (4D-Var line-search trial points, perturbed-friction members, meshes of uneven
// sizes) advances K steps in one launch of k_queue.  The work is a list of items
// (step, phase, member, tile): the phases of one step are the four of the SP step (slopes,
// edges, CFL bound, update; no slopes for Godunov), a tile is a block of consecutive cells (or
// edges) of one member.  CTAs take items in list order from an atomic ticket counter, so an
// item's prerequisites, which all come earlier in the list, were taken by CTAs that are already
// running: the queue cannot deadlock, whatever the number of resident CTAs.
//
// Order of the list: step by step, phase by phase, member by member, tile by tile.  An item
// waits (thread 0, bounded polls) for the phase it depends on to be complete for its member:
//   slopes(s)  on update(s-1)       edges(s)  on slopes(s) (Godunov: update(s-1))
//   cfl(s)     on edges(s)          update(s) on the member's dt of step s
// Each member counts its finished tiles per phase (monotonic over the launch, zeroed before
// it).  Its CFL tiles fold their minima into an order-preserving integer key (atomicMin); the
// tile that finishes the phase last snaps and clips dt (dt_finalize) and publishes it.  The
// arithmetic is that of the step kernels (sp_phases.cuh, read through L2 because other CTAs of
// the launch wrote the data), so every member's results are bit for bit those of the member run
// alone.  A wait that runs out sets the queue's status word; every CTA then leaves the queue,
// and the host reports the error.
//
// Memory ordering: an item's thread 0 takes the counter of its prerequisite with a gpu-scope
// acquire load and the CTA then passes a barrier; a finished item passes a barrier, and its
// thread 0 fences (gpu scope) and increments its counter.  That release/acquire chain orders
// every write of a prerequisite before every plain load of the item that depends on it.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "sp_phases.cuh"
#include "sw2d_internal.cuh"

namespace sw2d {

namespace {

constexpr int kPhaseSlopes = 0, kPhaseEdges = 1, kPhaseCfl = 2, kPhaseUpdate = 3;

// how the phases read what other CTAs of the launch wrote (sp_phases.cuh): plain loads after
// the item's acquire and barrier
using LdQ = LdCo;
constexpr unsigned kQueueTimeout = 1u;

struct QMember {
    DevMesh m;
    int n_cell_tiles;
    int n_edge_tiles;
    int friction;
    int head_loss;
};

struct QSync {
    unsigned done[4];   // tiles finished per phase during this launch
    unsigned dt_ready;  // steps of this launch whose dt is published
    unsigned pad[3];
};

struct QArgs {
    const QMember* mem;
    QSync* sync;
    unsigned long long* dmin;  // per member: running minimum key of the CFL bounds (kDminEmpty between steps)
    const unsigned* items;  // one step's items: phase << 30 | member << 20 | tile
    unsigned items_per_step;
    unsigned total;         // items of the launch (steps * items_per_step)
    int cells_per_tile;
    int edges_per_tile;
    unsigned* next;         // ticket counter
    unsigned* status;       // kQueueTimeout when a wait ran out
    long long max_polls;
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool active(const Ctrl* c) { return __ldcg(&c->t) < __ldcg(&c->t_max); }

// thread 0: wait until *p >= target, at most max_polls polls; false (and the queue's status set)
// when the wait ran out or another CTA's did
__device__ bool wait_at_least(const QArgs& q, const unsigned* p, unsigned target)
{
    long long polls = 0;
    while (ld_acquire(p) < target) {
        if (++polls > q.max_polls || ld_acquire(q.status) != 0u) {
            atomicOr(q.status, kQueueTimeout);
            return false;
        }
        __nanosleep(64);
    }
    return true;
}

// The phases of one tile, each a separate (not inlined) function over its element range with a
// stride of the CTA size: each gets its own register allocation, and a call is made once per
// item, not per element.
__device__ __noinline__ void q_slopes(const DevMesh& m, int c0, int c1, int stride)
{
    for (int c = c0; c < c1; c += stride) slopes_cell<LdQ>(m, c);
}

template <int kScheme, bool kBlending>
__device__ __noinline__ unsigned q_edges(const DevMesh& m, int i0, int i1, int stride)
{
    unsigned bad = 0;
    for (int i = i0; i < i1; i += stride)
        bad |= (i < m.ni) ? edge_internal<kScheme, kBlending, kModelSp, LdQ>(m, i)
                          : edge_boundary<kScheme, kModelSp, LdQ>(m, i - m.ni);
    return bad;
}

__device__ __noinline__ double q_cfl(const DevMesh& m, int c0, int c1, int stride, double best)
{
    for (int c = c0; c < c1; c += stride) {
        const double x = cfl_cell<LdQ>(m, c);
        if (x < best) best = x;
    }
    return best;
}

template <int kFriction, bool kHeadLoss>
__device__ __noinline__ void q_update(const DevMesh& m, int c0, int c1, int stride, double dt)
{
    for (int c = c0; c < c1; c += stride) update_cell<kFriction, kHeadLoss, false, false, LdQ>(m, c, dt);
}

template <int kFriction>
__device__ __forceinline__ void q_update_h(const DevMesh& m, int c0, int c1, int stride, double dt, bool hl)
{
    if (hl) q_update<kFriction, true>(m, c0, c1, stride, dt);
    else q_update<kFriction, false>(m, c0, c1, stride, dt);
}

template <int kScheme, bool kBlending, int kThreads, int kMinB>
__global__ void __launch_bounds__(kThreads, kMinB) k_queue(QArgs q)
{
    constexpr bool kMuscl = kScheme == SW2D_SCHEME_MUSCL_EVR;
    __shared__ DevMesh sm;
    __shared__ unsigned s_item;
    __shared__ int s_mem, s_ok, s_go;
    __shared__ double s_dt;
    __shared__ double wmin[kThreads / 32];
    if (threadIdx.x == 0) s_mem = -1;
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(q.next, 1u);
        __syncthreads();
        const unsigned it = s_item;
        if (it >= q.total) break;
        const unsigned s = it / q.items_per_step;
        const unsigned code = __ldg(&q.items[it % q.items_per_step]);
        const int phase = (int)(code >> 30), mi = (int)((code >> 20) & 1023u), tile = (int)(code & 0xfffffu);
        const QMember& qm = q.mem[mi];
        QSync* sy = q.sync + mi;
        const unsigned nct = (unsigned)__ldg(&qm.n_cell_tiles), net = (unsigned)__ldg(&qm.n_edge_tiles);
        // the member's mesh view, into shared memory when the member changes (s_mem is written
        // by thread 0 only after the last barrier of an item)
        if (mi != s_mem) {
            const int* src = reinterpret_cast<const int*>(&qm.m);
            int* dst = reinterpret_cast<int*>(&sm);
            for (int k = threadIdx.x; k < (int)(sizeof(DevMesh) / sizeof(int)); k += kThreads) dst[k] = __ldg(src + k);
        }
        if (threadIdx.x == 0) {
            bool ok;
            if (phase == kPhaseSlopes) ok = wait_at_least(q, &sy->done[kPhaseUpdate], s * nct);
            else if (phase == kPhaseEdges)
                ok = kMuscl ? wait_at_least(q, &sy->done[kPhaseSlopes], (s + 1) * nct)
                            : wait_at_least(q, &sy->done[kPhaseUpdate], s * nct);
            else if (phase == kPhaseCfl) ok = wait_at_least(q, &sy->done[kPhaseEdges], (s + 1) * net);
            else ok = wait_at_least(q, &sy->dt_ready, s + 1);
            s_ok = ok;
            if (ok && phase == kPhaseUpdate) {
                s_go = __ldcg(&qm.m.ctrl->go);
                s_dt = __ldcg(&qm.m.ctrl->dt);
            }
        }
        __syncthreads();
        if (!s_ok) break;
        const DevMesh& m = sm;
        Ctrl* ctrl = m.ctrl;
        const int c0 = tile * q.cells_per_tile + threadIdx.x, c1 = min(m.nc, (tile + 1) * q.cells_per_tile);
        if (phase == kPhaseSlopes) {
            if (active(ctrl)) q_slopes(m, c0, c1, kThreads);
        } else if (phase == kPhaseEdges) {
            if (active(ctrl)) {
                const int i1 = min(m.ni + m.nb, (tile + 1) * q.edges_per_tile);
                const unsigned bad = q_edges<kScheme, kBlending>(m, tile * q.edges_per_tile + threadIdx.x, i1, kThreads);
                if (bad) atomicOr(&ctrl->status, bad);
            }
        } else if (phase == kPhaseCfl) {
            const bool act = active(ctrl);
            double best = m.dt_max;
            if (act) best = q_cfl(m, c0, c1, kThreads, best);
            for (int off = 16; off > 0; off >>= 1) best = min_keep(best, __shfl_down_sync(0xffffffffu, best, off));
            if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = best;
            __syncthreads();
            if (threadIdx.x == 0) {
                for (int w = 1; w < kThreads / 32; w++) best = min_keep(best, wmin[w]);
                if (act) atomicMin(&q.dmin[mi], dmin_key((unsigned long long)__double_as_longlong(best)));
            }
        } else if (s_go) {
            const double dt = s_dt;
            if (tile == 0 && threadIdx.x == 0) {
                ctrl->t = __ldcg(&ctrl->t) + dt;  // swSp.cpp:592
                ctrl->steps = __ldcg(&ctrl->steps) + 1;
            }
            const bool hl = __ldg(&qm.head_loss) != 0;
            switch (__ldg(&qm.friction)) {
                case SW2D_FRICTION_CHEZY: q_update_h<SW2D_FRICTION_CHEZY>(m, c0, c1, kThreads, dt, hl); break;
                case SW2D_FRICTION_MANNING: q_update_h<SW2D_FRICTION_MANNING>(m, c0, c1, kThreads, dt, hl); break;
                case SW2D_FRICTION_STRICKLER: q_update_h<SW2D_FRICTION_STRICKLER>(m, c0, c1, kThreads, dt, hl); break;
                default: q_update_h<SW2D_FRICTION_NONE>(m, c0, c1, kThreads, dt, hl); break;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            const unsigned done = atomicAdd(&sy->done[phase], 1u);
            if (phase == kPhaseCfl && done == (s + 1) * nct - 1) {
                // the member's last CFL tile of step s: publish its dt (or stop the member)
                __threadfence();
                const unsigned long long key = atomicExch(&q.dmin[mi], kDminEmpty);
                if (active(ctrl)) dt_finalize<false, LdQ>(m, ctrl, __longlong_as_double((long long)dmin_bits(key)));
                else ctrl->go = 0;
                __threadfence();
                atomicExch(&sy->dt_ready, s + 1);
            }
            s_mem = mi;
        }
    }
}

struct QueueVariant {
    int threads, minb;
};
constexpr QueueVariant kQueueVariants[] = {{256, 2}, {256, 3}, {128, 4}, {128, 6}, {512, 1}};
constexpr int kNumQueueVariants = (int)(sizeof(kQueueVariants) / sizeof(QueueVariant));

template <int kScheme, bool kBlending, int V>
void* queue_fn()
{
    return reinterpret_cast<void*>(&k_queue<kScheme, kBlending, kQueueVariants[V].threads, kQueueVariants[V].minb>);
}

template <int kScheme, bool kBlending>
void* queue_fn_v(int v)
{
    switch (v) {
        case 1: return queue_fn<kScheme, kBlending, 1>();
        case 2: return queue_fn<kScheme, kBlending, 2>();
        case 3: return queue_fn<kScheme, kBlending, 3>();
        case 4: return queue_fn<kScheme, kBlending, 4>();
        default: return queue_fn<kScheme, kBlending, 0>();
    }
}

void* queue_kernel(int scheme, bool blending, int v)
{
    if (scheme == SW2D_SCHEME_GODUNOV) return blending ? queue_fn_v<SW2D_SCHEME_GODUNOV, true>(v) : queue_fn_v<SW2D_SCHEME_GODUNOV, false>(v);
    return blending ? queue_fn_v<SW2D_SCHEME_MUSCL_EVR, true>(v) : queue_fn_v<SW2D_SCHEME_MUSCL_EVR, false>(v);
}

}  // namespace

struct QueueState {
    int scheme = 0;
    bool blending = false;
    int variant = 0;
    int cells_per_tile = 0, edges_per_tile = 0;
    int grid = 0;
    int n = 0;
    unsigned items_per_step = 0;
    long long max_polls = 1ll << 25;
    QMember* d_mem = nullptr;
    QSync* d_sync = nullptr;
    unsigned long long* d_dmin = nullptr;
    unsigned* d_items = nullptr;
    unsigned* d_next = nullptr;    // ticket counter, then the status word
    std::vector<QMember> h_mem;
};

int queue_eligible(sw2d_handle* const* members, int n, std::string& why)
{
    if (n <= 0 || n > 1024) {
        why = "the queue takes 1 to 1024 members";
        return 0;
    }
    for (int i = 0; i < n; i++) {
        const sw2d_handle* h = members[i];
        if (h->model != kModelSp) why = "member " + std::to_string(i) + " is not an SP model";
        else if (h->closure) why = "member " + std::to_string(i) + " has a learned closure";
        else if (h->p.scheme != members[0]->p.scheme) why = "members differ in scheme";
        else if (h->p.topo != members[0]->p.topo) why = "members differ in topography discretisation";
        if (!why.empty()) return 0;
    }
    return 1;
}

void queue_release(QueueState* q)
{
    if (!q) return;
    cudaFree(q->d_mem);
    cudaFree(q->d_sync);
    cudaFree(q->d_dmin);
    cudaFree(q->d_items);
    cudaFree(q->d_next);
    delete q;
}

// (Re)builds the item table and the members' views for the given tile sizes and variant.
int queue_build(QueueState*& q, sw2d_handle* const* members, int n, int variant, int cells_per_tile, int edges_per_tile,
                std::string& why)
{
    if (variant < 0 || variant >= kNumQueueVariants) {
        why = "queue variant outside the variants";
        return SW2D_E_ARG;
    }
    if (cells_per_tile < 32 || edges_per_tile < 32 || cells_per_tile > (1 << 16) || edges_per_tile > (1 << 16)) {
        why = "queue tile sizes outside 32..65536";
        return SW2D_E_ARG;
    }
    if (!q) q = new QueueState();
    q->scheme = members[0]->p.scheme;
    q->blending = members[0]->p.topo == SW2D_TOPO_BLENDING;
    q->variant = variant;
    q->cells_per_tile = cells_per_tile;
    q->edges_per_tile = edges_per_tile;
    const bool muscl = q->scheme == SW2D_SCHEME_MUSCL_EVR;
    q->h_mem.assign(n, QMember{});
    std::vector<unsigned> items;
    for (int i = 0; i < n; i++) {
        const sw2d_handle* h = members[i];
        QMember& qm = q->h_mem[i];
        qm.m = h->m;
        qm.n_cell_tiles = (int)((h->nc + cells_per_tile - 1) / cells_per_tile);
        qm.n_edge_tiles = (int)((h->ni + h->nb + edges_per_tile - 1) / edges_per_tile);
        qm.friction = h->p.friction;
        qm.head_loss = h->p.singular_head_loss ? 1 : 0;
        if (qm.n_cell_tiles > (1 << 20) || qm.n_edge_tiles > (1 << 20)) {
            why = "member " + std::to_string(i) + " has more than 2^20 tiles";
            return SW2D_E_ARG;
        }
    }
    for (int p = muscl ? kPhaseSlopes : kPhaseEdges; p <= kPhaseUpdate; p++)
        for (int i = 0; i < n; i++) {
            const int nt = (p == kPhaseEdges) ? q->h_mem[i].n_edge_tiles : q->h_mem[i].n_cell_tiles;
            for (int t = 0; t < nt; t++) items.push_back((unsigned)p << 30 | (unsigned)i << 20 | (unsigned)t);
        }
    q->items_per_step = (unsigned)items.size();
    cudaFree(q->d_mem);
    cudaFree(q->d_sync);
    cudaFree(q->d_dmin);
    cudaFree(q->d_items);
    q->d_mem = nullptr;
    q->d_sync = nullptr;
    q->d_dmin = nullptr;
    q->d_items = nullptr;
    q->n = n;
    cudaError_t e = cudaMalloc(&q->d_mem, n * sizeof(QMember));
    if (e == cudaSuccess) e = cudaMalloc(&q->d_sync, n * sizeof(QSync));
    if (e == cudaSuccess) e = cudaMalloc(&q->d_dmin, n * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&q->d_items, items.size() * sizeof(unsigned));
    if (e == cudaSuccess && !q->d_next) e = cudaMalloc(&q->d_next, 2 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemcpy(q->d_mem, q->h_mem.data(), n * sizeof(QMember), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(q->d_items, items.data(), items.size() * sizeof(unsigned), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(q->d_next, 0, 2 * sizeof(unsigned));
    // a persistent grid: as many CTAs as can be resident at once
    const void* fn = queue_kernel(q->scheme, q->blending, variant);
    int per_sm = 0, sms = 0, dev = 0;
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kQueueVariants[variant].threads, 0);
    if (e != cudaSuccess) {
        why = std::string("queue set-up: ") + cudaGetErrorString(e);
        return SW2D_E_CUDA;
    }
    q->grid = std::max(1, per_sm) * sms;
    return SW2D_OK;
}

// Enqueues on `stream` the launch that advances every member by `steps` steps: the members'
// counters and the ticket counter are zeroed first (both captured in a graph by the caller).
int queue_launch(QueueState* q, int steps, cudaStream_t stream)
{
    cudaError_t e = cudaMemsetAsync(q->d_sync, 0, q->n * sizeof(QSync), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(q->d_dmin, 0xff, q->n * sizeof(unsigned long long), stream);  // kDminEmpty
    if (e == cudaSuccess) e = cudaMemsetAsync(q->d_next, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return SW2D_E_CUDA;
    QArgs a;
    a.mem = q->d_mem;
    a.sync = q->d_sync;
    a.dmin = q->d_dmin;
    a.items = q->d_items;
    a.items_per_step = q->items_per_step;
    const unsigned long long total = (unsigned long long)steps * q->items_per_step;
    if (total >= (1ull << 32)) return SW2D_E_ARG;
    a.total = (unsigned)total;
    a.cells_per_tile = q->cells_per_tile;
    a.edges_per_tile = q->edges_per_tile;
    a.next = q->d_next;
    a.status = q->d_next + 1;
    a.max_polls = q->max_polls;
    void* args[] = {&a};
    e = cudaLaunchKernel(queue_kernel(q->scheme, q->blending, q->variant), dim3(q->grid),
                         dim3(kQueueVariants[q->variant].threads), args, 0, stream);
    return e == cudaSuccess ? SW2D_OK : SW2D_E_CUDA;
}

unsigned queue_read_status(QueueState* q)
{
    unsigned st = 0;
    cudaMemcpy(&st, q->d_next + 1, sizeof(unsigned), cudaMemcpyDeviceToHost);
    return st;
}

void queue_clear_status(QueueState* q) { cudaMemset(q->d_next + 1, 0, sizeof(unsigned)); }

int queue_variants() { return kNumQueueVariants; }

std::string queue_variant_label(int v)
{
    return std::to_string(kQueueVariants[v].threads) + "x" + std::to_string(kQueueVariants[v].minb);
}

void queue_set_polls(QueueState* q, long long polls) { q->max_polls = polls; }

int queue_grid(const QueueState* q) { return q->grid; }

}  // namespace sw2d
