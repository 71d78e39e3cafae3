// adjoint_common.cuh — device and host helpers shared by the reverse sweeps of the native step
// (sw2d_adjoint.cu) and of the differentiated step (sw2d_assim.cu): numbering transfers, the
// mirror table of internal-neighbour entries, the observation cost and its reverse, the
// reverse of the MUSCL slope limiter, the non-finite clean-up and device allocation lists.
// Everything sits in an anonymous namespace: each translation unit keeps its own copy.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "sw2d_internal.cuh"
#include "sp_adjoint.cuh"

namespace {

using namespace sw2d;

constexpr int kCostBlocks = 256;

// dst[i*stride + offset] = src[perm[i]]: a caller-numbered array into one component of an
// internal-numbered record array
__global__ void k_gather_component(const double* __restrict__ src, const int* __restrict__ perm, double* dst, int stride,
                                   int offset, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[(size_t)i * stride + offset] = src[perm[i]];
}


// out[perm[i]] = src[i*stride + offset]: an internal-numbered array back to the caller's numbering
__global__ void k_scatter_cells(const double* __restrict__ src, int stride, int offset, const int* __restrict__ perm,
                                double* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[perm[i]] = src[(size_t)i * stride + offset];
}


// mirror[k] = the entry of the same internal edge in the neighbour's list
__global__ void k_mirror(const int2* __restrict__ coff, const int2* __restrict__ cint, int* mirror, int nc)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    for (int k = coff[c].x; k < coff[c + 1].x; k++) {
        const int2 e = cint[k];
        const int want = e.x ^ 1;
        int found = -1;
        for (int kk = coff[e.y].x; kk < coff[e.y + 1].x; kk++)
            if (cint[kk].x == want) found = kk;
        mirror[k] = found;
    }
}


// ------------------------------------------------------------------------------------------
// cost: per-block partial sums in a fixed tree, then one thread adds them in block order
// ------------------------------------------------------------------------------------------
struct ObsView {
    const int* pts;
    const double *wh, *wq;       // wq may be null
    const double *hobs, *qobs, *robs;  // this observation's values
    int n;
    double scale;                // 1 or 1 / n_obs
    int wdh;                     // term (w dh) dh instead of w (dh dh) (the reference's gauge cost)
};


__device__ __forceinline__ double obs_term(const ObsView& o, const double4* st, int i)
{
    const double4 s = st[o.pts[i]];
    const double dh = s.x - o.hobs[i];
    double v = o.wdh ? (o.wh[i] * dh) * dh : o.wh[i] * (dh * dh);
    if (o.wq) {
        const double dq = s.y - o.qobs[i], dr = s.z - o.robs[i];
        v += o.wq[i] * ((dq * dq) + (dr * dr));
    }
    return v;
}


__global__ void __launch_bounds__(kBlock) k_obs_cost(ObsView o, const double4* st, double* part)
{
    __shared__ double sh[kBlock];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < o.n; i += gridDim.x * blockDim.x) acc += obs_term(o, st, i);
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kBlock / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}


__global__ void k_obs_finish(const double* part, int nblocks, double scale, double* J_obs)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < nblocks; b++) s += part[b];
        *J_obs = s * scale;
    }
}


// d(scale * term)/d(state) at the observed cells; cells are distinct, so no two threads meet
__global__ void k_obs_rev(ObsView o, const double4* st, double4* lam)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= o.n) return;
    const int c = o.pts[i];
    const double4 s = st[c];
    double4 l = lam[c];
    l.x += 2.0 * o.wh[i] * (s.x - o.hobs[i]) * o.scale;
    if (o.wq) {
        l.y += 2.0 * o.wq[i] * (s.y - o.qobs[i]) * o.scale;
        l.z += 2.0 * o.wq[i] * (s.z - o.robs[i]) * o.scale;
    }
    lam[c] = l;
}


// Reverse of the slope limiter of cell c with up to N neighbours (entries e0 .. e0+cnt of
// cint), N fixed so that the per-neighbour values stay in registers: the cell's own z
// contribution is returned, the neighbours' go to znb.
template <int N>
__device__ __forceinline__ double slope_rev_cell(const DevMesh& m, int e0, int cnt, double zc, double2 xy, double sxb,
                                                 double syb, double* znb)
{
    constexpr int kU = N <= 4 ? N : 1;
    SlopeNbr nb[N];
    SW2D_UNROLL_KU
    for (int i = 0; i < N; i++) {
        if (i < cnt) {
            const int2 en = ld(&m.cint[e0 + i]);
            const double2 xj = ld(&m.cxy[en.y]);
            const double2 mp = ld(&m.mxy[en.x >> 1]);
            nb[i].zj = m.st[en.y].w;
            nb[i].dx = xj.x - xy.x;
            nb[i].dy = xj.y - xy.y;
            nb[i].ax = mp.x - xy.x;
            nb[i].ay = mp.y - xy.y;
            nb[i].c_is_r = (en.x & 1) != 0;
        }
    }
    double zcb = 0.0, zjb[N];
    slopes_rev_t<N>(zc, cnt, nb, sxb, syb, zcb, zjb);
    SW2D_UNROLL_KU
    for (int i = 0; i < N; i++)
        if (i < cnt) znb[e0 + i] = zjb[i];
    return zcb;
}


// Reverse of each cell's slope limiter (MUSCL-EVR): the cell's own z contribution is applied
// here, the neighbours' go to znb (one value per internal-neighbour entry).
__global__ void __launch_bounds__(kBlock) k_limiter_rev(DevMesh m, const double2* __restrict__ sgb, double4* lam,
                                                        double* gzb, double* znb)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const int e0 = ld(&m.coff[c].x), e1 = ld(&m.coff[c + 1].x);
    const int cnt = e1 - e0;
    const double2 b = sgb[c];
    if (b.x == 0.0 && b.y == 0.0) {
        for (int i = e0; i < e1; i++) znb[i] = 0.0;
        return;
    }
    const double zc = m.st[c].w;
    const double2 xy = ld(&m.cxy[c]);
    double zcb = 0.0;
    if (cnt <= 3) zcb = slope_rev_cell<3>(m, e0, cnt, zc, xy, b.x, b.y, znb);
    else if (cnt == 4) zcb = slope_rev_cell<4>(m, e0, cnt, zc, xy, b.x, b.y, znb);
    else if (cnt <= kMaxNbr) zcb = slope_rev_cell<kMaxNbr>(m, e0, cnt, zc, xy, b.x, b.y, znb);
    else atomicOr(&m.ctrl->status, kStatusUnsupported);  // degree beyond the reverse's table
    lam[c].x += zcb;
    gzb[c] += zcb;
}


// z contributions of the neighbours' slope limiters, gathered in the cell's entry order (the
// first kPre entries' loads in flight together)
__global__ void __launch_bounds__(kBlock) k_nbr_rev(DevMesh m, const int* __restrict__ mirror,
                                                    const double* __restrict__ znb, double4* lam, double* gzb)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    constexpr int kPre = 4;
    const int e0 = ld(&m.coff[c].x), e1 = ld(&m.coff[c + 1].x);
    int mk[kPre];
    double z[kPre];
#pragma unroll
    for (int i = 0; i < kPre; i++)
        if (e0 + i < e1) mk[i] = ld_now(&mirror[e0 + i]);  // every internal edge has an entry on both sides
#pragma unroll
    for (int i = 0; i < kPre; i++)
        if (e0 + i < e1 && mk[i] >= 0) z[i] = ld_now(&znb[mk[i]]);
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < kPre; i++)
        if (e0 + i < e1 && mk[i] >= 0) s += z[i];
    for (int k = e0 + kPre; k < e1; k++) {
        const int mk = ld(&mirror[k]);  // every internal edge has an entry on both sides
        if (mk >= 0) s += znb[mk];
    }
    lam[c].x += s;
    gzb[c] += s;
}


// Non-finite gradient entries -> 0, counted per control (h0, q0, r0, z_b, friction_1,
// friction_2): the reference's final clean-up of its gradient (assim/swSpE_checkpoint.cpp:
// 1196-1207).  Near-dry cells carry the 1/max(h, 1e-16) factors of the wave speeds and
// velocities; over long windows their adjoint can overflow, in the reference as here.
// keep = true counts them without zeroing (the option "adjoint_keep_nonfinite", to locate them).
__device__ __forceinline__ void clean(double& v, unsigned long long* count, bool keep = false)
{
    if (!isfinite(v)) {
        if (!keep) v = 0.0;
        atomicAdd(count, 1ull);
    }
}

// ------------------------------------------------------------------------------------------
// device allocations owned by a list
// ------------------------------------------------------------------------------------------
template <class T>
int adj_alloc(sw2d_handle* h, std::vector<void*>& list, size_t n, T** out)
{
    void* p = nullptr;
    CK(cudaMalloc(&p, std::max<size_t>(1, n) * sizeof(T)));
    list.push_back(p);
    CK(cudaMemsetAsync(p, 0, std::max<size_t>(1, n) * sizeof(T), h->stream));
    *out = static_cast<T*>(p);
    return SW2D_OK;
}

void free_list(std::vector<void*>& list)
{
    for (void* p : list) cudaFree(p);
    list.clear();
}

}  // namespace
