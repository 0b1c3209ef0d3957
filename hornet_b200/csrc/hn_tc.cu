// TriangleCounting2 (hornetsnest/src/Static/TriangleCounting/triangle2.cu:75-171
// with forAllAdjUnions, primitives/Operator++.i.cuh:319-522).
//
// The reference counts on a graph read with DIRECTED_BY_DEGREE | SORT
// (hornetsnest/test/TriangleTest2.cu:86-87): every undirected edge is kept
// once, from the lower-(degree, id) endpoint (xlib/src/Graph/GraphStd.cpp:
// 247-268), so each triangle is found exactly once.  It then bins all
// directed edges by log-degree pair with 64-bit global atomics (two passes)
// and runs ~37 intersection launches.
//
// Here the orientation is built on the device from the (always sorted)
// undirected adjacency in two merge-path balanced passes around one scan:
//   pass 1  keep flag of every edge (needs deg(v): one 16-byte record read),
//   scan    flag positions = the oriented CSR,
//   pass 2  compact the kept neighbours (lists stay sorted).
// The intersection then runs one thread per oriented edge (u,v): the
// shorter of N+(u), N+(v) is walked and each element is found in the
// longer one by a binary search whose lower bound only moves forward.
#include <cub/cub.cuh>

#include "hn_graph.cuh"
#include "hn_tc.cuh"

namespace hn {

namespace {

constexpr int kB = 256;
using Tile = LbTile<kB, 4>;

__device__ __forceinline__ bool oriented_before(int du, int u, int dv, int v) {
    return du < dv || (du == dv && u < v);
}

__global__ void __launch_bounds__(kB)
k_orient_flags(const long long* __restrict__ prefix, int nV, const VRec* __restrict__ vtab,
               const int32_t* __restrict__ pool, int32_t* __restrict__ flag) {
    __shared__ Tile t;
    __shared__ long long s_base[Tile::TILE + 1];
    __shared__ int s_deg[Tile::TILE + 1];
    const long long total = prefix[nV];
    const long long ntiles = (total + nV + Tile::TILE - 1) / Tile::TILE;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int n = lb_tile_load(t, prefix, (long long)nV, total, tile);
        for (int b = threadIdx.x; b <= t.nends; b += kB) {
            long long u = t.seg0 + b;
            if (u < nV) {
                VRec r = vtab[u];
                s_base[b] = r.off - t.seg_start(b);
                s_deg[b] = r.deg;
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += kB) {
            long long e = t.item0 + i;
            int b = t.seg[i];
            int u = (int)(t.seg0 + b);
            int v = pool[s_base[b] + e];
            flag[e] = oriented_before(s_deg[b], u, vtab[v].deg, v) ? 1 : 0;
        }
        __syncthreads();
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) flag[total] = 0;
}

__global__ void __launch_bounds__(kB)
k_orient_fill(const long long* __restrict__ prefix, int nV, const VRec* __restrict__ vtab,
              const int32_t* __restrict__ pool, const int32_t* __restrict__ pos,
              int32_t* __restrict__ fwd, long long* __restrict__ offp) {
    __shared__ Tile t;
    __shared__ long long s_base[Tile::TILE + 1];
    const long long total = prefix[nV];
    const long long ntiles = (total + nV + Tile::TILE - 1) / Tile::TILE;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int n = lb_tile_load(t, prefix, (long long)nV, total, tile);
        for (int b = threadIdx.x; b <= t.nends; b += kB) {
            long long u = t.seg0 + b;
            if (u < nV) s_base[b] = vtab[u].off - t.seg_start(b);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += kB) {
            long long e = t.item0 + i;
            int p = pos[e];
            if (pos[e + 1] != p) fwd[p] = pool[s_base[t.seg[i]] + e];
        }
        __syncthreads();
    }
    // offp[u] = pos[prefix[u]]
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u <= nV;
         u += (long long)gridDim.x * blockDim.x)
        offp[u] = pos[prefix[u]];
}

// |A ∩ B| for sorted A (shorter) and B; optional per-match callback.
template <bool PER_VERTEX>
__device__ __forceinline__ long long intersect_count(const int32_t* A, long long la,
                                                     const int32_t* B, long long lb,
                                                     unsigned long long* per_vertex) {
    long long cnt = 0, lo = 0;
    if (la == 0 || lb == 0) return 0;
    if (A[la - 1] < B[0] || B[lb - 1] < A[0]) return 0;
    for (long long i = 0; i < la && lo < lb; i++) {
        int x = A[i];
        // galloping-free binary search in B[lo, lb)
        long long l = lo, h = lb;
        while (l < h) {
            long long m = (l + h) >> 1;
            if (B[m] < x) l = m + 1; else h = m;
        }
        lo = l;
        if (l < lb && B[l] == x) {
            cnt++;
            lo = l + 1;
            if (PER_VERTEX) atomicAdd(per_vertex + x, 1ull);
        }
    }
    return cnt;
}

template <bool PER_VERTEX>
__global__ void __launch_bounds__(kB)
k_tc_count(const long long* __restrict__ offp, int nV, const int32_t* __restrict__ fwd,
           unsigned long long* __restrict__ per_vertex, unsigned long long* __restrict__ total_out) {
    __shared__ Tile t;
    __shared__ unsigned long long s_sum[kB / 32];
    const long long total = offp[nV];
    const long long ntiles = (total + nV + Tile::TILE - 1) / Tile::TILE;
    unsigned long long mine = 0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int n = lb_tile_load(t, offp, (long long)nV, total, tile);
        for (int i = threadIdx.x; i < n; i += kB) {
            long long e = t.item0 + i;
            int b = t.seg[i];
            int u = (int)(t.seg0 + b);
            long long ua = t.seg_start(b);
            long long la = (b < t.nends ? t.ends[b] : offp[u + 1]) - ua;
            int v = fwd[e];
            long long vb = offp[v], lbn = offp[v + 1] - vb;
            const int32_t* A = fwd + ua;
            const int32_t* B = fwd + vb;
            long long c = la <= lbn ? intersect_count<PER_VERTEX>(A, la, B, lbn, per_vertex)
                                    : intersect_count<PER_VERTEX>(B, lbn, A, la, per_vertex);
            if (PER_VERTEX && c) {
                atomicAdd(per_vertex + u, (unsigned long long)c);
                atomicAdd(per_vertex + v, (unsigned long long)c);
            }
            mine += (unsigned long long)c;
        }
        __syncthreads();
    }
    for (int o = 16; o; o >>= 1) mine += __shfl_down_sync(0xFFFFFFFFu, mine, o);
    if ((threadIdx.x & 31) == 0) s_sum[threadIdx.x >> 5] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long tsum = 0;
        for (int w = 0; w < kB / 32; w++) tsum += s_sum[w];
        if (tsum) atomicAdd(total_out, tsum);
    }
}

// ---------------------------------------------------------------------------
// Vertex-centric counting: N+(u) is staged in shared memory once, then all
// (v, w) pairs with v in N+(u), w in N+(v) are flattened over the lanes
// (warp prefix of d+(v) over 32 v's at a time) and each w is looked up in
// the staged list by binary search.  N+(v) lists are read coalesced; N+(u)
// is read once per u instead of once per edge.
//   k_tc_warp: one warp per vertex, d+(u) <= kWarpCap, vertices handed out
//              in chunks by an atomic counter (dynamic balance);
//   k_tc_cta:  one CTA per vertex with d+(u) > kWarpCap; the list sits in
//              dynamic shared memory when it fits, else it is searched in
//              global memory.
// ---------------------------------------------------------------------------
constexpr int kTcWarps = 8;
constexpr int kWarpCap = 512;
constexpr int kChunk = 16;

__device__ __forceinline__ int smem_lower_bound(const int32_t* a, int n, int x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// One warp: all (v, w) pairs of u against the sorted list L (length du).
template <bool PER_VERTEX>
__device__ __forceinline__ unsigned long long tc_vertex_warp(
    int u, const int32_t* __restrict__ L, int du, int v_begin, int v_step,
    const long long* __restrict__ offp, const int32_t* __restrict__ fwd,
    long long* s_pref /*33*/, long long* s_vb /*32*/, int* s_v /*32*/,
    unsigned long long* __restrict__ per_vertex) {
    const int lane = threadIdx.x & 31;
    const int lo_w = L[0], hi_w = L[du - 1];
    unsigned long long cnt = 0;
    for (int c0 = v_begin * 32; c0 < du; c0 += v_step * 32) {
        int idx = c0 + lane;
        long long dv = 0, vb = 0;
        int v = 0;
        if (idx < du) {
            v = L[idx];
            vb = offp[v];
            dv = offp[v + 1] - vb;
        }
        long long incl = dv;
        for (int o = 1; o < 32; o <<= 1) {
            long long x = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += x;
        }
        s_pref[lane + 1] = incl;
        if (lane == 0) s_pref[0] = 0;
        s_vb[lane] = vb;
        s_v[lane] = v;
        __syncwarp();
        const long long T = s_pref[32];
        for (long long k = lane; k < T; k += 32) {
            // slot of pair k: last s with s_pref[s] <= k
            int a = 0, b = 32;
            while (b - a > 1) {
                int mid = (a + b) >> 1;
                if (s_pref[mid] <= k) a = mid; else b = mid;
            }
            int w = fwd[s_vb[a] + (k - s_pref[a])];
            if (w < lo_w || w > hi_w) continue;
            int p = smem_lower_bound(L, du, w);
            if (p < du && L[p] == w) {
                cnt++;
                if (PER_VERTEX) {
                    atomicAdd(per_vertex + w, 1ull);
                    atomicAdd(per_vertex + u, 1ull);
                    atomicAdd(per_vertex + s_v[a], 1ull);
                }
            }
        }
        __syncwarp();
    }
    return cnt;
}

template <bool PER_VERTEX>
__global__ void __launch_bounds__(kTcWarps * 32)
k_tc_warp(const long long* __restrict__ offp, int nV, const int32_t* __restrict__ fwd,
          unsigned long long* __restrict__ per_vertex, unsigned long long* __restrict__ total_out,
          int* __restrict__ next_u) {
    __shared__ int32_t s_list[kTcWarps][kWarpCap];
    __shared__ long long s_pref[kTcWarps][33];
    __shared__ long long s_vb[kTcWarps][32];
    __shared__ int s_v[kTcWarps][32];
    __shared__ unsigned long long s_sum[kTcWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long mine = 0;
    while (true) {
        int u0 = 0;
        if (lane == 0) u0 = atomicAdd(next_u, kChunk);
        u0 = __shfl_sync(0xFFFFFFFFu, u0, 0);
        if (u0 >= nV) break;
        int u1 = u0 + kChunk < nV ? u0 + kChunk : nV;
        for (int u = u0; u < u1; u++) {
            long long ub = offp[u];
            int du = (int)(offp[u + 1] - ub);
            if (du == 0 || du > kWarpCap) continue;
            for (int i = lane; i < du; i += 32) s_list[warp][i] = fwd[ub + i];
            __syncwarp();
            mine += tc_vertex_warp<PER_VERTEX>(u, s_list[warp], du, 0, 1, offp, fwd,
                                               s_pref[warp], s_vb[warp], s_v[warp], per_vertex);
            __syncwarp();
        }
    }
    for (int o = 16; o; o >>= 1) mine += __shfl_down_sync(0xFFFFFFFFu, mine, o);
    if (lane == 0) s_sum[warp] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kTcWarps; w++) t += s_sum[w];
        if (t) atomicAdd(total_out, t);
    }
}

// Vertices with d+(u) > kWarpCap (few): one CTA each.
template <bool PER_VERTEX>
__global__ void __launch_bounds__(kTcWarps * 32)
k_tc_cta(const long long* __restrict__ offp, int nV, const int32_t* __restrict__ fwd,
         unsigned long long* __restrict__ per_vertex, unsigned long long* __restrict__ total_out,
         int smem_cap) {
    extern __shared__ int32_t s_dyn[];
    __shared__ long long s_pref[kTcWarps][33];
    __shared__ long long s_vb[kTcWarps][32];
    __shared__ int s_v[kTcWarps][32];
    __shared__ unsigned long long s_sum[kTcWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long mine = 0;
    for (long long u = blockIdx.x; u < nV; u += gridDim.x) {
        long long ub = offp[u];
        int du = (int)(offp[u + 1] - ub);
        if (du <= kWarpCap) continue;
        const int32_t* L = fwd + ub;
        if (du <= smem_cap) {
            for (int i = threadIdx.x; i < du; i += blockDim.x) s_dyn[i] = fwd[ub + i];
            L = s_dyn;
        }
        __syncthreads();
        mine += tc_vertex_warp<PER_VERTEX>((int)u, L, du, warp, kTcWarps, offp, fwd, s_pref[warp],
                                           s_vb[warp], s_v[warp], per_vertex);
        __syncthreads();
    }
    for (int o = 16; o; o >>= 1) mine += __shfl_down_sync(0xFFFFFFFFu, mine, o);
    if (lane == 0) s_sum[warp] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kTcWarps; w++) t += s_sum[w];
        if (t) atomicAdd(total_out, t);
    }
}

}  // namespace

void build_oriented(hn_graph* g, Oriented& o) {
    cudaStream_t s = g->stream;
    const int nV = g->nV;
    const long long m = g->nE;
    o.prefix.alloc((size_t)nV + 1, s);
    degree_prefix(g, nullptr, nV, o.prefix.get());
    DevBuf<int32_t> pos((size_t)m + 1, s);
    const long long grid = (long long)g->info.sms * 8;
    HN_LAUNCH(k_orient_flags, grid, kB, 0, s, o.prefix.get(), nV, g->vtab, g->pool, pos.get());
    {
        size_t tb = 0;
        HN_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, pos.get(), pos.get(), (int)(m + 1), s));
        DevBuf<char> tmp(tb, s);
        HN_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tb, pos.get(), pos.get(), (int)(m + 1), s));
        count_launch();
    }
    o.offp.alloc((size_t)nV + 1, s);
    o.fwd.alloc((size_t)(m / 2 + 4), s);
    HN_LAUNCH(k_orient_fill, grid, kB, 0, s, o.prefix.get(), nV, g->vtab, g->pool, pos.get(),
              o.fwd.get(), o.offp.get());
}

unsigned long long count_triangles(hn_graph* g, const Oriented& o, unsigned long long* d_per_vertex) {
    cudaStream_t s = g->stream;
    unsigned long long* d_total = (unsigned long long*)g->d_scalar;
    HN_CUDA(cudaMemsetAsync(d_total, 0, sizeof(unsigned long long), s));
    int* next_u = (int*)(g->d_scalar + 1);
    HN_CUDA(cudaMemsetAsync(next_u, 0, sizeof(int), s));
    const long long gw = (long long)g->info.sms * 8;
    // dynamic shared memory for the CTA path: up to 160 KB of list
    const int smem_cap = 40 * 1024;
    const size_t dyn = (size_t)smem_cap * sizeof(int32_t);
    static bool attr_set = false;
    if (!attr_set) {
        HN_CUDA(cudaFuncSetAttribute(k_tc_cta<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)dyn));
        HN_CUDA(cudaFuncSetAttribute(k_tc_cta<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)dyn));
        attr_set = true;
    }
    const long long gc = (long long)g->info.sms * 2;
    if (d_per_vertex) {
        HN_CUDA(cudaMemsetAsync(d_per_vertex, 0, sizeof(unsigned long long) * g->nV, s));
        HN_LAUNCH(k_tc_warp<true>, gw, kTcWarps * 32, 0, s, o.offp.get(), g->nV, o.fwd.get(),
                  d_per_vertex, d_total, next_u);
        HN_LAUNCH(k_tc_cta<true>, gc, kTcWarps * 32, dyn, s, o.offp.get(), g->nV, o.fwd.get(),
                  d_per_vertex, d_total, smem_cap);
    } else {
        HN_LAUNCH(k_tc_warp<false>, gw, kTcWarps * 32, 0, s, o.offp.get(), g->nV, o.fwd.get(),
                  (unsigned long long*)nullptr, d_total, next_u);
        HN_LAUNCH(k_tc_cta<false>, gc, kTcWarps * 32, dyn, s, o.offp.get(), g->nV, o.fwd.get(),
                  (unsigned long long*)nullptr, d_total, smem_cap);
    }
    read_scalars(g, 1);
    return (unsigned long long)g->h_scalar[0];
}

}  // namespace hn

using namespace hn;

extern "C" int hn_tc(hn_graph_t* g, uint64_t* per_vertex, int mem, uint64_t* total) {
    HN_API_BEGIN
    HN_REQUIRE(g != nullptr, "graph is null");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    if (g->nV == 0) {
        if (total) *total = 0;
        return HN_OK;
    }
    Oriented o;
    build_oriented(g, o);
    DevBuf<unsigned long long> pv;
    unsigned long long* d_pv = nullptr;
    if (per_vertex) {
        if (mem == HN_MEM_HOST) {
            pv.alloc((size_t)g->nV, s);
            d_pv = pv.get();
        } else {
            d_pv = (unsigned long long*)per_vertex;
        }
    }
    unsigned long long t = count_triangles(g, o, d_pv);
    if (per_vertex && mem == HN_MEM_HOST)
        HN_CUDA(cudaMemcpyAsync(per_vertex, d_pv, sizeof(unsigned long long) * g->nV,
                                cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    if (total) *total = t;
    HN_API_END
}
