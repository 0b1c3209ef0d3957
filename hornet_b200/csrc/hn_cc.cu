// Connected components (hornetsnest/src/Static/ConnectedComponents/CC.cu:133-156).
//
// Reference: BFS-colour the giant component from max_degree_id() with 0,
// colour every other vertex id+1, queue the (src > dst) vertex pairs and
// propagate the MAX colour over them until a host-read flag stays false —
// one host round trip per propagation sweep.
//
// Here: lock-free union-find in the style of ECL-CC (Jaiganesh & Burtscher,
// "A High-Performance Connected Components Implementation for GPUs",
// HPDC 2018): every undirected edge (u > v) hooks the larger root under the
// smaller one with atomicCAS, finds use intermediate pointer jumping, and
// a final pass points every vertex at its root.  Parents only ever point to
// smaller ids, so each root is the minimum id of its component: the labels
// come out canonical with no relabelling.  One merge-path balanced pass over
// the edges, two grid-stride passes over the vertices, no host round trips.
// The reference's own colouring is produced from the same roots on request
// (giant component of max_degree_id -> 0, others max(id)+1).
#include "hn_graph.cuh"

namespace hn {
namespace {

constexpr int kB = 256;
using Tile = LbTile<kB, 8>;

__device__ __forceinline__ int find_root(int* __restrict__ parent, int v) {
    int cur = parent[v];
    if (cur != v) {
        int prev = v, next;
        while (cur > (next = parent[cur])) {
            parent[prev] = next;  // pointer jumping; values only decrease
            prev = cur;
            cur = next;
        }
    }
    return cur;
}

__global__ void k_cc_init(int* __restrict__ parent, int nV) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x)
        parent[v] = (int)v;
}

__global__ void __launch_bounds__(kB)
k_cc_hook(const long long* __restrict__ prefix, int nV, const VRec* __restrict__ vtab,
          const int32_t* __restrict__ pool, int* __restrict__ parent) {
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
            int b = t.seg[i];
            int u = (int)(t.seg0 + b);
            int v = pool[s_base[b] + e];
            if (v >= u) continue;  // each undirected edge once
            int ru = find_root(parent, u);
            int rv = find_root(parent, v);
            while (ru != rv) {
                if (ru < rv) { int x = ru; ru = rv; rv = x; }
                // ru > rv: hang ru under rv if ru is still a root
                int old = atomicCAS(parent + ru, ru, rv);
                if (old == ru) break;
                ru = find_root(parent, old);
            }
        }
        __syncthreads();
    }
}

__global__ void k_cc_finish(int* __restrict__ parent, int nV, int* __restrict__ ncomp) {
    int mine = 0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x) {
        int r = find_root(parent, (int)v);
        parent[v] = r;
        mine += (r == v);
    }
    for (int o = 16; o; o >>= 1) mine += __shfl_down_sync(0xFFFFFFFFu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(ncomp, mine);
}

__global__ void k_cc_maxid(const int* __restrict__ label, int nV, int* __restrict__ mx) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x)
        atomicMax(mx + label[v], (int)v);
}

// giant: the component of the max-degree vertex (lowest id on ties) -> 0
__global__ void k_cc_refcolor(const int* __restrict__ label, const int* __restrict__ mx, int nV,
                              const unsigned long long* __restrict__ maxkey,
                              int* __restrict__ color) {
    unsigned long long k = *maxkey;
    int giant_v = k ? (int)(0xFFFFFFFFu - (unsigned)(k & 0xFFFFFFFFu)) : 0;
    int giant = label[giant_v];
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x) {
        int l = label[v];
        color[v] = l == giant ? 0 : mx[l] + 1;
    }
}

__global__ void k_max_degree_key(const VRec* __restrict__ vtab, int nV,
                                 unsigned long long* out) {
    unsigned long long best = 0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x) {
        unsigned long long k = ((unsigned long long)(unsigned)vtab[v].deg << 32) |
                               (unsigned)(0xFFFFFFFFu - (unsigned)v);
        best = k > best ? k : best;
    }
    for (int o = 16; o; o >>= 1) {
        unsigned long long x = __shfl_down_sync(0xFFFFFFFFu, best, o);
        best = x > best ? x : best;
    }
    if ((threadIdx.x & 31) == 0 && best) atomicMax(out, best);
}

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" int hn_cc(hn_graph_t* g, int mode, int32_t* labels, int mem, int32_t* n_components) {
    HN_API_BEGIN
    HN_REQUIRE(g && labels, "null argument");
    HN_REQUIRE(mode == HN_CC_MIN_ID || mode == HN_CC_REFERENCE, "bad CC mode");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    const int nV = g->nV;
    if (nV == 0) {
        if (n_components) *n_components = 0;
        return HN_OK;
    }
    DevBuf<int> parent((size_t)nV, s);
    DevBuf<long long> prefix((size_t)nV + 1, s);
    degree_prefix(g, nullptr, nV, prefix.get());
    HN_LAUNCH(k_cc_init, grid_for(g, nV, kB), kB, 0, s, parent.get(), nV);
    HN_LAUNCH(k_cc_hook, (long long)g->info.sms * 8, kB, 0, s, prefix.get(), nV, g->vtab, g->pool,
              parent.get());
    HN_CUDA(cudaMemsetAsync(g->d_scalar, 0, 2 * sizeof(long long), s));
    HN_LAUNCH(k_cc_finish, grid_for(g, nV, kB), kB, 0, s, parent.get(), nV, (int*)g->d_scalar);
    int32_t* out = mem == HN_MEM_DEVICE ? labels : nullptr;
    DevBuf<int32_t> tmp;
    if (!out) {
        tmp.alloc((size_t)nV, s);
        out = tmp.get();
    }
    if (mode == HN_CC_MIN_ID) {
        HN_CUDA(cudaMemcpyAsync(out, parent.get(), sizeof(int32_t) * nV, cudaMemcpyDeviceToDevice,
                                s));
    } else {
        DevBuf<int> mx((size_t)nV, s);
        HN_CUDA(cudaMemsetAsync(mx.get(), 0xFF, sizeof(int) * nV, s));
        HN_LAUNCH(k_cc_maxid, grid_for(g, nV, kB), kB, 0, s, parent.get(), nV, mx.get());
        unsigned long long* key = (unsigned long long*)(g->d_scalar + 1);
        HN_LAUNCH(k_max_degree_key, grid_for(g, nV, kB), kB, 0, s, g->vtab, nV, key);
        HN_LAUNCH(k_cc_refcolor, grid_for(g, nV, kB), kB, 0, s, parent.get(), mx.get(), nV, key,
                  out);
    }
    if (mem == HN_MEM_HOST)
        HN_CUDA(cudaMemcpyAsync(labels, out, sizeof(int32_t) * nV, cudaMemcpyDeviceToHost, s));
    read_scalars(g, 1);
    if (n_components) *n_components = (int32_t)(g->h_scalar[0] & 0xFFFFFFFF);
    HN_API_END
}
