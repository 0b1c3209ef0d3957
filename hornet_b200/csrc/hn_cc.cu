// Connected components (hornetsnest/src/Static/ConnectedComponents/CC.cu:133-156).
//
// Reference: BFS-colour the giant component from max_degree_id() with 0,
// colour every other vertex id+1, queue the (src > dst) vertex pairs and
// propagate the MAX colour over them until a host-read flag stays false —
// one host round trip per propagation sweep.
//
// Here: lock-free union-find in the style of ECL-CC (Jaiganesh & Burtscher,
// "A High-Performance Connected Components Implementation for GPUs",
// HPDC 2018) — a link hangs the larger root under the smaller one with
// atomicCAS, finds use intermediate pointer jumping — driven by the
// neighbour-sampling schedule of Afforest (Sutton, Ben-Nun & Barak,
// IPDPS 2018):
//   1. every vertex links with its first kSample neighbours;
//   2. compress; the most frequent root among 256 evenly spaced vertices
//      is taken as the giant component G;
//   3. only vertices outside G (with more than kSample neighbours) link
//      with the rest of their neighbours — an edge from G to a vertex
//      outside G is seen from the outside end, edges inside G are already
//      implied — so on power-law graphs most edges are never read;
//   4. compress and count roots.
// Parents only ever point to smaller ids, so each root is the minimum id of
// its component: the labels come out canonical with no relabelling, and no
// step waits on the host.
// The reference's own colouring is produced from the same roots on request
// (giant component of max_degree_id -> 0, others max(id)+1).
#include "hn_graph.cuh"

namespace hn {
namespace {

constexpr int kB = 256;

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

constexpr int kSample = 2;

__device__ __forceinline__ void cc_link(int* __restrict__ parent, int u, int v) {
    int ru = find_root(parent, u);
    int rv = find_root(parent, v);
    while (ru != rv) {
        if (ru < rv) { int x = ru; ru = rv; rv = x; }
        // ru > rv: hang ru under rv if ru is still a root
        int old = atomicCAS(parent + ru, ru, rv);
        if (old == ru) return;
        ru = find_root(parent, old);
    }
}

// 1. link every vertex with its first kSample neighbours.  Each thread
// takes kVerts vertices per round and issues all their record and
// neighbour loads before the first link (each link is a chain of dependent
// parent reads, so the loads of one vertex alone leave the SM waiting).
constexpr int kVerts = 4;
__global__ void k_cc_sample(const VRec* __restrict__ vtab, const int32_t* __restrict__ pool,
                            int nV, int* __restrict__ parent) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long v0 = blockIdx.x * (long long)blockDim.x + threadIdx.x; v0 < nV;
         v0 += kVerts * stride) {
        int deg[kVerts];
        long long off[kVerts];
#pragma unroll
        for (int j = 0; j < kVerts; j++) {
            const long long v = v0 + j * stride;
            deg[j] = 0;
            off[j] = 0;
            if (v < nV) {
                const VRec r = vtab[v];
                deg[j] = r.deg < kSample ? r.deg : kSample;
                off[j] = r.off;
            }
        }
        int nb[kVerts][kSample];
#pragma unroll
        for (int j = 0; j < kVerts; j++)
#pragma unroll
            for (int i = 0; i < kSample; i++) nb[j][i] = i < deg[j] ? __ldg(pool + off[j] + i) : -1;
#pragma unroll
        for (int j = 0; j < kVerts; j++)
#pragma unroll
            for (int i = 0; i < kSample; i++)
                if (nb[j][i] >= 0) cc_link(parent, (int)(v0 + j * stride), nb[j][i]);
    }
}

__global__ void k_cc_compress(int* __restrict__ parent, int nV) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x)
        parent[v] = find_root(parent, (int)v);
}

// 2. most frequent root among 256 evenly spaced vertices (one CTA of 256)
__global__ void k_cc_giant(const int* __restrict__ parent, int nV, int* __restrict__ giant) {
    __shared__ int s_r[256];
    int t = threadIdx.x;
    long long v = (long long)t * nV / 256;
    s_r[t] = parent[v < nV ? v : nV - 1];
    __syncthreads();
    int mine = s_r[t], c = 0;
    for (int i = 0; i < 256; i++) c += (s_r[i] == mine);
    // pack (count, -root) so ties pick the smaller root
    unsigned long long key = ((unsigned long long)c << 32) | (unsigned)(0x7FFFFFFF - mine);
    __shared__ unsigned long long s_key;
    if (t == 0) s_key = 0;
    __syncthreads();
    atomicMax(&s_key, key);
    __syncthreads();
    if (t == 0) *giant = 0x7FFFFFFF - (int)(s_key & 0xFFFFFFFFull);
}

// 3a. vertices outside the giant component with unread neighbours
__global__ void k_cc_worklist(const VRec* __restrict__ vtab, const int* __restrict__ parent,
                              int nV, const int* __restrict__ giant, int* __restrict__ list,
                              int* __restrict__ nlist) {
    const int gr = *giant;
    for (long long v0 = blockIdx.x * (long long)blockDim.x; v0 < nV;
         v0 += (long long)gridDim.x * blockDim.x) {
        long long v = v0 + threadIdx.x;
        bool take = v < nV && vtab[v].deg > kSample && parent[v] != gr;
        int p = warp_append(nlist, take);
        if (take) list[p] = (int)v;
    }
}

// 3b. one warp per listed vertex: link with neighbours kSample..deg-1
__global__ void k_cc_rest(const VRec* __restrict__ vtab, const int32_t* __restrict__ pool,
                          const int* __restrict__ list, const int* __restrict__ nlist,
                          int* __restrict__ parent) {
    const int n = *nlist;
    const int lane = threadIdx.x & 31;
    long long wid = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long i = wid; i < n; i += nw) {
        int v = list[i];
        VRec r = vtab[v];
        for (int k = kSample + lane; k < r.deg; k += 32) cc_link(parent, v, pool[r.off + k]);
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
    HandleUse use(g);
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    const int nV = g->nV;
    if (nV == 0) {
        if (n_components) *n_components = 0;
        return HN_OK;
    }
    DevBuf<int> parent((size_t)nV, s), list((size_t)nV, s);
    int* cnt = (int*)(g->d_scalar + 2);  // [0] giant root, [1] worklist size
    HN_CUDA(cudaMemsetAsync(cnt, 0, 2 * sizeof(int), s));
    HN_LAUNCH(k_cc_init, grid_for(g, nV, kB), kB, 0, s, parent.get(), nV);
    HN_LAUNCH(k_cc_sample, grid_for(g, nV, kB), kB, 0, s, g->vtab, g->pool, nV, parent.get());
    HN_LAUNCH(k_cc_compress, grid_for(g, nV, kB), kB, 0, s, parent.get(), nV);
    HN_LAUNCH(k_cc_giant, 1, 256, 0, s, parent.get(), nV, cnt);
    HN_LAUNCH(k_cc_worklist, grid_for(g, nV, kB), kB, 0, s, g->vtab, parent.get(), nV, cnt,
              list.get(), cnt + 1);
    HN_LAUNCH(k_cc_rest, (long long)g->info.sms * 8, kB, 0, s, g->vtab, g->pool, list.get(),
              cnt + 1, parent.get());
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
