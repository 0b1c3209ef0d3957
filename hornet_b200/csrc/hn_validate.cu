// Device-side result certificates behind StaticAlgorithm::validate().
//
// The reference's validate() methods are stubs that return true
// (hornetsnest/src/Static/BreadthFirstSearch/TopDown.cu:113-128,
// ConnectedComponents/CC.cu:163-203).  Here a result is checked on the
// device, without the oracle and without recomputing it the same way:
//
//   BFS distances from src (directed or undirected graph) are exactly the
//   BFS distances iff dist[src] == 0, every edge u -> v leaving a reached u
//   reaches v with dist[v] <= dist[u] + 1, and every reached v != src has an
//   in-edge u -> v with dist[u] == dist[v] - 1.
//
//   Edge truss numbers (sorted-COO order) of a simple undirected graph: the
//   lower-bound half of the truss certificate -- every number in [2, max_K],
//   equal on both directions of an edge, max_K attained, and every edge of
//   truss number t >= 3 lies in at least t - 2 triangles whose other two
//   edges have truss numbers >= t (so the edges numbered >= t do form a
//   t-truss).  That no edge belongs to a larger truss than its number is
//   not checked.
//
//   Minimum-id component labels of an undirected graph are correct iff they
//   are constant along every edge, labels[v] <= v, labels[labels[v]] ==
//   labels[v], and propagating the labels of the roots (v == labels[v])
//   along edges alone gives back the same labels (two components sharing a
//   label would leave the second one without it).
#include "hn_graph.cuh"

namespace hn {
namespace {

constexpr int kVB = 256;

// one warp per vertex: edge conditions of the BFS certificate; a parent of
// v is recorded in has_parent[v]
__global__ void k_bfs_cert_edges(const VRec* __restrict__ vtab, const int32_t* __restrict__ pool,
                                 int nV, const int32_t* __restrict__ dist,
                                 unsigned char* __restrict__ has_parent,
                                 unsigned long long* __restrict__ bad) {
    const int lane = threadIdx.x & 31;
    const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    unsigned long long nbad = 0;
    for (long long u = w0; u < nV; u += nw) {
        const int du = dist[u];
        if (du == kInf) continue;
        const VRec r = vtab[u];
        for (int i = lane; i < r.deg; i += 32) {
            const int v = pool[r.off + i];
            const int dv = dist[v];
            if (dv == kInf || dv > du + 1) nbad++;
            else if (dv == du + 1) has_parent[v] = 1;
        }
    }
    for (int o = 16; o; o >>= 1) nbad += __shfl_down_sync(0xFFFFFFFFu, nbad, o);
    if (lane == 0 && nbad) atomicAdd(bad, nbad);
}

__global__ void k_bfs_cert_vertices(int nV, int src, const int32_t* __restrict__ dist,
                                    const unsigned char* __restrict__ has_parent,
                                    unsigned long long* __restrict__ bad) {
    unsigned long long nbad = 0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x) {
        const int d = dist[v];
        if (v == src) nbad += d != 0;
        else if (d != kInf && (d <= 0 || !has_parent[v])) nbad++;
    }
    if (nbad) atomicAdd(bad, nbad);
}

// CC: constancy along edges, label <= id, fixed points; roots seed prop[]
__global__ void k_cc_cert_local(const VRec* __restrict__ vtab, const int32_t* __restrict__ pool,
                                int nV, const int32_t* __restrict__ lab,
                                int32_t* __restrict__ prop, unsigned long long* __restrict__ bad) {
    const int lane = threadIdx.x & 31;
    const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    unsigned long long nbad = 0;
    for (long long u = w0; u < nV; u += nw) {
        const int lu = lab[u];
        if (lane == 0) {
            if (lu < 0 || lu > u || lab[lu] != lu) nbad++;
            prop[u] = lu == u ? lu : kInf;
        }
        const VRec r = vtab[u];
        for (int i = lane; i < r.deg; i += 32)
            if (lab[pool[r.off + i]] != lu) nbad++;
    }
    for (int o = 16; o; o >>= 1) nbad += __shfl_down_sync(0xFFFFFFFFu, nbad, o);
    if (lane == 0 && nbad) atomicAdd(bad, nbad);
}

// one round of root-label propagation: prop[v] = min over in-edges
__global__ void k_cc_cert_prop(const VRec* __restrict__ vtab, const int32_t* __restrict__ pool,
                               int nV, int32_t* __restrict__ prop, int* __restrict__ changed) {
    const int lane = threadIdx.x & 31;
    const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    bool ch = false;
    for (long long u = w0; u < nV; u += nw) {
        const int pu = prop[u];
        if (pu == kInf) continue;
        const VRec r = vtab[u];
        for (int i = lane; i < r.deg; i += 32) {
            const int v = pool[r.off + i];
            if (prop[v] > pu && atomicMin(prop + v, pu) > pu) ch = true;
        }
    }
    if (__any_sync(0xFFFFFFFFu, ch) && lane == 0) *changed = 1;
}

__global__ void k_cc_cert_compare(int nV, const int32_t* __restrict__ lab,
                                  const int32_t* __restrict__ prop,
                                  unsigned long long* __restrict__ bad) {
    unsigned long long nbad = 0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x)
        nbad += prop[v] != lab[v];
    if (nbad) atomicAdd(bad, nbad);
}

__device__ __forceinline__ long long find_in(const int32_t* __restrict__ adj, long long lo,
                                             long long hi, int x) {
    long long e = hi;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (adj[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo < e && adj[lo] == x ? lo : -1;
}

// a thread per stored edge (u, v): range, symmetry and triangle support of
// its truss number
__global__ void k_ktruss_cert(const long long* __restrict__ off, const int32_t* __restrict__ adj,
                              int nV, long long nE, const int32_t* __restrict__ et, int maxk,
                              unsigned long long* __restrict__ bad, int* __restrict__ seen_max) {
    unsigned long long nbad = 0;
    int mx = 0;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < nE;
         p += (long long)gridDim.x * blockDim.x) {
        // source of position p: last u with off[u] <= p
        int lo = 0, hi = nV;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (off[mid] <= p) lo = mid; else hi = mid;
        }
        const int u = lo, v = adj[p], t = et[p];
        mx = t > mx ? t : mx;
        if (t < 2 || t > maxk || u == v) { nbad++; continue; }
        const long long q = find_in(adj, off[v], off[v + 1], u);
        if (q < 0 || et[q] != t) { nbad++; continue; }
        if (u > v || t < 3) continue;
        // triangles through (u, v) whose other edges are numbered >= t
        const bool us = off[u + 1] - off[u] <= off[v + 1] - off[v];
        const int a = us ? u : v, b = us ? v : u;
        int cnt = 0;
        for (long long i = off[a]; i < off[a + 1] && cnt < t - 2; i++) {
            const int w = adj[i];
            if (et[i] < t) continue;
            const long long j = find_in(adj, off[b], off[b + 1], w);
            if (j >= 0 && et[j] >= t) cnt++;
        }
        if (cnt < t - 2) nbad++;
    }
    if (nbad) atomicAdd(bad, nbad);
    if (mx) atomicMax(seen_max, mx);
}

// Copies a host array to the device when mem is HN_MEM_HOST.
const int32_t* device_input(hn_graph* g, const int32_t* p, int mem, DevBuf<int32_t>& tmp,
                            long long n = -1) {
    if (n < 0) n = g->nV;
    if (mem == HN_MEM_DEVICE) return p;
    tmp.alloc((size_t)(n > 0 ? n : 1), g->stream);
    if (n > 0)
        HN_CUDA(cudaMemcpyAsync(tmp.get(), p, sizeof(int32_t) * n, cudaMemcpyHostToDevice,
                                g->stream));
    return tmp.get();
}

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" {

int hn_bfs_validate(hn_graph_t* g, int32_t src, const int32_t* dist, int mem, int64_t* violations) {
    HN_API_BEGIN
    HN_REQUIRE(g && dist && violations, "null argument");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    HN_REQUIRE(src >= 0 && src < g->nV, "BFS source outside [0, nV)");
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    DevBuf<int32_t> tmp;
    const int32_t* d = device_input(g, dist, mem, tmp);
    DevBuf<unsigned char> hp((size_t)g->nV, s);
    DevBuf<unsigned long long> bad(1, s);
    HN_CUDA(cudaMemsetAsync(hp.get(), 0, (size_t)g->nV, s));
    HN_CUDA(cudaMemsetAsync(bad.get(), 0, sizeof(unsigned long long), s));
    HN_LAUNCH(k_bfs_cert_edges, grid_for(g, (long long)g->nV * 32, kVB), kVB, 0, s, g->vtab,
              g->pool, g->nV, d, hp.get(), bad.get());
    HN_LAUNCH(k_bfs_cert_vertices, grid_for(g, g->nV, kVB), kVB, 0, s, g->nV, src, d, hp.get(),
              bad.get());
    unsigned long long h = 0;
    HN_CUDA(cudaMemcpyAsync(&h, bad.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    *violations = (int64_t)h;
    HN_API_END
}

int hn_cc_validate(hn_graph_t* g, const int32_t* labels, int mem, int64_t* violations) {
    HN_API_BEGIN
    HN_REQUIRE(g && labels && violations, "null argument");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    DevBuf<int32_t> tmp;
    const int32_t* lab = device_input(g, labels, mem, tmp);
    DevBuf<int32_t> prop((size_t)g->nV, s);
    DevBuf<unsigned long long> bad(1, s);
    DevBuf<int> changed(1, s);
    HN_CUDA(cudaMemsetAsync(bad.get(), 0, sizeof(unsigned long long), s));
    const long long gw = grid_for(g, (long long)g->nV * 32, kVB);
    HN_LAUNCH(k_cc_cert_local, gw, kVB, 0, s, g->vtab, g->pool, g->nV, lab, prop.get(), bad.get());
    unsigned long long h = 0;
    HN_CUDA(cudaMemcpyAsync(&h, bad.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    if (h == 0) {
        // propagation rounds until nothing changes (at most nV rounds: every
        // round that changes something lowers some entry)
        for (long long it = 0; it <= g->nV; it++) {
            int hc = 0;
            HN_CUDA(cudaMemsetAsync(changed.get(), 0, sizeof(int), s));
            HN_LAUNCH(k_cc_cert_prop, gw, kVB, 0, s, g->vtab, g->pool, g->nV, prop.get(),
                      changed.get());
            HN_CUDA(cudaMemcpyAsync(&hc, changed.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
            HN_CUDA(cudaStreamSynchronize(s));
            if (!hc) break;
        }
        HN_LAUNCH(k_cc_cert_compare, grid_for(g, g->nV, kVB), kVB, 0, s, g->nV, lab, prop.get(),
                  bad.get());
        HN_CUDA(cudaMemcpyAsync(&h, bad.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
        HN_CUDA(cudaStreamSynchronize(s));
    }
    *violations = (int64_t)h;
    HN_API_END
}

int hn_ktruss_validate(hn_graph_t* g, int32_t max_k, const int32_t* edge_truss, int mem,
                       int64_t* violations) {
    HN_API_BEGIN
    HN_REQUIRE(g && violations && (edge_truss || g->nE == 0), "null argument");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    *violations = 0;
    if (g->nE == 0) {
        *violations = max_k == 2 ? 0 : 1;
        return HN_OK;
    }
    DevBuf<int32_t> tmp;
    const int32_t* et = device_input(g, edge_truss, mem, tmp, g->nE);
    DevBuf<long long> off((size_t)g->nV + 1, s);
    DevBuf<int32_t> adj((size_t)g->nE, s);
    export_csr64(g, off.get(), adj.get());
    DevBuf<unsigned long long> bad(1, s);
    DevBuf<int> seen(1, s);
    HN_CUDA(cudaMemsetAsync(bad.get(), 0, sizeof(unsigned long long), s));
    HN_CUDA(cudaMemsetAsync(seen.get(), 0, sizeof(int), s));
    HN_LAUNCH(k_ktruss_cert, grid_for(g, g->nE, kVB), kVB, 0, s, off.get(), adj.get(), g->nV,
              (long long)g->nE, et, max_k, bad.get(), seen.get());
    unsigned long long h = 0;
    int mx = 0;
    HN_CUDA(cudaMemcpyAsync(&h, bad.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaMemcpyAsync(&mx, seen.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    *violations = (int64_t)h + (mx != max_k ? 1 : 0);
    HN_API_END
}

}  // extern "C"
