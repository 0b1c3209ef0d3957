// BFS TopDown (hornetsnest/src/Static/BreadthFirstSearch/TopDown.cu:49-106).
//
// Reference: per level, forAllEdges(queue, BFSOperator, BinarySearch) =
// computeWorkKernel + CUB scan + D2H total + binarySearchKernel with a
// non-atomic `dist[dst] == INF` test (duplicate enqueues possible), then a
// <<<1,1>>> swap kernel and another D2H (TwoLevelQueue.i.cuh:158-179).
//
// Here, per level: the frontier carries each vertex's degree (written when
// it is enqueued), one device scan turns it into the merge-path prefix, and
// one persistent expand kernel walks the frontier's edges with the
// merge-path load balancer.  A vertex is claimed with atomicOr on a visited
// bitmap (nV/8 bytes: L2-resident), so it is enqueued exactly once and its
// distance written once; the next frontier is filled with warp-aggregated
// appends.  The only host round trip per level is the 8-byte frontier size.
// Distances equal the reference's: level-synchronous, INF = INT32_MAX.
#include <cub/cub.cuh>

#include "hn_graph.cuh"

namespace hn {
namespace {

constexpr int kB = 256;
constexpr int kItems = 8;
using Tile = LbTile<kB, kItems>;

__global__ void k_bfs_init(int32_t* __restrict__ dist, unsigned* __restrict__ visited, int nV,
                           int src, const VRec* __restrict__ vtab, int32_t* __restrict__ q,
                           long long* __restrict__ qdeg, int* __restrict__ counters) {
    long long nwords = ((long long)nV + 31) / 32;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nV || i < nwords;
         i += (long long)gridDim.x * blockDim.x) {
        if (i < nV) dist[i] = i == src ? 0 : kInf;
        if (i < nwords) {
            unsigned w = 0;
            if (i == src / 32) w = 1u << (src & 31);
            visited[i] = w;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        q[0] = src;
        qdeg[0] = vtab[src].deg;
        qdeg[1] = 0;
        counters[0] = 1;  // current frontier size
        counters[1] = 0;  // next frontier size
    }
}

// One BFS level: edges of frontier q (prefix over its degrees) -> next
// frontier nq.  Vertices newly reached get distance `level`.
__global__ void __launch_bounds__(kB)
k_bfs_expand(const long long* __restrict__ prefix, const int32_t* __restrict__ q,
             long long nq, const VRec* __restrict__ vtab, const int32_t* __restrict__ pool,
             unsigned* __restrict__ visited, int32_t* __restrict__ dist, int level,
             int32_t* __restrict__ nqv, long long* __restrict__ nqdeg,
             int* __restrict__ ncount) {
    __shared__ Tile t;
    __shared__ long long s_base[Tile::TILE + 1];
    const long long total = prefix[nq];
    const long long ntiles = (total + nq + Tile::TILE - 1) / Tile::TILE;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int n = lb_tile_load(t, prefix, nq, total, tile);
        for (int b = threadIdx.x; b <= t.nends; b += kB) {
            long long s = t.seg0 + b;
            if (s < nq) s_base[b] = vtab[q[s]].off - t.seg_start(b);
        }
        __syncthreads();
        // round the loop up to a whole number of passes so every lane of a
        // warp reaches the warp-aggregated append together
        for (int i0 = 0; i0 < n; i0 += kB) {
            int i = i0 + threadIdx.x;
            bool claim = false;
            int w = 0;
            if (i < n) {
                w = pool[s_base[t.seg[i]] + t.item0 + i];
                unsigned bit = 1u << (w & 31);
                unsigned* word = visited + (w >> 5);
                if (!(__ldcg(word) & bit)) claim = !(atomicOr(word, bit) & bit);
            }
            int pos = warp_append(ncount, claim);
            if (claim) {
                dist[w] = level;
                nqv[pos] = w;
                nqdeg[pos] = vtab[w].deg;
            }
        }
        __syncthreads();
    }
}

__global__ void k_set_sentinel(long long* __restrict__ qdeg, const int* __restrict__ count) {
    qdeg[*count] = 0;
}

struct BfsWork {
    DevBuf<int32_t> q[2];
    DevBuf<long long> qdeg[2];
    DevBuf<long long> prefix;
    DevBuf<unsigned> visited;
    DevBuf<int> counters;
    DevBuf<char> scan_tmp;
    size_t scan_bytes = 0;
};

void bfs_one(hn_graph* g, BfsWork& w, int src, int32_t* d_dist, hn_bfs_stats_t* stats) {
    cudaStream_t s = g->stream;
    const int nV = g->nV;
    HN_LAUNCH(k_bfs_init, grid_for(g, nV, kB), kB, 0, s, d_dist, w.visited.get(), nV, src,
              g->vtab, w.q[0].get(), w.qdeg[0].get(), w.counters.get());
    long long nq = 1;
    int cur = 0;
    int level = 1;
    long long visited = 1, scanned = 0;
    const long long grid = (long long)g->info.sms * 8;
    while (nq > 0) {
        // prefix over the frontier's degrees (qdeg[nq] is the 0 sentinel)
        HN_CUDA(cub::DeviceScan::ExclusiveSum(w.scan_tmp.get(), w.scan_bytes, w.qdeg[cur].get(),
                                              w.prefix.get(), (int)(nq + 1), s));
        count_launch();
        int* ncount = w.counters.get() + 1 - cur;  // counter of the next queue
        HN_CUDA(cudaMemsetAsync(ncount, 0, sizeof(int), s));
        HN_LAUNCH(k_bfs_expand, grid, kB, 0, s, w.prefix.get(), w.q[cur].get(), nq, g->vtab,
                  g->pool, w.visited.get(), d_dist, level, w.q[1 - cur].get(),
                  w.qdeg[1 - cur].get(), ncount);
        HN_LAUNCH(k_set_sentinel, 1, 1, 0, s, w.qdeg[1 - cur].get(), ncount);
        HN_CUDA(cudaMemcpyAsync(g->h_scalar, w.prefix.get() + nq, sizeof(long long),
                                cudaMemcpyDeviceToHost, s));
        HN_CUDA(cudaMemcpyAsync(g->h_scalar + 1, ncount, sizeof(int), cudaMemcpyDeviceToHost, s));
        HN_CUDA(cudaStreamSynchronize(s));
        scanned += g->h_scalar[0];
        nq = *(int*)(g->h_scalar + 1);
        visited += nq;
        cur = 1 - cur;
        level++;
    }
    if (stats) {
        stats->levels = level - 1;
        stats->pad = 0;
        stats->visited = visited;
        stats->edges_scanned = scanned;
    }
}

void bfs_run(hn_graph* g, const int32_t* sources, int k, int32_t* dist, int mem,
             hn_bfs_stats_t* stats) {
    cudaStream_t s = g->stream;
    const int nV = g->nV;
    for (int i = 0; i < k; i++)
        if (sources[i] < 0 || sources[i] >= nV)
            throw Error(HN_ERR_INVALID, "BFS source outside [0, nV)");
    BfsWork w;
    for (int i = 0; i < 2; i++) {
        w.q[i].alloc((size_t)nV + 1, s);
        w.qdeg[i].alloc((size_t)nV + 2, s);
    }
    w.prefix.alloc((size_t)nV + 2, s);
    w.visited.alloc(((size_t)nV + 31) / 32 + 1, s);
    w.counters.alloc(4, s);
    HN_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, w.scan_bytes, w.qdeg[0].get(), w.prefix.get(),
                                          nV + 1, s));
    w.scan_tmp.alloc(w.scan_bytes, s);
    DevBuf<int32_t> d_dist;
    if (mem == HN_MEM_HOST) d_dist.alloc((size_t)nV, s);
    for (int i = 0; i < k; i++) {
        int32_t* out = mem == HN_MEM_HOST ? d_dist.get() : dist + (size_t)i * nV;
        bfs_one(g, w, sources[i], out, stats ? stats + i : nullptr);
        if (mem == HN_MEM_HOST)
            HN_CUDA(cudaMemcpyAsync(dist + (size_t)i * nV, out, sizeof(int32_t) * nV,
                                    cudaMemcpyDeviceToHost, s));
    }
    HN_CUDA(cudaStreamSynchronize(s));
}

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" {

int hn_bfs(hn_graph_t* g, int32_t src, int32_t* dist, int mem, hn_bfs_stats_t* stats) {
    HN_API_BEGIN
    HN_REQUIRE(g && dist, "null argument");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    HN_REQUIRE(g->nV > 0, "empty graph");
    HN_CUDA(cudaSetDevice(g->device));
    bfs_run(g, &src, 1, dist, mem, stats);
    HN_API_END
}

int hn_bfs_multi(hn_graph_t* g, const int32_t* sources, int32_t k, int32_t* dist, int mem,
                 hn_bfs_stats_t* stats) {
    HN_API_BEGIN
    HN_REQUIRE(g && sources && dist, "null argument");
    HN_REQUIRE(k >= 0, "negative source count");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    HN_REQUIRE(g->nV > 0 || k == 0, "empty graph");
    HN_CUDA(cudaSetDevice(g->device));
    bfs_run(g, sources, k, dist, mem, stats);
    HN_API_END
}

}  // extern "C"
