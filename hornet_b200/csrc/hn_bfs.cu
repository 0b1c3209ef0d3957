// BFS TopDown (hornetsnest/src/Static/BreadthFirstSearch/TopDown.cu:49-106).
//
// Reference: per level, forAllEdges(queue, BFSOperator, BinarySearch) =
// computeWorkKernel + CUB scan + D2H total + binarySearchKernel with a
// non-atomic `dist[dst] == INF` test (duplicate enqueues possible), then a
// <<<1,1>>> swap kernel and another D2H (TwoLevelQueue.i.cuh:158-179): at
// least three host synchronisations per level.
//
// Here a whole BFS is ONE CUDA-graph launch: an init kernel, then a
// conditional WHILE node whose body is a single persistent expand kernel.
//   * The frontier carries, next to each vertex, the exclusive prefix of the
//     frontier's degrees.  It is produced by the enqueue itself: one 64-bit
//     atomicAdd of (degree << 32 | 1) per warp hands out the queue slot (low
//     word) and the edge offset (high word) together, so the offsets are
//     ordered like the slots and no scan pass is needed.
//   * The expand kernel walks the frontier's edges with the merge-path load
//     balancer (tiles over edges + vertex boundaries, segment ends and
//     adjacency bases staged in shared memory).
//   * A vertex is claimed with atomicOr on a visited bitmap (nV/8 bytes,
//     L2-resident), so it is enqueued exactly once and its distance written
//     once.
//   * The last CTA to finish a level (ticket counter) seals the next
//     frontier and sets the WHILE condition with cudaGraphSetConditional, so
//     the host never waits between levels.  The loop also stops after nV
//     levels, so it always terminates.
// Distances equal the reference's: level-synchronous, INF = INT32_MAX.
#include <cub/cub.cuh>

#include "hn_graph.cuh"

namespace hn {

constexpr int kBfsBlock = 256;
constexpr int kBfsItems = 8;

struct BfsState {
    unsigned long long cnt[3];   // frontier counters: (edge total << 32) | size
    int level;                   // distance given to vertices found now
    unsigned ticket;             // CTAs finished with the current level
    long long visited;
    long long scanned;
    int src;
    int nV;
    int32_t* dist;
    const VRec* vtab;
    const int32_t* pool;
    int32_t* q[2];               // frontier vertices
    unsigned* qoff[2];           // exclusive degree prefix of the frontier
    unsigned* bitmap;            // visited bits
};

struct BfsGraph {
    int nV = -1;
    BfsState* state = nullptr;      // device
    BfsState* h_state = nullptr;    // pinned
    int32_t* qbuf = nullptr;
    unsigned* qoffbuf = nullptr;
    unsigned* bitmap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

using Tile = LbTile<kBfsBlock, kBfsItems>;

__global__ void k_bfs2_init(BfsState* st) {
    const int nV = st->nV;
    const int src = st->src;
    int32_t* dist = st->dist;
    unsigned* bm = st->bitmap;
    long long nwords = ((long long)nV + 31) / 32;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nV;
         i += (long long)gridDim.x * blockDim.x) {
        dist[i] = i == src ? 0 : kInf;
        if (i < nwords) bm[i] = (i == src / 32) ? (1u << (src & 31)) : 0u;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        unsigned d = (unsigned)st->vtab[src].deg;
        st->q[0][0] = src;
        st->qoff[0][0] = 0;
        st->qoff[0][1] = d;
        st->cnt[0] = ((unsigned long long)d << 32) | 1ull;
        st->cnt[1] = 0;
        st->cnt[2] = 0;
        st->level = 1;
        st->ticket = 0;
        st->visited = 1;
        st->scanned = 0;
    }
}

__global__ void __launch_bounds__(kBfsBlock)
k_bfs2_expand(BfsState* st, cudaGraphConditionalHandle cond) {
    __shared__ Tile t;
    __shared__ long long s_base[Tile::TILE + 1];
    const int level = st->level;
    const int it = level - 1;
    const unsigned long long cin = st->cnt[it % 3];
    unsigned long long* cout = &st->cnt[(it + 1) % 3];
    if (blockIdx.x == 0 && threadIdx.x == 0) st->cnt[(it + 2) % 3] = 0;
    const long long nq = (long long)(cin & 0xFFFFFFFFull);
    const long long total = (long long)(cin >> 32);
    const int32_t* q = st->q[it & 1];
    const unsigned* prefix = st->qoff[it & 1];
    int32_t* nqv = st->q[(it + 1) & 1];
    unsigned* nqoff = st->qoff[(it + 1) & 1];
    const VRec* vtab = st->vtab;
    const int32_t* pool = st->pool;
    unsigned* bm = st->bitmap;
    int32_t* dist = st->dist;
    const int lane = threadIdx.x & 31;

    const long long ntiles = (total + nq + Tile::TILE - 1) / Tile::TILE;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int n = lb_tile_load(t, prefix, nq, total, tile);
        for (int b = threadIdx.x; b <= t.nends; b += kBfsBlock) {
            long long s = t.seg0 + b;
            if (s < nq) s_base[b] = vtab[q[s]].off - t.seg_start(b);
        }
        __syncthreads();
        for (int i0 = 0; i0 < n; i0 += kBfsBlock) {
            int i = i0 + threadIdx.x;
            bool claim = false;
            int w = 0;
            unsigned d = 0;
            if (i < n) {
                w = pool[s_base[t.seg[i]] + t.item0 + i];
                unsigned bit = 1u << (w & 31);
                unsigned* word = bm + (w >> 5);
                if (!(__ldcg(word) & bit)) claim = !(atomicOr(word, bit) & bit);
                if (claim) d = (unsigned)vtab[w].deg;
            }
            // warp-aggregated enqueue: slot and edge offset from one atomic
            unsigned ballot = __ballot_sync(0xFFFFFFFFu, claim);
            if (ballot) {
                unsigned incl = d;
                for (int o = 1; o < 32; o <<= 1) {
                    unsigned x = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                    if (lane >= o) incl += x;
                }
                unsigned wsum = __shfl_sync(0xFFFFFFFFu, incl, 31);
                int leader = __ffs(ballot) - 1;
                unsigned long long base = 0;
                if (lane == leader)
                    base = atomicAdd(cout, ((unsigned long long)wsum << 32) |
                                               (unsigned long long)__popc(ballot));
                base = __shfl_sync(0xFFFFFFFFu, base, leader);
                if (claim) {
                    unsigned pos = (unsigned)(base & 0xFFFFFFFFull) +
                                   __popc(ballot & ((1u << lane) - 1));
                    nqv[pos] = w;
                    nqoff[pos] = (unsigned)(base >> 32) + incl - d;
                    dist[w] = level;
                }
            }
        }
        __syncthreads();
    }
    // the last CTA seals the next frontier and decides whether to loop
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned tk = atomicAdd(&st->ticket, 1u);
        if (tk == gridDim.x - 1) {
            __threadfence();
            unsigned long long c = atomicAdd(cout, 0ull);
            unsigned nn = (unsigned)(c & 0xFFFFFFFFull);
            nqoff[nn] = (unsigned)(c >> 32);
            st->ticket = 0;
            st->visited += nn;
            st->scanned += total;
            st->level = level + 1;
            cudaGraphSetConditional(cond, (nn > 0 && level < st->nV) ? 1u : 0u);
        }
    }
}

void build_bfs_graph(hn_graph* g, BfsGraph& bg) {
    const int nV = g->nV;
    HN_CUDA(cudaMalloc((void**)&bg.state, sizeof(BfsState)));
    HN_CUDA(cudaMallocHost((void**)&bg.h_state, sizeof(BfsState)));
    HN_CUDA(cudaMalloc((void**)&bg.qbuf, sizeof(int32_t) * 2 * ((size_t)nV + 1)));
    HN_CUDA(cudaMalloc((void**)&bg.qoffbuf, sizeof(unsigned) * 2 * ((size_t)nV + 2)));
    HN_CUDA(cudaMalloc((void**)&bg.bitmap, sizeof(unsigned) * (((size_t)nV + 31) / 32 + 1)));
    bg.nV = nV;

    HN_CUDA(cudaGraphCreate(&bg.graph, 0));
    // init node
    cudaGraphNode_t init_node, cond_node, body_node;
    {
        void* args[] = {&bg.state};
        cudaKernelNodeParams p = {};
        p.func = (void*)k_bfs2_init;
        p.gridDim = dim3((unsigned)grid_for(g, nV, 256));
        p.blockDim = dim3(256);
        p.kernelParams = args;
        HN_CUDA(cudaGraphAddKernelNode(&init_node, bg.graph, nullptr, 0, &p));
    }
    cudaGraphConditionalHandle handle;
    HN_CUDA(cudaGraphConditionalHandleCreate(&handle, bg.graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    HN_CUDA(cudaGraphAddNode(&cond_node, bg.graph, &init_node, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    {
        void* args[] = {&bg.state, &handle};
        cudaKernelNodeParams p = {};
        p.func = (void*)k_bfs2_expand;
        p.gridDim = dim3((unsigned)g->info.sms * 4);
        p.blockDim = dim3(kBfsBlock);
        p.kernelParams = args;
        HN_CUDA(cudaGraphAddKernelNode(&body_node, body, nullptr, 0, &p));
    }
    HN_CUDA(cudaGraphInstantiate(&bg.exec, bg.graph, 0));
}

}  // namespace

void free_bfs_graph(BfsGraph* bg) {
    if (!bg) return;
    if (bg->exec) cudaGraphExecDestroy(bg->exec);
    if (bg->graph) cudaGraphDestroy(bg->graph);
    if (bg->state) cudaFree(bg->state);
    if (bg->h_state) cudaFreeHost(bg->h_state);
    if (bg->qbuf) cudaFree(bg->qbuf);
    if (bg->qoffbuf) cudaFree(bg->qoffbuf);
    if (bg->bitmap) cudaFree(bg->bitmap);
    delete bg;
}

namespace {

BfsGraph& bfs_graph_of(hn_graph* g) {
    if (g->bfs && g->bfs->nV != g->nV) {
        HN_CUDA(cudaStreamSynchronize(g->stream));
        free_bfs_graph(g->bfs);
        g->bfs = nullptr;
    }
    if (!g->bfs) {
        g->bfs = new BfsGraph();
        try {
            build_bfs_graph(g, *g->bfs);
        } catch (...) {
            free_bfs_graph(g->bfs);
            g->bfs = nullptr;
            throw;
        }
    }
    return *g->bfs;
}

void bfs_run(hn_graph* g, const int32_t* sources, int k, int32_t* dist, int mem,
             hn_bfs_stats_t* stats) {
    cudaStream_t s = g->stream;
    const int nV = g->nV;
    for (int i = 0; i < k; i++)
        if (sources[i] < 0 || sources[i] >= nV)
            throw Error(HN_ERR_INVALID, "BFS source outside [0, nV)");
    if (g->nE >= 0xFFFFFFFFll) throw Error(HN_ERR_CAPACITY, "BFS needs nE < 2^32");
    BfsGraph& bg = bfs_graph_of(g);
    DevBuf<int32_t> d_dist;
    if (mem == HN_MEM_HOST) d_dist.alloc((size_t)nV, s);
    std::vector<BfsState> snap(k > 0 ? k : 1);
    for (int i = 0; i < k; i++) {
        int32_t* out = mem == HN_MEM_HOST ? d_dist.get() : dist + (size_t)i * nV;
        BfsState& h = *bg.h_state;
        HN_CUDA(cudaStreamSynchronize(s));  // h_state is reused per source
        h = BfsState{};
        h.src = sources[i];
        h.nV = nV;
        h.dist = out;
        h.vtab = g->vtab;
        h.pool = g->pool;
        h.q[0] = bg.qbuf;
        h.q[1] = bg.qbuf + nV + 1;
        h.qoff[0] = bg.qoffbuf;
        h.qoff[1] = bg.qoffbuf + nV + 2;
        h.bitmap = bg.bitmap;
        HN_CUDA(cudaMemcpyAsync(bg.state, &h, sizeof(BfsState), cudaMemcpyHostToDevice, s));
        HN_CUDA(cudaGraphLaunch(bg.exec, s));
        count_launch(2);
        HN_CUDA(cudaMemcpyAsync(bg.h_state, bg.state, sizeof(BfsState), cudaMemcpyDeviceToHost, s));
        if (mem == HN_MEM_HOST)
            HN_CUDA(cudaMemcpyAsync(dist + (size_t)i * nV, out, sizeof(int32_t) * nV,
                                    cudaMemcpyDeviceToHost, s));
        HN_CUDA(cudaStreamSynchronize(s));
        snap[i] = *bg.h_state;
    }
    if (stats)
        for (int i = 0; i < k; i++) {
            stats[i].levels = snap[i].level - 1;
            stats[i].pad = 0;
            stats[i].visited = snap[i].visited;
            stats[i].edges_scanned = snap[i].scanned;
        }
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
