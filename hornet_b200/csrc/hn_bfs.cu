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
//   * Frontier entries are (vertex, adjacency base, edge offset).  The edge
//     offset is the exclusive prefix of the frontier's degrees; it comes out
//     of the enqueue itself: one 64-bit atomicAdd of (degree << 32 | 1) per
//     warp hands out the queue slot (low word) and the edge offset (high
//     word) together, so offsets are ordered like slots and no scan runs.
//   * The frontier's edge space is cut into chunks of kChunk edges.  The
//     vertex that covers the first edge of each chunk records itself in
//     chunk_seg[] when it is enqueued, so the expand kernel finds a chunk's
//     vertex window with two loads — no search in global memory.  Only
//     vertices with at least one edge are queued, so a chunk spans at most
//     kChunk + 1 queue entries.
//   * Visited-bitmap probes go through L1 (ld.ca): on power-law graphs most
//     edges point at a few hubs, and L2-only probes of their bitmap words
//     turn into a hot spot on a few L2 slices.  A stale L1 copy can only
//     miss bits set during this level (bits never clear), which costs an
//     extra atomicOr and never a wrong claim.
//   * A CTA stages the window's (edge offset, adjacency base) pairs in
//     shared memory; each thread takes kIpt consecutive edges, finds its
//     first vertex by a shared-memory binary search, then issues all kIpt
//     neighbour loads and all kIpt visited-bitmap probes back to back (high
//     memory-level parallelism), and claims new vertices with atomicOr on
//     the bitmap (nV/8 bytes, L2-resident): each vertex is enqueued and its
//     distance written exactly once.
//   * The last CTA of a level (ticket counter) seals the next frontier and
//     sets the WHILE condition with cudaGraphSetConditional; the loop also
//     stops after nV levels, so it always terminates.
// Distances equal the reference's: level-synchronous, INF = INT32_MAX.
//
// hn_bfs_do runs the same graph with a level kernel that may switch to
// bottom-up steps (Beamer's direction-optimising BFS, the counterpart of
// hornetsnest's BottomUpBFS, src/Static/BottomUpBreadthFirstSearch/
// BottomUpBFS.cu); distances are identical, fewer edges are read.
#include "hn_graph.cuh"

namespace hn {

constexpr int kBfsBlock = 128;
constexpr int kIpt = 8;                          // edges per thread per chunk
constexpr int kChunk = kBfsBlock * kIpt;         // edges per chunk

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
    long long* qbase[2];         // their adjacency base in the pool
    unsigned* qoff[2];           // exclusive degree prefix (edge offset)
    int32_t* chunk[2];           // queue slot covering each chunk's first edge
    unsigned* bitmap;            // visited bits
    int mode;                    // direction-optimising: 0 top-down, 1 bottom-up
    int pad;
    long long m_total;           // edges of the graph
    long long edges_visited;     // sum of degrees of vertices reached so far
    int alpha;                   // direction-optimising switch thresholds
    int beta;
    int dynamic_chunks;          // 1: CTAs take chunks from next_chunk
    unsigned next_chunk;         // chunk counter of the current level
    int warp_strided;            // 1: a warp's edges are lane-strided (coalesced loads)
    int cont;                    // 1 while another level follows (host-driven loop)
    int host_driven;             // 1: no conditional node (levels launched by the host)
    int pad3;
};

struct BfsGraph {
    int nV = -1;
    long long nchunk_cap = 0;
    BfsState* state = nullptr;      // device
    BfsState* h_state = nullptr;    // pinned
    int32_t* qbuf = nullptr;
    long long* qbasebuf = nullptr;
    unsigned* qoffbuf = nullptr;
    int32_t* chunkbuf = nullptr;
    unsigned* bitmap = nullptr;
    cudaGraph_t graph[2] = {nullptr, nullptr};      // [0] top-down, [1] direction-optimising
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    unsigned grid = 0;                              // level-kernel CTAs baked in
    // multi-source calls: pinned per-source states (the next source's state
    // is staged while the previous BFS runs), a copy stream and events so a
    // host-bound distance array is copied out while the next BFS runs
    static constexpr int kRing = 64;
    BfsState* h_ring = nullptr;                     // pinned, kRing entries
    cudaStream_t copy = nullptr;
    cudaEvent_t done[2] = {nullptr, nullptr};       // BFS into buffer b finished
    cudaEvent_t copied[2] = {nullptr, nullptr};     // buffer b copied to the host
};

namespace {

// Record queue slot `pos` as the owner of every chunk whose first edge lies
// in [off, off + d).
__device__ __forceinline__ void mark_chunks(int32_t* chunk, unsigned off, unsigned d, int pos) {
    unsigned c0 = (off + kChunk - 1) / kChunk;
    unsigned c1 = (off + d - 1) / kChunk;
    for (unsigned c = c0; c <= c1; c++) chunk[c] = pos;
}

__global__ void k_bfs3_init(BfsState* st) {
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
    VRec r = st->vtab[src];
    unsigned d = (unsigned)r.deg;
    // chunk marks of a high-degree source are spread over the grid
    if (d > 0) {
        unsigned nc = (d - 1) / kChunk + 1;
        for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc;
             c += (long long)gridDim.x * blockDim.x)
            st->chunk[0][c] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->q[0][0] = src;
        st->qbase[0][0] = r.off;
        st->qoff[0][0] = 0;
        st->qoff[0][d > 0 ? 1 : 0] = d;
        st->cnt[0] = d > 0 ? (((unsigned long long)d << 32) | 1ull) : 0ull;
        st->cnt[1] = 0;
        st->cnt[2] = 0;
        st->level = 1;
        st->ticket = 0;
        st->visited = 1;
        st->scanned = 0;
        st->mode = 0;
        st->edges_visited = d;
    }
}

// Per-level shared memory of the level kernel.
struct BfsSmem {
    unsigned start[kChunk + 2];   // window edge offsets (+ end)
    long long base[kChunk + 1];   // pool index = base + edge
    int claimed[kChunk];          // vertices claimed in this chunk
    int nclaimed;
    int nw;
    unsigned next;                // this CTA's next chunk
    unsigned long long wsum[kBfsBlock / 32];
    unsigned long long cbase;
};

// CTA-wide enqueue of the chunk's claimed vertices.  The claims are first
// gathered into shared memory (one shared atomic per warp), then each thread
// takes an equal contiguous share of them: distance written, and vertices
// with edges appended to the next frontier with their adjacency base and
// edge offset; ONE atomic per call reserves both the queue slots and the
// edge range.  Holding no per-claim arrays keeps the kernel's register
// count, and so its residency, down.  Must be called by all threads.
__device__ __forceinline__ void bfs_enqueue(BfsSmem& sm, const int (&w)[kIpt],
                                            const bool (&claim)[kIpt], int level,
                                            const VRec* __restrict__ vtab, int32_t* dist,
                                            unsigned long long* cout, int32_t* nqv,
                                            long long* nqbase, unsigned* nqoff, int32_t* nchunk,
                                            int& found) {
    const int lane = threadIdx.x & 31;
    if (threadIdx.x == 0) sm.nclaimed = 0;
    __syncthreads();
    {
        int mine = 0;
#pragma unroll
        for (int k = 0; k < kIpt; k++) mine += claim[k] ? 1 : 0;
        int incl = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int x = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += x;
        }
        const int wtot = __shfl_sync(0xFFFFFFFFu, incl, 31);
        int wbase = 0;
        if (lane == 31 && wtot) wbase = atomicAdd(&sm.nclaimed, wtot);
        wbase = __shfl_sync(0xFFFFFFFFu, wbase, 31);
        int at = wbase + incl - mine;
#pragma unroll
        for (int k = 0; k < kIpt; k++)
            if (claim[k]) sm.claimed[at++] = w[k];
    }
    __syncthreads();
    const int n = sm.nclaimed;
    if (n == 0) return;   // uniform: every thread read the same count
    const int per = (n + kBfsBlock - 1) / kBfsBlock;
    const int i0 = threadIdx.x * per;
    const int i1 = i0 + per < n ? i0 + per : n;
    unsigned long long mine = 0;   // (degree sum << 32) | queued count
    for (int i = i0; i < i1; i++) {
        const int v = sm.claimed[i];
        const int d = vtab[v].deg;
        dist[v] = level;
        found++;
        if (d) mine += ((unsigned long long)d << 32) | 1ull;
    }
    unsigned long long incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long x = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += x;
    }
    const int warp = threadIdx.x >> 5;
    if (lane == 31) sm.wsum[warp] = incl;
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned long long v = threadIdx.x < kBfsBlock / 32 ? sm.wsum[threadIdx.x] : 0ull;
        unsigned long long vi = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long x = __shfl_up_sync(0xFFFFFFFFu, vi, o);
            if (lane >= o) vi += x;
        }
        if (threadIdx.x < kBfsBlock / 32) sm.wsum[threadIdx.x] = vi - v;   // exclusive
        unsigned long long tot = __shfl_sync(0xFFFFFFFFu, vi, 31);
        if (threadIdx.x == 0) sm.cbase = tot ? atomicAdd(cout, tot) : 0ull;
    }
    __syncthreads();
    unsigned long long at = sm.cbase + sm.wsum[warp] + (incl - mine);
    int pos = (int)(at & 0xFFFFFFFFull);
    unsigned off = (unsigned)(at >> 32);
    for (int i = i0; i < i1; i++) {
        const int v = sm.claimed[i];
        const VRec r = vtab[v];   // second read of the record: an L1 hit
        if (r.deg) {
            nqv[pos] = v;
            nqbase[pos] = r.off;
            nqoff[pos] = off;
            mark_chunks(nchunk, off, (unsigned)r.deg, pos);
            pos++;
            off += (unsigned)r.deg;
        }
    }
    __syncthreads();
}

// One BFS level.  TopDown (always, or while st->mode == 0 when DO): the
// frontier's edges in chunks.  BottomUp (DO and st->mode == 1): every
// unvisited vertex scans its sorted neighbours for one at distance level-1
// and stops at the first (Beamer, Asanovic & Patterson, "Direction-Optimizing
// Breadth-First Search", SC 2012).  Both produce the next frontier queue, so
// the direction may change at any level; distances are the same either way.
template <bool DO>
__global__ void __launch_bounds__(kBfsBlock, 9)
k_bfs_level(BfsState* st, cudaGraphConditionalHandle cond) {
    __shared__ BfsSmem sm;
    const int level = st->level;
    const int it = level - 1;
    const unsigned long long cin = st->cnt[it % 3];
    unsigned long long* cout = &st->cnt[(it + 1) % 3];
    if (blockIdx.x == 0 && threadIdx.x == 0) st->cnt[(it + 2) % 3] = 0;
    const int nq = (int)(cin & 0xFFFFFFFFull);
    const unsigned total = (unsigned)(cin >> 32);
    const int cur = it & 1, nxt = cur ^ 1;
    int32_t* nqv = st->q[nxt];
    long long* nqbase = st->qbase[nxt];
    unsigned* nqoff = st->qoff[nxt];
    int32_t* nchunk = st->chunk[nxt];
    const VRec* vtab = st->vtab;
    const int32_t* pool = st->pool;
    unsigned* bm = st->bitmap;
    int32_t* dist = st->dist;
    const int lane = threadIdx.x & 31;
    const int mode = DO ? st->mode : 0;
    int found = 0;

    if (mode == 0) {
        const long long* qbase = st->qbase[cur];
        const unsigned* qoff = st->qoff[cur];
        const int32_t* chunk = st->chunk[cur];
        const unsigned nchunks = (total + kChunk - 1) / kChunk;
        const bool dyn = st->dynamic_chunks != 0;
        const bool warp_strided = st->warp_strided != 0;
        if (threadIdx.x == 0) sm.next = dyn ? atomicAdd(&st->next_chunk, 1u) : blockIdx.x;
        __syncthreads();
        for (unsigned c = sm.next; c < nchunks; c = sm.next) {
            const unsigned e0 = c * kChunk;
            const unsigned e1 = e0 + kChunk < total ? e0 + kChunk : total;
            const int s0 = chunk[c];
            const int s1 = c + 1 < nchunks ? chunk[c + 1] : nq - 1;   // inclusive
            const int nw = s1 - s0 + 1;
            for (int j = threadIdx.x; j <= nw; j += kBfsBlock) {
                int s = s0 + j;
                unsigned so = qoff[s];        // qoff[nq] is the sealed total
                sm.start[j] = so;
                if (j < nw) sm.base[j] = qbase[s] - (long long)so;
            }
            if (threadIdx.x == 0) sm.nw = nw;
            __syncthreads();
            int w[kIpt];
            bool claim[kIpt];
#pragma unroll
            for (int k = 0; k < kIpt; k++) { w[k] = -1; claim[k] = false; }
            bool mine_any = false;
            if (warp_strided) {
                // the warp's 32*kIpt edges, lane-strided: each load reads 32
                // consecutive edges (one window for high-degree vertices);
                // windows are searched inside the warp's own window range
                const unsigned wb = e0 + (threadIdx.x >> 5) * (32 * kIpt);
                if (wb < e1) {
                    const unsigned wl = wb + 32 * kIpt - 1 < e1 - 1 ? wb + 32 * kIpt - 1 : e1 - 1;
                    int jw0 = 0, jw1 = 0;
                    {
                        int lo = 0, hi = sm.nw;   // last j with start[j] <= wb
                        while (hi - lo > 1) {
                            int mid = (lo + hi) >> 1;
                            if (sm.start[mid] <= wb) lo = mid; else hi = mid;
                        }
                        jw0 = lo;
                        hi = sm.nw;               // last j with start[j] <= wl
                        while (hi - lo > 1) {
                            int mid = (lo + hi) >> 1;
                            if (sm.start[mid] <= wl) lo = mid; else hi = mid;
                        }
                        jw1 = lo;
                    }
#pragma unroll
                    for (int k = 0; k < kIpt; k++) {
                        const unsigned e = wb + k * 32 + (threadIdx.x & 31);
                        if (e < e1) {
                            int lo = jw0, hi = jw1 + 1;
                            while (hi - lo > 1) {
                                int mid = (lo + hi) >> 1;
                                if (sm.start[mid] <= e) lo = mid; else hi = mid;
                            }
                            w[k] = __ldg(pool + sm.base[lo] + e);
                            mine_any = true;
                        }
                    }
                }
            } else {
                // this thread's edges [a, b)
                const unsigned a = e0 + threadIdx.x * kIpt;
                const unsigned b = a + kIpt < e1 ? a + kIpt : e1;
                if (a < b) {
                    mine_any = true;
                    int lo = 0, hi = sm.nw;        // last j with start[j] <= a
                    while (hi - lo > 1) {
                        int mid = (lo + hi) >> 1;
                        if (sm.start[mid] <= a) lo = mid; else hi = mid;
                    }
                    int j = lo;
#pragma unroll
                    for (int k = 0; k < kIpt; k++) {
                        unsigned e = a + k;
                        if (e < b) {
                            while (sm.start[j + 1] <= e) j++;
                            w[k] = __ldg(pool + sm.base[j] + e);
                        }
                    }
                }
            }
            if (mine_any) {
                unsigned word[kIpt];
#pragma unroll
                for (int k = 0; k < kIpt; k++)
                    word[k] = w[k] >= 0 ? __ldca(bm + (w[k] >> 5)) : 0xFFFFFFFFu;
#pragma unroll
                for (int k = 0; k < kIpt; k++) {
                    if (w[k] >= 0 && !(word[k] & (1u << (w[k] & 31)))) {
                        unsigned bit = 1u << (w[k] & 31);
                        claim[k] = !(atomicOr(bm + (w[k] >> 5), bit) & bit);
                    }
                }
            }
            bfs_enqueue(sm, w, claim, level, vtab, dist, cout, nqv, nqbase, nqoff, nchunk, found);
            // bfs_enqueue ends with a barrier, so every thread has read sm.next
            if (threadIdx.x == 0) sm.next = dyn ? atomicAdd(&st->next_chunk, 1u) : c + gridDim.x;
            __syncthreads();
        }
    } else {
        // bottom-up over all vertices, kIpt per thread, striped
        const int nV = st->nV;
        const int per = kBfsBlock * kIpt;
        const int nvc = (nV + per - 1) / per;
        for (int c = blockIdx.x; c < nvc; c += gridDim.x) {
            int w[kIpt];
            bool claim[kIpt];
            int dv[kIpt];
#pragma unroll
            for (int k = 0; k < kIpt; k++) {
                int v = c * per + k * kBfsBlock + threadIdx.x;
                w[k] = v < nV ? v : -1;
                claim[k] = false;
                dv[k] = w[k] >= 0 ? __ldcg(dist + v) : 0;
            }
#pragma unroll
            for (int k = 0; k < kIpt; k++) {
                if (w[k] >= 0 && dv[k] == kInf) {
                    VRec r = vtab[w[k]];
                    const int32_t* nb = pool + r.off;
                    for (int i = 0; i < r.deg; i++) {
                        if (__ldca(dist + nb[i]) == level - 1) { claim[k] = true; break; }
                    }
                    if (claim[k]) atomicOr(bm + (w[k] >> 5), 1u << (w[k] & 31));
                }
            }
            bfs_enqueue(sm, w, claim, level, vtab, dist, cout, nqv, nqbase, nqoff, nchunk, found);
        }
    }
    // visited count: one atomic per warp
    for (int o = 16; o; o >>= 1) found += __shfl_down_sync(0xFFFFFFFFu, found, o);
    if (lane == 0 && found) atomicAdd((unsigned long long*)&st->visited, (unsigned long long)found);
    // the last CTA seals the next frontier, picks the next direction and
    // decides whether to loop
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned tk = atomicAdd(&st->ticket, 1u);
        if (tk == gridDim.x - 1) {
            __threadfence();
            unsigned long long cn = atomicAdd(cout, 0ull);
            unsigned nn = (unsigned)(cn & 0xFFFFFFFFull);
            unsigned long long mf = cn >> 32;
            nqoff[nn] = (unsigned)mf;
            st->ticket = 0;
            st->next_chunk = 0;
            st->scanned += total;
            st->level = level + 1;
            if (DO) {
                // Beamer's switch: to bottom-up when the next frontier's edges
                // exceed 1/alpha of the unexplored edges (alpha = 14 by
                // default), back to top-down when the frontier falls below
                // nV/beta vertices (beta = 24) and is shrinking
                st->edges_visited += (long long)mf;
                long long mu = st->m_total - st->edges_visited;
                if (st->mode == 0) {
                    if ((long long)mf * st->alpha > mu) st->mode = 1;
                } else {
                    if ((long long)nn * st->beta < st->nV && nn < (unsigned)nq) st->mode = 0;
                }
            }
            const unsigned more = (nn > 0 && level < st->nV) ? 1u : 0u;
            st->cont = (int)more;
            if (!st->host_driven) cudaGraphSetConditional(cond, more);
        }
    }
}

void build_bfs_graph(hn_graph* g, BfsGraph& bg) {
    const int nV = g->nV;
    const long long nchunk_cap = g->nE / kChunk + 4;
    HN_CUDA(cudaMalloc((void**)&bg.state, sizeof(BfsState)));
    HN_CUDA(cudaMallocHost((void**)&bg.h_state, sizeof(BfsState)));
    HN_CUDA(cudaMalloc((void**)&bg.qbuf, sizeof(int32_t) * 2 * ((size_t)nV + 1)));
    HN_CUDA(cudaMalloc((void**)&bg.qbasebuf, sizeof(long long) * 2 * ((size_t)nV + 1)));
    HN_CUDA(cudaMalloc((void**)&bg.qoffbuf, sizeof(unsigned) * 2 * ((size_t)nV + 2)));
    HN_CUDA(cudaMalloc((void**)&bg.chunkbuf, sizeof(int32_t) * 2 * (size_t)nchunk_cap));
    HN_CUDA(cudaMalloc((void**)&bg.bitmap, sizeof(unsigned) * (((size_t)nV + 31) / 32 + 1)));
    bg.nV = nV;
    bg.nchunk_cap = nchunk_cap;

    for (int variant = 0; variant < 2; variant++) {
        cudaGraph_t& graph = bg.graph[variant];
        HN_CUDA(cudaGraphCreate(&graph, 0));
        cudaGraphNode_t init_node, cond_node, body_node;
        {
            void* args[] = {&bg.state};
            cudaKernelNodeParams p = {};
            p.func = (void*)k_bfs3_init;
            p.gridDim = dim3((unsigned)grid_for(g, nV, 256));
            p.blockDim = dim3(256);
            p.kernelParams = args;
            HN_CUDA(cudaGraphAddKernelNode(&init_node, graph, nullptr, 0, &p));
        }
        cudaGraphConditionalHandle handle;
        HN_CUDA(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        HN_CUDA(cudaGraphAddNode(&cond_node, graph, &init_node, 1, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        {
            void* args[] = {&bg.state, &handle};
            cudaKernelNodeParams p = {};
            p.func = variant ? (void*)k_bfs_level<true> : (void*)k_bfs_level<false>;
            p.gridDim = dim3(bg.grid);
            p.blockDim = dim3(kBfsBlock);
            p.kernelParams = args;
            HN_CUDA(cudaGraphAddKernelNode(&body_node, body, nullptr, 0, &p));
        }
        HN_CUDA(cudaGraphInstantiate(&bg.exec[variant], graph, 0));
    }
}

}  // namespace

void free_bfs_graph(BfsGraph* bg) {
    if (!bg) return;
    for (int i = 0; i < 2; i++) {
        if (bg->exec[i]) cudaGraphExecDestroy(bg->exec[i]);
        if (bg->graph[i]) cudaGraphDestroy(bg->graph[i]);
    }
    if (bg->copy) cudaStreamSynchronize(bg->copy);
    for (int i = 0; i < 2; i++) {
        if (bg->done[i]) cudaEventDestroy(bg->done[i]);
        if (bg->copied[i]) cudaEventDestroy(bg->copied[i]);
    }
    if (bg->copy) cudaStreamDestroy(bg->copy);
    if (bg->h_ring) cudaFreeHost(bg->h_ring);
    if (bg->state) cudaFree(bg->state);
    if (bg->h_state) cudaFreeHost(bg->h_state);
    if (bg->qbuf) cudaFree(bg->qbuf);
    if (bg->qbasebuf) cudaFree(bg->qbasebuf);
    if (bg->qoffbuf) cudaFree(bg->qoffbuf);
    if (bg->chunkbuf) cudaFree(bg->chunkbuf);
    if (bg->bitmap) cudaFree(bg->bitmap);
    delete bg;
}

namespace {

BfsGraph& bfs_graph_of(hn_graph* g) {
    // rebuilt when the vertex count changes, the edge count outgrows the
    // chunk table or the bfs.ctas_per_sm knob changes the level grid
    const unsigned grid = (unsigned)(g->info.sms * knob(kKnobBfsCtasPerSm));
    if (g->bfs && (g->bfs->nV != g->nV || g->nE / kChunk + 4 > g->bfs->nchunk_cap ||
                   g->bfs->grid != grid)) {
        HN_CUDA(cudaStreamSynchronize(g->stream));
        free_bfs_graph(g->bfs);
        g->bfs = nullptr;
    }
    if (!g->bfs) {
        g->bfs = new BfsGraph();
        g->bfs->grid = grid;
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
             hn_bfs_stats_t* stats, bool direction_optimizing) {
    cudaStream_t s = g->stream;
    const int nV = g->nV;
    for (int i = 0; i < k; i++)
        if (sources[i] < 0 || sources[i] >= nV)
            throw Error(HN_ERR_INVALID, "BFS source outside [0, nV)");
    if (g->nE >= 0xFFFFFFFFll) throw Error(HN_ERR_CAPACITY, "BFS needs nE < 2^32");
    BfsGraph& bg = bfs_graph_of(g);
    if (!bg.h_ring) {
        HN_CUDA(cudaMallocHost((void**)&bg.h_ring, sizeof(BfsState) * BfsGraph::kRing));
        HN_CUDA(cudaStreamCreateWithFlags(&bg.copy, cudaStreamNonBlocking));
        for (int b = 0; b < 2; b++) {
            HN_CUDA(cudaEventCreateWithFlags(&bg.done[b], cudaEventDisableTiming));
            HN_CUDA(cudaEventCreateWithFlags(&bg.copied[b], cudaEventDisableTiming));
        }
    }
    const bool host_out = mem == HN_MEM_HOST;
    // host output: two device buffers; BFS i writes buffer i % 2 while the
    // copy stream drains buffer (i - 1) % 2 to the host
    DevBuf<int32_t> d_dist;
    if (host_out) d_dist.alloc((size_t)2 * nV, s);
    const bool host_driven = knob(kKnobBfsHostLevels) != 0;
    std::vector<BfsState> snap(k > 0 ? k : 1);
    HN_CUDA(cudaStreamSynchronize(s));   // the ring's previous contents are read
    for (int i = 0; i < k; i++) {
        const int r = i % BfsGraph::kRing;
        if (i > 0 && r == 0) {
            // ring wrapped: collect the snapshots of the last kRing sources
            HN_CUDA(cudaStreamSynchronize(s));
            for (int j = 0; j < BfsGraph::kRing; j++) snap[i - BfsGraph::kRing + j] = bg.h_ring[j];
        }
        const int b = i & 1;
        int32_t* out = host_out ? d_dist.get() + (size_t)b * nV : dist + (size_t)i * nV;
        if (host_out && i >= 2) HN_CUDA(cudaStreamWaitEvent(s, bg.copied[b], 0));
        BfsState& h = bg.h_ring[r];
        h = BfsState{};
        h.src = sources[i];
        h.nV = nV;
        h.dist = out;
        h.vtab = g->vtab;
        h.pool = g->pool;
        h.q[0] = bg.qbuf;
        h.q[1] = bg.qbuf + nV + 1;
        h.qbase[0] = bg.qbasebuf;
        h.qbase[1] = bg.qbasebuf + nV + 1;
        h.qoff[0] = bg.qoffbuf;
        h.qoff[1] = bg.qoffbuf + nV + 2;
        h.chunk[0] = bg.chunkbuf;
        h.chunk[1] = bg.chunkbuf + bg.nchunk_cap;
        h.bitmap = bg.bitmap;
        h.m_total = g->nE;
        h.alpha = (int)knob(kKnobBfsDoAlpha);
        h.beta = (int)knob(kKnobBfsDoBeta);
        h.dynamic_chunks = (int)knob(kKnobBfsDynamicChunks);
        h.warp_strided = (int)knob(kKnobBfsWarpStrided);
        h.host_driven = host_driven ? 1 : 0;
        h.next_chunk = 0;
        HN_CUDA(cudaMemcpyAsync(bg.state, &h, sizeof(BfsState), cudaMemcpyHostToDevice, s));
        // profiling records the whole graph (one init + one expand per
        // level) under the name of its dominant kernel
        cudaEvent_t ev0 = nullptr;
        if (g_profiling) profile_begin(s, &ev0);
        if (host_driven) {
            // host-driven levels: one ordinary launch per level (each level
            // can be profiled on its own), one host round trip per level
            k_bfs3_init<<<(unsigned)grid_for(g, nV, 256), 256, 0, s>>>(bg.state);
            HN_CUDA(cudaGetLastError());
            count_launch();
            for (int lv = 0; lv <= nV; lv++) {
                if (direction_optimizing)
                    k_bfs_level<true><<<bg.grid, kBfsBlock, 0, s>>>(bg.state, 0);
                else
                    k_bfs_level<false><<<bg.grid, kBfsBlock, 0, s>>>(bg.state, 0);
                HN_CUDA(cudaGetLastError());
                count_launch();
                HN_CUDA(cudaMemcpyAsync(&bg.h_state->cont, &bg.state->cont, sizeof(int),
                                        cudaMemcpyDeviceToHost, s));
                HN_CUDA(cudaStreamSynchronize(s));
                if (!bg.h_state->cont) break;
            }
        } else {
            HN_CUDA(cudaGraphLaunch(bg.exec[direction_optimizing ? 1 : 0], s));
            count_launch(2);
        }
        if (ev0)
            profile_end(direction_optimizing ? "k_bfs_level<true>" : "k_bfs_level<false>", s, ev0);
        // the finished state back into this source's ring slot (ordered
        // before the next source's state upload on the same stream)
        HN_CUDA(cudaMemcpyAsync(&h, bg.state, sizeof(BfsState), cudaMemcpyDeviceToHost, s));
        if (host_out) {
            HN_CUDA(cudaEventRecord(bg.done[b], s));
            HN_CUDA(cudaStreamWaitEvent(bg.copy, bg.done[b], 0));
            HN_CUDA(cudaMemcpyAsync(dist + (size_t)i * nV, out, sizeof(int32_t) * nV,
                                    cudaMemcpyDeviceToHost, bg.copy));
            HN_CUDA(cudaEventRecord(bg.copied[b], bg.copy));
        }
    }
    HN_CUDA(cudaStreamSynchronize(s));
    if (host_out) HN_CUDA(cudaStreamSynchronize(bg.copy));
    if (k > 0) {
        const int first = ((k - 1) / BfsGraph::kRing) * BfsGraph::kRing;
        for (int i = first; i < k; i++) snap[i] = bg.h_ring[i - first];
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
    bfs_run(g, &src, 1, dist, mem, stats, false);
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
    bfs_run(g, sources, k, dist, mem, stats, false);
    HN_API_END
}

int hn_bfs_do(hn_graph_t* g, const int32_t* sources, int32_t k, int32_t* dist, int mem,
              hn_bfs_stats_t* stats) {
    HN_API_BEGIN
    HN_REQUIRE(g && sources && dist, "null argument");
    HN_REQUIRE(k >= 0, "negative source count");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    HN_REQUIRE(g->nV > 0 || k == 0, "empty graph");
    HN_CUDA(cudaSetDevice(g->device));
    bfs_run(g, sources, k, dist, mem, stats, true);
    HN_API_END
}

}  // extern "C"
