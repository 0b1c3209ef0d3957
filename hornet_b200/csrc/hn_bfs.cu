// BFS TopDown (hornetsnest/src/Static/BreadthFirstSearch/TopDown.cu:49-106).
//
// Reference: per level, forAllEdges(queue, BFSOperator, BinarySearch) =
// computeWorkKernel + CUB scan + D2H total + binarySearchKernel with a
// non-atomic `dist[dst] == INF` test (duplicate enqueues possible), then a
// <<<1,1>>> swap kernel and another D2H (TwoLevelQueue.i.cuh:158-179): at
// least three host synchronisations per level.
//
// Here a whole BFS is ONE CUDA-graph launch: an init kernel, then a
// conditional WHILE node whose body is a single persistent level kernel.
//   * Frontier entries are (vertex, adjacency base, edge offset).  The edge
//     offset is the exclusive prefix of the frontier's degrees; it comes out
//     of the enqueue itself: one 64-bit atomicAdd of (degree sum << 32 |
//     count) hands out the queue slots (low word) and the edge offsets (high
//     word) together, so offsets are ordered like slots and no scan runs.
//   * The frontier's edge space is cut into chunks of 2^cshift edges.  The
//     vertex that covers the first edge of each chunk records itself in
//     chunk[] when it is enqueued, so a chunk finds its vertex window with
//     two loads -- no search in global memory.  Only vertices with at least
//     one edge are queued, so a chunk of E edges spans at most E + 1 queue
//     entries.
//   * Visited-bitmap probes go through L1 (ld.ca): on power-law graphs most
//     edges point at a few hubs, and L2-only probes of their bitmap words
//     turn into a hot spot on a few L2 slices.  A stale L1 copy can only
//     miss bits set during this level (bits never clear), which costs an
//     extra atomicOr and never a wrong claim.  New vertices are claimed with
//     atomicOr on the bitmap (nV/8 bytes, L2-resident), so each vertex is
//     enqueued and its distance written exactly once.
//   * The last CTA of a level (ticket counter) seals the next frontier and
//     sets the WHILE condition with cudaGraphSetConditional; the loop also
//     stops after nV levels, so it always terminates.
//
// Two level kernels share this frontier format (knob bfs.kernel):
//   * k_bfs_wlevel (default): every WARP runs on its own.  It takes 256-edge
//     chunks round-robin, reads its window, loads its 8 x 32 neighbours
//     lane-strided (each load instruction reads 32 consecutive edges),
//     probes and claims, and appends the claims to a warp-private list in
//     shared memory.  The list is enqueued 32 vertices at a time with one
//     atomic per 32 claims.  There is no CTA barrier inside a level, so the
//     resident warps are independent chains of loads.  Windows of at most
//     32 vertices stay in registers: a lane finds the vertex of each of its
//     edges with one OR-reduction, one ballot and one shuffle.
//   * k_bfs_level: a CTA of 128 threads per 1024-edge chunk, with the window
//     staged in shared memory and a CTA-wide enqueue (one atomic per chunk).
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
constexpr int kChunk = kBfsBlock * kIpt;         // edges per CTA chunk (k_bfs_level)
constexpr int kChunkShiftCta = 10;               // log2(kChunk)
constexpr int kWBlock = 256;                     // k_bfs_wlevel: threads per CTA
constexpr int kWIpt = 8;                         // edges per lane per warp chunk
constexpr int kWChunk = 32 * kWIpt;              // edges per warp chunk
constexpr int kChunkShiftWarp = 8;               // log2(kWChunk)
constexpr int kWList = kWChunk + 32;             // claim list capacity per warp
static_assert(kChunk == 1 << kChunkShiftCta && kWChunk == 1 << kChunkShiftWarp, "chunk sizes");

constexpr int kTraceLevels = 32;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

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
    int cshift;                  // log2 of the chunk size of chunk[]
    // level trace: global timer (ns) at the start and at the end of each of
    // the first kTraceLevels levels, and the frontier edges each one scanned
    unsigned long long t_start;
    unsigned long long t_end[kTraceLevels];
    unsigned long long lvl_edges[kTraceLevels];
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
    int kernel = -1;                                // bfs.kernel baked in
    int per_sm = 0;                                 // CTAs per SM baked in
    // multi-source calls: pinned per-source states (the next source's state
    // is staged while the previous BFS runs), a copy stream and events so a
    // host-bound distance array is copied out while the next BFS runs
    static constexpr int kRing = 64;
    BfsState* h_ring = nullptr;                     // pinned, kRing entries
    cudaStream_t copy = nullptr;
    cudaEvent_t done[2] = {nullptr, nullptr};       // BFS into buffer b finished
    cudaEvent_t copied[2] = {nullptr, nullptr};     // buffer b copied to the host
    BfsState last = {};                             // final state of the latest BFS
    bool have_last = false;
};

namespace {

// Record queue slot `pos` as the owner of every chunk (2^cs edges) whose
// first edge lies in [off, off + d).
__device__ __forceinline__ void mark_chunks(int32_t* chunk, unsigned off, unsigned d, int pos,
                                            int cs) {
    unsigned c0 = (off + (1u << cs) - 1) >> cs;
    unsigned c1 = (off + d - 1) >> cs;
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
        unsigned nc = ((d - 1) >> st->cshift) + 1;
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
        st->t_start = global_ns();
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
                                            int cs, int& found) {
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
            mark_chunks(nchunk, off, (unsigned)r.deg, pos, cs);
            pos++;
            off += (unsigned)r.deg;
        }
    }
    __syncthreads();
}

// End of a level, called by every thread of every CTA: the visited count
// (one atomic per warp), then the last CTA seals the next frontier, picks the
// next direction and decides whether to loop.
template <bool DO>
__device__ __forceinline__ void bfs_level_end(BfsState* st, cudaGraphConditionalHandle cond,
                                              int found, int level, int nq, unsigned total,
                                              unsigned long long* cout, unsigned* nqoff) {
    const int lane = threadIdx.x & 31;
    for (int o = 16; o; o >>= 1) found += __shfl_down_sync(0xFFFFFFFFu, found, o);
    if (lane == 0 && found) atomicAdd((unsigned long long*)&st->visited, (unsigned long long)found);
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
            if (level <= kTraceLevels) {
                st->t_end[level - 1] = global_ns();
                st->lvl_edges[level - 1] = total;
            }
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

// Warp-private shared memory of k_bfs_wlevel.
struct WarpSmem {
    long long base[kWList];        // window: pool index = base + edge (large windows);
                                   // flush: adjacency base of each listed vertex
    unsigned start[kWList];        // window edge offsets (+ end); flush: degrees
    int list[kWList];              // claimed vertices not yet enqueued
};

// Where a level's claims go (per CTA, in shared memory: the enqueue is rare
// next to the edge loop, so these do not hold registers there).
struct LevelOut {
    const VRec* vtab;
    int32_t* dist;
    unsigned long long* cout;
    int32_t* nqv;
    long long* nqbase;
    unsigned* nqoff;
    int32_t* nchunk;
    int level;
};

// Enqueue all n vertices of the warp's claim list in one pass: every lane
// reads the records of up to ceil(n / 32) listed vertices (loads issued
// together) into the warp's shared memory and writes their distances, then
// one warp scan and ONE 64-bit atomicAdd reserve the queue slots and the
// edge range of all of them, and each lane writes its consecutive share of
// queue entries.  A vertex that spans many chunks has its chunk marks
// written by the whole warp.  Called by all 32 lanes with the same n.
__device__ __forceinline__ void warp_flush(WarpSmem& sm, int n, const LevelOut& lo, int& found) {
    const int lane = threadIdx.x & 31;
    const VRec* __restrict__ vtab = lo.vtab;
    int32_t* dist = lo.dist;
    const int level = lo.level;
    const unsigned kFull = 0xFFFFFFFFu;
    // records of the listed vertices, four loads in flight per lane
    for (int i0 = 0; i0 < n; i0 += 128) {
        VRec r[4];
        int v[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int i = i0 + u * 32 + lane;
            v[u] = i < n ? sm.list[i] : -1;
            if (v[u] >= 0) r[u] = vtab[v[u]];
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int i = i0 + u * 32 + lane;
            if (v[u] >= 0) {
                dist[v[u]] = level;
                found++;
                sm.base[i] = r[u].off;
                sm.start[i] = (unsigned)r[u].deg;
            }
        }
    }
    __syncwarp();
    // lane L owns list entries [L * per, L * per + per)
    const int per = (n + 31) >> 5;
    const int i0 = lane * per;
    const int i1 = i0 + per < n ? i0 + per : n;
    unsigned long long mine = 0;   // (degree sum << 32) | vertices with edges
    for (int i = i0; i < i1; i++) {
        const unsigned d = sm.start[i];
        if (d) mine += ((unsigned long long)d << 32) | 1ull;
    }
    unsigned long long incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long x = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += x;
    }
    unsigned long long base = 0;
    if (lane == 31 && incl) base = atomicAdd(lo.cout, incl);
    base = __shfl_sync(kFull, base, 31);
    unsigned long long at = base + incl - mine;
    bool has_big = false;
    int32_t* nqv = lo.nqv;
    long long* nqbase = lo.nqbase;
    unsigned* nqoff = lo.nqoff;
    int32_t* nchunk = lo.nchunk;
    for (int i = i0; i < i1; i++) {
        const unsigned d = sm.start[i];
        if (!d) continue;
        const int pos = (int)(at & 0xFFFFFFFFull);
        const unsigned off = (unsigned)(at >> 32);
        nqv[pos] = sm.list[i];
        nqbase[pos] = sm.base[i];
        nqoff[pos] = off;
        const unsigned c0 = (off + kWChunk - 1) >> kChunkShiftWarp;
        const unsigned c1 = (off + d - 1) >> kChunkShiftWarp;
        if (c1 < c0 + 8) {
            for (unsigned c = c0; c <= c1; c++) nchunk[c] = pos;
        } else {
            // marked below by the whole warp: keep its (slot, offset)
            sm.base[i] = (long long)at;
            sm.start[i] = d | 0x80000000u;
            has_big = true;
        }
        at += ((unsigned long long)d << 32) | 1ull;
    }
    // vertices spanning many chunks: their chunk marks written by the warp
    unsigned bigm = __ballot_sync(kFull, has_big);
    __syncwarp();
    while (bigm) {
        const int src = __ffs(bigm) - 1;
        bigm &= bigm - 1;
        const int j0 = src * per;
        const int j1 = j0 + per < n ? j0 + per : n;
        for (int i = j0; i < j1; i++) {
            const unsigned f = sm.start[i];
            if (!(f & 0x80000000u)) continue;
            const unsigned d = f & 0x7FFFFFFFu;
            const unsigned long long a2 = (unsigned long long)sm.base[i];
            const int pos = (int)(a2 & 0xFFFFFFFFull);
            const unsigned off = (unsigned)(a2 >> 32);
            const unsigned c0 = (off + kWChunk - 1) >> kChunkShiftWarp;
            const unsigned c1 = (off + d - 1) >> kChunkShiftWarp;
            for (unsigned c = c0 + lane; c <= c1; c += 32) nchunk[c] = pos;
        }
    }
    __syncwarp();
}

// Append the lanes' claimed vertices (bit k of `claim` set: w[k] claimed) to
// the warp list and flush whole groups of 32.
__device__ __forceinline__ void warp_claims(WarpSmem& sm, int& nlist, const int (&w)[kWIpt],
                                            unsigned claim, const LevelOut& lo, int& found) {
    const int lane = threadIdx.x & 31;
    const unsigned kFull = 0xFFFFFFFFu;
    if (!__any_sync(kFull, claim != 0u)) return;
    const int mine = __popc(claim);
    int incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int x = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += x;
    }
    const int tot = __shfl_sync(kFull, incl, 31);
    if (tot == 0) return;
    int at = nlist + incl - mine;
#pragma unroll
    for (int k = 0; k < kWIpt; k++)
        if (claim >> k & 1u) sm.list[at++] = w[k];
    nlist += tot;
    __syncwarp();
    if (nlist >= 32) {
        warp_flush(sm, nlist, lo, found);
        nlist = 0;
    }
}

// One BFS level, warp-independent form (bfs.kernel = 1).  Top-down: warps
// take 256-edge chunks round-robin.  Bottom-up (DO and st->mode == 1): warps
// take 256 vertices; every unvisited one scans its sorted neighbours for one
// at distance level-1 and stops at the first (Beamer, Asanovic & Patterson,
// "Direction-Optimizing Breadth-First Search", SC 2012).  Both append their
// claims to the warp's list; there is no CTA barrier before the level end.
template <bool DO, int MINB>
__global__ void __launch_bounds__(kWBlock, MINB)
k_bfs_wlevel(BfsState* st, cudaGraphConditionalHandle cond) {
    __shared__ WarpSmem wsm[kWBlock / 32];
    __shared__ LevelOut lo;
    const unsigned kFull = 0xFFFFFFFFu;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    WarpSmem& sm = wsm[warp];
    const int level = st->level;
    const int it = level - 1;
    const unsigned long long cin = st->cnt[it % 3];
    unsigned long long* cout = &st->cnt[(it + 1) % 3];
    const int nq = (int)(cin & 0xFFFFFFFFull);
    const unsigned total = (unsigned)(cin >> 32);
    const int cur = it & 1, nxt = cur ^ 1;
    if (threadIdx.x == 0) {
        if (blockIdx.x == 0) st->cnt[(it + 2) % 3] = 0;
        lo.vtab = st->vtab;
        lo.dist = st->dist;
        lo.cout = cout;
        lo.nqv = st->q[nxt];
        lo.nqbase = st->qbase[nxt];
        lo.nqoff = st->qoff[nxt];
        lo.nchunk = st->chunk[nxt];
        lo.level = level;
    }
    __syncthreads();
    const int32_t* __restrict__ pool = st->pool;
    unsigned* bm = st->bitmap;
    const int mode = DO ? st->mode : 0;
    const unsigned gw = blockIdx.x * (kWBlock / 32) + warp;
    const unsigned nwarps = gridDim.x * (kWBlock / 32);
    int found = 0;
    int nlist = 0;

    if (mode == 0) {
        const long long* __restrict__ qbase = st->qbase[cur];
        const unsigned* __restrict__ qoff = st->qoff[cur];
        const int32_t* __restrict__ chunk = st->chunk[cur];
        const unsigned nchunks = (total + kWChunk - 1) >> kChunkShiftWarp;
        // A chunk's window: its first queue entry s0 and its size nw; with
        // at most 32 entries, lane j holds entry s0 + j (start sj, base bj).
        int s0 = 0, nw = 0;
        unsigned sj = 0xFFFFFFFFu;
        long long bj = 0;
        auto load_window = [&](unsigned cc) {
            s0 = 0;
            nw = 0;
            sj = 0xFFFFFFFFu;
            bj = 0;
            if (cc < nchunks) {
                s0 = chunk[cc];
                nw = (cc + 1 < nchunks ? chunk[cc + 1] : nq - 1) - s0 + 1;
                if (nw <= 32 && lane < nw) {
                    sj = qoff[s0 + lane];
                    bj = qbase[s0 + lane] - (long long)sj;
                }
            }
        };
        // the neighbours of chunk cc (window loaded) into v[], lane-strided
        // (-1 past the frontier's end)
        auto load_adj = [&](unsigned cc, int (&v)[kWIpt]) {
#pragma unroll
            for (int k = 0; k < kWIpt; k++) v[k] = -1;
            if (cc >= nchunks) return;
            const unsigned e0 = cc << kChunkShiftWarp;
            const unsigned e1 = e0 + kWChunk < total ? e0 + kWChunk : total;
            if (nw == 1) {
                // one vertex covers the chunk (hubs): no owner search
                const long long b = __shfl_sync(kFull, bj, 0);
#pragma unroll
                for (int k = 0; k < kWIpt; k++) {
                    const unsigned e = e0 + 32u * k + lane;
                    if (e < e1) v[k] = __ldg(pool + b + e);
                }
            } else if (nw <= 32) {
                // the vertex of edge e is the last entry starting at or
                // before e: entries started before the row (ballot) plus
                // starts inside the row up to this lane (OR-reduced bits)
#pragma unroll
                for (int k = 0; k < kWIpt; k++) {
                    const unsigned rs = e0 + 32u * k;
                    const unsigned rel = sj - rs;   // wraps for entries before the row
                    const unsigned bits = __reduce_or_sync(kFull, lane < nw && sj >= rs && rel < 32u
                                                                      ? 1u << rel : 0u);
                    const int before = __popc(__ballot_sync(kFull, lane < nw && sj < rs));
                    const int j = before - 1 + __popc(bits & (kFull >> (31 - lane)));
                    const long long b = __shfl_sync(kFull, bj, j & 31);
                    const unsigned e = rs + lane;
                    if (e < e1) v[k] = __ldg(pool + b + e);
                }
            } else {
                // larger window: staged in the warp's shared memory, one
                // search per lane over 8 consecutive edges
                for (int j = lane; j <= nw; j += 32) {
                    const unsigned so = qoff[s0 + j];   // qoff[nq] is the sealed total
                    sm.start[j] = so;
                    if (j < nw) sm.base[j] = qbase[s0 + j] - (long long)so;
                }
                __syncwarp();
                const unsigned a = e0 + lane * kWIpt;
                int lo2 = 0, hi = nw;                   // last j with start[j] <= a
                while (hi - lo2 > 1) {
                    const int mid = (lo2 + hi) >> 1;
                    if (sm.start[mid] <= a) lo2 = mid; else hi = mid;
                }
                int j = lo2;
#pragma unroll
                for (int k = 0; k < kWIpt; k++) {
                    const unsigned e = a + k;
                    if (e < e1) {
                        while (sm.start[j + 1] <= e) j++;
                        v[k] = __ldg(pool + sm.base[j] + e);
                    }
                }
                __syncwarp();
            }
        };
        // The next chunk's window is read while this chunk's neighbour loads
        // are in flight, so a chunk waits on three round trips (neighbours,
        // bitmap, claims), not five.
        load_window(gw);
        for (unsigned c = gw; c < nchunks; c += nwarps) {
            const unsigned cn = c + nwarps;
            int ns0 = 0, ns1 = -1;
            if (cn < nchunks) {
                ns0 = chunk[cn];
                ns1 = cn + 1 < nchunks ? chunk[cn + 1] : nq - 1;   // inclusive
            }
            int w[kWIpt];
            load_adj(c, w);
            // the next chunk's register window
            s0 = ns0;
            nw = ns1 - ns0 + 1;
            sj = 0xFFFFFFFFu;
            bj = 0;
            if (nw <= 32 && lane < nw) {
                sj = qoff[s0 + lane];
                bj = qbase[s0 + lane] - (long long)sj;
            }
            unsigned word[kWIpt];
#pragma unroll
            for (int k = 0; k < kWIpt; k++)
                word[k] = w[k] >= 0 ? __ldca(bm + (w[k] >> 5)) : 0xFFFFFFFFu;
            unsigned claim = 0;
#pragma unroll
            for (int k = 0; k < kWIpt; k++) {
                if (w[k] >= 0 && !(word[k] & (1u << (w[k] & 31)))) {
                    const unsigned bit = 1u << (w[k] & 31);
                    if (!(atomicOr(bm + (w[k] >> 5), bit) & bit)) claim |= 1u << k;
                }
            }
            warp_claims(sm, nlist, w, claim, lo, found);
        }
    } else {
        // bottom-up over all vertices, 256 per warp, lane-strided
        const VRec* __restrict__ vtab = st->vtab;
        const int32_t* dist = st->dist;
        const int nV = st->nV;
        const unsigned nvc = ((unsigned)nV + kWChunk - 1) >> kChunkShiftWarp;
        for (unsigned c = gw; c < nvc; c += nwarps) {
            int w[kWIpt];
            int dv[kWIpt];
#pragma unroll
            for (int k = 0; k < kWIpt; k++) {
                const long long v = ((long long)c << kChunkShiftWarp) + 32 * k + lane;
                w[k] = v < nV ? (int)v : -1;
                dv[k] = w[k] >= 0 ? __ldcg(dist + v) : 0;
            }
            unsigned claim = 0;
#pragma unroll
            for (int k = 0; k < kWIpt; k++) {
                if (w[k] >= 0 && dv[k] == kInf) {
                    const VRec r = vtab[w[k]];
                    const int32_t* nb = pool + r.off;
                    for (int i = 0; i < r.deg; i++) {
                        if (__ldca(dist + nb[i]) == level - 1) { claim |= 1u << k; break; }
                    }
                    if (claim >> k & 1u) atomicOr(bm + (w[k] >> 5), 1u << (w[k] & 31));
                }
            }
            warp_claims(sm, nlist, w, claim, lo, found);
        }
    }
    if (nlist > 0) warp_flush(sm, nlist, lo, found);
    (void)kFull;
    bfs_level_end<DO>(st, cond, found, level, nq, total, cout, st->qoff[nxt]);
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
            bfs_enqueue(sm, w, claim, level, vtab, dist, cout, nqv, nqbase, nqoff, nchunk,
                        kChunkShiftCta, found);
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
            bfs_enqueue(sm, w, claim, level, vtab, dist, cout, nqv, nqbase, nqoff, nchunk,
                        kChunkShiftCta, found);
        }
    }
    bfs_level_end<DO>(st, cond, found, level, nq, total, cout, nqoff);
}

// The level kernel for bfs.kernel = `kernel` (top-down or direction-
// optimising).  The warp kernel is compiled for 3, 4 and 5 resident CTAs per
// SM (80, 64 and 48 registers); `per_sm` (bfs.warp_ctas_per_sm) picks the
// build that lets that many CTAs reside.
void* level_kernel(int kernel, bool dir_opt, int per_sm) {
    if (kernel) {
        if (per_sm >= 5)
            return dir_opt ? (void*)k_bfs_wlevel<true, 5> : (void*)k_bfs_wlevel<false, 5>;
        if (per_sm == 4)
            return dir_opt ? (void*)k_bfs_wlevel<true, 4> : (void*)k_bfs_wlevel<false, 4>;
        return dir_opt ? (void*)k_bfs_wlevel<true, 3> : (void*)k_bfs_wlevel<false, 3>;
    }
    return dir_opt ? (void*)k_bfs_level<true> : (void*)k_bfs_level<false>;
}

const char* level_kernel_name(int kernel, bool dir_opt) {
    if (kernel) return dir_opt ? "k_bfs_wlevel<true>" : "k_bfs_wlevel<false>";
    return dir_opt ? "k_bfs_level<true>" : "k_bfs_level<false>";
}

void build_bfs_graph(hn_graph* g, BfsGraph& bg) {
    const int nV = g->nV;
    // the finer of the two granularities, with room for the graph to grow
    // by a quarter before the table (and the CUDA graph) is rebuilt
    const long long nchunk_cap = (g->nE + g->nE / 4) / kWChunk + 1024;
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
            p.func = level_kernel(bg.kernel, variant != 0, bg.per_sm);
            p.gridDim = dim3(bg.grid);
            p.blockDim = dim3(bg.kernel ? kWBlock : kBfsBlock);
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
    // chunk table or a knob changes the level kernel or its grid
    const int kernel = (int)knob(kKnobBfsKernel);
    const int per_sm = (int)knob(kernel ? kKnobBfsWarpCtasPerSm : kKnobBfsCtasPerSm);
    const unsigned grid = (unsigned)(g->info.sms * per_sm);
    if (g->bfs && (g->bfs->nV != g->nV || g->nE / kWChunk + 4 > g->bfs->nchunk_cap ||
                   g->bfs->grid != grid || g->bfs->kernel != kernel)) {
        HN_CUDA(cudaStreamSynchronize(g->stream));
        free_bfs_graph(g->bfs);
        g->bfs = nullptr;
    }
    if (!g->bfs) {
        g->bfs = new BfsGraph();
        g->bfs->grid = grid;
        g->bfs->kernel = kernel;
        g->bfs->per_sm = per_sm;
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
    // edge offsets are 32-bit, and a chunk's end (offset + 256) must not wrap
    if (g->nE > 0xFFFFFE00ll) throw Error(HN_ERR_CAPACITY, "BFS needs nE < 2^32 - 512");
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
        h.cshift = bg.kernel ? kChunkShiftWarp : kChunkShiftCta;
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
                cudaGraphConditionalHandle none = 0;
                void* args[] = {&bg.state, &none};
                HN_CUDA(cudaLaunchKernel(level_kernel(bg.kernel, direction_optimizing, bg.per_sm),
                                         dim3(bg.grid), dim3(bg.kernel ? kWBlock : kBfsBlock),
                                         args, 0, s));
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
        if (ev0) profile_end(level_kernel_name(bg.kernel, direction_optimizing), s, ev0);
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
    if (k > 0) {
        bg.last = snap[k - 1];
        bg.have_last = true;
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
    HandleUse use(g);
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
    HandleUse use(g);
    HN_CUDA(cudaSetDevice(g->device));
    bfs_run(g, sources, k, dist, mem, stats, false);
    HN_API_END
}

int hn_bfs_level_trace(hn_graph_t* g, int32_t max_levels, double* us, int64_t* edges,
                       int32_t* n_levels) {
    HN_API_BEGIN
    HN_REQUIRE(g && n_levels && max_levels >= 0, "null argument");
    *n_levels = 0;
    if (!g->bfs || !g->bfs->h_ring || !g->bfs->have_last) return HN_OK;
    const BfsState& t = g->bfs->last;
    const int lv = t.level - 1 < kTraceLevels ? t.level - 1 : kTraceLevels;
    const int n = lv < max_levels ? lv : max_levels;
    unsigned long long prev = t.t_start;
    for (int i = 0; i < n; i++) {
        if (us) us[i] = (double)(t.t_end[i] - prev) / 1e3;
        if (edges) edges[i] = (int64_t)t.lvl_edges[i];
        prev = t.t_end[i];
    }
    *n_levels = n;
    HN_API_END
}

int hn_bfs_do(hn_graph_t* g, const int32_t* sources, int32_t k, int32_t* dist, int mem,
              hn_bfs_stats_t* stats) {
    HN_API_BEGIN
    HN_REQUIRE(g && sources && dist, "null argument");
    HN_REQUIRE(k >= 0, "negative source count");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    HN_REQUIRE(g->nV > 0 || k == 0, "empty graph");
    HandleUse use(g);
    HN_CUDA(cudaSetDevice(g->device));
    bfs_run(g, sources, k, dist, mem, stats, true);
    HN_API_END
}

}  // extern "C"
