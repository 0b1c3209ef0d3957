// Batched BFS: up to 64 BFS "slots" in one traversal (bit-parallel
// multi-source BFS after Then et al., "The More the Merrier: Efficient
// Multi-Source Graph Traversal", VLDB 2015).
//
// Batching: many BFS sources (and, on a disjoint union, many small graphs)
// in one persistent launch captured in a CUDA graph.  Each vertex carries three 64-bit masks:
//   seen[v]  slots that have reached v,
//   front[v] slots for which v is on the current frontier,
//   nxt[v]   slots that reach v at this level (OR-accumulated).
// One level is two kernels inside the graph's WHILE body:
//   push:  the frontier's edges (u, v), load-balanced in chunks exactly as
//          the single-source top-down kernel does, OR front[u] & ~seen[v]
//          into nxt[v]; the first writer of nxt[v] records v as touched;
//   apply: every touched v takes its new bits, writes dist[slot][v] = level
//          for each, and joins the next frontier once (whatever the number
//          of slots) with its edge offset from one packed atomic per CTA.
// An edge is read once per level for ALL slots on it, so a 64-source batch
// reads each vertex's adjacency about as many times as there are distinct
// distances to it, instead of 64 times.  Distances per slot equal a
// single-source BFS from that slot's source; slots shared by several sources
// give the distance to the nearest of them, which is each source's own
// distance when they sit in different components (a disjoint union of
// graphs, one source per graph per slot).
#include "hn_graph.cuh"

namespace hn {

constexpr int kSeedBlock = 256;       // the single seeding CTA
constexpr int kMsChunk = 2048;        // edges per chunk (block x items per thread)
constexpr int kMaxSlots = 64;

struct MsState {
    unsigned long long cnt[3];      // frontier counters: (edge total << 32) | size
    unsigned long long tcnt;        // touched vertices this level
    int level;
    unsigned ticket;
    int nV;
    int nslots;
    const VRec* vtab;
    const int32_t* pool;
    int32_t* q[2];
    long long* qbase[2];
    unsigned* qoff[2];
    int32_t* chunk[2];
    unsigned long long* seen;
    unsigned long long* front[2];
    unsigned long long* nxt;
    int32_t* touched;
    int32_t* dist;                  // nslots x nV, slot-major
    const int32_t* src;
    const int32_t* slot;
    int nsrc;
    int mode;                       // 0 top-down (push + apply), 1 bottom-up (apply scans)
    unsigned long long* stat;       // [3*kMaxSlots]: visited, scanned, last level per slot
    int prev_nq;                    // size of the previous frontier (its fronts are cleared)
    int bottom_up;                  // bottom-up levels allowed
    int alpha, beta;                // direction switch thresholds
    long long m_total;              // edges of the graph
    unsigned long long all_mask;    // slots that hold at least one source
};

struct MsGraph {
    int nV = -1;
    long long nchunk_cap = 0;
    MsState* state = nullptr;
    MsState* h_state = nullptr;
    int32_t* qbuf = nullptr;
    long long* qbasebuf = nullptr;
    unsigned* qoffbuf = nullptr;
    int32_t* chunkbuf = nullptr;
    unsigned long long* masks = nullptr;   // seen, front0, front1, nxt
    int32_t* touched = nullptr;
    unsigned long long* stat = nullptr;
    unsigned long long* h_stat = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int block = 256;      // msbfs.block knob baked into the graph
    unsigned grid = 0;    // msbfs.ctas_per_sm x SMs
};

namespace {

__device__ __forceinline__ void ms_mark_chunks(int32_t* chunk, unsigned off, unsigned d, int pos) {
    unsigned c0 = (off + kMsChunk - 1) / kMsChunk;
    unsigned c1 = (off + d - 1) / kMsChunk;
    for (unsigned c = c0; c <= c1; c++) chunk[c] = pos;
}

// CTA-wide exclusive scan of a packed (degree << 32 | count) value and one
// atomic on `counter`; returns this thread's (slot, edge offset) base.
// Must be called by all threads of a BLOCK-thread CTA.
template <int BLOCK>
__device__ __forceinline__ unsigned long long ms_cta_reserve(unsigned long long mine,
                                                             unsigned long long* counter,
                                                             unsigned long long* s_wsum,
                                                             unsigned long long* s_base) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long x = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += x;
    }
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned long long v = threadIdx.x < BLOCK / 32 ? s_wsum[threadIdx.x] : 0ull;
        unsigned long long vi = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long x = __shfl_up_sync(0xFFFFFFFFu, vi, o);
            if (lane >= o) vi += x;
        }
        if (threadIdx.x < BLOCK / 32) s_wsum[threadIdx.x] = vi - v;
        unsigned long long tot = __shfl_sync(0xFFFFFFFFu, vi, 31);
        if (threadIdx.x == 0) *s_base = tot ? atomicAdd(counter, tot) : 0ull;
    }
    __syncthreads();
    unsigned long long r = *s_base + s_wsum[warp] + (incl - mine);
    __syncthreads();   // s_wsum / s_base are reused by the next call
    return r;
}

__global__ void k_ms_fill(MsState* st) {
    const long long n = st->nV;
    const long long nd = n * st->nslots;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nd;
         i += (long long)gridDim.x * blockDim.x) {
        st->dist[i] = kInf;
        if (i < n) {
            st->seen[i] = 0;
            st->front[0][i] = 0;
            st->front[1][i] = 0;
            st->nxt[i] = 0;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x < 3 * kMaxSlots) st->stat[threadIdx.x] = 0;
}

// one CTA: seed every source, build the first frontier
__global__ void __launch_bounds__(kSeedBlock) k_ms_seed(MsState* st) {
    __shared__ unsigned long long s_wsum[kSeedBlock / 32];
    __shared__ unsigned long long s_base;
    __shared__ unsigned long long s_stat[2 * kMaxSlots];
    for (int i = threadIdx.x; i < 2 * kMaxSlots; i += kSeedBlock) s_stat[i] = 0;
    if (threadIdx.x == 0) {
        st->cnt[0] = 0;
        st->cnt[1] = 0;
        st->cnt[2] = 0;
        st->tcnt = 0;
        st->level = 1;
        st->ticket = 0;
    }
    __syncthreads();
    const int nV = st->nV;
    for (int j0 = 0; j0 < st->nsrc; j0 += kSeedBlock) {
        int j = j0 + threadIdx.x;
        bool first = false;
        int v = 0;
        VRec r;
        r.deg = 0;
        r.off = 0;
        if (j < st->nsrc) {
            v = st->src[j];
            int b = st->slot ? st->slot[j] : j;
            unsigned long long bit = 1ull << b;
            atomicOr(&st->all_mask, bit);
            unsigned long long old = atomicOr(st->front[0] + v, bit);
            unsigned long long olds = atomicOr(st->seen + v, bit);
            first = old == 0;
            r = st->vtab[v];
            if (!(olds & bit)) {
                st->dist[(long long)b * nV + v] = 0;
                atomicAdd(&s_stat[b], 1ull);
                atomicAdd(&s_stat[kMaxSlots + b], (unsigned long long)r.deg);
            }
        }
        bool q = first && r.deg > 0;
        unsigned long long mine = q ? (((unsigned long long)r.deg << 32) | 1ull) : 0ull;
        unsigned long long at = ms_cta_reserve<kSeedBlock>(mine, &st->cnt[0], s_wsum, &s_base);
        if (q) {
            int pos = (int)(at & 0xFFFFFFFFull);
            unsigned off = (unsigned)(at >> 32);
            st->q[0][pos] = v;
            st->qbase[0][pos] = r.off;
            st->qoff[0][pos] = off;
            ms_mark_chunks(st->chunk[0], off, (unsigned)r.deg, pos);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long c = st->cnt[0];
        st->qoff[0][c & 0xFFFFFFFFull] = (unsigned)(c >> 32);
    }
    for (int i = threadIdx.x; i < 2 * kMaxSlots; i += kSeedBlock)
        if (s_stat[i]) atomicAdd(st->stat + i, s_stat[i]);
}

// push: OR frontier masks along the frontier's edges
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK) k_ms_push(MsState* st) {
    constexpr int IPT = kMsChunk / BLOCK;
    __shared__ unsigned s_start[kMsChunk + 2];
    __shared__ long long s_base[kMsChunk + 1];
    __shared__ unsigned long long s_front[kMsChunk + 1];
    __shared__ int s_nw;
    __shared__ unsigned long long s_wsum[BLOCK / 32];
    __shared__ unsigned long long s_cb;
    const int it = st->level - 1;
    const unsigned long long cin = st->cnt[it % 3];
    if (blockIdx.x == 0 && threadIdx.x == 0) st->cnt[(it + 2) % 3] = 0;
    const int nq = (int)(cin & 0xFFFFFFFFull);
    const unsigned total = (unsigned)(cin >> 32);
    const int cur = it & 1;
    {
        // the previous frontier's masks are spent: its buffer is the one this
        // level's apply writes, and bottom-up levels read every vertex's mask
        const int pn = st->prev_nq;
        const int32_t* pq = st->q[cur ^ 1];
        unsigned long long* pf = st->front[cur ^ 1];
        for (long long i = blockIdx.x * (long long)BLOCK + threadIdx.x; i < pn;
             i += (long long)gridDim.x * BLOCK)
            pf[pq[i]] = 0ull;
    }
    if (st->mode == 1) return;   // bottom-up level: apply does the work
    const int32_t* q = st->q[cur];
    const long long* qbase = st->qbase[cur];
    const unsigned* qoff = st->qoff[cur];
    const int32_t* chunk = st->chunk[cur];
    const unsigned long long* front = st->front[cur];
    const unsigned long long* seen = st->seen;
    unsigned long long* nxt = st->nxt;
    const int32_t* pool = st->pool;
    const unsigned nchunks = (total + kMsChunk - 1) / kMsChunk;
    for (unsigned c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const unsigned e0 = c * kMsChunk;
        const unsigned e1 = e0 + kMsChunk < total ? e0 + kMsChunk : total;
        const int s0 = chunk[c];
        const int s1 = c + 1 < nchunks ? chunk[c + 1] : nq - 1;
        const int nw = s1 - s0 + 1;
        for (int j = threadIdx.x; j <= nw; j += BLOCK) {
            int s = s0 + j;
            unsigned so = qoff[s];
            s_start[j] = so;
            if (j < nw) {
                s_base[j] = qbase[s] - (long long)so;
                s_front[j] = front[q[s]];
            }
        }
        if (threadIdx.x == 0) s_nw = nw;
        __syncthreads();
        const unsigned a = e0 + threadIdx.x * IPT;
        const unsigned b = a + IPT < e1 ? a + IPT : e1;
        int touched_here[IPT];
        int nt = 0;
        if (a < b) {
            int lo = 0, hi = s_nw;
            while (hi - lo > 1) {
                int mid = (lo + hi) >> 1;
                if (s_start[mid] <= a) lo = mid; else hi = mid;
            }
            int j = lo;
            int w[IPT];
            unsigned long long fm[IPT];
#pragma unroll
            for (int k = 0; k < IPT; k++) {
                unsigned e = a + k;
                w[k] = -1;
                fm[k] = 0;
                if (e < b) {
                    while (s_start[j + 1] <= e) j++;
                    w[k] = __ldg(pool + s_base[j] + e);
                    fm[k] = s_front[j];
                }
            }
            unsigned long long sv[IPT];
#pragma unroll
            for (int k = 0; k < IPT; k++) sv[k] = w[k] >= 0 ? __ldca(seen + w[k]) : ~0ull;
#pragma unroll
            for (int k = 0; k < IPT; k++) {
                unsigned long long m = fm[k] & ~sv[k];
                if (m) {
                    unsigned long long old = atomicOr(nxt + w[k], m);
                    if (old == 0) touched_here[nt++] = w[k];
                }
            }
        }
        // nothing newly touched in the whole chunk (common late in the
        // traversal): skip the scan; the barrier still guards the window
        if (__syncthreads_or(nt > 0)) {
            unsigned long long at =
                ms_cta_reserve<BLOCK>((unsigned long long)nt, &st->tcnt, s_wsum, &s_cb);
            int pos = (int)at;
            for (int k = 0; k < nt; k++) st->touched[pos + k] = touched_here[k];
        }
    }
}

// apply: new bits of every touched vertex; next frontier; clear the old one
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_ms_apply(MsState* st, cudaGraphConditionalHandle cond) {
    __shared__ unsigned long long s_wsum[BLOCK / 32];
    __shared__ unsigned long long s_cb;
    __shared__ unsigned long long s_stat[2 * kMaxSlots];
    __shared__ int s_last[kMaxSlots];   // written only with this level's number
    for (int i = threadIdx.x; i < 2 * kMaxSlots; i += BLOCK) s_stat[i] = 0;
    for (int i = threadIdx.x; i < kMaxSlots; i += BLOCK) s_last[i] = 0;
    __syncthreads();
    const int level = st->level;
    const int it = level - 1;
    const int nx = (it & 1) ^ 1;
    unsigned long long* cout = &st->cnt[(it + 1) % 3];
    const long long nt = (long long)st->tcnt;
    const int nV = st->nV;
    const VRec* vtab = st->vtab;
    unsigned long long* seen = st->seen;
    unsigned long long* nxt = st->nxt;
    unsigned long long* nfront = st->front[nx];
    const long long stride = (long long)gridDim.x * blockDim.x;
    const bool bu = st->mode == 1;
    const unsigned long long* cfront = st->front[nx ^ 1];
    const unsigned long long all = st->all_mask;
    const int nq_in = (int)(st->cnt[it % 3] & 0xFFFFFFFFull);
    const long long n_items = bu ? (long long)nV : nt;
    for (long long i0 = blockIdx.x * (long long)blockDim.x; i0 < n_items; i0 += stride) {
        long long i = i0 + threadIdx.x;
        bool q = false;
        int v = 0;
        VRec r;
        r.deg = 0;
        r.off = 0;
        unsigned long long nw = 0;
        if (bu && i < n_items) {
            // bottom-up: v takes, for every slot it still misses, the first
            // neighbour on that slot's frontier; stops once nothing is missing
            v = (int)i;
            unsigned long long todo = all & ~seen[v];
            if (todo) {
                r = vtab[v];
                const int32_t* nb = st->pool + r.off;
                for (int e = 0; e < r.deg && todo; e++) {
                    const unsigned long long m = cfront[__ldg(nb + e)] & todo;
                    nw |= m;
                    todo &= ~m;
                }
                if (nw) {
                    seen[v] |= nw;
                    nfront[v] = nw;
                }
            }
        } else if (!bu && i < nt) {
            v = st->touched[i];
            unsigned long long x = nxt[v];
            nxt[v] = 0;
            nw = x & ~seen[v];
            seen[v] |= nw;
            nfront[v] = nw;
            r = vtab[v];
        }
        if (nw) {
            while (nw) {
                int bb = __ffsll((long long)nw) - 1;
                nw &= nw - 1;
                st->dist[(long long)bb * nV + v] = level;
                atomicAdd(&s_stat[bb], 1ull);
                atomicAdd(&s_stat[kMaxSlots + bb], (unsigned long long)r.deg);
                s_last[bb] = level;
            }
            q = r.deg > 0;
        }
        unsigned long long mine = q ? (((unsigned long long)r.deg << 32) | 1ull) : 0ull;
        unsigned long long at = ms_cta_reserve<BLOCK>(mine, cout, s_wsum, &s_cb);
        if (q) {
            int pos = (int)(at & 0xFFFFFFFFull);
            unsigned off = (unsigned)(at >> 32);
            st->q[nx][pos] = v;
            st->qbase[nx][pos] = r.off;
            st->qoff[nx][pos] = off;
            ms_mark_chunks(st->chunk[nx], off, (unsigned)r.deg, pos);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * kMaxSlots; i += BLOCK)
        if (s_stat[i]) atomicAdd(st->stat + i, s_stat[i]);
    for (int i = threadIdx.x; i < kMaxSlots; i += BLOCK)
        if (s_last[i]) st->stat[2 * kMaxSlots + i] = (unsigned long long)level;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned tk = atomicAdd(&st->ticket, 1u);
        if (tk == gridDim.x - 1) {
            __threadfence();
            unsigned long long c = atomicAdd(cout, 0ull);
            unsigned nn = (unsigned)(c & 0xFFFFFFFFull);
            st->qoff[nx][nn] = (unsigned)(c >> 32);
            st->ticket = 0;
            st->tcnt = 0;
            st->level = level + 1;
            st->prev_nq = nq_in;
            if (st->bottom_up) {
                // bottom-up while the next frontier's edges exceed m/alpha;
                // back to top-down once it holds fewer than nV/beta vertices
                const long long mf = (long long)(c >> 32);
                if (st->mode == 0) {
                    if (mf * st->alpha > st->m_total) st->mode = 1;
                } else if ((long long)nn * st->beta < nV) {
                    st->mode = 0;
                }
            }
            cudaGraphSetConditional(cond, (nn > 0 && level < nV) ? 1u : 0u);
        }
    }
}

void build_ms_graph(hn_graph* g, MsGraph& mg) {
    const int nV = g->nV;
    // room for the graph to grow by a quarter before a rebuild
    const long long nchunk_cap = (g->nE + g->nE / 4) / kMsChunk + 1024;
    HN_CUDA(cudaMalloc((void**)&mg.state, sizeof(MsState)));
    HN_CUDA(cudaMallocHost((void**)&mg.h_state, sizeof(MsState)));
    HN_CUDA(cudaMalloc((void**)&mg.qbuf, sizeof(int32_t) * 2 * ((size_t)nV + 1)));
    HN_CUDA(cudaMalloc((void**)&mg.qbasebuf, sizeof(long long) * 2 * ((size_t)nV + 1)));
    HN_CUDA(cudaMalloc((void**)&mg.qoffbuf, sizeof(unsigned) * 2 * ((size_t)nV + 2)));
    HN_CUDA(cudaMalloc((void**)&mg.chunkbuf, sizeof(int32_t) * 2 * (size_t)nchunk_cap));
    HN_CUDA(cudaMalloc((void**)&mg.masks, sizeof(unsigned long long) * 4 * (size_t)nV));
    HN_CUDA(cudaMalloc((void**)&mg.touched, sizeof(int32_t) * ((size_t)nV + 1)));
    HN_CUDA(cudaMalloc((void**)&mg.stat, sizeof(unsigned long long) * 3 * kMaxSlots));
    HN_CUDA(cudaMallocHost((void**)&mg.h_stat, sizeof(unsigned long long) * 3 * kMaxSlots));
    mg.nV = nV;
    mg.nchunk_cap = nchunk_cap;

    HN_CUDA(cudaGraphCreate(&mg.graph, 0));
    cudaGraphNode_t fill, seed, condn, push, apply;
    {
        void* args[] = {&mg.state};
        cudaKernelNodeParams p = {};
        p.func = (void*)k_ms_fill;
        p.gridDim = dim3((unsigned)g->info.sms * 8);
        p.blockDim = dim3(256);
        p.kernelParams = args;
        HN_CUDA(cudaGraphAddKernelNode(&fill, mg.graph, nullptr, 0, &p));
        p.func = (void*)k_ms_seed;
        p.gridDim = dim3(1);
        p.blockDim = dim3(kSeedBlock);
        HN_CUDA(cudaGraphAddKernelNode(&seed, mg.graph, &fill, 1, &p));
    }
    cudaGraphConditionalHandle handle;
    HN_CUDA(cudaGraphConditionalHandleCreate(&handle, mg.graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    HN_CUDA(cudaGraphAddNode(&condn, mg.graph, &seed, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    {
        void* args[] = {&mg.state};
        cudaKernelNodeParams p = {};
        p.func = mg.block == 128 ? (void*)k_ms_push<128>
               : mg.block == 512 ? (void*)k_ms_push<512> : (void*)k_ms_push<256>;
        p.gridDim = dim3(mg.grid);
        p.blockDim = dim3(mg.block);
        p.kernelParams = args;
        HN_CUDA(cudaGraphAddKernelNode(&push, body, nullptr, 0, &p));
        void* args2[] = {&mg.state, &handle};
        p.func = mg.block == 128 ? (void*)k_ms_apply<128>
               : mg.block == 512 ? (void*)k_ms_apply<512> : (void*)k_ms_apply<256>;
        p.gridDim = dim3(mg.grid);
        p.kernelParams = args2;
        HN_CUDA(cudaGraphAddKernelNode(&apply, body, &push, 1, &p));
    }
    HN_CUDA(cudaGraphInstantiate(&mg.exec, mg.graph, 0));
}

}  // namespace

void free_ms_graph(MsGraph* mg) {
    if (!mg) return;
    if (mg->exec) cudaGraphExecDestroy(mg->exec);
    if (mg->graph) cudaGraphDestroy(mg->graph);
    if (mg->state) cudaFree(mg->state);
    if (mg->h_state) cudaFreeHost(mg->h_state);
    if (mg->qbuf) cudaFree(mg->qbuf);
    if (mg->qbasebuf) cudaFree(mg->qbasebuf);
    if (mg->qoffbuf) cudaFree(mg->qoffbuf);
    if (mg->chunkbuf) cudaFree(mg->chunkbuf);
    if (mg->masks) cudaFree(mg->masks);
    if (mg->touched) cudaFree(mg->touched);
    if (mg->stat) cudaFree(mg->stat);
    if (mg->h_stat) cudaFreeHost(mg->h_stat);
    delete mg;
}

}  // namespace hn

using namespace hn;

extern "C" int hn_bfs_batch(hn_graph_t* g, const int32_t* sources, const int32_t* slots,
                            int32_t k, int32_t nslots, int32_t* dist, int mem,
                            hn_bfs_stats_t* slot_stats) {
    HN_API_BEGIN
    HN_REQUIRE(g && dist && (sources || k == 0), "null argument");
    HN_REQUIRE(nslots >= 1 && nslots <= kMaxSlots, "nslots must be in [1, 64]");
    HN_REQUIRE(k >= 0, "negative source count");
    HN_REQUIRE(slots || k <= nslots, "without slots, source j uses slot j (k <= nslots)");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    HN_REQUIRE(g->nV > 0, "empty graph");
    HN_REQUIRE(g->nE < 0xFFFFFFFFll, "batched BFS needs nE < 2^32");
    HandleUse use(g);
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    const int nV = g->nV;
    for (int j = 0; j < k; j++) {
        if (sources[j] < 0 || sources[j] >= nV) throw Error(HN_ERR_INVALID, "source outside [0, nV)");
        if (slots && (slots[j] < 0 || slots[j] >= nslots))
            throw Error(HN_ERR_INVALID, "slot outside [0, nslots)");
    }
    const int block = (int)knob(kKnobMsBlock);
    const unsigned grid = (unsigned)(g->info.sms * knob(kKnobMsCtasPerSm));
    if (g->ms && (g->ms->nV != nV || g->nE / kMsChunk + 4 > g->ms->nchunk_cap ||
                  g->ms->block != block || g->ms->grid != grid)) {
        HN_CUDA(cudaStreamSynchronize(s));
        free_ms_graph(g->ms);
        g->ms = nullptr;
    }
    if (!g->ms) {
        g->ms = new MsGraph();
        g->ms->block = block;
        g->ms->grid = grid;
        try {
            build_ms_graph(g, *g->ms);
        } catch (...) {
            free_ms_graph(g->ms);
            g->ms = nullptr;
            throw;
        }
    }
    MsGraph& mg = *g->ms;
    DevBuf<int32_t> d_src((size_t)k + 1, s), d_slot((size_t)k + 1, s), d_dist;
    if (k) {
        HN_CUDA(cudaMemcpyAsync(d_src.get(), sources, sizeof(int32_t) * k, cudaMemcpyHostToDevice, s));
        if (slots)
            HN_CUDA(cudaMemcpyAsync(d_slot.get(), slots, sizeof(int32_t) * k,
                                    cudaMemcpyHostToDevice, s));
    }
    int32_t* out = dist;
    if (mem == HN_MEM_HOST) {
        d_dist.alloc((size_t)nslots * nV, s);
        out = d_dist.get();
    }
    HN_CUDA(cudaStreamSynchronize(s));
    MsState& h = *mg.h_state;
    h = MsState{};
    h.nV = nV;
    h.nslots = nslots;
    h.vtab = g->vtab;
    h.pool = g->pool;
    h.q[0] = mg.qbuf;
    h.q[1] = mg.qbuf + nV + 1;
    h.qbase[0] = mg.qbasebuf;
    h.qbase[1] = mg.qbasebuf + nV + 1;
    h.qoff[0] = mg.qoffbuf;
    h.qoff[1] = mg.qoffbuf + nV + 2;
    h.chunk[0] = mg.chunkbuf;
    h.chunk[1] = mg.chunkbuf + mg.nchunk_cap;
    h.seen = mg.masks;
    h.front[0] = mg.masks + nV;
    h.front[1] = mg.masks + 2 * (size_t)nV;
    h.nxt = mg.masks + 3 * (size_t)nV;
    h.touched = mg.touched;
    h.dist = out;
    h.src = d_src.get();
    h.slot = slots ? d_slot.get() : nullptr;
    h.nsrc = k;
    h.stat = mg.stat;
    h.bottom_up = (int)knob(kKnobMsBottomUp);
    h.alpha = (int)knob(kKnobBfsDoAlpha);
    h.beta = (int)knob(kKnobBfsDoBeta);
    h.m_total = g->nE;
    HN_CUDA(cudaMemcpyAsync(mg.state, &h, sizeof(MsState), cudaMemcpyHostToDevice, s));
    cudaEvent_t ev0 = nullptr;
    if (g_profiling) profile_begin(s, &ev0);
    HN_CUDA(cudaGraphLaunch(mg.exec, s));
    if (ev0) profile_end("k_ms_push+apply", s, ev0);
    count_launch(3);
    HN_CUDA(cudaMemcpyAsync(mg.h_stat, mg.stat, sizeof(unsigned long long) * 3 * kMaxSlots,
                            cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaMemcpyAsync(mg.h_state, mg.state, sizeof(MsState), cudaMemcpyDeviceToHost, s));
    if (mem == HN_MEM_HOST)
        HN_CUDA(cudaMemcpyAsync(dist, out, sizeof(int32_t) * (size_t)nslots * nV,
                                cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    if (slot_stats)
        for (int b = 0; b < nslots; b++) {
            slot_stats[b].levels =
                mg.h_stat[b] ? (int32_t)mg.h_stat[2 * kMaxSlots + b] + 1 : 0;
            slot_stats[b].pad = 0;
            slot_stats[b].visited = (int64_t)mg.h_stat[b];
            slot_stats[b].edges_scanned = (int64_t)mg.h_stat[kMaxSlots + b];
        }
    HN_API_END
}
