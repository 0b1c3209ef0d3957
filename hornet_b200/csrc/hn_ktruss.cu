// k-truss (hornetsnest/src/Static/KTruss/KTruss.cu:90-174,
// KTrussSupport.cu:375-468, KTrussOperators.cuh:16-38).
//
// Reference semantics: max_K starts at 3; findTrussOfK repeatedly
// recomputes every edge's support (triangles through it) from scratch and
// deletes all edges with support < max_K - 2 through a BatchUpdate erase,
// until a pass deletes nothing; if no edge is left max_K-- and stop,
// otherwise max_K++ on the peeled graph.  (The reference k-truss does not
// compile against the current core; the definition is what is kept.)
//
// Here the supports are computed once and then maintained incrementally:
// a round deletes the current frontier F (edges with support < K-2) and,
// for every triangle (e, e1, e2) of a frontier edge e whose other two edges
// are still alive, decrements the supports it destroys exactly once — if
// neither e1 nor e2 is in F both lose one; if exactly one of them is in F
// the remaining edge loses one, charged to the smaller of the two frontier
// edges; if both are in F nothing remains to update.  An edge whose support
// crosses from K-2 to K-3 joins the next frontier.  After the rounds the
// supports equal the from-scratch supports of the peeled graph, so the
// surviving edge sets, truss numbers and max_K are those of the reference
// loop.  Edge ids are positions in the sorted CSR; undirected edge state
// lives on the (u < v) position.
#include <optional>

#include <algorithm>
#include <climits>

#include "hn_graph.cuh"
#include "hn_tc.cuh"

namespace hn {
namespace {

constexpr int kB = 256;

// Device state of the peel rounds.  Every kernel of a round reads its
// arrays and counts from here, so one instantiated CUDA graph (a WHILE node
// around the round's kernels) serves every round of every K: the frontier
// buffers swap, the lists shrink and K advances on the device or between
// graph launches, never as baked-in kernel arguments.
struct KtPeel {
    const long long* off;     // current adjacency lists (rebuilt as edges die)
    const int32_t* adj;
    const int32_t* canon;
    int32_t* F;               // this round's frontier (canonical edge ids)
    int32_t* NF;              // the next round's frontier
    int nf;                   // |F|
    int nNF;                  // |NF| (appended atomically)
    int nheavy;               // frontier edges left to the heavy kernel
    int K;
    long long remaining;      // alive edges
    long long rounds;         // peel rounds run
};

__global__ void k_kt_src(const long long* __restrict__ off, int nV, int32_t* __restrict__ src) {
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < nV;
         u += (long long)gridDim.x * blockDim.x)
        for (long long e = off[u]; e < off[u + 1]; e++) src[e] = (int)u;
}

// canonical (u < v) position of every directed edge; checks simplicity and
// symmetry.
__global__ void k_kt_canon(const long long* __restrict__ off, const int32_t* __restrict__ adj,
                           const int32_t* __restrict__ src, long long m,
                           int32_t* __restrict__ canon, int* __restrict__ err) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m;
         e += (long long)gridDim.x * blockDim.x) {
        int u = src[e], v = adj[e];
        bool bad = (u == v) || (e > off[u] && adj[e - 1] == v);
        long long c = e;
        if (u > v) {
            long long p = off[v] + lower_bound_dev(adj + off[v], off[v + 1] - off[v], u);
            if (p >= off[v + 1] || adj[p] != u) bad = true;
            c = p;
        }
        canon[e] = (int)c;
        if (bad) atomicExch(err, 1);
    }
}

// Canonical edges (u < v) start alive (their supports come from the
// triangle enumeration: every triangle, found once, credits its three edges).
__global__ void k_kt_init(const int32_t* __restrict__ adj, const int32_t* __restrict__ src,
                          long long m, unsigned char* __restrict__ alive,
                          int* __restrict__ nalive) {
    int mine = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m;
         e += (long long)gridDim.x * blockDim.x) {
        const bool canon = src[e] < adj[e];
        alive[e] = canon ? 1 : 0;
        mine += canon ? 1 : 0;
    }
    for (int o = 16; o; o >>= 1) mine += __shfl_down_sync(0xFFFFFFFFu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(nalive, mine);
}

// Positions of the current lists whose (canonical) edge is still alive.
__global__ void k_kt_live_pos(const int32_t* __restrict__ canon, long long n,
                              const unsigned char* __restrict__ alive,
                              int32_t* __restrict__ flag) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x)
        flag[p] = alive[canon[p]] ? 1 : 0;
}

// List shrinking: a vertex's new offset is the new slot of its first old
// entry (noff[v] = pos[off[v]], v = 0..nV), and every live entry moves to
// its new slot, in order.
__global__ void k_kt_shrink_off(const long long* __restrict__ off, int nV,
                                const long long* __restrict__ pos, long long* __restrict__ noff) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v <= nV;
         v += (long long)gridDim.x * blockDim.x)
        noff[v] = pos[off[v]];
}

__global__ void k_kt_shrink_copy(const int32_t* __restrict__ adj, const int32_t* __restrict__ canon,
                                 const int32_t* __restrict__ flag, const long long* __restrict__ pos,
                                 long long m, int32_t* __restrict__ nadj,
                                 int32_t* __restrict__ ncanon) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
         i += (long long)gridDim.x * blockDim.x)
        if (flag[i]) {
            nadj[pos[i]] = adj[i];
            ncanon[pos[i]] = canon[i];
        }
}

// Frontier of round K: alive edges of the list L with support < K - 2.
__global__ void k_kt_frontier(const int32_t* __restrict__ L, int nL,
                              const int32_t* __restrict__ sup,
                              const unsigned char* __restrict__ alive,
                              unsigned char* __restrict__ inF, KtPeel* st) {
    const int K = st->K;
    int32_t* F = st->F;
    int* nF = &st->nf;
    for (long long i0 = blockIdx.x * (long long)blockDim.x; i0 < nL;
         i0 += (long long)gridDim.x * blockDim.x) {
        long long i = i0 + threadIdx.x;
        int e = i < nL ? L[i] : 0;
        bool take = i < nL && alive[e] && sup[e] < K - 2;
        int p = warp_append(nF, take);
        if (take) {
            F[p] = e;
            inF[e] = 1;
        }
    }
}

// Alive-edge list: from all canonical edges (L == nullptr, n = m) or from
// the previous list, dropping peeled edges; *minsup receives the smallest
// support left, so the next round can start at the first K that peels.
__global__ void k_kt_compact(const int32_t* __restrict__ L, long long n,
                             const unsigned char* __restrict__ alive,
                             const int32_t* __restrict__ sup, int32_t* __restrict__ out,
                             int* __restrict__ nout, int* __restrict__ minsup) {
    int mn = 0x7FFFFFFF;
    for (long long i0 = blockIdx.x * (long long)blockDim.x; i0 < n;
         i0 += (long long)gridDim.x * blockDim.x) {
        long long i = i0 + threadIdx.x;
        int e = i < n ? (L ? L[i] : (int)i) : 0;
        bool take = i < n && alive[e];
        int p = warp_append(nout, take);
        if (take) {
            out[p] = e;
            mn = min(mn, sup[e]);
        }
    }
    for (int o = 16; o; o >>= 1) mn = min(mn, __shfl_down_sync(0xFFFFFFFFu, mn, o));
    if ((threadIdx.x & 31) == 0 && mn != 0x7FFFFFFF) atomicMin(minsup, mn);
}

__device__ __forceinline__ void kt_dec(int x, int K, int32_t* sup, int32_t* NF, int* nNF) {
    int old = atomicSub(sup + x, 1);
    if (old == K - 2) NF[atomicAdd(nNF, 1)] = x;
}

// One common neighbour w of a frontier edge e = (u, v): e1 = (u, w) or
// (v, w) and e2 the other, in canonical ids.  Each destroyed triangle is
// charged exactly once (see the decrement rule above).
__device__ __forceinline__ void kt_triangle(int e, int e1, int e2, int K,
                                            const unsigned char* __restrict__ alive,
                                            const unsigned char* __restrict__ inF,
                                            int32_t* sup, int32_t* NF, int* nNF) {
    if (!alive[e1] || !alive[e2]) return;
    bool f1 = inF[e1], f2 = inF[e2];
    if (!f1 && !f2) {
        kt_dec(e1, K, sup, NF, nNF);
        kt_dec(e2, K, sup, NF, nNF);
    } else if (f1 && !f2) {
        if (e < e1) kt_dec(e2, K, sup, NF, nNF);
    } else if (!f1 && f2) {
        if (e < e2) kt_dec(e1, K, sup, NF, nNF);
    }
}

// Frontier edges whose shorter list has at most 32 entries: a thread each.
// Longer ones go to a list for k_kt_peel_heavy (a CTA each): the dense
// core's hub-hub edges would otherwise run one long intersection per thread.
__global__ void k_kt_peel(KtPeel* st, const int32_t* __restrict__ src,
                          const int32_t* __restrict__ eadj,
                          const unsigned char* __restrict__ alive,
                          const unsigned char* __restrict__ inF, int32_t* __restrict__ sup,
                          int32_t* __restrict__ heavy) {
    const long long* __restrict__ off = st->off;
    const int32_t* __restrict__ adj = st->adj;
    const int32_t* __restrict__ canon = st->canon;
    const int32_t* __restrict__ F = st->F;
    const int nF = st->nf, K = st->K;
    int32_t* NF = st->NF;
    int* nNF = &st->nNF;
    int* nheavy = &st->nheavy;
    for (long long f0 = blockIdx.x * (long long)blockDim.x; f0 < nF;
         f0 += (long long)gridDim.x * blockDim.x) {
        const long long f = f0 + threadIdx.x;
        bool big = false;
        int e = 0;
        if (f < nF) {
            e = F[f];
            int u = src[e], v = eadj[e];
            long long au = off[u], la = off[u + 1] - au;
            long long bv = off[v], lb = off[v + 1] - bv;
            bool swapped = la > lb;
            long long pa = swapped ? bv : au, pb = swapped ? au : bv;
            long long na = swapped ? lb : la, nb = swapped ? la : lb;
            if (na > 32) {
                big = true;
            } else {
                long long lo = 0;
                for (long long i = 0; i < na && lo < nb; i++) {
                    int w = adj[pa + i];
                    long long p = lo + lower_bound_dev(adj + pb + lo, nb - lo, w);
                    lo = p;
                    if (p >= nb || adj[pb + p] != w) continue;
                    lo = p + 1;
                    kt_triangle(e, canon[pa + i], canon[pb + p], K, alive, inF, sup, NF, nNF);
                }
            }
        }
        int slot = warp_append(nheavy, big);
        if (big) heavy[slot] = e;
    }
}

__global__ void k_kt_peel_heavy(KtPeel* st, const int32_t* __restrict__ src,
                                const int32_t* __restrict__ eadj,
                                const int32_t* __restrict__ heavy,
                                const unsigned char* __restrict__ alive,
                                const unsigned char* __restrict__ inF, int32_t* __restrict__ sup) {
    const long long* __restrict__ off = st->off;
    const int32_t* __restrict__ adj = st->adj;
    const int32_t* __restrict__ canon = st->canon;
    const int K = st->K;
    int32_t* NF = st->NF;
    int* nNF = &st->nNF;
    // a CTA per heavy edge: its shorter list is searched by all threads,
    // so a round whose frontier is a few hub-hub edges still spreads them
    const long long nh = st->nheavy;
    for (long long h = blockIdx.x; h < nh; h += gridDim.x) {
        const int e = heavy[h];
        const int u = src[e], v = eadj[e];
        const long long au = off[u], la = off[u + 1] - au;
        const long long bv = off[v], lb = off[v + 1] - bv;
        const bool swapped = la > lb;
        const long long pa = swapped ? bv : au, pb = swapped ? au : bv;
        const long long na = swapped ? lb : la, nb = swapped ? la : lb;
        for (long long i = threadIdx.x; i < na; i += blockDim.x) {
            const int w = adj[pa + i];
            const long long p = lower_bound_dev(adj + pb, nb, w);
            if (p < nb && adj[pb + p] == w)
                kt_triangle(e, canon[pa + i], canon[pb + p], K, alive, inF, sup, NF, nNF);
        }
    }
}

__global__ void k_kt_retire(const KtPeel* st, unsigned char* __restrict__ alive,
                            unsigned char* __restrict__ inF, int32_t* __restrict__ truss) {
    const int32_t* __restrict__ F = st->F;
    const int nF = st->nf, K = st->K;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nF;
         i += (long long)gridDim.x * blockDim.x) {
        int e = F[i];
        alive[e] = 0;
        inF[e] = 0;
        truss[e] = K - 1;
    }
}

__global__ void k_kt_mark(const KtPeel* st, unsigned char* __restrict__ inF) {
    const int32_t* __restrict__ NF = st->NF;
    const int nn = st->nNF;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nn;
         i += (long long)gridDim.x * blockDim.x)
        inF[NF[i]] = 1;
}

// End of a round (one thread): the peeled edges leave the alive count, the
// next frontier becomes the current one, and the WHILE loop continues while
// it is non-empty.
__global__ void k_kt_advance(KtPeel* st, cudaGraphConditionalHandle cond, int in_graph) {
    st->remaining -= st->nf;
    st->rounds++;
    int32_t* t = st->F;
    st->F = st->NF;
    st->NF = t;
    st->nf = st->nNF;
    st->nNF = 0;
    st->nheavy = 0;
    if (in_graph) cudaGraphSetConditional(cond, st->nf > 0 ? 1u : 0u);
}

// Start of a K (one thread): its value, empty frontier counters.
__global__ void k_kt_begin(KtPeel* st, int K) {
    st->K = K;
    st->nf = 0;
    st->nNF = 0;
    st->nheavy = 0;
}

__global__ void k_kt_out(const int32_t* __restrict__ canon, const int32_t* __restrict__ truss,
                         long long m, int32_t* __restrict__ out) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m;
         e += (long long)gridDim.x * blockDim.x)
        out[e] = truss[canon[e]];
}

// Edges (in sorted-COO order) whose truss number is below K, compacted
// into an erase batch: keep[e] = truss[e] < K, pos = exclusive scan of keep.
__global__ void k_kt_below(const int32_t* __restrict__ truss, long long m, int K,
                           int32_t* __restrict__ flag) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m;
         e += (long long)gridDim.x * blockDim.x)
        flag[e] = truss[e] < K ? 1 : 0;
}

__global__ void k_kt_gather(const int32_t* __restrict__ flag, const int32_t* __restrict__ pos,
                            const int32_t* __restrict__ src, const int32_t* __restrict__ dst,
                            long long m, int32_t* __restrict__ osrc, int32_t* __restrict__ odst,
                            long long* __restrict__ total) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m;
         e += (long long)gridDim.x * blockDim.x) {
        if (flag[e]) {
            osrc[pos[e]] = src[e];
            odst[pos[e]] = dst[e];
        }
        if (e == m - 1) *total = (long long)pos[e] + flag[e];
    }
}

int ktruss_run(hn_graph* g, int32_t* d_edge_truss) {
    cudaStream_t s = g->stream;
    const int nV = g->nV;
    const long long m = g->nE;
    if (m > 0x7FFFFFFF) throw Error(HN_ERR_INVALID, "k-truss needs nE < 2^31");
    if (m == 0) return 2;
    DevBuf<long long> off((size_t)nV + 1, s);
    DevBuf<int32_t> adj((size_t)m, s), src((size_t)m, s), canon((size_t)m, s), sup((size_t)m, s),
        truss((size_t)m, s), F((size_t)m, s), NF((size_t)m, s);
    DevBuf<unsigned char> alive((size_t)m, s), inF((size_t)m, s);
    int* cnt = (int*)g->d_scalar;  // [0] err/alive, [1] nF, [2] nNF
    export_csr64(g, off.get(), adj.get());
    HN_LAUNCH(k_kt_src, grid_for(g, nV, kB), kB, 0, s, off.get(), nV, src.get());
    HN_CUDA(cudaMemsetAsync(cnt, 0, 4 * sizeof(int), s));
    HN_LAUNCH(k_kt_canon, grid_for(g, m, kB), kB, 0, s, off.get(), adj.get(), src.get(), m,
              canon.get(), cnt);
    read_scalars(g, 1);
    if (((int*)g->h_scalar)[0])
        throw Error(HN_ERR_INVALID, "k-truss needs a simple symmetric graph");
    HN_CUDA(cudaMemsetAsync(cnt, 0, 4 * sizeof(int), s));
    HN_CUDA(cudaMemsetAsync(inF.get(), 0, (size_t)m, s));
    DevBuf<int32_t> H((size_t)m, s);   // heavy frontier edges of each peel round
    {
        // supports: each triangle of the degree-oriented graph credits its
        // three canonical edges once (uses the graph's scalars, so it runs
        // before the counters below are set)
        HN_CUDA(cudaMemsetAsync(sup.get(), 0, sizeof(int32_t) * (size_t)m, s));
        Oriented o;
        build_oriented(g, o, canon.get());
        edge_support(g, o, sup.get());
    }
    HN_CUDA(cudaMemsetAsync(cnt, 0, 4 * sizeof(int), s));
    HN_LAUNCH(k_kt_init, grid_for(g, m, kB), kB, 0, s, adj.get(), src.get(), m, alive.get(), cnt);
    // truss numbers start at 2 (0x02020202 per int is not 2; fill by kernel-free memset of 0
    // then write on retirement: every edge is retired exactly once)
    read_scalars(g, 1);
    long long remaining = ((int*)g->h_scalar)[0];
    int K = 3;
    int* nL = cnt + 4;      // alive-list length
    int* minsup = cnt + 5;  // smallest support on the alive list
    // the frontier of each K scans only the alive edges, and K jumps to the
    // first value that peels anything (min support + 3): R-MAT graphs reach
    // max K in the hundreds while most edges leave at small K
    DevBuf<int32_t> L((size_t)remaining + 1, s), L2((size_t)remaining + 1, s);
    auto compact = [&](const int32_t* in, long long n) {
        HN_CUDA(cudaMemsetAsync(nL, 0, sizeof(int), s));
        const int big = 0x7FFFFFFF;
        HN_CUDA(cudaMemcpyAsync(minsup, &big, sizeof(int), cudaMemcpyHostToDevice, s));
        HN_LAUNCH(k_kt_compact, grid_for(g, n, kB), kB, 0, s, in, n, alive.get(), sup.get(),
                  L2.get(), nL, minsup);
        std::swap(L.p, L2.p);
        HN_CUDA(cudaMemcpyAsync(g->h_scalar, cnt, 8 * sizeof(int), cudaMemcpyDeviceToHost, s));
        HN_CUDA(cudaStreamSynchronize(s));
        return ((int*)g->h_scalar)[4];
    };
    int n_alive = compact(nullptr, m);
    // the peel intersects adjacency lists; once most edges are gone the
    // lists are rebuilt from the alive edges only (hubs of the dense core
    // otherwise keep their full original lists)
    long long* loff = off.get();
    int32_t* ladj = adj.get();
    int32_t* lcanon = canon.get();
    long long lm = m;
    DevBuf<long long> coff;
    DevBuf<int32_t> cadj, ccanon, cflag;
    auto shrink_lists = [&]() {
        const long long keep = 2LL * n_alive;
        if (keep * 2 > lm) return;
        cflag.alloc((size_t)lm + 1, s);
        HN_CUDA(cudaMemsetAsync(cflag.get() + lm, 0, sizeof(int32_t), s));
        HN_LAUNCH(k_kt_live_pos, grid_for(g, lm, kB), kB, 0, s, (const int32_t*)lcanon, lm,
                  alive.get(), cflag.get());
        // new slot of every live entry: an exclusive scan of the live flags;
        // a vertex's new offset is the new slot of its first old entry
        DevBuf<long long> pos((size_t)lm + 1, s), noff((size_t)nV + 1, s);
        exclusive_scan(g, (const int32_t*)cflag.get(), pos.get(), lm + 1, s);
        DevBuf<int32_t> nadj((size_t)keep + 1, s), ncanon((size_t)keep + 1, s);
        HN_LAUNCH(k_kt_shrink_off, grid_for(g, (long long)nV + 1, kB), kB, 0, s,
                  (const long long*)loff, nV, (const long long*)pos.get(), noff.get());
        HN_LAUNCH(k_kt_shrink_copy, grid_for(g, lm, kB), kB, 0, s, (const int32_t*)ladj,
                  (const int32_t*)lcanon, (const int32_t*)cflag.get(), (const long long*)pos.get(),
                  lm, nadj.get(), ncanon.get());
        coff = std::move(noff);
        cadj = std::move(nadj);
        ccanon = std::move(ncanon);
        loff = coff.get();
        ladj = cadj.get();
        lcanon = ccanon.get();
        lm = keep;
        cflag.release();
    };
    // the peel rounds of one K: a CUDA graph whose WHILE node repeats
    // peel -> heavy peel -> retire -> mark -> advance until a round finds no
    // new frontier, with no host round trip between rounds
    DevBuf<KtPeel> st(1, s);
    KtPeel* h_st = nullptr;
    HN_CUDA(cudaMallocHost((void**)&h_st, sizeof(KtPeel)));
    struct HostFree {
        KtPeel* p;
        ~HostFree() { cudaFreeHost(p); }
    } h_st_free{h_st};
    *h_st = KtPeel{loff, ladj, lcanon, F.get(), NF.get(), 0, 0, 0, K, remaining, 0};
    HN_CUDA(cudaMemcpyAsync(st.get(), h_st, sizeof(KtPeel), cudaMemcpyHostToDevice, s));
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    struct GraphFree {
        cudaGraph_t* g;
        cudaGraphExec_t* e;
        ~GraphFree() {
            if (*e) cudaGraphExecDestroy(*e);
            if (*g) cudaGraphDestroy(*g);
        }
    } graph_free{&graph, &exec};
    const bool device_rounds = knob(kKnobKtDeviceRounds) != 0;
    if (device_rounds) {
        HN_CUDA(cudaGraphCreate(&graph, 0));
        cudaGraphConditionalHandle cond;
        HN_CUDA(cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cnode;
        HN_CUDA(cudaGraphAddNode(&cnode, graph, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        KtPeel* a_st = st.get();
        const int32_t* a_src = src.get();
        const int32_t* a_eadj = adj.get();
        const unsigned char* a_alive_c = alive.get();
        unsigned char* a_alive = alive.get();
        const unsigned char* a_inF_c = inF.get();
        unsigned char* a_inF = inF.get();
        int32_t* a_sup = sup.get();
        int32_t* a_heavy = H.get();
        const int32_t* a_heavy_c = H.get();
        int32_t* a_truss = truss.get();
        const unsigned sms = (unsigned)g->info.sms;
        void* peel_args[] = {&a_st, &a_src, &a_eadj, &a_alive_c, &a_inF_c, &a_sup, &a_heavy};
        void* heavy_args[] = {&a_st, &a_src, &a_eadj, &a_heavy_c, &a_alive_c, &a_inF_c, &a_sup};
        void* retire_args[] = {&a_st, &a_alive, &a_inF, &a_truss};
        void* mark_args[] = {&a_st, &a_inF};
        int one = 1;
        void* adv_args[] = {&a_st, &cond, &one};
        struct N {
            void* f;
            unsigned grid, block;
            void** args;
        } nodes[] = {{(void*)k_kt_peel, sms * 16, 128, peel_args},
                     {(void*)k_kt_peel_heavy, sms * 8, 256, heavy_args},
                     {(void*)k_kt_retire, sms * 8, kB, retire_args},
                     {(void*)k_kt_mark, sms * 8, kB, mark_args},
                     {(void*)k_kt_advance, 1, 1, adv_args}};
        cudaGraphNode_t prev = nullptr;
        for (const N& n : nodes) {
            cudaKernelNodeParams p = {};
            p.func = n.f;
            p.gridDim = dim3(n.grid);
            p.blockDim = dim3(n.block);
            p.kernelParams = n.args;
            cudaGraphNode_t node;
            HN_CUDA(cudaGraphAddKernelNode(&node, body, prev ? &prev : nullptr, prev ? 1 : 0, &p));
            prev = node;
        }
        HN_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    }
    while (true) {
        if (remaining <= 0) { K--; break; }
        const int ms = ((int*)g->h_scalar)[5];
        if (ms + 3 > K) K = ms + 3;
        HN_LAUNCH(k_kt_begin, 1, 1, 0, s, st.get(), K);
        HN_LAUNCH(k_kt_frontier, grid_for(g, n_alive, kB), kB, 0, s, L.get(), n_alive,
                  sup.get(), alive.get(), inF.get(), st.get());
        const long long rounds_before = h_st->rounds;
        if (device_rounds) {
            HN_CUDA(cudaGraphLaunch(exec, s));
        } else {
            // host-driven rounds: launches sized to each frontier, one
            // read-back of the next frontier's size per round
            HN_CUDA(cudaMemcpyAsync(&h_st->nf, &st.get()->nf, sizeof(int), cudaMemcpyDeviceToHost,
                                    s));
            HN_CUDA(cudaStreamSynchronize(s));
            int nf = h_st->nf;
            while (nf > 0) {
                HN_LAUNCH(k_kt_peel, grid_for(g, nf, 128), 128, 0, s, st.get(), src.get(),
                          (const int32_t*)adj.get(), (const unsigned char*)alive.get(),
                          (const unsigned char*)inF.get(), sup.get(), H.get());
                HN_LAUNCH(k_kt_peel_heavy, std::min<long long>(nf, (long long)g->info.sms * 8),
                          256, 0, s, st.get(), src.get(), (const int32_t*)adj.get(),
                          (const int32_t*)H.get(), (const unsigned char*)alive.get(),
                          (const unsigned char*)inF.get(), sup.get());
                HN_LAUNCH(k_kt_retire, grid_for(g, nf, kB), kB, 0, s, (const KtPeel*)st.get(),
                          alive.get(), inF.get(), truss.get());
                HN_LAUNCH(k_kt_mark, grid_for(g, nf, kB), kB, 0, s, (const KtPeel*)st.get(),
                          inF.get());
                HN_LAUNCH(k_kt_advance, 1, 1, 0, s, st.get(), (cudaGraphConditionalHandle)0, 0);
                HN_CUDA(cudaMemcpyAsync(&h_st->nf, &st.get()->nf, sizeof(int),
                                        cudaMemcpyDeviceToHost, s));
                HN_CUDA(cudaStreamSynchronize(s));
                nf = h_st->nf;
            }
        }
        // the state comes back with the alive-list compaction's read-back
        HN_CUDA(cudaMemcpyAsync(h_st, st.get(), sizeof(KtPeel), cudaMemcpyDeviceToHost, s));
        n_alive = compact(L.get(), n_alive);
        remaining = h_st->remaining;
        if (device_rounds)
            count_launch((int)(5 * (h_st->rounds - rounds_before)));   // kernels the WHILE node ran
        if (remaining <= 0) { K--; break; }
        const long long* old_off = loff;
        shrink_lists();
        if (loff != old_off) {
            h_st->off = loff;
            h_st->adj = ladj;
            h_st->canon = lcanon;
            HN_CUDA(cudaMemcpyAsync(st.get(), h_st, 3 * sizeof(void*), cudaMemcpyHostToDevice, s));
            HN_CUDA(cudaStreamSynchronize(s));   // h_st is the copy's source
        }
        K++;
    }
    if (d_edge_truss)
        HN_LAUNCH(k_kt_out, grid_for(g, m, kB), kB, 0, s, canon.get(), truss.get(), m,
                  d_edge_truss);
    HN_CUDA(cudaStreamSynchronize(s));
    return K;
}

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" int hn_ktruss(hn_graph_t* g, int32_t* max_k, int32_t* edge_truss, int mem) {
    HN_API_BEGIN
    HN_REQUIRE(g != nullptr, "graph is null");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    HandleUse use(g);
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    DevBuf<int32_t> tmp;
    int32_t* d_out = edge_truss;
    if (edge_truss && mem == HN_MEM_HOST) {
        tmp.alloc((size_t)g->nE, s);
        d_out = tmp.get();
    }
    int K = ktruss_run(g, d_out);
    if (edge_truss && mem == HN_MEM_HOST && g->nE)
        HN_CUDA(cudaMemcpyAsync(edge_truss, d_out, sizeof(int32_t) * g->nE,
                                cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    if (max_k) *max_k = K;
    HN_API_END
}

extern "C" int hn_ktruss_keep(hn_graph_t* g, int32_t K, int32_t* max_k, int64_t* removed) {
    HN_API_BEGIN
    HN_REQUIRE(g != nullptr, "graph is null");
    HN_REQUIRE(K >= 2, "K must be at least 2");
    require_owner(g);
    std::optional<HandleUse> use;   // released before the erase call below takes it
    use.emplace(g);
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    if (removed) *removed = 0;
    const long long m = g->nE;
    if (m == 0) {
        if (max_k) *max_k = 2;
        return HN_OK;
    }
    DevBuf<int32_t> truss((size_t)m, s), src((size_t)m, s), dst((size_t)m, s), flag((size_t)m, s),
        pos((size_t)m, s);
    const int kmax = ktruss_run(g, truss.get());
    int rc = hn_graph_export_coo(g, 1, src.get(), dst.get(), HN_MEM_DEVICE);
    if (rc != HN_OK) return rc;
    HN_LAUNCH(k_kt_below, grid_for(g, m, kB), kB, 0, s, truss.get(), m, K, flag.get());
    exclusive_scan(g, (const int32_t*)flag.get(), pos.get(), m, s);
    DevBuf<int32_t> esrc((size_t)m, s), edst((size_t)m, s);
    long long* total = (long long*)(g->d_scalar + 6);
    HN_LAUNCH(k_kt_gather, grid_for(g, m, kB), kB, 0, s, flag.get(), pos.get(), src.get(),
              dst.get(), m, esrc.get(), edst.get(), total);
    HN_CUDA(cudaMemcpyAsync(g->h_scalar + 6, total, sizeof(long long), cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    const long long nrem = g->h_scalar[6];
    if (max_k) *max_k = kmax;
    if (nrem == 0) return HN_OK;
    // the below-K edges leave the graph through the ordinary erase pipeline
    use.reset();
    hn_batch_t* b = nullptr;
    rc = hn_batch_create(g, nrem, esrc.get(), edst.get(), HN_MEM_DEVICE, &b);
    if (rc != HN_OK) return rc;
    int64_t n = 0;
    rc = hn_erase(g, b, HN_DEDUP_BATCH, &n);
    hn_batch_destroy(b);
    if (rc != HN_OK) return rc;
    if (removed) *removed = n;
    HN_API_END
}
