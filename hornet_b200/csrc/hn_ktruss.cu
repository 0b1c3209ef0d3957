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
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>

#include "hn_graph.cuh"
#include "hn_tc.cuh"

namespace hn {
namespace {

constexpr int kB = 256;

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

// Frontier of round K: alive edges of the list L with support < K - 2.
__global__ void k_kt_frontier(const int32_t* __restrict__ L, int nL, int K,
                              const int32_t* __restrict__ sup,
                              const unsigned char* __restrict__ alive,
                              unsigned char* __restrict__ inF, int32_t* __restrict__ F,
                              int* __restrict__ nF) {
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
__global__ void k_kt_peel(const long long* __restrict__ off, const int32_t* __restrict__ adj,
                          const int32_t* __restrict__ src, const int32_t* __restrict__ canon,
                          const int32_t* __restrict__ eadj,
                          const int32_t* __restrict__ F, int nF, int K,
                          const unsigned char* __restrict__ alive,
                          const unsigned char* __restrict__ inF, int32_t* __restrict__ sup,
                          int32_t* __restrict__ NF, int* __restrict__ nNF,
                          int32_t* __restrict__ heavy, int* __restrict__ nheavy) {
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

__global__ void k_kt_peel_heavy(const long long* __restrict__ off,
                                const int32_t* __restrict__ adj,
                                const int32_t* __restrict__ src,
                                const int32_t* __restrict__ canon,
                                const int32_t* __restrict__ eadj,
                                const int32_t* __restrict__ heavy, const int* __restrict__ nheavy,
                                int K, const unsigned char* __restrict__ alive,
                                const unsigned char* __restrict__ inF, int32_t* __restrict__ sup,
                                int32_t* __restrict__ NF, int* __restrict__ nNF) {
    // a CTA per heavy edge: its shorter list is searched by all threads,
    // so a round whose frontier is a few hub-hub edges still spreads them
    const long long nh = *nheavy;
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

__global__ void k_kt_retire(const int32_t* __restrict__ F, int nF, const int32_t* __restrict__ NF,
                            const int* __restrict__ nNF, int K, unsigned char* __restrict__ alive,
                            unsigned char* __restrict__ inF, int32_t* __restrict__ truss) {
    int nn = *nNF;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nF || i < nn;
         i += (long long)gridDim.x * blockDim.x) {
        if (i < nF) {
            int e = F[i];
            alive[e] = 0;
            inF[e] = 0;
            truss[e] = K - 1;
        }
    }
}

__global__ void k_kt_mark(const int32_t* __restrict__ NF, const int* __restrict__ nNF,
                          unsigned char* __restrict__ inF) {
    int nn = *nNF;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nn;
         i += (long long)gridDim.x * blockDim.x)
        inF[NF[i]] = 1;
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
    int* nF = cnt + 1;
    int* nNF = cnt + 2;
    int* nheavy = cnt + 3;  // frontier edges left to k_kt_peel_heavy (right after nNF)
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
        cflag.alloc((size_t)lm, s);
        HN_LAUNCH(k_kt_live_pos, grid_for(g, lm, kB), kB, 0, s, (const int32_t*)lcanon, lm,
                  alive.get(), cflag.get());
        DevBuf<long long> noff((size_t)nV + 1, s);
        {
            size_t tb = 0;
            HN_CUDA(cub::DeviceSegmentedReduce::Sum(nullptr, tb, cflag.get(), noff.get(), nV, loff,
                                                    loff + 1, s));
            DevBuf<char> tmp(tb, s);
            HN_CUDA(cub::DeviceSegmentedReduce::Sum(tmp.get(), tb, cflag.get(), noff.get(), nV,
                                                    loff, loff + 1, s));
            HN_CUDA(cudaMemsetAsync(noff.get() + nV, 0, sizeof(long long), s));
            tb = 0;
            HN_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, noff.get(), noff.get(), nV + 1, s));
            DevBuf<char> tmp2(tb, s);
            HN_CUDA(cub::DeviceScan::ExclusiveSum(tmp2.get(), tb, noff.get(), noff.get(), nV + 1,
                                                  s));
            count_launch(2);
        }
        DevBuf<int32_t> nadj((size_t)keep + 1, s), ncanon((size_t)keep + 1, s);
        {
            int* nsel = cnt + 6;
            size_t tb = 0;
            HN_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, ladj, cflag.get(), nadj.get(), nsel,
                                               lm, s));
            DevBuf<char> tmp(tb, s);
            HN_CUDA(cub::DeviceSelect::Flagged(tmp.get(), tb, ladj, cflag.get(), nadj.get(), nsel,
                                               lm, s));
            HN_CUDA(cub::DeviceSelect::Flagged(tmp.get(), tb, lcanon, cflag.get(), ncanon.get(),
                                               nsel, lm, s));
            count_launch(2);
        }
        coff = std::move(noff);
        cadj = std::move(nadj);
        ccanon = std::move(ncanon);
        loff = coff.get();
        ladj = cadj.get();
        lcanon = ccanon.get();
        lm = keep;
        cflag.release();
    };
    while (true) {
        if (remaining <= 0) { K--; break; }
        const int ms = ((int*)g->h_scalar)[5];
        if (ms + 3 > K) K = ms + 3;
        HN_CUDA(cudaMemsetAsync(nF, 0, sizeof(int), s));
        HN_LAUNCH(k_kt_frontier, grid_for(g, n_alive, kB), kB, 0, s, L.get(), n_alive, K,
                  sup.get(), alive.get(), inF.get(), F.get(), nF);
        HN_CUDA(cudaMemcpyAsync(g->h_scalar, nF, sizeof(int), cudaMemcpyDeviceToHost, s));
        HN_CUDA(cudaStreamSynchronize(s));
        int nf = ((int*)g->h_scalar)[0];
        while (nf > 0) {
            HN_CUDA(cudaMemsetAsync(nNF, 0, 2 * sizeof(int), s));   // nNF, nheavy
            HN_LAUNCH(k_kt_peel, grid_for(g, nf, 128), 128, 0, s, (const long long*)loff,
                      (const int32_t*)ladj, src.get(), (const int32_t*)lcanon,
                      (const int32_t*)adj.get(), F.get(), nf, K, alive.get(), inF.get(), sup.get(),
                      NF.get(), nNF, H.get(), nheavy);
            HN_LAUNCH(k_kt_peel_heavy, std::min<long long>(nf, (long long)g->info.sms * 8), 256, 0, s,
                      (const long long*)loff, (const int32_t*)ladj, src.get(),
                      (const int32_t*)lcanon, (const int32_t*)adj.get(), (const int32_t*)H.get(),
                      (const int*)nheavy, K, alive.get(), inF.get(), sup.get(), NF.get(), nNF);
            HN_LAUNCH(k_kt_retire, grid_for(g, nf, kB), kB, 0, s, F.get(), nf, NF.get(), nNF, K,
                      alive.get(), inF.get(), truss.get());
            HN_LAUNCH(k_kt_mark, grid_for(g, nf, kB), kB, 0, s, NF.get(), nNF, inF.get());
            remaining -= nf;
            HN_CUDA(cudaMemcpyAsync(g->h_scalar, nNF, sizeof(int), cudaMemcpyDeviceToHost, s));
            HN_CUDA(cudaStreamSynchronize(s));
            nf = ((int*)g->h_scalar)[0];
            std::swap(F.p, NF.p);
        }
        if (remaining <= 0) { K--; break; }
        n_alive = compact(L.get(), n_alive);
        shrink_lists();
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
    {
        size_t tb = 0;
        HN_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag.get(), pos.get(), (int)m, s));
        DevBuf<char> tmp(tb, s);
        HN_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tb, flag.get(), pos.get(), (int)m, s));
        count_launch();
    }
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
