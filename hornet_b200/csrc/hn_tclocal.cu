// Local triangle counts of a seed set: for every seed v, the number of
// triangles of the graph that contain v — the per-vertex count that
// TriangleCounting2 accumulates for every vertex
// (hornetsnest/src/Static/TriangleCounting/triangle2.cu:30-59, one credit to
// each of a triangle's three vertices), computed for the seeds only:
//     t(v) = 1/2 * sum over u in N(v) of |N(v) ∩ N(u)|
// on a simple undirected graph with sorted adjacency (each triangle {v,u,w}
// is found from u and from w).
//
// Work items are the seeds' (v, u) adjacency pairs, load-balanced over the
// seeds' degree prefix.  A lane intersects its pair alone when the shorter
// list has at most kLaneMax entries (probing each entry of the shorter list
// in the longer one by a binary search narrowed from the previous hit);
// longer pairs are appended to a list that a second kernel spreads over the
// whole grid, one warp per pair, lanes striding the shorter list.  (The
// heavy pairs of one seed sit side by side in the pair order, so leaving
// them to the warp that met them would serialise them.)  Per-seed sums are
// warp-aggregated before one atomic.
#include "hn_graph.cuh"

namespace hn {
namespace {

constexpr int kTclBlock = 256;
constexpr int kLaneMax = 8;

// entries of a[0..na) that occur in b[0..nb) (both sorted, no duplicates)
__device__ __forceinline__ unsigned common_seq(const int32_t* __restrict__ a, int na,
                                               const int32_t* __restrict__ b, int nb) {
    unsigned c = 0;
    int lo = 0;
    for (int i = 0; i < na && lo < nb; i++) {
        const int32_t x = __ldg(a + i);
        int hi = nb;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (__ldg(b + mid) < x) lo = mid + 1; else hi = mid;
        }
        if (lo < nb && __ldg(b + lo) == x) {
            c++;
            lo++;
        }
    }
    return c;
}

__device__ __forceinline__ bool find_sorted(const int32_t* __restrict__ b, int nb, int32_t x) {
    int lo = 0, hi = nb;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (__ldg(b + mid) < x) lo = mid + 1; else hi = mid;
    }
    return lo < nb && __ldg(b + lo) == x;
}

__global__ void __launch_bounds__(kTclBlock) k_tcl_pairs(const VRec* __restrict__ vtab,
                                                         const int32_t* __restrict__ pool,
                                                         const int32_t* __restrict__ seeds,
                                                         const long long* __restrict__ prefix,
                                                         int n, unsigned long long* counts,
                                                         long long* heavy_list,
                                                         unsigned long long* heavy_n) {
    const int lane = threadIdx.x & 31;
    const long long total = prefix[n];
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < total;
         base += stride) {
        const long long p = base + lane;
        int i = -1;
        unsigned c = 0;
        bool heavy = false;
        const int32_t* a = nullptr;
        const int32_t* b = nullptr;
        int na = 0, nb = 0;
        if (p < total) {
            int lo = 0, hi = n;   // last i with prefix[i] <= p
            while (hi - lo > 1) {
                int mid = (lo + hi) >> 1;
                if (__ldg(prefix + mid) <= p) lo = mid; else hi = mid;
            }
            i = lo;
            const VRec rv = vtab[seeds[i]];
            const int32_t u = __ldg(pool + rv.off + (p - __ldg(prefix + i)));
            const VRec ru = vtab[u];
            a = pool + rv.off;
            na = rv.deg;
            b = pool + ru.off;
            nb = ru.deg;
            if (na > nb) {
                const int32_t* t = a; a = b; b = t;
                int tn = na; na = nb; nb = tn;
            }
            if (na <= kLaneMax) c = common_seq(a, na, b, nb);
            else heavy = true;
        }
        const unsigned hm = __ballot_sync(0xFFFFFFFFu, heavy);
        if (hm) {
            unsigned long long at = 0;
            if (lane == 0) at = atomicAdd(heavy_n, (unsigned long long)__popc(hm));
            at = __shfl_sync(0xFFFFFFFFu, at, 0);
            if (heavy) heavy_list[at + __popc(hm & ((1u << lane) - 1u))] = p;
        }
        // lanes of one seed are contiguous: one atomic per run of equal i,
        // issued by the run's last lane with the run's sum
        unsigned long long incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long x = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += x;
        }
        const int prev = __shfl_up_sync(0xFFFFFFFFu, i, 1);
        const int next = __shfl_down_sync(0xFFFFFFFFu, i, 1);
        const bool head = lane == 0 || prev != i;
        const bool tail = lane == 31 || next != i;
        const unsigned heads = __ballot_sync(0xFFFFFFFFu, head);
        const unsigned upto = lane == 31 ? 0xFFFFFFFFu : ((2u << lane) - 1u);
        const int h = 31 - __clz(heads & upto);
        const unsigned long long ex = __shfl_sync(0xFFFFFFFFu, incl - c, h);
        if (tail && i >= 0 && incl > ex) atomicAdd(counts + i, incl - ex);
    }
}

// One warp per listed heavy pair: lanes stride the shorter list and probe
// the longer one.
__global__ void __launch_bounds__(kTclBlock) k_tcl_heavy(const VRec* __restrict__ vtab,
                                                         const int32_t* __restrict__ pool,
                                                         const int32_t* __restrict__ seeds,
                                                         const long long* __restrict__ prefix,
                                                         int n, unsigned long long* counts,
                                                         const long long* __restrict__ heavy_list,
                                                         const unsigned long long* heavy_n) {
    const int lane = threadIdx.x & 31;
    const long long nh = (long long)*heavy_n;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long h = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); h < nh;
         h += warps) {
        const long long p = heavy_list[h];
        int lo = 0, hi = n;   // last i with prefix[i] <= p
        while (hi - lo > 1) {
            int mid = (lo + hi) >> 1;
            if (__ldg(prefix + mid) <= p) lo = mid; else hi = mid;
        }
        const int i = lo;
        const VRec rv = vtab[seeds[i]];
        const int32_t u = __ldg(pool + rv.off + (p - __ldg(prefix + i)));
        const VRec ru = vtab[u];
        const int32_t* a = pool + rv.off;
        const int32_t* b = pool + ru.off;
        int na = rv.deg, nb = ru.deg;
        if (na > nb) {
            const int32_t* t = a; a = b; b = t;
            int tn = na; na = nb; nb = tn;
        }
        unsigned c = 0;
        for (int j = lane; j < na; j += 32) c += find_sorted(b, nb, __ldg(a + j)) ? 1u : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
        if (lane == 0 && c) atomicAdd(counts + i, (unsigned long long)c);
    }
}

__global__ void k_tcl_half(unsigned long long* counts, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        counts[i] >>= 1;
}

__global__ void k_tcl_check(const int32_t* seeds, int n, int nV, int* bad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (seeds[i] < 0 || seeds[i] >= nV) atomicExch(bad, 1);
}

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" int hn_tc_local(hn_graph_t* g, const int32_t* seeds, int32_t k, uint64_t* counts,
                           int mem) {
    HN_API_BEGIN
    HN_REQUIRE(g && (seeds || k == 0) && (counts || k == 0), "null argument");
    HN_REQUIRE(k >= 0, "negative seed count");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    if (k == 0) return HN_OK;
    HandleUse use(g);
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    const int32_t* d_seeds = seeds;
    DevBuf<int32_t> sbuf;
    if (mem == HN_MEM_HOST) {
        for (int j = 0; j < k; j++)
            if (seeds[j] < 0 || seeds[j] >= g->nV) throw Error(HN_ERR_INVALID, "seed outside [0, nV)");
        sbuf.alloc((size_t)k, s);
        HN_CUDA(cudaMemcpyAsync(sbuf.get(), seeds, sizeof(int32_t) * k, cudaMemcpyHostToDevice, s));
        d_seeds = sbuf.get();
    } else {
        int* bad = (int*)(g->d_scalar + 3);
        HN_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
        HN_LAUNCH(k_tcl_check, grid_for(g, k, 256), 256, 0, s, d_seeds, k, g->nV, bad);
        HN_CUDA(cudaMemcpyAsync(g->h_scalar + 3, g->d_scalar + 3, sizeof(long long),
                                cudaMemcpyDeviceToHost, s));
        HN_CUDA(cudaStreamSynchronize(s));
        if ((int)g->h_scalar[3] != 0) throw Error(HN_ERR_INVALID, "seed outside [0, nV)");
    }
    DevBuf<long long> prefix((size_t)k + 1, s);
    degree_prefix(g, d_seeds, k, prefix.get());
    DevBuf<unsigned long long> cbuf;
    unsigned long long* d_counts = (unsigned long long*)counts;
    if (mem == HN_MEM_HOST) {
        cbuf.alloc((size_t)k, s);
        d_counts = cbuf.get();
    }
    HN_CUDA(cudaMemsetAsync(d_counts, 0, sizeof(unsigned long long) * k, s));
    // the pair count sizes the heavy-pair list
    HN_CUDA(cudaMemcpyAsync(g->h_scalar + 4, prefix.get() + k, sizeof(long long),
                            cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    const long long pairs = g->h_scalar[4];
    DevBuf<long long> heavy((size_t)pairs + 1, s);
    unsigned long long* heavy_n = (unsigned long long*)(g->d_scalar + 5);
    HN_CUDA(cudaMemsetAsync(heavy_n, 0, sizeof(unsigned long long), s));
    HN_LAUNCH(k_tcl_pairs, (long long)g->info.sms * 8, kTclBlock, 0, s, g->vtab, g->pool, d_seeds,
              prefix.get(), k, d_counts, heavy.get(), heavy_n);
    HN_LAUNCH(k_tcl_heavy, (long long)g->info.sms * 8, kTclBlock, 0, s, g->vtab, g->pool,
              d_seeds, prefix.get(), k, d_counts, (const long long*)heavy.get(),
              (const unsigned long long*)heavy_n);
    HN_LAUNCH(k_tcl_half, grid_for(g, k, 256), 256, 0, s, d_counts, k);
    if (mem == HN_MEM_HOST)
        HN_CUDA(cudaMemcpyAsync(counts, d_counts, sizeof(unsigned long long) * k,
                                cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    HN_API_END
}
