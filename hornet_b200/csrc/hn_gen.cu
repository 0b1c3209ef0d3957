// Synthetic inputs: R-MAT edge pairs and an undirected CSR builder.
//
// The reference has no R-MAT or ER generator (its random batch generator
// hornet/include/Util/RandomGraphData.cuh:230-245 yields only self-loops),
// so this is new code.  Pair i is a pure function of (seed, i): each level
// of the recursion draws a 32-bit uniform from SplitMix64 (S. Vigna's
// published mixing function) over a per-pair counter, so the host
// (multi-threaded) and device generators produce identical arrays.
// Endpoints >= n (non-power-of-two vertex counts) redraw the whole pair with
// the next attempt counter.
//
// The CSR builder follows GraphStd's undirected COOtoCSR
// (xlib/src/Graph/GraphStd.cpp:174-206): mirror every pair, drop self
// loops, sort, remove duplicates — as one radix sort of packed keys, one
// unique pass and one offsets pass on the device.

#include <algorithm>
#include <thread>
#include <vector>

#include "hn_graph.cuh"

namespace hn {
namespace {

__host__ __device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

struct RmatParams {
    int scale;
    int n;
    unsigned long long ta, tb, tc;  // cumulative thresholds * 2^32
    unsigned long long seed;
};

__host__ __device__ __forceinline__ void rmat_pair(const RmatParams& p, long long i, int* su,
                                                   int* sv) {
    unsigned long long base = splitmix64(p.seed ^ ((unsigned long long)i * 0xD1B54A32D192ED03ull));
    for (int attempt = 0; attempt < 64; attempt++) {
        unsigned long long ctr = base + (unsigned long long)attempt * 0x10000ull;
        unsigned u = 0, v = 0;
        unsigned long long bits = 0;
        for (int l = 0; l < p.scale; l++) {
            if ((l & 1) == 0) bits = splitmix64(ctr + (unsigned long long)(l >> 1));
            unsigned long long r = (l & 1) ? (bits >> 32) : (bits & 0xFFFFFFFFull);
            unsigned ub = 0, vb = 0;
            if (r < p.ta) {
            } else if (r < p.tb) {
                vb = 1;
            } else if (r < p.tc) {
                ub = 1;
            } else {
                ub = 1;
                vb = 1;
            }
            u = (u << 1) | ub;
            v = (v << 1) | vb;
        }
        if ((int)u < p.n && (int)v < p.n) {
            *su = (int)u;
            *sv = (int)v;
            return;
        }
    }
    // astronomically unlikely for n >= 2^(scale-1): fold into range
    *su = (int)(base % (unsigned long long)p.n);
    *sv = (int)((base >> 32) % (unsigned long long)p.n);
}

__global__ void k_rmat(RmatParams p, long long np, int32_t* __restrict__ src,
                       int32_t* __restrict__ dst) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < np;
         i += (long long)gridDim.x * blockDim.x) {
        int u, v;
        rmat_pair(p, i, &u, &v);
        src[i] = u;
        dst[i] = v;
    }
}

RmatParams make_params(int scale, int n, double a, double b, double c, unsigned long long seed) {
    if (scale < 1 || scale > 31) throw Error(HN_ERR_INVALID, "scale must be in [1, 31]");
    if (n <= 0 || (long long)n > (1ll << scale)) throw Error(HN_ERR_INVALID, "n outside (0, 2^scale]");
    if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) throw Error(HN_ERR_INVALID, "bad R-MAT params");
    RmatParams p;
    p.scale = scale;
    p.n = n;
    const double two32 = 4294967296.0;
    p.ta = (unsigned long long)(a * two32);
    p.tb = (unsigned long long)((a + b) * two32);
    p.tc = (unsigned long long)((a + b + c) * two32);
    p.seed = seed;
    return p;
}

// keys = u << S | v with S = L+1 field bits; self loops -> all-ones sentinel
__global__ void k_sym_keys(const int32_t* __restrict__ src, const int32_t* __restrict__ dst,
                           long long np, int nV, int S, unsigned long long* __restrict__ keys,
                           int* __restrict__ err) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < np;
         i += (long long)gridDim.x * blockDim.x) {
        int u = src[i], v = dst[i];
        if (u < 0 || u >= nV || v < 0 || v >= nV) {
            atomicExch(err, 1);
            u = v = 0;
        }
        if (u == v) {
            keys[2 * i] = ~0ull;
            keys[2 * i + 1] = ~0ull;
        } else {
            keys[2 * i] = ((unsigned long long)u << S) | (unsigned)v;
            keys[2 * i + 1] = ((unsigned long long)v << S) | (unsigned)u;
        }
    }
}

// mark[i] = 1 where a run of equal sorted keys starts.
__global__ void k_run_starts(const unsigned long long* __restrict__ k, long long n,
                             int* __restrict__ mark) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        mark[i] = i == 0 || k[i] != k[i - 1];
}

// The first key of each run to its slot (pos: the exclusive scan of the
// run starts); the run count to *nsel.
__global__ void k_keep_run_starts(const unsigned long long* __restrict__ k, long long n,
                                  const int* __restrict__ pos, unsigned long long* __restrict__ out,
                                  long long* __restrict__ nsel) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const bool head = i == 0 || k[i] != k[i - 1];
        if (head) out[pos[i]] = k[i];
        if (i == n - 1) *nsel = (long long)pos[i] + (head ? 1 : 0);
    }
}

__global__ void k_csr_from_keys(const unsigned long long* __restrict__ keys, long long m, int nV,
                                int S, int32_t* __restrict__ off, int32_t* __restrict__ adj) {
    const unsigned long long mask = (1ull << S) - 1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i <= m;
         i += (long long)gridDim.x * blockDim.x) {
        int s = i < m ? (int)(keys[i] >> S) : nV;
        int sp = i > 0 ? (int)(keys[i - 1] >> S) : -1;
        for (int v = sp + 1; v <= s; v++) off[v] = (int)i;
        if (i < m) adj[i] = (int)(keys[i] & mask);
    }
}

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" {

int hn_gen_rmat_host(int32_t scale, int32_t n_vertices, int64_t np, double a, double b, double c,
                     uint64_t seed, int32_t* src, int32_t* dst) {
    HN_API_BEGIN
    HN_REQUIRE(np >= 0 && (np == 0 || (src && dst)), "bad arguments");
    RmatParams p = make_params(scale, n_vertices, a, b, c, seed);
    unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    if (np < 65536) nt = 1;
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; t++) {
        th.emplace_back([&, t]() {
            long long lo = np * t / nt, hi = np * (t + 1) / nt;
            for (long long i = lo; i < hi; i++) {
                int u, v;
                rmat_pair(p, i, &u, &v);
                src[i] = u;
                dst[i] = v;
            }
        });
    }
    for (auto& x : th) x.join();
    HN_API_END
}

int hn_gen_rmat_device(int32_t scale, int32_t n_vertices, int64_t np, double a, double b,
                       double c, uint64_t seed, int32_t* src, int32_t* dst, int device) {
    HN_API_BEGIN
    HN_REQUIRE(np >= 0 && (np == 0 || (src && dst)), "bad arguments");
    RmatParams p = make_params(scale, n_vertices, a, b, c, seed);
    HN_CUDA(cudaSetDevice(device));
    int sms = 148;
    HN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    long long grid = std::min<long long>((np + 255) / 256, (long long)sms * 16);
    HN_LAUNCH(k_rmat, grid, 256, 0, (cudaStream_t)0, p, (long long)np, src, dst);
    HN_CUDA(cudaDeviceSynchronize());
    HN_API_END
}

int hn_coo_to_csr_device(int32_t nV, int64_t np, const int32_t* src, const int32_t* dst,
                         int device, int32_t** off_out, int32_t** adj_out, int64_t* nE_out) {
    HN_API_BEGIN
    HN_REQUIRE(off_out && adj_out && nE_out, "null output");
    HN_REQUIRE(nV > 0 && np >= 0 && (np == 0 || (src && dst)), "bad arguments");
    HN_REQUIRE(2 * np <= 0x7FFFFFFF, "too many pairs for one radix sort");
    *off_out = nullptr;
    *adj_out = nullptr;
    *nE_out = 0;
    HN_CUDA(cudaSetDevice(device));
    cudaStream_t s = 0;
    int sms = 148;
    HN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int L = nV > 1 ? ceil_log2_u64((unsigned long long)nV) : 1;
    const int S = L + 1;
    const long long n2 = 2 * np;
    DevBuf<unsigned long long> k1((size_t)n2 + 1, s), k2((size_t)n2 + 1, s);
    DevBuf<int> err(2, s);
    HN_CUDA(cudaMemsetAsync(err.get(), 0, 2 * sizeof(int), s));
    long long grid = std::min<long long>((np + 255) / 256, (long long)sms * 16);
    HN_LAUNCH(k_sym_keys, grid, 256, 0, s, src, dst, (long long)np, nV, S, k1.get(), err.get());
    // the library's radix sort (the sentinel of a self loop has every key
    // bit set, so it sorts last), then the first key of every run of equal
    // keys kept: its slot is an exclusive scan of the run-start marks
    unsigned long long* sorted = k1.get();
    unsigned long long* alt = k2.get();
    {
        uint32_t* nv = nullptr;
        uint32_t* nva = nullptr;
        radix_sort_u64(nullptr, sorted, alt, nv, nva, n2, 2 * S, err.get() + 1, s);
    }
    unsigned long long* uniq = alt;
    DevBuf<long long> nsel(1, s);
    if (n2 > 0) {
        DevBuf<int> mark((size_t)n2, s);
        HN_LAUNCH(k_run_starts, grid, 256, 0, s, (const unsigned long long*)sorted, n2,
                  mark.get());
        exclusive_scan(nullptr, (const int*)mark.get(), mark.get(), n2, s);
        HN_LAUNCH(k_keep_run_starts, grid, 256, 0, s, (const unsigned long long*)sorted, n2,
                  (const int*)mark.get(), uniq, nsel.get());
    } else {
        HN_CUDA(cudaMemsetAsync(nsel.get(), 0, sizeof(long long), s));
    }
    long long nu = 0;
    int herr = 0;
    HN_CUDA(cudaMemcpyAsync(&nu, nsel.get(), sizeof(long long), cudaMemcpyDeviceToHost, s));
    int herr2 = 0;
    HN_CUDA(cudaMemcpyAsync(&herr, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaMemcpyAsync(&herr2, err.get() + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    if (herr) throw Error(HN_ERR_INVALID, "pair id outside [0, nV)");
    if (herr2) throw Error(HN_ERR_TIMEOUT, "pair sort: a bounded wait gave up");
    unsigned long long last = 0;
    if (nu > 0) {
        HN_CUDA(cudaMemcpy(&last, uniq + nu - 1, sizeof(last), cudaMemcpyDeviceToHost));
        if (last == ~0ull) nu--;  // the self-loop sentinel
    }
    int32_t* off = nullptr;
    int32_t* adj = nullptr;
    HN_CUDA(cudaMalloc((void**)&off, sizeof(int32_t) * ((size_t)nV + 1)));
    HN_CUDA(cudaMalloc((void**)&adj, sizeof(int32_t) * ((size_t)nu + 1)));
    grid = std::min<long long>((nu + 256) / 256, (long long)sms * 16);
    HN_LAUNCH(k_csr_from_keys, grid, 256, 0, s, uniq, nu, nV, S, off, adj);
    HN_CUDA(cudaStreamSynchronize(s));
    *off_out = off;
    *adj_out = adj;
    *nE_out = nu;
    HN_API_END
}

}  // extern "C"
