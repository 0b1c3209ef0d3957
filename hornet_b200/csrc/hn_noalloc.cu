// Connected components over a caller-owned device CSR, with no device
// allocation at all.
//
// Who needs this: callers that must not call cudaMalloc / cudaFree or any
// allocating library routine — plugins running inside a host framework
// that owns every byte of device memory and hands out fixed buffers,
// services that reserve their whole memory budget up front so that no
// request can fail for lack of memory halfway through, and latency-critical
// loops where the implicit device synchronisation of cudaMalloc / cudaFree
// is not acceptable.  Such a caller already holds its graph as a CSR in
// device memory and a device buffer for the result; this entry point needs
// nothing else.
//
// Set-up: the first call on a device looks up the device address of the
// scratch array (cudaGetSymbolAddress) with that device current; make that
// first call before any stream capture of your own.  Every call on a device
// shares the one scratch array and it keeps the previous call's contents
// (the counters are cleared at the start of each call): calls that overlap
// on the GPU — from two host threads, or on two streams — race and give
// wrong results, so serialise them.
//
// The only working memory beyond the caller's buffers is a file-scope
// __device__ array (g_cc_scratch below): a worklist of at most
// kNoAllocMaxVertices vertices plus a few counters, 16 MiB in all.  Every
// GPU that loads this library holds it until the process exits.  The
// result array doubles as the union-find parent array.
//
// The algorithm is the one hn_cc uses (ECL-CC style union-find on an
// Afforest schedule, hn_cc.cu), written here a second time against a plain
// CSR so that the existing path stays untouched.  Like hn_cc it needs an
// undirected graph stored symmetrically (every edge in both endpoints'
// lists): vertices of the giant component skip their remaining neighbours,
// so an edge stored only in a giant-component vertex's list would be lost.
// The CSR is validated first (offsets start at 0 and never decrease, every
// id is a vertex) by one pass over off[] and adj[]; the union-find kernels
// are skipped when the offsets are malformed.
#include <mutex>

#include "hn_graph.cuh"

namespace hn {
namespace {

constexpr int kNoAllocMaxVertices = 1 << 22;        // 4,194,304 vertices
constexpr int kNoAllocCounters = 64;                // [0] giant root, [1] list size,
                                                    // [2] components, [3] bad-id flag,
                                                    // [4] bad-offsets flag
static __device__ __align__(256) int g_cc_scratch[kNoAllocMaxVertices + kNoAllocCounters];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
int* g_scratch_addr[kMaxDevices] = {};

constexpr int kB = 256;
constexpr int kSampleNa = 2;

__device__ __forceinline__ int na_find(int* __restrict__ parent, int v) {
    int cur = parent[v];
    if (cur != v) {
        int prev = v, next;
        while (cur > (next = parent[cur])) {
            parent[prev] = next;
            prev = cur;
            cur = next;
        }
    }
    return cur;
}

__device__ __forceinline__ void na_link(int* __restrict__ parent, int u, int v) {
    int ru = na_find(parent, u);
    int rv = na_find(parent, v);
    while (ru != rv) {
        if (ru < rv) { int x = ru; ru = rv; rv = x; }
        int old = atomicCAS(parent + ru, ru, rv);
        if (old == ru) return;
        ru = na_find(parent, old);
    }
}

// Validation of the caller's CSR before anything follows it: off[0] == 0
// and off non-decreasing (ctr[4]); then, only when the offsets are sound,
// every id of adj[0, off[nV]) inside [0, nV) (ctr[3]).  The kernels after
// them return at once when ctr[4] is set, so a malformed offset array is
// never used to address adj.
__global__ void k_na_check_off(const int32_t* __restrict__ off, int nV, int* __restrict__ ctr) {
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    bool bad = t0 == 0 && off[0] != 0;
    for (long long v = t0; v < nV; v += (long long)gridDim.x * blockDim.x)
        if (off[v + 1] < off[v]) bad = true;
    if (__any_sync(0xFFFFFFFFu, bad) && (threadIdx.x & 31) == 0) ctr[4] = 1;
}

__global__ void k_na_check_ids(const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                               int nV, int* __restrict__ ctr) {
    if (ctr[4]) return;
    const long long m = off[nV];
    bool bad = false;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
         i += (long long)gridDim.x * blockDim.x) {
        const int u = adj[i];
        if (u < 0 || u >= nV) bad = true;
    }
    if (__any_sync(0xFFFFFFFFu, bad) && (threadIdx.x & 31) == 0) ctr[3] = 1;
}

__global__ void k_na_init(int* __restrict__ parent, int nV, const int* __restrict__ ctr) {
    if (ctr[4]) return;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x)
        parent[v] = (int)v;
}

// first kSampleNa neighbours of every vertex; ids outside [0,nV) are
// skipped (k_na_check has flagged them)
__global__ void k_na_sample(const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                            int nV, int* __restrict__ parent, int* __restrict__ ctr) {
    if (ctr[4]) return;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x) {
        int b = off[v], e = off[v + 1];
        int k = e - b < kSampleNa ? e - b : kSampleNa;
        for (int i = 0; i < k; i++) {
            int u = adj[b + i];
            if (u < 0 || u >= nV) continue;
            na_link(parent, (int)v, u);
        }
    }
}

__global__ void k_na_compress(int* __restrict__ parent, int nV, const int* __restrict__ ctr) {
    if (ctr[4]) return;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x)
        parent[v] = na_find(parent, (int)v);
}

// most frequent root among 256 evenly spaced vertices (one CTA of 256)
__global__ void k_na_giant(const int* __restrict__ parent, int nV, int* __restrict__ ctr) {
    if (ctr[4]) return;
    __shared__ int s_r[256];
    __shared__ unsigned long long s_key;
    int t = threadIdx.x;
    long long v = (long long)t * nV / 256;
    s_r[t] = parent[v < nV ? v : nV - 1];
    if (t == 0) s_key = 0;
    __syncthreads();
    int mine = s_r[t], c = 0;
    for (int i = 0; i < 256; i++) c += (s_r[i] == mine);
    atomicMax(&s_key, ((unsigned long long)c << 32) | (unsigned)(0x7FFFFFFF - mine));
    __syncthreads();
    if (t == 0) ctr[0] = 0x7FFFFFFF - (int)(s_key & 0xFFFFFFFFull);
}

__global__ void k_na_worklist(const int32_t* __restrict__ off, const int* __restrict__ parent,
                              int nV, int* __restrict__ list, int* __restrict__ ctr) {
    if (ctr[4]) return;
    const int gr = ctr[0];
    for (long long v0 = blockIdx.x * (long long)blockDim.x; v0 < nV;
         v0 += (long long)gridDim.x * blockDim.x) {
        long long v = v0 + threadIdx.x;
        bool take = v < nV && off[v + 1] - off[v] > kSampleNa && parent[v] != gr;
        int p = warp_append(ctr + 1, take);
        if (take) list[p] = (int)v;
    }
}

__global__ void k_na_rest(const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                          int nV, const int* __restrict__ list, int* __restrict__ parent,
                          int* __restrict__ ctr) {
    if (ctr[4]) return;
    const int n = ctr[1];
    const int lane = threadIdx.x & 31;
    long long wid = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long i = wid; i < n; i += nw) {
        int v = list[i];
        int b = off[v], e = off[v + 1];
        for (int k = b + kSampleNa + lane; k < e; k += 32) {
            int u = adj[k];
            if (u < 0 || u >= nV) continue;
            na_link(parent, v, u);
        }
    }
}

__global__ void k_na_finish(int* __restrict__ parent, int nV, int* __restrict__ ctr) {
    if (ctr[4]) return;
    int mine = 0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x) {
        int r = na_find(parent, (int)v);
        parent[v] = r;
        mine += (r == v);
    }
    for (int o = 16; o; o >>= 1) mine += __shfl_down_sync(0xFFFFFFFFu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(ctr + 2, mine);
}

// Device address of the scratch array on the current device, looked up
// once per device (the host-side symbol g_cc_scratch is only a stand-in
// and must never be handed to a kernel).
int* scratch_on_current_device() {
    int dev = 0;
    HN_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw Error(HN_ERR_INVALID, "device ordinal too large");
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        int* p = nullptr;
        HN_CUDA(cudaGetSymbolAddress((void**)&p, g_cc_scratch));
        g_scratch_addr[dev] = p;
    }
    return g_scratch_addr[dev];
}

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" int hn_cc_csr_noalloc(int32_t nV, const int32_t* off, const int32_t* adj,
                                 int32_t* labels, int32_t* n_components, void* stream) {
    HN_API_BEGIN
    HN_REQUIRE(nV >= 0, "negative vertex count");
    if (nV > kNoAllocMaxVertices)
        throw Error(HN_ERR_CAPACITY,
                    "hn_cc_csr_noalloc handles at most 4194304 vertices (static scratch)");
    HN_REQUIRE(off && labels && (adj || nV == 0), "null CSR or label pointer");
    cudaStream_t s = (cudaStream_t)stream;
    int* scratch = scratch_on_current_device();
    int* list = scratch;
    int* ctr = scratch + kNoAllocMaxVertices;
    // the array keeps the previous call's contents: clear the counters
    HN_CUDA(cudaMemsetAsync(ctr, 0, sizeof(int) * 5, s));
    if (nV > 0) {
        int dev = 0, sms = 148;
        HN_CUDA(cudaGetDevice(&dev));
        HN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        long long gv = ((long long)nV + kB - 1) / kB;
        if (gv > (long long)sms * 8) gv = (long long)sms * 8;
        HN_LAUNCH(k_na_check_off, gv, kB, 0, s, off, nV, ctr);
        HN_LAUNCH(k_na_check_ids, (long long)sms * 8, kB, 0, s, off, adj, nV, ctr);
        HN_LAUNCH(k_na_init, gv, kB, 0, s, labels, nV, ctr);
        HN_LAUNCH(k_na_sample, gv, kB, 0, s, off, adj, nV, labels, ctr);
        HN_LAUNCH(k_na_compress, gv, kB, 0, s, labels, nV, ctr);
        HN_LAUNCH(k_na_giant, 1, 256, 0, s, labels, nV, ctr);
        HN_LAUNCH(k_na_worklist, gv, kB, 0, s, off, labels, nV, list, ctr);
        HN_LAUNCH(k_na_rest, (long long)sms * 8, kB, 0, s, off, adj, nV, list, labels, ctr);
        HN_LAUNCH(k_na_finish, gv, kB, 0, s, labels, nV, ctr);
    }
    int host_ctr[5] = {0, 0, 0, 0, 0};
    HN_CUDA(cudaMemcpyAsync(host_ctr, ctr, sizeof(host_ctr), cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    if (host_ctr[4])
        throw Error(HN_ERR_INVALID, "CSR offsets must start at 0 and never decrease");
    if (host_ctr[3]) throw Error(HN_ERR_INVALID, "CSR neighbour id outside [0, nV)");
    if (n_components) *n_components = host_ctr[2];
    HN_API_END
}
