// Exclusive prefix sums for the library's pipelines (the batch update's
// keep / segment counters and work prefixes, the triangle count's candidate
// offsets, the k-truss compactions), in place or not.
//
// Three kernels, none of which waits on another CTA:
//   1. k_scan_reduce: the sum of each tile of kTile inputs;
//   2. k_scan_tiles: one CTA turns the tile sums into their exclusive prefix
//      (in chunks of 4 x 1024, with a carry);
//   3. k_scan_down: each tile stages its inputs in shared memory (coalesced
//      loads), scans them (eight consecutive per thread, a warp scan, then
//      the warps' sums), adds its tile prefix and stores coalesced.
// A tile reads all its inputs before it writes, and writes only its own
// range, so out may equal in.
#include "hn_graph.cuh"

namespace hn {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanIpt = 8;
constexpr int kScanTile = kScanThreads * kScanIpt;
constexpr int kTopThreads = 1024;

template <typename T>
__device__ __forceinline__ T warp_incl_t(T x, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

template <typename InT, typename OutT>
__global__ void __launch_bounds__(kScanThreads)
k_scan_reduce(const InT* __restrict__ in, long long n, OutT* __restrict__ sums) {
    __shared__ OutT s_w[kScanThreads / 32];
    // order does not matter for a sum: striped, so every load is coalesced
    const long long base = (long long)blockIdx.x * kScanTile + threadIdx.x;
    OutT acc = 0;
#pragma unroll
    for (int j = 0; j < kScanIpt; j++)
        if (base + j * kScanThreads < n) acc += (OutT)in[base + j * kScanThreads];
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        OutT t = 0;
#pragma unroll
        for (int w = 0; w < kScanThreads / 32; w++) t += s_w[w];
        sums[blockIdx.x] = t;
    }
}

template <typename T>
__global__ void __launch_bounds__(kTopThreads) k_scan_tiles(T* __restrict__ sums, long long nt) {
    __shared__ T s_w[kTopThreads / 32];
    __shared__ T s_carry;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (long long c0 = 0; c0 < nt; c0 += (long long)kTopThreads * 4) {
        const long long b = c0 + (long long)threadIdx.x * 4;
        T v[4];
#pragma unroll
        for (int j = 0; j < 4; j++) v[j] = b + j < nt ? sums[b + j] : (T)0;
        const T mine = v[0] + v[1] + v[2] + v[3];
        const T incl = warp_incl_t(mine, lane);
        if (lane == 31) s_w[w] = incl;
        __syncthreads();
        if (w == 0) {
            T x = s_w[lane];
            x = warp_incl_t(x, lane);
            s_w[lane] = x;   // inclusive over warps
        }
        __syncthreads();
        const T carry = s_carry;
        T run = carry + (w ? s_w[w - 1] : (T)0) + incl - mine;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (b + j < nt) sums[b + j] = run;
            run += v[j];
        }
        __syncthreads();   // every thread has read s_carry and s_w
        if (threadIdx.x == 0) s_carry = carry + s_w[kTopThreads / 32 - 1];
        __syncthreads();
    }
}

// Slot of tile element i in shared memory: one pad slot per 32 elements, so
// that a thread's 8 consecutive elements do not all fall on a few banks.
__device__ __forceinline__ int scan_slot(int i) { return i + (i >> 5); }

template <typename InT, typename OutT>
__global__ void __launch_bounds__(kScanThreads)
k_scan_down(const InT* in, OutT* out, long long n, const OutT* __restrict__ prefix) {
    __shared__ OutT s_buf[kScanTile + kScanTile / 32];
    __shared__ OutT s_w[kScanThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long t0 = (long long)blockIdx.x * kScanTile;
    // coalesced (striped) loads into shared memory, then each thread takes
    // 8 consecutive elements
#pragma unroll
    for (int j = 0; j < kScanIpt; j++) {
        const int i = j * kScanThreads + threadIdx.x;
        s_buf[scan_slot(i)] = t0 + i < n ? (OutT)in[t0 + i] : (OutT)0;
    }
    __syncthreads();
    OutT v[kScanIpt];
    OutT mine = 0;
#pragma unroll
    for (int j = 0; j < kScanIpt; j++) {
        v[j] = s_buf[scan_slot(threadIdx.x * kScanIpt + j)];
        mine += v[j];
    }
    const OutT incl = warp_incl_t(mine, lane);
    if (lane == 31) s_w[w] = incl;
    __syncthreads();
    OutT run = prefix[blockIdx.x] + incl - mine;
#pragma unroll
    for (int ww = 0; ww < kScanThreads / 32; ww++)
        if (ww < w) run += s_w[ww];
#pragma unroll
    for (int j = 0; j < kScanIpt; j++) {
        s_buf[scan_slot(threadIdx.x * kScanIpt + j)] = run;
        run += v[j];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kScanIpt; j++) {
        const int i = j * kScanThreads + threadIdx.x;
        if (t0 + i < n) out[t0 + i] = s_buf[scan_slot(i)];
    }
}

}  // namespace

template <typename InT, typename OutT>
void exclusive_scan(hn_graph* g, const InT* in, OutT* out, long long n, cudaStream_t s) {
    if (n <= 0) return;
    const long long nt = (n + kScanTile - 1) / kScanTile;
    if (nt > 0x7FFFFFFFll) throw Error(HN_ERR_CAPACITY, "prefix sum over too many elements");
    (void)g;
    DevBuf<OutT> sums((size_t)nt, s);
    HN_LAUNCH((k_scan_reduce<InT, OutT>), nt, kScanThreads, 0, s, in, n, sums.get());
    HN_LAUNCH(k_scan_tiles<OutT>, 1, kTopThreads, 0, s, sums.get(), nt);
    HN_LAUNCH((k_scan_down<InT, OutT>), nt, kScanThreads, 0, s, in, out, n,
              (const OutT*)sums.get());
}

template void exclusive_scan<int, int>(hn_graph*, const int*, int*, long long, cudaStream_t);
template void exclusive_scan<int, long long>(hn_graph*, const int*, long long*, long long,
                                             cudaStream_t);
template void exclusive_scan<long long, long long>(hn_graph*, const long long*, long long*,
                                                   long long, cudaStream_t);
template void exclusive_scan<unsigned long long, unsigned long long>(
    hn_graph*, const unsigned long long*, unsigned long long*, long long, cudaStream_t);

}  // namespace hn
