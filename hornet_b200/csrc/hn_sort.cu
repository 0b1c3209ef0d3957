// Stable LSD radix sort of the packed update keys (src << L | dst), with an
// optional 32-bit value per key, for the batch-update pipeline.
//
// The reference sorts a batch with two stable thrust sorts
// (hornet/include/Core/SoA/impl/SoAPtr.i.cuh:560-613, called from
// BatchUpdate.i.cuh).  Here the key is one 64-bit word of 2L significant bits,
// sorted 8 bits per pass (ceil(2L / 8) passes: 6 at 2^24 vertices), ONE kernel
// per pass over tiles of 8 keys per thread (4096 keys, or 2048 with values;
// 1024 threads per SM either way: the pass waits on memory, so occupancy
// pays):
//   * tiles take their numbers from a counter as they start, so every
//     lower-numbered tile is already running;
//   * a tile ranks its keys stably by digit (warp by warp, 32 keys a round in
//     key order, equal digits found with eight ballots), publishes its digit
//     counts, then finds how many keys of each digit the tiles before it hold
//     by looking back over their published counts until it meets a tile that
//     has published its inclusive prefix (decoupled look-back: Merrill and
//     Garland, "Single-pass Parallel Prefix Scan with Decoupled Look-back",
//     NVIDIA technical report NVR-2016-002), and publishes its own;
//   * it reorders its keys by digit in shared memory and writes each digit's
//     run to (keys of smaller digits) + (keys of this digit in earlier tiles);
//   * while its keys are in registers it also counts the NEXT pass's digits
//     into the global histogram that pass needs (the first pass's histogram
//     comes from a separate counting kernel).
// A wait for a lower-numbered tile is bounded: after kWaitLimit polls the
// tile records HN_ERR_TIMEOUT in the caller's error word and writes nothing;
// the update pipeline's later kernels see the error word and do nothing, and
// the host reports the error at its synchronisation.  (The wait cannot
// actually run out: a lower-numbered tile took its number, so it is running,
// and it publishes its counts before any wait of its own.)
#include "hn_graph.cuh"

namespace hn {
namespace {

constexpr int kOsThreads = 256;   // the first pass's counting kernel
constexpr int kOsIpt = 8;          // keys per thread of a pass
constexpr int kBins = 256;
constexpr int kMaxPasses = 8;
constexpr long long kWaitLimit = 1 << 22;
constexpr int kLook = 4;   // statuses a look-back step reads at once

constexpr unsigned long long kFlagAgg = 1ull << 62;    // the tile's own counts
constexpr unsigned long long kFlagIncl = 2ull << 62;   // counts of tiles 0..t
constexpr unsigned long long kValMask = (1ull << 62) - 1;

struct SortState {
    unsigned ghist[kMaxPasses][kBins];   // keys per digit, per pass
    int tile_ctr[kMaxPasses];            // next tile number, per pass
};

__device__ __forceinline__ unsigned digit_of(unsigned long long k, int shift) {
    return (unsigned)(k >> shift) & 0xFFu;
}

// Lanes (among `active`) whose digit equals this lane's: eight ballots.
__device__ __forceinline__ unsigned same_digit_lanes(unsigned d, unsigned active) {
    unsigned peers = active;
#pragma unroll
    for (int b = 0; b < 8; b++) {
        const unsigned bal = __ballot_sync(0xFFFFFFFFu, (d >> b) & 1u);
        peers &= ((d >> b) & 1u) ? bal : ~bal;
    }
    return peers;
}

// First pass's digit counts over all keys.
__global__ void __launch_bounds__(kOsThreads)
k_rs_hist0(const unsigned long long* __restrict__ keys, long long n, SortState* ss) {
    __shared__ unsigned cnt[kBins];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    for (long long i = blockIdx.x * (long long)kOsThreads + threadIdx.x; i < n;
         i += (long long)gridDim.x * kOsThreads)
        atomicAdd(&cnt[digit_of(keys[i], 0)], 1u);
    __syncthreads();
    if (cnt[threadIdx.x]) atomicAdd(&ss->ghist[0][threadIdx.x], cnt[threadIdx.x]);
}

// Inclusive warp scan.
__device__ __forceinline__ unsigned warp_incl(unsigned x, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// One pass over one tile of NT * kOsIpt keys (NT threads, NT >= kBins);
// threads 0..255 also act for the 256 digits.
template <bool VALS, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT)
k_rs_pass(const unsigned long long* __restrict__ kin, const uint32_t* __restrict__ vin,
          unsigned long long* __restrict__ kout, uint32_t* __restrict__ vout, long long n,
          int pass, int shift, int next_shift, unsigned long long* status, SortState* ss,
          int* err) {
    constexpr int NW = NT / 32;
    constexpr int TILE = NT * kOsIpt;
    constexpr int DW = kBins / 32;   // warps acting for the digits
    __shared__ unsigned long long skey[TILE];
    __shared__ uint32_t sval[VALS ? TILE : 1];
    __shared__ unsigned short wcnt[NW][kBins];   // per warp, then warp prefix
    __shared__ unsigned s_start[kBins];   // first slot of digit d in the reordered tile
    __shared__ unsigned s_out[kBins];     // output slot of the tile's first key of digit d
    __shared__ unsigned s_next[kBins];    // next pass's digit counts of this tile
    __shared__ unsigned s_wsum[DW], s_bsum[DW];
    __shared__ int s_tile, s_fail;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int d = threadIdx.x;   // the digit a thread acts for (d < kBins)
    if (threadIdx.x == 0) {
        s_tile = atomicAdd(&ss->tile_ctr[pass], 1);
        s_fail = 0;
    }
    for (int i = threadIdx.x; i < NW * kBins; i += NT) (&wcnt[0][0])[i] = 0;
    if (d < kBins) s_next[d] = 0;
    __syncthreads();
    const int tile = s_tile;
    // warp w: keys tile*TILE + w*32*kOsIpt + r*32 + lane, r = 0..kOsIpt-1
    const long long t0 = (long long)tile * TILE + w * (32 * kOsIpt);
    unsigned long long k[kOsIpt];
    uint32_t v[kOsIpt];
    unsigned short rank[kOsIpt];
#pragma unroll
    for (int r = 0; r < kOsIpt; r++) {
        const long long i = t0 + r * 32 + lane;
        k[r] = i < n ? kin[i] : 0ull;
        if (VALS) v[r] = i < n ? vin[i] : 0u;
    }
#pragma unroll
    for (int r = 0; r < kOsIpt; r++) {
        const bool valid = t0 + r * 32 + lane < n;
        const unsigned active = __ballot_sync(0xFFFFFFFFu, valid);
        const unsigned dg = digit_of(k[r], shift);
        const unsigned peers = same_digit_lanes(dg, active);
        const int leader = valid ? __ffs(peers) - 1 : lane;
        unsigned base = 0;
        if (valid && lane == leader) base = wcnt[w][dg];
        base = __shfl_sync(0xFFFFFFFFu, base, leader);
        if (valid) {
            rank[r] = (unsigned short)(base + __popc(peers & ((1u << lane) - 1u)));
            if (lane == leader) wcnt[w][dg] = (unsigned short)(base + __popc(peers));
            if (next_shift >= 0) atomicAdd(&s_next[digit_of(k[r], next_shift)], 1u);
        }
        __syncwarp();
    }
    __syncthreads();
    unsigned cnt = 0, tot = 0, ci = 0, ti = 0;
    unsigned long long excl = 0;
    if (d < kBins) {
        // digit d's count in this tile (warp counts -> warp prefixes)
#pragma unroll
        for (int ww = 0; ww < NW; ww++) {
            const unsigned c = wcnt[ww][d];
            wcnt[ww][d] = (unsigned short)cnt;
            cnt += c;
        }
        // publish the counts now; the look-back for the earlier tiles'
        // counts waits until this tile's keys are reordered, so that the
        // tiles before it have had that long to publish theirs
        *(volatile unsigned long long*)(status + (long long)tile * kBins + d) =
            (tile == 0 ? kFlagIncl : kFlagAgg) | cnt;
        // this tile's digit starts (exclusive scan of cnt over d) and the
        // digits' bases in the output (exclusive scan of the pass histogram)
        tot = ss->ghist[pass][d];
        ci = warp_incl(cnt, lane);
        ti = warp_incl(tot, lane);
        if (lane == 31) {
            s_wsum[w] = ci;
            s_bsum[w] = ti;
        }
    }
    __syncthreads();
    unsigned tpre = 0;
    if (d < kBins) {
        unsigned cpre = 0;
        for (int ww = 0; ww < w; ww++) {
            cpre += s_wsum[ww];
            tpre += s_bsum[ww];
        }
        s_start[d] = cpre + ci - cnt;
    }
    __syncthreads();
    // reorder in shared memory
#pragma unroll
    for (int r = 0; r < kOsIpt; r++) {
        if (t0 + r * 32 + lane < n) {
            const unsigned dd = digit_of(k[r], shift);
            const unsigned at = s_start[dd] + wcnt[w][dd] + rank[r];
            skey[at] = k[r];
            if (VALS) sval[at] = v[r];
        }
    }
    if (d < kBins) {
        bool fail = false;
        if (tile > 0) {
            // kLook statuses read at once (tiles j, j-1, ...), consumed in
            // order up to the first inclusive one, or up to the first that
            // is not ready, which is then polled; tile 0 is always
            // inclusive, so the walk never passes it
            long long j = tile - 1;
            long long polls = 0;
            bool done = false;
            while (!done) {
                unsigned long long sv[kLook];
#pragma unroll
                for (int q = 0; q < kLook; q++)
                    sv[q] = j - q >= 0
                                ? *(volatile const unsigned long long*)(status + (j - q) * kBins + d)
                                : kFlagIncl;
                int q = 0;
                for (; q < kLook; q++) {
                    const unsigned f = (unsigned)(sv[q] >> 62);
                    if (f == 0) break;
                    excl += sv[q] & kValMask;
                    if (f == 2) {
                        done = true;
                        break;
                    }
                }
                if (done) break;
                j -= q;
                if (q < kLook) {   // tile j has not published yet
                    if (++polls > kWaitLimit) {
                        fail = true;
                        break;
                    }
                    __nanosleep(32);
                }
            }
            *(volatile unsigned long long*)(status + (long long)tile * kBins + d) =
                kFlagIncl | (excl + cnt);
        }
        if (fail) s_fail = 1;
        s_out[d] = tpre + ti - tot + (unsigned)excl;
    }
    __syncthreads();
    if (s_fail) {
        if (threadIdx.x == 0) atomicExch(err, HN_ERR_TIMEOUT);
        return;
    }
    const long long rem = n - (long long)tile * TILE;
    const int tile_n = rem < TILE ? (int)rem : TILE;
    for (int j = threadIdx.x; j < tile_n; j += NT) {
        const unsigned long long key = skey[j];
        const unsigned dd = digit_of(key, shift);
        const long long at = (long long)s_out[dd] + (j - (long long)s_start[dd]);
        if (at < n) {   // always: the counts add up to n
            kout[at] = key;
            if (VALS) vout[at] = sval[j];
        }
    }
    if (d < kBins && next_shift >= 0 && s_next[d])
        atomicAdd(&ss->ghist[pass + 1][d], s_next[d]);
}

// SMs of the graph's device, or of the current device without a graph.
int sm_count(const hn_graph* g) {
    if (g) return g->info.sms;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

}  // namespace

// Sorts keys[0, n) by their low `bits` bits, stably, carrying vals (may be
// null).  keys_alt / vals_alt are buffers of the same size; on return keys
// and vals point at the sorted data (the pointers of a pair may have been
// swapped).  A bounded wait that gave up sets *err to HN_ERR_TIMEOUT (the
// keys are then not sorted).  n < 2^32.
void radix_sort_u64(hn_graph* g, unsigned long long*& keys, unsigned long long*& keys_alt,
                    uint32_t*& vals, uint32_t*& vals_alt, long long n, int bits, int* err,
                    cudaStream_t s) {
    if (n <= 1 || bits <= 0) return;
    if (n >= (1ll << 32)) throw Error(HN_ERR_CAPACITY, "radix sort of 2^32 keys or more");
    const int passes = (bits + 7) / 8;
    if (passes > kMaxPasses) throw Error(HN_ERR_INVALID, "radix sort keys wider than 64 bits");
    // keys alone: 512-thread tiles of 4096 keys; with values: 256-thread
    // tiles of 2048 (the values' staging keeps it within static shared memory)
    const int nt = vals ? 256 : 512;
    const long long tile = (long long)nt * kOsIpt;
    const long long ntiles = (n + tile - 1) / tile;
    DevBuf<SortState> ss(1, s);
    DevBuf<unsigned long long> status((size_t)ntiles * kBins, s);
    HN_CUDA(cudaMemsetAsync(ss.get(), 0, sizeof(SortState), s));
    const long long grid0 = std::min<long long>((n + kOsThreads - 1) / kOsThreads,
                                                (long long)sm_count(g) * 8);
    HN_LAUNCH(k_rs_hist0, grid0, kOsThreads, 0, s, keys, n, ss.get());
    for (int p = 0; p < passes; p++) {
        const int shift = 8 * p;
        const int next = p + 1 < passes ? shift + 8 : -1;
        HN_CUDA(cudaMemsetAsync(status.get(), 0, sizeof(unsigned long long) * ntiles * kBins, s));
        if (vals)
            HN_LAUNCH((k_rs_pass<true, 256>), ntiles, 256, 0, s, keys, vals, keys_alt, vals_alt,
                      n, p, shift, next, status.get(), ss.get(), err);
        else
            HN_LAUNCH((k_rs_pass<false, 512>), ntiles, 512, 0, s, keys,
                      (const uint32_t*)nullptr, keys_alt, (uint32_t*)nullptr, n, p, shift, next,
                      status.get(), ss.get(), err);
        std::swap(keys, keys_alt);
        if (vals) std::swap(vals, vals_alt);
    }
}

}  // namespace hn
