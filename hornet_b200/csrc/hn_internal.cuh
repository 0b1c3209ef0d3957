// Internal definitions shared by the sm_100a kernels and the C ABI layer.
//
// Storage model (replaces the reference's per-degree BlockArray pools,
// hornet/include/Core/MemoryManager/BlockArray/BlockArray.i.cuh:111-173):
//   * one device edge pool `pool` of int32 neighbour ids;
//   * a 16-byte vertex record {int64 off; int32 deg; int32 cap} per vertex
//     (cap is a power of two or 0) — the reference keeps
//     {degree, edge_block_ptr, vertex_offset, edges_per_block} in an SoA
//     (hornet/include/Core/Hornet.cuh:90-93);
//   * adjacency lists are kept SORTED at all times, so graph de-duplication
//     and erase locate by binary search and triangle counting needs no
//     re-sort;
//   * blocks of 2^c slots come from per-class device free lists or a bump
//     pointer; blocks with cap >= 4 start on a 16-byte boundary.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <stdexcept>
#include <string>

#include "../../include/hornet_b200.h"
#include "../../include/hornet_b200/detail/MergePathLB.cuh"

namespace hn {

constexpr int kNumClasses = 32;       // block classes 2^0 .. 2^31
constexpr int kInf = 2147483647;      // unreachable BFS distance (TopDown.cu:42)

struct __align__(16) VRec {
    long long off;  // first slot of the vertex's block in the pool
    int deg;        // number of neighbours stored
    int cap;        // block capacity (power of two) or 0 when no block
};
static_assert(sizeof(VRec) == 16, "vertex record must be 16 bytes");

// Device-resident allocator state (one per graph).
struct AllocState {
    unsigned long long bump;        // next never-used slot
    unsigned long long pool_cap;    // slots in the pool
    int fl_count[kNumClasses];      // blocks on each free list
    int need[kNumClasses];          // blocks requested in this update
    int push[kNumClasses];          // blocks released in this update
    int take[kNumClasses];          // requests served from the free list
    int rank[kNumClasses];          // per-class request counter (assign pass)
    int prank[kNumClasses];         // per-class push counter (release pass)
    unsigned long long bump_base[kNumClasses];
    unsigned long long bump_demand; // slots the bump pointer must advance
    int error;                      // HN_ERR_* raised on the device
    int pad;
};

// Host-side exception carrying an HN_ERR_* status.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char* what, const char* file, int line);
#define HN_CUDA(x) ::hn::cuda_check((x), #x, __FILE__, __LINE__)

void set_last_error(const std::string& s);

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------

__host__ __device__ inline int ceil_log2_u64(unsigned long long x) {
    int c = 0;
    while ((1ull << c) < x) c++;
    return c;
}

__device__ __forceinline__ int cap_class(int cap) { return 31 - __clz(cap); }

// Warp-aggregated append: every active lane that passes `pred` receives a
// distinct slot of `counter`.  One atomic per warp (ballot/popc/shfl), the
// same idea as the reference's TwoLevelQueue::insert
// (primitives/Queue/TwoLevelQueue.i.cuh:126-137) written for 32-lane warps.
__device__ __forceinline__ int warp_append(int* counter, bool pred) {
    unsigned mask = __activemask();
    unsigned ballot = __ballot_sync(mask, pred);
    if (!ballot) return -1;
    int leader = __ffs(ballot) - 1;
    int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(ballot));
    base = __shfl_sync(mask, base, leader);
    return pred ? base + __popc(ballot & ((1u << lane) - 1)) : -1;
}

// First index i in [0,n) with a[i] >= x (n when none).
template <typename T>
__device__ __forceinline__ long long lower_bound_dev(const T* a, long long n, T x) {
    long long lo = 0, hi = n;
    while (lo < hi) {
        long long mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// First index i in [0,n) with a[i] > x (n when none).
template <typename T>
__device__ __forceinline__ long long upper_bound_dev(const T* a, long long n, T x) {
    long long lo = 0, hi = n;
    while (lo < hi) {
        long long mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Merge-path load-balancing search (public so user operators share it).
using hornet_b200::detail::LbTile;
using hornet_b200::detail::lb_tile_load;
using hornet_b200::detail::merge_path_items;
using hornet_b200::detail::lb_partition;

}  // namespace hn
