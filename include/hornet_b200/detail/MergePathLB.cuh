// Merge-path load-balancing search shared by the library kernels and the
// header-only operator templates (<hornet_b200/Operator++.cuh>).
//
// The B200 replacement for xlib::binarySearchLB
// (xlib/include/Device/Primitives/impl/BinarySearchLB.i.cuh:227-299), which
// each CTA runs as a global upper_bound of its first item, a staged window of
// the prefix and ITEMS_PER_THREAD sequential (pos, offset) pairs.
#pragma once

#include <cuda_runtime.h>

namespace hornet_b200 {
namespace detail {

// ---------------------------------------------------------------------------
// Merge-path load-balancing search (the B200 replacement for
// xlib::binarySearchLB, xlib/include/Device/Primitives/impl/
// BinarySearchLB.i.cuh:227-299).
//
// Work items [0, total) are split into nseg segments by an exclusive prefix
// `prefix` (prefix[0] = 0, prefix[nseg] = total).  Items and segment ENDS are
// merged into one sequence of total + nseg elements, which is cut into
// equal tiles, so a tile never holds more than TILE segment boundaries even
// when many segments are empty.  The segment ends of a tile are staged in
// shared memory; each thread then finds its own split there and walks its
// ITEMS elements, and the (item -> segment) map is written to shared memory
// so that the operator runs item-striped (coalesced across the warp).
// ---------------------------------------------------------------------------

// Number of items among the first `diag` merged elements.
template <typename P>
__device__ __forceinline__ long long merge_path_items(const P* ends, long long nseg,
                                                      long long total, long long diag) {
    long long lo = diag - nseg > 0 ? diag - nseg : 0;
    long long hi = diag < total ? diag : total;
    while (lo < hi) {
        long long mid = (lo + hi) >> 1;
        // item `mid` precedes boundary ends[diag-1-mid] iff mid < that end
        if ((long long)ends[diag - 1 - mid] > mid) lo = mid + 1; else hi = mid;
    }
    return lo;
}

template <int BLOCK, int ITEMS>
struct LbTile {
    static constexpr int TILE = BLOCK * ITEMS;
    long long ends[TILE + 1];   // staged segment ends of this tile
    int seg[TILE];              // segment (relative to seg0) of each item
    long long item0, seg0;      // first item / first segment of the tile
    long long start0;           // prefix[seg0]: first item of segment seg0
    int nitems, nends;

    // First item of local segment b.
    __device__ __forceinline__ long long seg_start(int b) const {
        return b == 0 ? start0 : ends[b - 1];
    }
};

// Fill `t` for tile `tile_id`.  Must be called by all BLOCK threads.
// Returns the number of items in the tile.
// Split of every tile boundary (one thread each; all searches run in
// parallel with independent loads): splits[t] = items among the first
// t * tile merged elements, t = 0 .. ntiles.  `total` is read from
// prefix[nseg] so the work size may be known only on the device; at most
// max_tiles tiles are described.
template <typename P>
__global__ void lb_partition(const P* __restrict__ prefix, long long nseg, int tile,
                             long long max_tiles, long long* __restrict__ splits) {
    const long long total = (long long)prefix[nseg];
    long long ntiles = (total + nseg + tile - 1) / tile;
    if (ntiles > max_tiles) ntiles = max_tiles;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t <= ntiles;
         t += (long long)gridDim.x * blockDim.x) {
        long long d = t * tile;
        if (d > total + nseg) d = total + nseg;
        splits[t] = merge_path_items(prefix + 1, nseg, total, d);
    }
}

template <int BLOCK, int ITEMS, typename P>
__device__ int lb_tile_load(LbTile<BLOCK, ITEMS>& t, const P* prefix, long long nseg,
                            long long total, long long tile_id,
                            const long long* splits = nullptr, long long split_tiles = 0) {
    constexpr int TILE = BLOCK * ITEMS;
    const P* ends = prefix + 1;
    long long d0 = tile_id * TILE;
    long long d1 = d0 + TILE;
    if (d1 > total + nseg) d1 = total + nseg;
    if (threadIdx.x == 0) {
        // precomputed splits cover tiles [0, split_tiles); beyond them (a
        // work size above the caller's bound) the tile searches for itself
        const bool pre = splits && tile_id < split_tiles;
        long long a0 = pre ? splits[tile_id] : merge_path_items(ends, nseg, total, d0);
        long long a1 = pre ? splits[tile_id + 1] : merge_path_items(ends, nseg, total, d1);
        t.item0 = a0;
        t.seg0 = d0 - a0;
        t.nitems = (int)(a1 - a0);
        t.nends = (int)((d1 - a1) - (d0 - a0));
        t.start0 = (long long)prefix[d0 - a0];
    }
    __syncthreads();
    const long long seg0 = t.seg0;
    const int nends = t.nends;
    // stage ends[seg0 .. seg0+nends] (one extra for the walk's look-ahead)
    for (int i = threadIdx.x; i <= nends; i += BLOCK) {
        long long s = seg0 + i;
        t.ends[i] = s < nseg ? (long long)ends[s] : (long long)total;
    }
    __syncthreads();
    // each thread: its own split inside the tile, then walk ITEMS elements
    const long long item0 = t.item0;
    const int nitems = t.nitems;
    int dl = threadIdx.x * ITEMS;                 // local diagonal
    if (dl < nitems + nends) {
        // local merge path over (items item0.., staged ends)
        int lo = dl - nends > 0 ? dl - nends : 0;
        int hi = dl < nitems ? dl : nitems;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (t.ends[dl - 1 - mid] > item0 + mid) lo = mid + 1; else hi = mid;
        }
        int a = lo, b = dl - lo;
        for (int k = 0; k < ITEMS && a + b < nitems + nends; k++) {
            if (b < nends && t.ends[b] <= item0 + a) {
                b++;
            } else {
                t.seg[a] = b;
                a++;
            }
        }
    }
    __syncthreads();
    return nitems;
}

}  // namespace detail
}  // namespace hornet_b200
