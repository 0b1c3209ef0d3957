// BatchUpdate insert / erase: a fused sort -> dedup -> block (re)allocation
// -> scatter-merge pipeline with sorted adjacency lists.
//
// Reference pipeline (hornet/include/Core/BatchUpdate/BatchUpdate.i.cuh and
// BatchUpdateKernels.cuh): two stable thrust sorts, unique_copy, a
// load-balanced scan of every touched adjacency list for graph duplicates,
// host allocator loops for reallocated vertices, append at old_degree
// (insert) or tail-refill of holes (erase), with >= 6 host round trips.
//
// Here (one host synchronisation per batch, to size the pool):
//   1. pack (src,dst) into one key of 2*key_bits bits; stable LSD radix sort
//      (hn_sort.cu);
//   2. mark: batch / graph duplicates (insert) or per-run deletions
//      (erase) — graph membership by binary search in the SORTED adjacency;
//   3. one scan of packed (kept, source-head) counters gives compacted
//      positions and touched-vertex segments in a single pass;
//   4. plan: per touched vertex the new degree and block class
//      (cap = next power of two, the reference's Vertex::limit());
//   5. host: serve block requests from the per-class free lists, the rest
//      from the bump pointer (largest class first, so blocks >= 4 slots stay
//      16-byte aligned); grow the pool / lists if needed;
//   6. assign blocks (warp-aggregated per-class ranks);
//   7. scatter-merge into the new block: old element A[r] goes to
//      r + |{B < A[r]}|, batch element B[j] to j + |{A <= B[j]}| (insert);
//      for erase a kept A[r] goes to r - |{B <= A[r]}|;
//   8. commit vertex records and push old blocks on their free lists.
// Every touched vertex is rewritten out of place, so no kernel ever reads
// a slot another thread of the same launch writes.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>

#include "hn_graph.cuh"

namespace hn {
namespace {

constexpr int kB = 256;

struct Plan {
    int take[kNumClasses];                    // served from the free list
    int pop_top[kNumClasses];                 // free-list size before pops
    int push_base[kNumClasses];               // free-list size after pops
    unsigned long long bump_base[kNumClasses];
};

__device__ __forceinline__ int pow2_ceil(int d) {
    return d <= 1 ? d : (int)(1u << (32 - __clz(d - 1)));
}

// keys = src << L | dst; ids outside [0,nV) raise HN_ERR_INVALID.
__global__ void k_pack(const int32_t* __restrict__ src, const int32_t* __restrict__ dst,
                       long long n, int nV, int L, unsigned long long* __restrict__ keys,
                       AllocState* st) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        int u = src[i], v = dst[i];
        if (u < 0 || u >= nV || v < 0 || v >= nV) {
            atomicExch(&st->error, HN_ERR_INVALID);
            u = 0;
            v = 0;
        }
        keys[i] = ((unsigned long long)(unsigned)u << L) | (unsigned)v;
    }
}

// Insert marking.  Packed counter value per element: (head << 32) | keep.
//   keep = (first-of-run || !DEDUP_BATCH) && !(DEDUP_GRAPH && first-of-run
//          && (u,x) already in the graph)
// which is the reference's behaviour: remove_batch_duplicates keeps the
// first of each run (thrust::unique_copy) and mark_duplicate_edges clears the
// flag of the FIRST batch entry equal to each graph edge
// (BatchUpdateKernels.cuh:27-58 with xlib lower_bound_left).
//
// apos[i] = the number of old-list entries <= x, so that a kept entry's
// place in the merged list (its rank among the kept batch entries of its
// vertex + apos) is known before any old list is rewritten in place.
__global__ void k_mark_insert(const unsigned long long* __restrict__ keys, long long n, int L,
                              unsigned flags, const VRec* __restrict__ vtab,
                              const int32_t* __restrict__ pool,
                              unsigned long long* __restrict__ val, int32_t* __restrict__ apos,
                              const AllocState* st) {
    const unsigned long long mask = (1ull << L) - 1;
    const bool failed = st->error != 0;   // bad ids or a failed sort: the batch is refused
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (failed) {
            val[i] = 0;
            continue;
        }
        unsigned long long k = keys[i];
        unsigned long long kp = i ? keys[i - 1] : ~0ull;
        bool first = (i == 0) || (k != kp);
        bool head = (i == 0) || ((k >> L) != (kp >> L));
        bool keep = first || !(flags & HN_DEDUP_BATCH);
        if (keep) {
            int u = (int)(k >> L);
            int x = (int)(k & mask);
            VRec r = vtab[u];
            const int32_t* a = pool + r.off;
            const long long ub = upper_bound_dev(a, (long long)r.deg, x);
            if (first && (flags & HN_DEDUP_GRAPH) && ub > 0 && a[ub - 1] == x) keep = false;
            apos[i] = (int32_t)ub;
        }
        val[i] = ((unsigned long long)head << 32) | (unsigned long long)keep;
    }
}

// Erase marking: element i of a run of equal (u,x) deletes a copy iff its
// rank in the run (after batch de-duplication) is below the graph
// multiplicity c_g, so each run removes min(c_b, c_g) copies
// (BatchUpdateKernels.cuh:263-300, :335-393).  apos[i] = the old list's
// entries below x.
__global__ void k_mark_erase(const unsigned long long* __restrict__ keys, long long n, int L,
                             unsigned flags, const VRec* __restrict__ vtab,
                             const int32_t* __restrict__ pool,
                             unsigned long long* __restrict__ val, int32_t* __restrict__ apos,
                             const AllocState* st) {
    const unsigned long long mask = (1ull << L) - 1;
    const bool failed = st->error != 0;   // bad ids or a failed sort: the batch is refused
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (failed) {
            val[i] = 0;
            continue;
        }
        unsigned long long k = keys[i];
        unsigned long long kp = i ? keys[i - 1] : ~0ull;
        bool first = (i == 0) || (k != kp);
        bool head = (i == 0) || ((k >> L) != (kp >> L));
        bool del = false;
        if (first || !(flags & HN_DEDUP_BATCH)) {
            // rank inside the run of equal keys
            long long rank = 0;
            if (!first) rank = i - lower_bound_dev(keys, i, k);
            int u = (int)(k >> L);
            int x = (int)(k & mask);
            VRec r = vtab[u];
            const int32_t* a = pool + r.off;
            long long lo = lower_bound_dev(a, (long long)r.deg, x);
            long long cg = 0;
            if (lo < r.deg && a[lo] == x) cg = upper_bound_dev(a, (long long)r.deg, x) - lo;
            del = rank < cg;
            apos[i] = (int32_t)lo;   // the old list's first copy of x
        }
        val[i] = ((unsigned long long)head << 32) | (unsigned long long)del;
    }
}

// Compaction + segments from the exclusive scan of the packed counters.
//   kept element i  -> cdst[pos], cseg[pos]
//   head element i  -> seg_u[seg], seg_kstart[seg]
// Totals go to d_scalar[0] (kept) and d_scalar[1] (segments).
__global__ void k_compact(const unsigned long long* __restrict__ keys,
                          const unsigned long long* __restrict__ val,
                          const unsigned long long* __restrict__ scan, long long n, int L,
                          int32_t* __restrict__ cdst, int32_t* __restrict__ cseg,
                          int32_t* __restrict__ seg_u, int32_t* __restrict__ seg_kstart,
                          long long* __restrict__ totals, const uint32_t* __restrict__ wsorted,
                          uint32_t* __restrict__ cw, const int32_t* __restrict__ apos,
                          int32_t* __restrict__ capos) {
    const unsigned long long mask = (1ull << L) - 1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        unsigned long long v = val[i], s = scan[i];
        long long pos = (long long)(s & 0xFFFFFFFFull);
        long long seg = (long long)(s >> 32) + (long long)(v >> 32) - 1;  // inclusive heads - 1
        unsigned long long k = keys[i];
        if (v >> 32) {
            seg_u[seg] = (int)(k >> L);
            seg_kstart[seg] = (int)pos;
        }
        if (v & 1) {
            cdst[pos] = (int)(k & mask);
            cseg[pos] = (int)seg;
            if (cw) cw[pos] = wsorted[i];
            if (capos) capos[pos] = apos[i];
        }
        if (i == n - 1) {
            long long kept = pos + (long long)(v & 1);
            long long nseg = seg + 1;
            totals[0] = kept;
            totals[1] = nseg;
            seg_kstart[nseg] = (int)kept;
        }
    }
}

// Per touched vertex: new degree / class; request and release counts.
// A vertex whose block class does not change (pow2_ceil of the new degree
// equals its capacity, the reference's Vertex::limit() test,
// BatchUpdateKernels.cuh:150-198) is updated in place (seg_ncap = kInPlace):
// only the part of its list from the first entry that moves, [base, deg),
// is rewritten (insert: base = the old entries <= the smallest batch entry;
// erase: base = the old entries below the smallest deleted one); a list
// moved by the tiles only when that part has at most kInPlaceMax entries,
// so that one warp can stage it, a hub only when it has at most kHubSnap
// batch entries (the slots snapshotted per chunk boundary).  Other vertices move to a new block (seg_ncap = new capacity, 0 for
// an emptied list, -1 for a vertex without batch entries) and their whole
// list is the work.  seg_work[s] = entries the scatter moves (0 for hubs,
// which k_scatter_big moves).  The per-class counts are gathered in shared
// memory and added once per CTA (a global atomic per segment serialises on
// the few popular classes).
constexpr int kInPlace = -2;
constexpr int kInPlaceMax = 2048;
constexpr int kBigChunk = 4096;       // hub lists move in chunks of this many entries
constexpr int kHubSnap = 256;         // most batch entries of a hub updated in place

__global__ void __launch_bounds__(kB)
k_plan(const int32_t* __restrict__ seg_u, const int32_t* __restrict__ seg_kstart,
       const long long* __restrict__ totals, bool insert, const VRec* __restrict__ vtab,
       const int32_t* __restrict__ capos, bool in_place,
       long long* __restrict__ seg_work, int32_t* __restrict__ seg_ncap,
       int32_t* __restrict__ seg_base, long long* __restrict__ seg_old_off, AllocState* st,
       int big_min, int32_t* __restrict__ big_list, int* __restrict__ nbig,
       unsigned long long* __restrict__ snap_words) {
    __shared__ int s_need[kNumClasses], s_push[kNumClasses];
    for (int c = threadIdx.x; c < kNumClasses; c += blockDim.x) s_need[c] = s_push[c] = 0;
    __syncthreads();
    long long nseg = totals[1];
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s <= nseg;
         s += (long long)gridDim.x * blockDim.x) {
        if (s == nseg) { seg_work[s] = 0; continue; }
        const int k0 = seg_kstart[s];
        int k = seg_kstart[s + 1] - k0;
        int u = seg_u[s];
        VRec r = vtab[u];
        int ncap = -1;  // -1: vertex unchanged
        int base = 0;
        // long old lists (hubs) are moved by k_scatter_big, not by the tiles
        const bool big = k > 0 && r.deg >= big_min;
        if (k > 0) {
            int nd = insert ? r.deg + k : r.deg - k;
            ncap = pow2_ceil(nd);
            bool here = in_place && nd > 0 && ncap == r.cap && (!big || k <= kHubSnap);
            if (here) {
                // the smallest batch entry's place in the old list, recorded
                // at marking
                base = capos[k0];
                if (big) {
                    // hub chunk boundaries inside the moved part keep k
                    // slots each in the snapshot
                    const int nch = (r.deg - base + kBigChunk - 1) / kBigChunk;
                    if (nch > 1) atomicAdd(snap_words, (unsigned long long)(nch - 1) * k);
                } else {
                    here = r.deg - base <= kInPlaceMax;
                }
            }
            if (here) {
                ncap = kInPlace;
            } else {
                base = 0;
                if (ncap > 0) atomicAdd(&s_need[cap_class(ncap)], 1);
                if (r.cap > 0) atomicAdd(&s_push[cap_class(r.cap)], 1);
            }
        }
        seg_ncap[s] = ncap;
        seg_base[s] = base;
        seg_work[s] = k > 0 && !big ? r.deg - base : 0;
        seg_old_off[s] = r.off;   // the scatter reads it without the seg_u -> vtab chain
        const int at = warp_append(nbig, big);
        if (big) big_list[at] = (int)s;
    }
    __syncthreads();
    for (int c = threadIdx.x; c < kNumClasses; c += blockDim.x) {
        if (s_need[c]) atomicAdd(&st->need[c], s_need[c]);
        if (s_push[c]) atomicAdd(&st->push[c], s_push[c]);
    }
}

// Contiguous range of segments owned by this CTA.
__device__ __forceinline__ void cta_range(long long n, long long& s0, long long& s1) {
    const long long per = (n + gridDim.x - 1) / gridDim.x;
    s0 = (long long)blockIdx.x * per;
    s1 = s0 + per < n ? s0 + per : n;
}

// Block assignment: per class, the first take[c] requests pop the free list,
// the rest are carved from the bump region of the class.  Each CTA counts
// its range's requests per class, reserves its ranks with one atomic per
// class, then hands them out with shared atomics.
__global__ void __launch_bounds__(kB)
k_assign(const int32_t* __restrict__ seg_ncap, long long nseg, Plan plan,
         long long* const* __restrict__ fl, AllocState* st,
         const long long* __restrict__ seg_old_off, long long* __restrict__ seg_new_off) {
    __shared__ int s_cnt[kNumClasses], s_base[kNumClasses];
    for (int c = threadIdx.x; c < kNumClasses; c += blockDim.x) s_cnt[c] = 0;
    __syncthreads();
    long long s0, s1;
    cta_range(nseg, s0, s1);
    for (long long s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        int ncap = seg_ncap[s];
        if (ncap > 0) atomicAdd(&s_cnt[cap_class(ncap)], 1);
    }
    __syncthreads();
    for (int c = threadIdx.x; c < kNumClasses; c += blockDim.x) {
        s_base[c] = s_cnt[c] ? atomicAdd(&st->rank[c], s_cnt[c]) : 0;
        s_cnt[c] = 0;
    }
    __syncthreads();
    for (long long s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        int ncap = seg_ncap[s];
        long long off = ncap == kInPlace ? seg_old_off[s] : 0;
        if (ncap > 0) {
            int c = cap_class(ncap);
            int r = s_base[c] + atomicAdd(&s_cnt[c], 1);
            if (r < plan.take[c]) off = fl[c][plan.pop_top[c] - 1 - r];
            else off = (long long)(plan.bump_base[c] +
                                   ((unsigned long long)(r - plan.take[c]) << c));
        }
        seg_new_off[s] = off;
    }
}

// Scatter tiles: 256 threads x 4 items, five CTAs per SM (the shared-memory
// limit of a tile).  128 x 8, 128 x 4 (ten per SM) and 256 x 2 (eight per
// SM) measured 13-52 % slower on the 10M-edge batch.
constexpr int kSB = 256;
constexpr int kScatterCtas = 5;
using Tile = LbTile<kSB, 4>;
constexpr int kStage = 512;    // batch entries of a tile staged in shared memory

__device__ __forceinline__ int lower_bound32(const int32_t* a, int n, int32_t x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ int upper_bound32(const int32_t* a, int n, int32_t x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Old adjacency of every changed vertex -> its place in the new block, or
// in its own block for a vertex updated in place (only its entries from
// seg_base on are work items).  The batch entries the tile's segments search
// are one contiguous run of cdst (the segments are consecutive sources and
// cdst is sorted by source): when the run has at most kStage entries it is
// staged in shared memory, so the per-item searches do not wait on global
// loads.
//
// In place, an entry's new slot may be another entry's old slot, so every
// item's value and destination are read and computed before the barrier
// and stored after it.  That orders the reads before the writes within the
// CTA; a vertex updated in place whose items span two tiles (two CTAs)
// would not be ordered, so the tiles leave it alone and the tile holding
// its first item lists it for k_inplace_span, which moves it whole.
template <bool INSERT>
__global__ void __launch_bounds__(kSB, kScatterCtas)
k_scatter_old(const long long* __restrict__ prefix, long long nseg,
              const int32_t* __restrict__ seg_u, const int32_t* __restrict__ seg_kstart,
              const long long* __restrict__ seg_new_off, const int32_t* __restrict__ cdst,
              const long long* __restrict__ seg_old_off, const int32_t* __restrict__ seg_ncap,
              const int32_t* __restrict__ seg_base, int32_t* __restrict__ pool,
              const long long* __restrict__ splits, long long split_tiles,
              uint32_t* __restrict__ wpool, int32_t* __restrict__ span_list,
              int* __restrict__ nspan, long long span_cap) {
    __shared__ Tile t;
    __shared__ long long s_old[Tile::TILE + 1];   // old slot of item e: s_old[b] + e
    __shared__ long long s_new[Tile::TILE + 1];   // slot before the batch shift: s_new[b] + e
    __shared__ int s_k0[Tile::TILE + 1];   // the batch list of segment b, narrowed to
    __shared__ int s_k1[Tile::TILE + 1];   // the old values this tile holds: [k0, k1)
    __shared__ int s_kb[Tile::TILE + 1];   // batch entries of the segment before k0
    __shared__ int32_t s_cd[kStage];       // cdst[K0, K1) of this tile
    __shared__ int s_K0, s_K1;
    const long long total = prefix[nseg];
    long long ntiles = (total + nseg + Tile::TILE - 1) / Tile::TILE;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        if (threadIdx.x == 0) {   // the previous tile ended with a barrier
            s_K0 = INT_MAX;
            s_K1 = INT_MIN;
        }
        int n = lb_tile_load(t, prefix, nseg, total, tile, splits, split_tiles);
        for (int b = threadIdx.x; b <= t.nends; b += kSB) {
            long long s = t.seg0 + b;
            s_k0[b] = 0;
            s_k1[b] = -1;   // marks a segment this tile does not move
            if (s < nseg) {
                const long long st0 = t.seg_start(b);
                const long long en = t.ends[b], tend = t.item0 + n;
                if (seg_ncap[s] == kInPlace && (st0 < t.item0 || en > tend)) {
                    // in place and spanning tiles: listed once, by the tile
                    // holding its first item
                    if (st0 >= t.item0 && st0 < tend) {
                        // one vertex per tile boundary at most, so the
                        // list (one entry per tile) never fills
                        const int at = atomicAdd(nspan, 1);
                        if (at < span_cap) span_list[at] = (int)s;
                    }
                    continue;
                }
                const int base = seg_base[s];
                const long long old_off = seg_old_off[s] + base;
                s_old[b] = old_off - st0;
                s_new[b] = seg_new_off[s] + base - st0;
                const int k0 = seg_kstart[s], k1 = seg_kstart[s + 1];
                // a segment with a long batch list (a hub hit by many
                // updates) searches only the batch entries that can fall
                // between this tile's first and last old value; short lists
                // are searched whole
                const long long lo_e = st0 > t.item0 ? st0 : t.item0;
                const long long hi_e = en < tend ? en : tend;
                int blo = 0, bhi = k1 - k0;
                if (lo_e < hi_e && k1 - k0 > 8) {   // short batch lists: searched whole
                    const int32_t a_lo = pool[old_off + (lo_e - st0)];
                    const int32_t a_hi = pool[old_off + (hi_e - 1 - st0)];
                    blo = (int)lower_bound_dev(cdst + k0, (long long)(k1 - k0), a_lo);
                    bhi = (int)upper_bound_dev(cdst + k0, (long long)(k1 - k0), a_hi);
                }
                s_k0[b] = k0 + blo;
                s_k1[b] = k0 + bhi;
                s_kb[b] = blo;
                if (bhi > blo) {
                    atomicMin(&s_K0, k0 + blo);
                    atomicMax(&s_K1, k0 + bhi);
                }
            }
        }
        __syncthreads();
        // all of this thread's old-list loads first (the pool is both read
        // and written here, so a plain loop would wait for each store)
        constexpr int IPT = Tile::TILE / kSB;
        int xs[IPT], bs[IPT];
        uint32_t ws[IPT];
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            const int i = threadIdx.x + k * kSB;
            bs[k] = -1;
            ws[k] = 0;
            if (i < n) {
                const int b = t.seg[i];
                if (s_k1[b] >= s_k0[b]) {
                    bs[k] = b;
                    xs[k] = pool[s_old[b] + t.item0 + i];
                    if (wpool) ws[k] = wpool[s_old[b] + t.item0 + i];
                }
            }
        }
        // stage the tile's batch run while those loads are in flight
        const int K0 = s_K0, K1 = s_K1;
        const bool staged = K1 > K0 && K1 - K0 <= kStage;   // uniform in the CTA
        if (staged) {
            for (int i = threadIdx.x; i < K1 - K0; i += kSB) s_cd[i] = cdst[K0 + i];
            __syncthreads();
        }
        long long to[IPT];   // destination slot, -1 = the entry is deleted
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            to[k] = -1;
            if (bs[k] < 0) continue;
            const int b = bs[k];
            const int x = xs[k];
            const long long e = t.item0 + threadIdx.x + k * kSB;   // global item
            const int nb = s_k1[b] - s_k0[b];
            // read only when nb > 0, and then [s_k0[b], s_k1[b]) lies in [K0, K1)
            const int32_t* B = staged ? s_cd + (s_k0[b] - K0) : cdst + s_k0[b];
            if (INSERT) {
                to[k] = s_new[b] + e + s_kb[b] + lower_bound32(B, nb, x);
            } else {
                // every batch copy of x lies inside the narrowed range
                // batch entries below x, then its copies (few): one search
                const long long lbl = lower_bound32(B, nb, x);
                long long ubl = lbl;
                while (ubl < nb && B[ubl] == x) ubl++;
                long long cnt = ubl - lbl;  // copies of x to delete
                bool keep = true;
                if (cnt > 0) {
                    // rank of this copy among equal values of the old list
                    // (the entries before seg_base are all below x)
                    long long r = e - t.seg_start(b);
                    const int32_t* A = pool + s_old[b] + t.seg_start(b);
                    long long first = r;
                    if (r > 0 && A[r - 1] == x) first = lower_bound_dev(A, r, x);
                    keep = (r - first) >= cnt;
                }
                if (keep) to[k] = s_new[b] + e - (s_kb[b] + ubl);
            }
        }
        __syncthreads();   // every read of this tile's lists before any write
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            if (to[k] < 0) continue;
            pool[to[k]] = xs[k];
            if (wpool) wpool[to[k]] = ws[k];
        }
        __syncthreads();
    }
}

// Vertices updated in place whose moved entries span two or more scatter
// tiles: a warp each stages the moved part [base, deg) (at most kInPlaceMax
// entries) in shared memory, then writes every entry to its new slot, so
// all reads precede all writes.  Same slot rules as k_scatter_old.
constexpr int kSpanWarps = 4;

template <bool INSERT>
__global__ void __launch_bounds__(kSpanWarps * 32)
k_inplace_span(const int32_t* __restrict__ span_list, const int* __restrict__ nspan,
               const int32_t* __restrict__ seg_u, const int32_t* __restrict__ seg_kstart,
               const int32_t* __restrict__ seg_base, const long long* __restrict__ seg_old_off,
               const int32_t* __restrict__ cdst, const VRec* __restrict__ vtab,
               int32_t* __restrict__ pool, long long span_cap) {
    __shared__ int32_t sA[kSpanWarps][kInPlaceMax];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int32_t* A = sA[w];
    const int count = *nspan < span_cap ? *nspan : (int)span_cap;
    for (int i = blockIdx.x * kSpanWarps + w; i < count; i += gridDim.x * kSpanWarps) {
        const int s = span_list[i];
        const int base = seg_base[s];
        const int n = vtab[seg_u[s]].deg - base;   // the old degree: commit runs later
        const long long off = seg_old_off[s] + base;
        for (int j = lane; j < n; j += 32) A[j] = pool[off + j];
        __syncwarp();
        const int k0 = seg_kstart[s], nb = seg_kstart[s + 1] - k0;
        const int32_t* B = cdst + k0;
        for (int j = lane; j < n; j += 32) {
            const int32_t x = A[j];
            if (INSERT) {
                pool[off + j + lower_bound32(B, nb, x)] = x;
            } else {
                const int lbl = lower_bound32(B, nb, x);
                int ubl = lbl;
                while (ubl < nb && B[ubl] == x) ubl++;
                bool keep = true;
                if (ubl > lbl) {
                    int first = j;
                    if (j > 0 && A[j - 1] == x) first = lower_bound32(A, j, x);
                    keep = (j - first) >= ubl - lbl;
                }
                if (keep) pool[off + j - ubl] = x;
            }
        }
        __syncwarp();   // A is restaged for the next vertex
    }
}

// Old lists of at least update.big_min entries (hubs), in chunks of
// kBigChunk entries.  A chunk that no batch entry falls inside keeps one
// shift for all its entries (insert: + the batch entries below it; erase:
// - the deleted entries below it), so it is moved as a block: 16-byte
// loads into shared memory, 16-byte stores at the shifted place (scalar
// stores at the unaligned ends).  A chunk with batch entries inside places
// each entry by the merge rule, with the batch entries it needs staged in
// shared memory.  The hubs' chunks are numbered through an exclusive scan
// of their chunk counts, and CTAs take chunk numbers round-robin.
//
// A hub whose block class stays and that has at most kHubSnap batch entries
// is updated in place, its chunks covering only the moved part [base, deg).
// A chunk stages all its entries in shared memory before it writes, but a
// neighbouring chunk (another CTA) may write into its range first: on an
// insert an entry moves right by at most k (the hub's batch entries), so
// chunk c writes into at most the first k slots of chunk c+1; on an erase
// it moves left by at most k, into the last k slots of chunk c-1.  Those k
// slots of every chunk boundary are copied to a snapshot (k_big_snap)
// before any chunk moves, and the chunk whose slots they are reads them
// from there.  The erase rule for equal entries uses the old list's first
// copy of the value, recorded at marking, instead of reading old slots
// that may already be overwritten.  Packed per-hub prefix (chunk_pre):
// high 32 bits chunks, low 32 bits snapshot slots.

struct BigHub {   // one hub as the chunk kernels see it
    long long old_off, new_off;
    int deg, k0, nb, base, nch;
    bool in_place;
};

__device__ __forceinline__ BigHub big_hub(int sg, const int32_t* seg_u, const int32_t* seg_kstart,
                                          const int32_t* seg_ncap, const int32_t* seg_base,
                                          const long long* seg_old_off,
                                          const long long* seg_new_off, const VRec* vtab) {
    BigHub h;
    h.deg = vtab[seg_u[sg]].deg;   // the old degree: the commit runs later
    h.k0 = seg_kstart[sg];
    h.nb = seg_kstart[sg + 1] - h.k0;
    h.in_place = seg_ncap[sg] == kInPlace;
    h.base = h.in_place ? seg_base[sg] : 0;
    h.old_off = seg_old_off[sg];
    h.new_off = seg_new_off[sg];
    h.nch = (h.deg - h.base + kBigChunk - 1) / kBigChunk;
    return h;
}

__global__ void k_big_chunks(const int32_t* __restrict__ big_list, int nbig,
                             const int32_t* __restrict__ seg_u,
                             const int32_t* __restrict__ seg_kstart,
                             const int32_t* __restrict__ seg_ncap,
                             const int32_t* __restrict__ seg_base,
                             const long long* __restrict__ seg_old_off,
                             const long long* __restrict__ seg_new_off,
                             const VRec* __restrict__ vtab, unsigned long long* __restrict__ pre) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= nbig; i += gridDim.x * blockDim.x) {
        unsigned long long v = 0;
        if (i < nbig) {
            const BigHub h = big_hub(big_list[i], seg_u, seg_kstart, seg_ncap, seg_base,
                                     seg_old_off, seg_new_off, vtab);
            const unsigned long long snaps =
                h.in_place && h.nch > 1 ? (unsigned long long)(h.nch - 1) * h.nb : 0;
            v = ((unsigned long long)h.nch << 32) | snaps;
        }
        pre[i] = v;
    }
}

// The hub and chunk of global chunk number q: last i with pre[i].chunks <= q.
__device__ __forceinline__ int big_hub_of(const unsigned long long* pre, int nbig, int q) {
    int lo = 0, hi = nbig;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if ((int)(pre[mid] >> 32) <= q) lo = mid; else hi = mid;
    }
    return lo;
}

// Snapshot of every in-place hub's chunk boundaries: boundary c (between
// chunks c and c+1, at old slot r1 = base + (c+1) * kBigChunk) keeps k slots:
// insert [r1, r1 + k) clipped to the list, erase [r1 - k, r1).
template <bool INSERT>
__global__ void k_big_snap(const int32_t* __restrict__ big_list, int nbig,
                           const int32_t* __restrict__ seg_u,
                           const int32_t* __restrict__ seg_kstart,
                           const int32_t* __restrict__ seg_ncap,
                           const int32_t* __restrict__ seg_base,
                           const long long* __restrict__ seg_old_off,
                           const long long* __restrict__ seg_new_off,
                           const VRec* __restrict__ vtab, const unsigned long long* __restrict__ pre,
                           const int32_t* __restrict__ pool, int32_t* __restrict__ snap) {
    // a thread per chunk: a boundary keeps only k (<= kHubSnap) slots
    const int total = (int)(pre[nbig] >> 32);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x) {
        const int i = big_hub_of(pre, nbig, q);
        const int c = q - (int)(pre[i] >> 32);
        const BigHub h = big_hub(big_list[i], seg_u, seg_kstart, seg_ncap, seg_base, seg_old_off,
                                 seg_new_off, vtab);
        if (!h.in_place || c + 1 >= h.nch) continue;   // no boundary after this chunk
        const long long r1 = (long long)h.base + (long long)(c + 1) * kBigChunk;
        int32_t* out = snap + (pre[i] & 0xFFFFFFFFull) + (long long)c * h.nb;
        for (int t = 0; t < h.nb; t++) {
            const long long r = INSERT ? r1 + t : r1 - h.nb + t;
            if (r < h.deg) out[t] = pool[h.old_off + r];
        }
    }
}

template <bool INSERT>
__global__ void __launch_bounds__(kSB)
k_scatter_big(const int32_t* __restrict__ big_list, int nbig, const int32_t* __restrict__ seg_u,
              const int32_t* __restrict__ seg_kstart, const int32_t* __restrict__ seg_ncap,
              const int32_t* __restrict__ seg_base, const long long* __restrict__ seg_old_off,
              const long long* __restrict__ seg_new_off, const int32_t* __restrict__ cdst,
              const int32_t* __restrict__ capos, const VRec* __restrict__ vtab,
              int32_t* __restrict__ pool, const unsigned long long* __restrict__ pre,
              const int32_t* __restrict__ snap) {
    __shared__ __align__(16) int32_t sA[kBigChunk];   // the chunk's old entries
    __shared__ int32_t sB[kBigChunk];                 // the batch entries inside it
    const int total = (int)(pre[nbig] >> 32);
    for (int q = blockIdx.x; q < total; q += gridDim.x) {
        const int i = big_hub_of(pre, nbig, q);   // uniform in the CTA
        const int c = q - (int)(pre[i] >> 32);
        const BigHub h = big_hub(big_list[i], seg_u, seg_kstart, seg_ncap, seg_base,
                                 seg_old_off, seg_new_off, vtab);
        const int32_t* B = cdst + h.k0;
        const int32_t* A = pool + h.old_off;
        const int r0 = h.base + c * kBigChunk;
        const int n = h.deg - r0 < kBigChunk ? h.deg - r0 : kBigChunk;
        // stage the chunk (in place: the slots a neighbour may overwrite
        // come from the snapshot)
        int snap_lo = 0, snap_hi = 0;   // chunk-relative slots read from snap
        const int32_t* sn = nullptr;
        if (h.in_place) {
            const long long sbase = (long long)(pre[i] & 0xFFFFFFFFull);
            if (INSERT && c > 0) {
                snap_hi = h.nb < n ? h.nb : n;
                sn = snap + sbase + (long long)(c - 1) * h.nb;
            } else if (!INSERT && c + 1 < h.nch) {
                snap_lo = n - h.nb;
                snap_hi = n;
                sn = snap + sbase + (long long)c * h.nb - snap_lo;
            }
        }
        if ((((h.old_off + r0) & 3) == 0)) {
            const int4* a4 = reinterpret_cast<const int4*>(A + r0);
            for (int v = threadIdx.x; v < n / 4; v += kSB)
                reinterpret_cast<int4*>(sA)[v] = __ldcs(a4 + v);
            for (int v = (n & ~3) + threadIdx.x; v < n; v += kSB) sA[v] = A[r0 + v];
        } else {
            for (int v = threadIdx.x; v < n; v += kSB) sA[v] = A[r0 + v];
        }
        __syncthreads();
        for (int v = snap_lo + threadIdx.x; v < snap_hi; v += kSB) sA[v] = sn[v];
        __syncthreads();
        const int lo = lower_bound32(B, h.nb, sA[0]);       // batch entries below the chunk
        const int hi = upper_bound32(B, h.nb, sA[n - 1]);   // ... and up to its last entry
        const long long out0 = h.new_off + r0;             // the chunk's slot before the shift
        if (lo == hi) {
            // one shift for the whole chunk
            const long long d0 = out0 + (INSERT ? lo : -lo);
            const int lead = (int)((4 - (d0 & 3)) & 3) < n ? (int)((4 - (d0 & 3)) & 3) : n;
            if (threadIdx.x < lead) pool[d0 + threadIdx.x] = sA[threadIdx.x];
            const int nq = (n - lead) / 4;
            int4* o4 = reinterpret_cast<int4*>(pool + d0 + lead);
            for (int t = threadIdx.x; t < nq; t += kSB) {
                const int b = lead + 4 * t;
                o4[t] = make_int4(sA[b], sA[b + 1], sA[b + 2], sA[b + 3]);
            }
            for (int v = lead + 4 * nq + threadIdx.x; v < n; v += kSB) pool[d0 + v] = sA[v];
        } else {
            // batch entries inside the chunk: the merge rule on [lo, hi),
            // searched in shared memory when they fit there
            const int m = hi - lo;
            const bool staged = m <= kBigChunk;   // uniform in the CTA
            if (staged)
                for (int v = threadIdx.x; v < m; v += kSB) sB[v] = B[lo + v];
            __syncthreads();
            const int32_t* Bn = staged ? sB : B + lo;
            for (int v = threadIdx.x; v < n; v += kSB) {
                const int32_t x = sA[v];
                const long long r = (long long)r0 + v;   // old slot in the list
                if (INSERT) {
                    pool[h.new_off + r + lo + lower_bound32(Bn, m, x)] = x;
                } else {
                    const int lbl = lower_bound32(Bn, m, x);
                    int ubl = lbl;
                    while (ubl < m && Bn[ubl] == x) ubl++;
                    const int cnt = ubl - lbl;   // copies of x this batch deletes
                    // the first cnt copies of x go: keep this one if its rank
                    // among the old copies (from the first copy's slot,
                    // recorded at marking) is at least cnt
                    const bool keep = cnt == 0 || r - capos[h.k0 + lo + lbl] >= cnt;
                    if (keep) pool[h.new_off + r - (lo + ubl)] = x;
                }
            }
        }
        __syncthreads();   // sA / sB are restaged by the next chunk
    }
}

// Batch edges -> their slot in the merged list (insert only; after the old
// entries have moved): rank among the vertex's kept batch entries + the old
// entries <= it (capos, recorded at marking before any list moved).
__global__ void k_scatter_new(const int32_t* __restrict__ cdst, const int32_t* __restrict__ cseg,
                              const int32_t* __restrict__ capos,
                              const long long* __restrict__ totals,
                              const int32_t* __restrict__ seg_kstart,
                              const long long* __restrict__ seg_new_off,
                              int32_t* __restrict__ pool,
                              const uint32_t* __restrict__ cw, uint32_t* __restrict__ wpool) {
    long long kept = totals[0];
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < kept;
         p += (long long)gridDim.x * blockDim.x) {
        const int s = cseg[p];
        const long long at = seg_new_off[s] + (p - seg_kstart[s]) + capos[p];
        pool[at] = cdst[p];
        if (wpool) wpool[at] = cw ? cw[p] : 0u;
    }
}

// New vertex records; old blocks pushed on their class free list (ranks
// reserved per CTA and class, as in k_assign).
__global__ void __launch_bounds__(kB)
k_commit(const int32_t* __restrict__ seg_u, const int32_t* __restrict__ seg_kstart,
         const int32_t* __restrict__ seg_ncap, const long long* __restrict__ seg_new_off,
         long long nseg, bool insert, Plan plan, long long* const* __restrict__ fl,
         AllocState* st, VRec* __restrict__ vtab) {
    __shared__ int s_cnt[kNumClasses], s_base[kNumClasses];
    for (int c = threadIdx.x; c < kNumClasses; c += blockDim.x) s_cnt[c] = 0;
    __syncthreads();
    long long s0, s1;
    cta_range(nseg, s0, s1);
    for (long long s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        if (seg_ncap[s] < 0) continue;   // unchanged or in place: no block released
        int cap = vtab[seg_u[s]].cap;
        if (cap > 0) atomicAdd(&s_cnt[cap_class(cap)], 1);
    }
    __syncthreads();
    for (int c = threadIdx.x; c < kNumClasses; c += blockDim.x) {
        s_base[c] = s_cnt[c] ? atomicAdd(&st->prank[c], s_cnt[c]) : 0;
        s_cnt[c] = 0;
    }
    __syncthreads();
    for (long long s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        int ncap = seg_ncap[s];
        if (ncap == kInPlace) {
            const int u = seg_u[s];
            const int k = seg_kstart[s + 1] - seg_kstart[s];
            vtab[u].deg += insert ? k : -k;
            continue;
        }
        if (ncap < 0) continue;
        int u = seg_u[s];
        int k = seg_kstart[s + 1] - seg_kstart[s];
        VRec r = vtab[u];
        if (r.cap > 0) {
            int c = cap_class(r.cap);
            int p = s_base[c] + atomicAdd(&s_cnt[c], 1);
            fl[c][plan.push_base[c] + p] = r.off;
        }
        VRec nr;
        nr.deg = insert ? r.deg + k : r.deg - k;
        nr.cap = ncap;
        nr.off = ncap > 0 ? seg_new_off[s] : 0;
        vtab[u] = nr;
    }
}

// Keys (src << L | dst) of the edges an insert actually added, ascending.
__global__ void k_new_keys(const int32_t* __restrict__ cdst, const int32_t* __restrict__ cseg,
                           const int32_t* __restrict__ seg_u, long long kept, int L,
                           unsigned long long* __restrict__ nkeys) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < kept;
         i += (long long)gridDim.x * blockDim.x)
        nkeys[i] = ((unsigned long long)(unsigned)seg_u[cseg[i]] << L) | (unsigned)cdst[i];
}

__device__ __forceinline__ bool key_in(const unsigned long long* __restrict__ keys, long long n,
                                       unsigned long long k) {
    long long lo = 0, hi = n;
    while (lo < hi) {
        long long mid = (lo + hi) >> 1;
        if (keys[mid] < k) lo = mid + 1; else hi = mid;
    }
    return lo < n && keys[lo] == k;
}

// Triangles created by an insert, counted on the updated graph: every
// added edge (u, v) with u < v meets each w in N(u) ∩ N(v); the triangle
// {u, v, w} holds k = 1 + [uw added] + [vw added] added edges and is met k
// times, so tallies by k give  new = c1 + c2 / 2 + c3 / 3.  A lane takes an
// edge whose shorter list has at most 32 entries; longer ones are taken by
// the whole warp in turn.
__global__ void __launch_bounds__(kB) k_tc_delta(const VRec* __restrict__ vtab,
                                                 const int32_t* __restrict__ pool,
                                                 const unsigned long long* __restrict__ nkeys,
                                                 long long nk, int L,
                                                 unsigned long long* __restrict__ tally) {
    const int lane = threadIdx.x & 31;
    const unsigned long long mask = (1ull << L) - 1;
    unsigned long long c[3] = {0, 0, 0};
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < nk;
         base += stride) {
        const long long p = base + lane;
        bool heavy = false;
        int u = 0, v = 0, na = 0, nb = 0;
        const int32_t* a = nullptr;
        const int32_t* b = nullptr;
        if (p < nk) {
            const unsigned long long k = nkeys[p];
            u = (int)(k >> L);
            v = (int)(k & mask);
            if (u < v) {
                const VRec ru = vtab[u], rv = vtab[v];
                a = pool + ru.off;
                na = ru.deg;
                b = pool + rv.off;
                nb = rv.deg;
                if (na > nb) {
                    const int32_t* t = a; a = b; b = t;
                    int tn = na; na = nb; nb = tn;
                }
                if (na > 32) {
                    heavy = true;
                } else {
                    int lo = 0;
                    for (int i = 0; i < na && lo < nb; i++) {
                        const int32_t x = a[i];
                        int hi = nb;
                        while (lo < hi) {
                            int mid = (lo + hi) >> 1;
                            if (b[mid] < x) lo = mid + 1; else hi = mid;
                        }
                        if (lo < nb && b[lo] == x) {
                            lo++;
                            const int kk = (int)key_in(nkeys, nk, ((unsigned long long)(unsigned)u << L) | (unsigned)x) +
                                           (int)key_in(nkeys, nk, ((unsigned long long)(unsigned)v << L) | (unsigned)x);
                            c[kk]++;
                        }
                    }
                }
            }
        }
        unsigned hm = __ballot_sync(0xFFFFFFFFu, heavy);
        while (hm) {
            const int l = __ffs(hm) - 1;
            hm &= hm - 1;
            const int32_t* wa = (const int32_t*)__shfl_sync(0xFFFFFFFFu, (unsigned long long)a, l);
            const int32_t* wb = (const int32_t*)__shfl_sync(0xFFFFFFFFu, (unsigned long long)b, l);
            const int wna = __shfl_sync(0xFFFFFFFFu, na, l);
            const int wnb = __shfl_sync(0xFFFFFFFFu, nb, l);
            const int wu = __shfl_sync(0xFFFFFFFFu, u, l);
            const int wv = __shfl_sync(0xFFFFFFFFu, v, l);
            for (int j = lane; j < wna; j += 32) {
                const int32_t x = wa[j];
                int lo = 0, hi = wnb;
                while (lo < hi) {
                    int mid = (lo + hi) >> 1;
                    if (wb[mid] < x) lo = mid + 1; else hi = mid;
                }
                if (lo < wnb && wb[lo] == x) {
                    const int kk = (int)key_in(nkeys, nk, ((unsigned long long)(unsigned)wu << L) | (unsigned)x) +
                                   (int)key_in(nkeys, nk, ((unsigned long long)(unsigned)wv << L) | (unsigned)x);
                    c[kk]++;
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        unsigned long long x = c[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, o);
        if (lane == 0 && x) atomicAdd(tally + k, x);
    }
}

void run_update(hn_graph* g, hn_batch* b, unsigned flags, bool insert, int64_t* applied,
                unsigned long long* new_triangles = nullptr) {
    cudaStream_t s = g->stream;
    const long long n = b->n;
    if (applied) *applied = 0;
    if (n == 0) return;
    const int L = g->key_bits;
    AllocState* st = g->alloc;

    // 1. pack + sort
    DevBuf<unsigned long long> keys(n, s), keys2(n, s);
    HN_CUDA(cudaMemsetAsync(st, 0, sizeof(AllocState), s));
    HN_LAUNCH(k_pack, grid_for(g, n, kB), kB, 0, s, b->src, b->dst, n, g->nV, L, keys.get(), st);
    // weights travel with their keys (a stable sort keeps the batch order
    // of equal edges)
    const bool carry_w = insert && g->weighted && b->has_w;
    DevBuf<uint32_t> wv, wv2;
    if (carry_w) {
        wv.alloc(n, s);
        wv2.alloc(n, s);
        HN_CUDA(cudaMemcpyAsync(wv.get(), b->w, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
    }
    if (knob(kKnobUpdateOwnSort)) {
        unsigned long long* kc = keys.get();
        unsigned long long* ka = keys2.get();
        uint32_t* vc = carry_w ? wv.get() : nullptr;
        uint32_t* va = carry_w ? wv2.get() : nullptr;
        radix_sort_u64(g, kc, ka, vc, va, n, 2 * L, &st->error, s);
        if (kc != keys.get()) std::swap(keys.p, keys2.p);
        if (carry_w && vc != wv.get()) std::swap(wv.p, wv2.p);
    } else {
        // the library sort, kept for comparison (update.own_sort 0)
        ProfileScope ps("cub_sort_keys", s);
        cub::DoubleBuffer<unsigned long long> db(keys.get(), keys2.get());
        size_t tb = 0;
        if (carry_w) {
            cub::DoubleBuffer<uint32_t> dw(wv.get(), wv2.get());
            HN_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, db, dw, (int)n, 0, 2 * L, s));
            DevBuf<char> tmp(tb, s);
            HN_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, db, dw, (int)n, 0, 2 * L, s));
            if (dw.Current() != wv.get()) std::swap(wv.p, wv2.p);
        } else {
            HN_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, db, (int)n, 0, 2 * L, s));
            DevBuf<char> tmp(tb, s);
            HN_CUDA(cub::DeviceRadixSort::SortKeys(tmp.get(), tb, db, (int)n, 0, 2 * L, s));
        }
        count_launch();
        if (db.Current() != keys.get()) std::swap(keys.p, keys2.p);
    }
    wv2.release();
    // 2. mark  (keys2 reused as the counter values)
    unsigned long long* val = keys2.get();
    // each entry's place in its old list (insert: old entries <= it; erase:
    // old entries below it), kept for the compacted entries
    DevBuf<int32_t> apos(n, s), capos(n, s);
    if (insert)
        HN_LAUNCH(k_mark_insert, grid_for(g, n, kB), kB, 0, s, keys.get(), n, L, flags, g->vtab,
                  g->pool, val, apos.get(), (const AllocState*)st);
    else
        HN_LAUNCH(k_mark_erase, grid_for(g, n, kB), kB, 0, s, keys.get(), n, L, flags, g->vtab,
                  g->pool, val, apos.get(), (const AllocState*)st);
    // 3. scan + compact
    DevBuf<unsigned long long> scan(n, s);
    exclusive_scan(g, (const unsigned long long*)val, scan.get(), n, s);
    DevBuf<int32_t> cdst(n, s), cseg(n, s), seg_u(n, s), seg_kstart(n + 1, s), seg_ncap(n, s),
        seg_base(n, s);
    DevBuf<long long> seg_work(n + 1, s), seg_new_off(n, s), seg_old_off(n, s);
    long long* totals = g->d_scalar;
    DevBuf<uint32_t> cw;
    if (carry_w) cw.alloc(n, s);
    HN_LAUNCH(k_compact, grid_for(g, n, kB), kB, 0, s, keys.get(), val, scan.get(), n, L,
              cdst.get(), cseg.get(), seg_u.get(), seg_kstart.get(), totals,
              (const uint32_t*)wv.get(), cw.get(), (const int32_t*)apos.get(), capos.get());
    wv.release();
    apos.release();
    keys2.release();
    scan.release();
    // 4. plan (weighted graphs keep every list on the tile path, which moves
    // the weights with their neighbours)
    const int big_min = g->weighted ? INT_MAX : (int)knob(kKnobUpdateBigMin);
    DevBuf<int32_t> big_list(n + 1, s);
    DevBuf<unsigned long long> big_ctr(2, s);   // [0] hubs listed, [1] snapshot slots
    HN_CUDA(cudaMemsetAsync(big_ctr.get(), 0, 2 * sizeof(unsigned long long), s));
    // weighted graphs move every touched list (the weights travel with it)
    const bool in_place = !g->weighted && knob(kKnobUpdateInPlace) != 0;
    HN_LAUNCH(k_plan, grid_for(g, n + 1, kB), kB, 0, s, seg_u.get(), seg_kstart.get(), totals,
              insert, g->vtab, (const int32_t*)capos.get(), in_place,
              seg_work.get(), seg_ncap.get(), seg_base.get(), seg_old_off.get(), st, big_min,
              big_list.get(), (int*)big_ctr.get(), big_ctr.get() + 1);
    // 5. host plan (the one synchronisation of the batch)
    cudaEvent_t plan_ev = nullptr;   // profiled: the stream's idle time across the plan
    if (g_profiling) profile_begin(s, &plan_ev);
    HN_CUDA(cudaMemcpyAsync(g->h_scalar, totals, 2 * sizeof(long long), cudaMemcpyDeviceToHost,
                            s));
    HN_CUDA(cudaMemcpyAsync(g->h_alloc, st, sizeof(AllocState), cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaMemcpyAsync(g->h_scalar + 2, big_ctr.get(), 2 * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    const int nbig = *(const int*)(g->h_scalar + 2);
    const long long snap_words = g->h_scalar[3];
    if (const int e = g->h_alloc->error) {
        HN_CUDA(cudaMemsetAsync(&st->error, 0, sizeof(int), s));
        if (e == HN_ERR_TIMEOUT) throw Error(HN_ERR_TIMEOUT, "batch sort: a bounded wait gave up");
        throw Error(HN_ERR_INVALID, "batch vertex id outside [0, nV)");
    }
    const long long kept = g->h_scalar[0];
    const long long nseg = g->h_scalar[1];
    if (new_triangles) *new_triangles = 0;
    if (kept == 0) {
        if (plan_ev) profile_end("host_plan_round_trip", s, plan_ev);
        return;
    }
    DevBuf<unsigned long long> nkeys;
    if (new_triangles) {
        nkeys.alloc((size_t)kept, s);
        HN_LAUNCH(k_new_keys, grid_for(g, kept, kB), kB, 0, s, cdst.get(), cseg.get(), seg_u.get(),
                  kept, L, nkeys.get());
    }

    Plan plan;
    unsigned long long bump = (g->bump_host + 3) & ~3ull;
    for (int c = kNumClasses - 1; c >= 0; c--) {
        int need = g->h_alloc->need[c];
        int have = g->fl_count[c];
        int take = need < have ? need : have;
        plan.take[c] = take;
        plan.pop_top[c] = have;
        plan.push_base[c] = have - take;
        plan.bump_base[c] = bump;
        bump += (unsigned long long)(need - take) << c;
    }
    ensure_pool(g, bump);
    for (int c = 0; c < kNumClasses; c++) {
        long long after = (long long)plan.push_base[c] + g->h_alloc->push[c];
        ensure_free_list(g, c, after);
    }
    if (plan_ev) profile_end("host_plan_round_trip", s, plan_ev);
    // 6. assign blocks
    HN_LAUNCH(k_assign, grid_for(g, nseg, kB), kB, 0, s, seg_ncap.get(), nseg, plan,
              (long long* const*)g->d_fl, st, (const long long*)seg_old_off.get(),
              seg_new_off.get());
    // 7. scatter-merge
    exclusive_scan(g, (const long long*)seg_work.get(), seg_work.get(), nseg + 1, s);
    // tiles are read from the device prefix; the grid is persistent
    // five CTAs per SM (the shared-memory limit of the tile): each tile waits
    // on a short chain of dependent loads, so more resident tiles hide it
    const long long grid_sc = (long long)g->info.sms * kScatterCtas;
    DevBuf<long long> splits;
    lb_splits(g, seg_work.get(), nseg, g->nE, Tile::TILE, splits);
    DevBuf<unsigned long long> chunk_pre;
    DevBuf<int32_t> snap;
    if (nbig > 0) {
        chunk_pre.alloc((size_t)nbig + 1, s);
        HN_LAUNCH(k_big_chunks, grid_for(g, (long long)nbig + 1, kB), kB, 0, s, big_list.get(),
                  nbig, seg_u.get(), seg_kstart.get(), seg_ncap.get(), seg_base.get(),
                  seg_old_off.get(), seg_new_off.get(), g->vtab, chunk_pre.get());
        exclusive_scan(g, (const unsigned long long*)chunk_pre.get(), chunk_pre.get(),
                       (long long)nbig + 1, s);
        const long long grid_big = (long long)g->info.sms * 8;
        if (snap_words > 0) {
            snap.alloc((size_t)snap_words, s);
            const long long grid_snap = grid_for(g, nbig * 8ll, kB);   // ~8 chunks a hub
            if (insert)
                HN_LAUNCH(k_big_snap<true>, grid_snap, kB, 0, s, big_list.get(), nbig, seg_u.get(),
                          seg_kstart.get(), seg_ncap.get(), seg_base.get(), seg_old_off.get(),
                          seg_new_off.get(), g->vtab, (const unsigned long long*)chunk_pre.get(),
                          (const int32_t*)g->pool, snap.get());
            else
                HN_LAUNCH(k_big_snap<false>, grid_snap, kB, 0, s, big_list.get(), nbig,
                          seg_u.get(), seg_kstart.get(), seg_ncap.get(), seg_base.get(),
                          seg_old_off.get(), seg_new_off.get(), g->vtab,
                          (const unsigned long long*)chunk_pre.get(), (const int32_t*)g->pool,
                          snap.get());
        }
        if (insert)
            HN_LAUNCH(k_scatter_big<true>, grid_big, kSB, 0, s, big_list.get(), nbig, seg_u.get(),
                      seg_kstart.get(), seg_ncap.get(), seg_base.get(), seg_old_off.get(),
                      seg_new_off.get(), cdst.get(), (const int32_t*)capos.get(), g->vtab,
                      g->pool, (const unsigned long long*)chunk_pre.get(),
                      (const int32_t*)snap.get());
        else
            HN_LAUNCH(k_scatter_big<false>, grid_big, kSB, 0, s, big_list.get(), nbig,
                      seg_u.get(), seg_kstart.get(), seg_ncap.get(), seg_base.get(),
                      seg_old_off.get(), seg_new_off.get(), cdst.get(),
                      (const int32_t*)capos.get(), g->vtab, g->pool,
                      (const unsigned long long*)chunk_pre.get(), (const int32_t*)snap.get());
    }
    // in-place vertices whose moved entries span tiles: at most one per
    // tile boundary, and the work is at most nE entries
    const long long span_cap = (g->nE + nseg) / Tile::TILE + 2;
    DevBuf<int32_t> span_list(span_cap, s);
    DevBuf<int> nspan(1, s);
    HN_CUDA(cudaMemsetAsync(nspan.get(), 0, sizeof(int), s));
    const long long grid_span = (long long)g->info.sms * 8;
    if (insert) {
        HN_LAUNCH(k_scatter_old<true>, grid_sc, kSB, 0, s, seg_work.get(), nseg,
                  seg_u.get(), seg_kstart.get(), seg_new_off.get(), cdst.get(),
                  seg_old_off.get(), seg_ncap.get(), seg_base.get(), g->pool, splits.get(),
                  (long long)splits.n - 1, g->wpool, span_list.get(), nspan.get(), span_cap);
        HN_LAUNCH(k_inplace_span<true>, grid_span, kSpanWarps * 32, 0, s, span_list.get(),
                  nspan.get(), seg_u.get(), seg_kstart.get(), seg_base.get(), seg_old_off.get(),
                  cdst.get(), g->vtab, g->pool, span_cap);
        HN_LAUNCH(k_scatter_new, grid_for(g, kept, kB), kB, 0, s, cdst.get(), cseg.get(),
                  (const int32_t*)capos.get(), totals, seg_kstart.get(), seg_new_off.get(),
                  g->pool, (const uint32_t*)cw.get(), g->wpool);
    } else {
        HN_LAUNCH(k_scatter_old<false>, grid_sc, kSB, 0, s, seg_work.get(),
                  nseg, seg_u.get(), seg_kstart.get(), seg_new_off.get(), cdst.get(),
                  seg_old_off.get(), seg_ncap.get(), seg_base.get(), g->pool, splits.get(),
                  (long long)splits.n - 1, g->wpool, span_list.get(), nspan.get(), span_cap);
        HN_LAUNCH(k_inplace_span<false>, grid_span, kSpanWarps * 32, 0, s, span_list.get(),
                  nspan.get(), seg_u.get(), seg_kstart.get(), seg_base.get(), seg_old_off.get(),
                  cdst.get(), g->vtab, g->pool, span_cap);
    }
    // 8. commit
    HN_LAUNCH(k_commit, grid_for(g, nseg, kB), kB, 0, s, seg_u.get(), seg_kstart.get(),
              seg_ncap.get(), seg_new_off.get(), nseg, insert, plan, (long long* const*)g->d_fl,
              st, g->vtab);
    for (int c = 0; c < kNumClasses; c++)
        g->fl_count[c] = plan.push_base[c] + g->h_alloc->push[c];
    g->bump_host = bump;
    g->nE += insert ? kept : -kept;
    if (applied) *applied = kept;
    if (new_triangles) {
        unsigned long long* tally = (unsigned long long*)(g->d_scalar + 8);
        HN_CUDA(cudaMemsetAsync(tally, 0, 3 * sizeof(unsigned long long), s));
        HN_LAUNCH(k_tc_delta, grid_for(g, kept, kB), kB, 0, s, g->vtab, g->pool,
                  (const unsigned long long*)nkeys.get(), kept, L, tally);
        HN_CUDA(cudaMemcpyAsync(g->h_scalar + 8, tally, 3 * sizeof(long long),
                                cudaMemcpyDeviceToHost, s));
        HN_CUDA(cudaStreamSynchronize(s));
        const unsigned long long* t = (const unsigned long long*)(g->h_scalar + 8);
        *new_triangles = t[0] + t[1] / 2 + t[2] / 3;
    }
    HN_CUDA(cudaStreamSynchronize(s));
}

// Net effect of a mixed run of update batches: after a stable sort of
// the packed keys (ops carried as values), the last entry of each key's run
// holds the op that decides the edge's final presence.  Packed scan value:
// (erase << 32) | insert.
__global__ void k_widen_ops(const unsigned char* __restrict__ ops, long long n,
                            uint32_t* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = ops[i];
}

__global__ void k_net_mark(const unsigned long long* __restrict__ keys,
                           const uint32_t* __restrict__ ops, long long n,
                           unsigned long long* __restrict__ val, const AllocState* st) {
    const bool failed = st->error != 0;   // bad ids or a failed sort: the run is refused
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (failed) {
            val[i] = 0;
            continue;
        }
        const bool last = i == n - 1 || keys[i + 1] != keys[i];
        const unsigned long long ins = last && ops[i] != 0;
        const unsigned long long del = last && ops[i] == 0;
        val[i] = (del << 32) | ins;
    }
}

__global__ void k_net_split(const unsigned long long* __restrict__ keys,
                            const unsigned long long* __restrict__ val,
                            const unsigned long long* __restrict__ scan, long long n, int L,
                            int32_t* ins_src, int32_t* ins_dst, int32_t* del_src,
                            int32_t* del_dst, long long* totals) {
    const unsigned long long mask = (1ull << L) - 1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long v = val[i], at = scan[i];
        const int32_t u = (int32_t)(keys[i] >> L), w = (int32_t)(keys[i] & mask);
        if (v & 0xFFFFFFFFull) {
            ins_src[at & 0xFFFFFFFFull] = u;
            ins_dst[at & 0xFFFFFFFFull] = w;
        } else if (v >> 32) {
            del_src[at >> 32] = u;
            del_dst[at >> 32] = w;
        }
        if (i == n - 1) {
            totals[0] = (long long)((at + v) & 0xFFFFFFFFull);
            totals[1] = (long long)((at + v) >> 32);
        }
    }
}

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" {

int hn_batch_create(hn_graph_t* g, int64_t n, const int32_t* src, const int32_t* dst, int mem,
                    hn_batch_t** out) {
    return hn_batch_create_w(g, n, src, dst, nullptr, mem, out);
}

int hn_batch_create_w(hn_graph_t* g, int64_t n, const int32_t* src, const int32_t* dst,
                      const uint32_t* weights, int mem, hn_batch_t** out) {
    HN_API_BEGIN
    HN_REQUIRE(g && out, "null argument");
    *out = nullptr;
    hn_batch* b = new hn_batch();
    b->g = g;
    b->device = g->device;
    int rc = hn_batch_reset_w(b, n, src, dst, weights, mem);
    if (rc != HN_OK) {
        delete b;
        return rc;
    }
    *out = b;
    HN_API_END
}

int hn_batch_reset(hn_batch_t* b, int64_t n, const int32_t* src, const int32_t* dst, int mem) {
    return hn_batch_reset_w(b, n, src, dst, nullptr, mem);
}

int hn_batch_reset_w(hn_batch_t* b, int64_t n, const int32_t* src, const int32_t* dst,
                     const uint32_t* weights, int mem) {
    HN_API_BEGIN
    HN_REQUIRE(b != nullptr, "batch is null");
    HN_REQUIRE(n >= 0 && n <= 0x7FFFFFFF, "batch size must be in [0, 2^31)");
    HN_REQUIRE(n == 0 || (src && dst), "null batch arrays");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    hn_graph* g = b->g;
    HN_CUDA(cudaSetDevice(g->device));
    // stream-ordered from the device's memory pool: a batch per request
    // costs no device-wide synchronisation (cudaMalloc / cudaFree would)
    if ((size_t)n > b->cap) {
        if (b->src) HN_CUDA(cudaFreeAsync(b->src, g->stream));
        if (b->dst) HN_CUDA(cudaFreeAsync(b->dst, g->stream));
        b->src = b->dst = nullptr;
        b->cap = 0;
        HN_CUDA(cudaMallocAsync((void**)&b->src, sizeof(int32_t) * (size_t)n, g->stream));
        HN_CUDA(cudaMallocAsync((void**)&b->dst, sizeof(int32_t) * (size_t)n, g->stream));
        b->cap = (size_t)n;
    }
    if (weights && (size_t)n > b->wcap) {
        if (b->w) HN_CUDA(cudaFreeAsync(b->w, g->stream));
        b->w = nullptr;
        b->wcap = 0;
        HN_CUDA(cudaMallocAsync((void**)&b->w, sizeof(uint32_t) * (size_t)n, g->stream));
        b->wcap = (size_t)n;
    }
    b->n = n;
    b->has_w = weights != nullptr;
    if (n) {
        cudaMemcpyKind kind = mem == HN_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
        HN_CUDA(cudaMemcpyAsync(b->src, src, sizeof(int32_t) * (size_t)n, kind, g->stream));
        HN_CUDA(cudaMemcpyAsync(b->dst, dst, sizeof(int32_t) * (size_t)n, kind, g->stream));
        if (weights)
            HN_CUDA(cudaMemcpyAsync(b->w, weights, sizeof(uint32_t) * (size_t)n, kind, g->stream));
        HN_CUDA(cudaStreamSynchronize(g->stream));
    }
    HN_API_END
}

int hn_batch_size(const hn_batch_t* b, int64_t* n) {
    HN_API_BEGIN
    HN_REQUIRE(b && n, "null argument");
    *n = b->n;
    HN_API_END
}

int hn_batch_destroy(hn_batch_t* b) {
    HN_API_BEGIN
    if (!b) return HN_OK;
    // the batch may outlive its graph (garbage-collection order), so only
    // its own device id is used here.  Every call that read the buffers has
    // returned (calls are synchronous), so they go back to the memory pool
    // in the legacy stream's order, without a device-wide synchronisation.
    cudaSetDevice(b->device);
    if (b->src) cudaFreeAsync(b->src, 0);
    if (b->dst) cudaFreeAsync(b->dst, 0);
    if (b->w) cudaFreeAsync(b->w, 0);
    delete b;
    (void)cudaGetLastError();
    HN_API_END
}

int hn_insert(hn_graph_t* g, hn_batch_t* b, unsigned flags, int64_t* applied) {
    HN_API_BEGIN
    HN_REQUIRE(g && b, "null argument");
    HN_REQUIRE(b->g == g, "batch belongs to another graph");
    HN_REQUIRE((flags & ~(HN_DEDUP_BATCH | HN_DEDUP_GRAPH)) == 0, "unknown flags");
    require_owner(g);
    HandleUse use(g);
    HN_CUDA(cudaSetDevice(g->device));
    run_update(g, b, flags, true, applied);
    HN_API_END
}

int hn_insert_count_triangles(hn_graph_t* g, hn_batch_t* b, int64_t* applied,
                              uint64_t* new_triangles) {
    HN_API_BEGIN
    HN_REQUIRE(g && b && new_triangles, "null argument");
    HN_REQUIRE(b->g == g, "batch belongs to another graph");
    require_owner(g);
    HandleUse use(g);
    HN_CUDA(cudaSetDevice(g->device));
    unsigned long long t = 0;
    run_update(g, b, HN_DEDUP_BATCH | HN_DEDUP_GRAPH, true, applied, &t);
    *new_triangles = t;
    HN_API_END
}

int hn_erase(hn_graph_t* g, hn_batch_t* b, unsigned flags, int64_t* applied) {
    HN_API_BEGIN
    HN_REQUIRE(g && b, "null argument");
    HN_REQUIRE(b->g == g, "batch belongs to another graph");
    HN_REQUIRE((flags & ~HN_DEDUP_BATCH) == 0, "unknown flags");
    require_owner(g);
    HandleUse use(g);
    HN_CUDA(cudaSetDevice(g->device));
    run_update(g, b, flags, false, applied);
    HN_API_END
}

int hn_update_coalesced(hn_graph_t* g, int64_t n, const int32_t* src, const int32_t* dst,
                        const uint8_t* ops, int mem, int64_t* inserted, int64_t* erased) {
    HN_API_BEGIN
    HN_REQUIRE(g, "graph is null");
    HN_REQUIRE(n >= 0 && n <= 0x7FFFFFFF, "batch size must be in [0, 2^31)");
    HN_REQUIRE(n == 0 || (src && dst && ops), "null batch arrays");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    require_owner(g);
    if (inserted) *inserted = 0;
    if (erased) *erased = 0;
    if (n == 0) return HN_OK;
    HandleUse use(g);
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    const int L = g->key_bits;
    DevBuf<int32_t> hs, hd;
    DevBuf<unsigned char> hops;
    const int32_t* d_src = src;
    const int32_t* d_dst = dst;
    const unsigned char* d_ops = ops;
    if (mem == HN_MEM_HOST) {
        hs.alloc((size_t)n, s);
        hd.alloc((size_t)n, s);
        hops.alloc((size_t)n, s);
        HN_CUDA(cudaMemcpyAsync(hs.get(), src, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
        HN_CUDA(cudaMemcpyAsync(hd.get(), dst, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
        HN_CUDA(cudaMemcpyAsync(hops.get(), ops, (size_t)n, cudaMemcpyHostToDevice, s));
        d_src = hs.get();
        d_dst = hd.get();
        d_ops = hops.get();
    }
    AllocState* st = g->alloc;
    DevBuf<unsigned long long> keys((size_t)n, s), keys2((size_t)n, s);
    DevBuf<uint32_t> ops2((size_t)n, s), ops1((size_t)n, s);
    HN_CUDA(cudaMemsetAsync(st, 0, sizeof(AllocState), s));
    HN_LAUNCH(k_pack, grid_for(g, n, kB), kB, 0, s, d_src, d_dst, n, g->nV, L, keys.get(), st);
    HN_LAUNCH(k_widen_ops, grid_for(g, n, kB), kB, 0, s, d_ops, n, ops1.get());
    {
        // LSD radix sort is stable: equal keys keep their batch order
        unsigned long long* kc = keys.get();
        unsigned long long* ka = keys2.get();
        uint32_t* vc = ops1.get();
        uint32_t* va = ops2.get();
        radix_sort_u64(g, kc, ka, vc, va, n, 2 * L, &st->error, s);
        if (kc != keys.get()) std::swap(keys.p, keys2.p);
        if (vc != ops1.get()) std::swap(ops1.p, ops2.p);
    }
    unsigned long long* val = keys2.get();
    HN_LAUNCH(k_net_mark, grid_for(g, n, kB), kB, 0, s, keys.get(), ops1.get(), n, val,
              (const AllocState*)st);
    DevBuf<unsigned long long> scan((size_t)n, s);
    exclusive_scan(g, (const unsigned long long*)val, scan.get(), n, s);
    hn_batch bi, bd;
    bi.g = bd.g = g;
    bi.device = bd.device = g->device;
    DevBuf<int32_t> is((size_t)n, s), id((size_t)n, s), ds((size_t)n, s), dd((size_t)n, s);
    HN_LAUNCH(k_net_split, grid_for(g, n, kB), kB, 0, s, keys.get(), val, scan.get(), n, L,
              is.get(), id.get(), ds.get(), dd.get(), g->d_scalar);
    HN_CUDA(cudaMemcpyAsync(g->h_scalar, g->d_scalar, 2 * sizeof(long long),
                            cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaMemcpyAsync(g->h_alloc, st, sizeof(AllocState), cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    if (const int e = g->h_alloc->error) {
        HN_CUDA(cudaMemsetAsync(&st->error, 0, sizeof(int), s));
        if (e == HN_ERR_TIMEOUT) throw Error(HN_ERR_TIMEOUT, "batch sort: a bounded wait gave up");
        throw Error(HN_ERR_INVALID, "batch vertex id outside [0, nV)");
    }
    bi.n = g->h_scalar[0];
    bd.n = g->h_scalar[1];
    keys.release();
    keys2.release();
    scan.release();
    bd.src = ds.get();
    bd.dst = dd.get();
    bi.src = is.get();
    bi.dst = id.get();
    // the two sets are disjoint, so their order does not matter
    run_update(g, &bd, HN_DEDUP_BATCH, false, erased);
    run_update(g, &bi, HN_DEDUP_BATCH | HN_DEDUP_GRAPH, true, inserted);
    HN_API_END
}

}  // extern "C"
