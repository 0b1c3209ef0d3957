// TriangleCounting2 (hornetsnest/src/Static/TriangleCounting/triangle2.cu:75-171
// with forAllAdjUnions, primitives/Operator++.i.cuh:319-522).
//
// The reference counts on a graph read with DIRECTED_BY_DEGREE | SORT
// (hornetsnest/test/TriangleTest2.cu:86-87): every undirected edge is kept
// once, from the lower-(degree, id) endpoint (xlib/src/Graph/GraphStd.cpp:
// 247-268), so each triangle is found exactly once.  It then bins all
// directed edges by log-degree pair with 64-bit global atomics (two passes)
// and runs ~37 intersection launches.
//
// Here the orientation is built on the device from the (always sorted)
// undirected adjacency in two merge-path balanced passes around one scan:
//   pass 1  keep flag of every edge (needs deg(v): one 16-byte record read),
//   scan    flag positions = the oriented CSR,
//   pass 2  compact the kept neighbours (lists stay sorted).
// The intersection is vertex-centric with N+(u) in a shared-memory hash
// table (see the comment above k_tc_warp).
#include <cub/cub.cuh>

#include <type_traits>

#include "hn_graph.cuh"
#include "hn_tc.cuh"

namespace hn {

namespace {

constexpr int kB = 256;
using Tile = LbTile<kB, 4>;

__device__ __forceinline__ bool oriented_before(int du, int u, int dv, int v) {
    return du < dv || (du == dv && u < v);
}

__global__ void __launch_bounds__(kB)
k_orient_flags(const long long* __restrict__ prefix, int nV, const VRec* __restrict__ vtab,
               const int32_t* __restrict__ pool, int32_t* __restrict__ flag,
               const long long* __restrict__ splits, long long split_tiles) {
    __shared__ Tile t;
    __shared__ long long s_base[Tile::TILE + 1];
    __shared__ int s_deg[Tile::TILE + 1];
    const long long total = prefix[nV];
    const long long ntiles = (total + nV + Tile::TILE - 1) / Tile::TILE;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int n = lb_tile_load(t, prefix, (long long)nV, total, tile, splits, split_tiles);
        for (int b = threadIdx.x; b <= t.nends; b += kB) {
            long long u = t.seg0 + b;
            if (u < nV) {
                VRec r = vtab[u];
                s_base[b] = r.off - t.seg_start(b);
                s_deg[b] = r.deg;
            }
        }
        __syncthreads();
        // all of a thread's loads first: neighbours, then their degrees
        constexpr int IPT = Tile::TILE / kB;
        int bs[IPT], vs[IPT], dv[IPT];
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            const int i = threadIdx.x + k * kB;
            bs[k] = -1;
            if (i < n) {
                bs[k] = t.seg[i];
                vs[k] = pool[s_base[bs[k]] + t.item0 + i];
            }
        }
#pragma unroll
        for (int k = 0; k < IPT; k++)
            if (bs[k] >= 0) dv[k] = vtab[vs[k]].deg;
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            if (bs[k] < 0) continue;
            const int b = bs[k];
            const int u = (int)(t.seg0 + b);
            flag[t.item0 + threadIdx.x + k * kB] = oriented_before(s_deg[b], u, dv[k], vs[k]) ? 1 : 0;
        }
        __syncthreads();
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) flag[total] = 0;
}

__global__ void __launch_bounds__(kB)
k_orient_fill(const long long* __restrict__ prefix, int nV, const VRec* __restrict__ vtab,
              const int32_t* __restrict__ pool, const int32_t* __restrict__ pos,
              int32_t* __restrict__ fwd, long long* __restrict__ offp,
              const long long* __restrict__ splits, long long split_tiles,
              const int32_t* __restrict__ canon, int32_t* __restrict__ feid) {
    __shared__ Tile t;
    __shared__ long long s_base[Tile::TILE + 1];
    const long long total = prefix[nV];
    const long long ntiles = (total + nV + Tile::TILE - 1) / Tile::TILE;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int n = lb_tile_load(t, prefix, (long long)nV, total, tile, splits, split_tiles);
        for (int b = threadIdx.x; b <= t.nends; b += kB) {
            long long u = t.seg0 + b;
            if (u < nV) s_base[b] = vtab[u].off - t.seg_start(b);
        }
        __syncthreads();
        constexpr int IPT = Tile::TILE / kB;
        int ps[IPT], keep[IPT], vs[IPT];
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            const int i = threadIdx.x + k * kB;
            keep[k] = 0;
            if (i < n) {
                const long long e = t.item0 + i;
                ps[k] = pos[e];
                keep[k] = pos[e + 1] != ps[k];
                vs[k] = pool[s_base[t.seg[i]] + e];
            }
        }
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            if (!keep[k]) continue;
            const long long e = t.item0 + threadIdx.x + k * kB;
            fwd[ps[k]] = vs[k];
            if (feid) feid[ps[k]] = canon[e];   // edge id of the kept edge
        }
        __syncthreads();
    }
    // offp[u] = pos[prefix[u]]
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u <= nV;
         u += (long long)gridDim.x * blockDim.x)
        offp[u] = pos[prefix[u]];
}

// Candidate lists.  The oriented edge x -> y contributes |N+(x) ∩ N+(y)|
// triangles whichever endpoint counts it, so it is counted by the endpoint
// whose out-list is the longer: that list is the hash table, the shorter
// one is probed (cost min(d+(x), d+(y)) instead of d+(y)).  C(z) lists the
// other endpoint of every edge z counts, stored as ~x when z is the head of
// x -> z (owner counts credit the tail x).  Order inside C(z) is immaterial.
__device__ __forceinline__ bool cand_flip(long long dx, long long dy) { return dy > dx; }

template <bool FILL>
__global__ void __launch_bounds__(kB)
k_cand(const long long* __restrict__ offp, int nV, const int32_t* __restrict__ fwd,
       int* __restrict__ cnt /*count pass: sizes; fill pass: cursors*/,
       const long long* __restrict__ coff, int32_t* __restrict__ cand,
       const long long* __restrict__ splits, long long split_tiles,
       const int32_t* __restrict__ feid, int32_t* __restrict__ ceid) {
    constexpr int IPT = Tile::TILE / kB;   // items per thread, blocked
    using Scan = cub::BlockScan<int, kB>;
    __shared__ Tile t;
    __shared__ typename Scan::TempStorage scan_tmp;
    __shared__ int s_rank[Tile::TILE + 1];       // kept edges of the tile before item i
    __shared__ long long s_pos[Tile::TILE + 1];  // first slot of segment b's kept edges
    const long long total = offp[nV];
    const long long ntiles = (total + nV + Tile::TILE - 1) / Tile::TILE;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int n = lb_tile_load(t, offp, (long long)nV, total, tile, splits, split_tiles);
        int ys[IPT], keep[IPT], rank[IPT];
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            const int i = threadIdx.x * IPT + k;
            keep[k] = 0;
            ys[k] = -1;
            if (i < n) {
                const int b = t.seg[i];
                const long long dx = t.ends[b] - t.seg_start(b);
                const int y = fwd[t.item0 + i];
                const long long dy = offp[y + 1] - offp[y];
                ys[k] = y;
                keep[k] = cand_flip(dx, dy) ? 0 : 1;
            }
        }
        int kept_total;
        Scan(scan_tmp).ExclusiveSum(keep, rank, kept_total);
#pragma unroll
        for (int k = 0; k < IPT; k++) s_rank[threadIdx.x * IPT + k] = rank[k];
        if (threadIdx.x == 0) s_rank[Tile::TILE] = kept_total;
        __syncthreads();
        // per segment: its kept edges are the ones ranked [lo, hi) of the tile
        for (int b = threadIdx.x; b <= t.nends; b += kB) {
            const long long x = t.seg0 + b;
            if (x < nV) {
                const long long s0 = t.seg_start(b), s1 = t.ends[b];
                const int lo = (int)((s0 > t.item0 ? s0 : t.item0) - t.item0);
                const long long e1 = t.item0 + n;
                const int hi = (int)((s1 < e1 ? s1 : e1) - t.item0);
                const int kept = lo < hi ? (hi < n ? s_rank[hi] : kept_total) - s_rank[lo] : 0;
                if (kept) {
                    if (FILL) s_pos[b] = coff[x] + atomicAdd(cnt + x, kept) - s_rank[lo];
                    else atomicAdd(cnt + x, kept);
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            const int i = threadIdx.x * IPT + k;
            if (ys[k] < 0) continue;
            const int b = t.seg[i];
            long long q = -1;
            if (keep[k]) {
                if (FILL) q = s_pos[b] + rank[k];
                if (FILL) cand[q] = ys[k];
            } else {
                if (FILL) q = coff[ys[k]] + atomicAdd(cnt + ys[k], 1);
                if (FILL) cand[q] = ~(int)(t.seg0 + b);   // flipped: ~tail
                else atomicAdd(cnt + ys[k], 1);
            }
            if (FILL && ceid) ceid[q] = feid[t.item0 + i];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Vertex-centric counting.  For each vertex u, N+(u) goes into an
// open-addressing hash table in shared memory (multiplicative hash, linear
// probing, load factor <= 1/2, so every probe sequence ends at an empty
// slot).  Every oriented edge (u,v) is counted by its tail u: the elements
// of N+(v) are probed against table(u), after N+(v) is narrowed to
// [min N+(u), max N+(u)] by two binary searches.  The (v, w) pairs of 32
// candidates v at a time are dealt to the lanes round-robin (lane l takes
// pairs l, l+32, ...), so a warp's loads of w read consecutive words of the
// same list; each lane advances its candidate monotonically (no per-pair
// search).
//   k_tc_warp: one warp per vertex with d+(u) <= warp_cap (the tc.warp_cap
//              knob, at most kWarpCap, the table's capacity); vertices handed
//              out in chunks by an atomic counter; larger ones are listed;
//   k_tc_cta:  one CTA per listed vertex, table in dynamic shared memory
//              (up to kCtaCap entries), binary search of the sorted list in
//              global memory beyond that.
// ---------------------------------------------------------------------------
constexpr int kTcWarps = 8;
constexpr int kWarpCap = 512;
constexpr int kWarpTab = 2 * kWarpCap;
constexpr int kCtaCap = 16384;   // largest tc.cta_table_cap: 160 KB tables
#ifndef HN_TC_PAIR_ILP
#define HN_TC_PAIR_ILP 8
#endif
constexpr int kPairIlp = HN_TC_PAIR_ILP;   // pairs in flight per lane

// Slots of a table for up to `cap` entries: the power of two >= 2*cap that a
// vertex with d+(u) = cap asks for (and no fewer than 32).
__host__ __device__ constexpr int tc_table_slots(int cap) {
    int n = 32;
    while (n < 2 * cap) n <<= 1;
    return n;
}

// Candidates of one work item of a listed vertex with d+(u) = du: about
// item_work pairs (every list it probes is at most du long), a multiple of
// 32, at least 32.
__device__ __forceinline__ int item_cands(int du, long long item_work) {
    long long c = item_work / du;
    if (c > (1 << 20)) c = 1 << 20;
    c &= ~31LL;
    return c < 32 ? 32 : (int)c;
}

__device__ __forceinline__ unsigned tc_hash(int w, int bits) {
    return ((unsigned)w * 2654435761u) >> (32 - bits);
}

// Linear probing whose home slot is the first of a 4-slot bucket (16
// bytes): a lookup reads the whole home bucket with one 128-bit load and is
// decided there unless the bucket is full and does not hold w.  Slots are
// never emptied, so a key sits before the first empty slot of its probe
// sequence.
__device__ __forceinline__ unsigned tab_home(int w, int bits) {
    return tc_hash(w, bits - 2) << 2;
}

// Inserts w; returns its slot.
__device__ __forceinline__ unsigned tab_insert(int* tab, int bits, int w) {
    unsigned mask = (1u << bits) - 1;
    unsigned h = tab_home(w, bits);
    while (true) {
        int old = atomicCAS(tab + h, -1, w);
        if (old == -1 || old == w) return h;
        h = (h + 1) & mask;
    }
}

// Filter bit of w for a table of 2^bits slots: the top bits+3 bits of the
// same product, so a filter of 8 bits per slot (2^(bits-2) words) rejects
// most absent values with one shared-memory load and no probe loop.  Its
// word index is the home bucket of w.
__device__ __forceinline__ unsigned tc_fbit(int w, int bits) {
    return ((unsigned)w * 2654435761u) >> (32 - (bits + 3));
}

__device__ __forceinline__ unsigned tab_insert_f(int* tab, unsigned* filt, int bits, int w) {
    const unsigned h = tab_insert(tab, bits, w);
    const unsigned f = tc_fbit(w, bits);
    atomicOr(filt + (f >> 5), 1u << (f & 31));
    return h;
}

// Membership of w, for lanes whose filter bit is set (`maybe`), in the home
// bucket.  `more`: the bucket is full and does not hold w, so the answer is
// tab_rest's.  `slot`: where w is, on a hit.
__device__ __forceinline__ bool tab_bucket(const int* tab, int bits, int w, bool maybe,
                                           bool& more, unsigned& slot) {
    const unsigned h = tab_home(w, bits);
    int4 q = make_int4(-1, -1, -1, -1);
    if (maybe) q = *reinterpret_cast<const int4*>(tab + h);
    const bool hit = (q.x == w) | (q.y == w) | (q.z == w) | (q.w == w);
    slot = h + (q.x == w ? 0 : q.y == w ? 1 : q.z == w ? 2 : 3);
    // slots hold vertex ids (>= 0) or -1: the bucket is full iff the OR of
    // its slots is non-negative
    more = maybe & !hit & ((q.x | q.y | q.z | q.w) >= 0);
    return hit;
}

// The probe after a full home bucket, slot by slot (the table is at most
// half full, so it meets an empty slot): w's slot, or -1.
__device__ __forceinline__ int tab_rest(const int* tab, int bits, int w) {
    const unsigned mask = (1u << bits) - 1;
    for (unsigned p = (tab_home(w, bits) + 4) & mask;; p = (p + 1) & mask) {
        const int x = tab[p];
        if (x == w) return (int)p;
        if (x == -1) return -1;
    }
}

// Owner credit: the warp's triangles found from u, added to counts[u] once
// (each triangle is found once, from its lowest vertex in the orientation).
__device__ __forceinline__ void tc_credit_owner(unsigned long long* counts, int u,
                                                unsigned long long c) {
    for (int o = 16; o; o >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(counts + u, c);
}

struct TcView {
    const long long* offp;   // oriented offsets
    const int32_t* fwd;      // oriented lists
    const long long* coff;   // candidate-list offsets
    const int32_t* cand;     // candidate lists C(z)
    // edge-support mode (MODE 3) only:
    const int32_t* feid;     // edge id of each fwd entry
    const int32_t* ceid;     // edge id of each candidate entry
    int* esup;               // per-edge triangle counts
};

// One triangle {u, v, w} found from u: credit its three edges (MODE 3).
__device__ __forceinline__ void tc_credit_edges(int* esup, int e_uv, int e_vw, int e_uw) {
    atomicAdd(esup + e_uv, 1);
    atomicAdd(esup + e_vw, 1);
    atomicAdd(esup + e_uw, 1);
}

// One warp: every (v, w) pair of u, w in N+(v) for v in the candidate
// list C of u, probed against L = N+(u) (hash table `tab`, or binary search
// of the sorted global list L when tab == nullptr).  Candidates v are taken
// 32 at a time (in order, or groups claimed from the CTA's counter `s_next`
// when several warps share u); each lane first narrows N+(v) to
// [min N+(u), max N+(u)] by two binary searches, then the group's pairs are
// dealt round-robin to the lanes (one search over the 33-entry prefix per
// lane per group).
template <int MODE, bool TAB>
__device__ __forceinline__ unsigned long long tc_vertex_warp(
    int u, const int32_t* __restrict__ L, int du, const int32_t* __restrict__ C, int dc,
    const int* tab, const unsigned* filt, const int* teid, int bits,
    int narrow_min, int* s_next, const TcView& g, int* s_pref /*33*/, long long* s_vb /*32*/,
    int* s_v /*32*/, unsigned* s_fc /*32*/, unsigned long long* __restrict__ per_vertex) {
    const int lane = threadIdx.x & 31;
    const int lo_w = L[0], hi_w = L[du - 1];
    unsigned long long cnt = 0, cnt_u = 0;   // all hits; MODE 2: hits owned by u
    auto claim = [&](int c) {
        if (!s_next) return c + 32;
        int t = 0;
        if (lane == 0) t = atomicAdd(s_next, 1);
        return __shfl_sync(0xFFFFFFFFu, t, 0) * 32;
    };
    for (int c0 = claim(-32); c0 < dc; c0 = claim(c0)) {
        int idx = c0 + lane;
        int dx = 0, v = 0;
        bool flp = false;   // u is the head of v -> u
        long long xb = 0;
        if (idx < dc) {
            v = C[idx];
            flp = v < 0;
            if (flp) v = ~v;
            long long b0 = g.offp[v], b1 = g.offp[v + 1];
            const int32_t* lst = g.fwd + b0;
            int n = (int)(b1 - b0);
            // [first element >= lo_w, first element > hi_w); lists of at most
            // narrow_min entries are probed whole (two dependent searches
            // cost more than the few extra filter probes)
            int lo = 0, hi = n;
            int s0 = 0;
            if (n > narrow_min) {
                while (lo < hi) { int m = (lo + hi) >> 1; if (lst[m] < lo_w) lo = m + 1; else hi = m; }
                s0 = lo;
                hi = n;
                while (lo < hi) { int m = (lo + hi) >> 1; if (lst[m] <= hi_w) lo = m + 1; else hi = m; }
            } else {
                lo = n;
            }
            xb = b0 + s0;
            dx = lo - s0;
        }
        int incl = dx;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        s_pref[lane + 1] = incl;
        if (lane == 0) s_pref[0] = 0;
        s_vb[lane] = xb;
        // MODE 3 keeps the candidate's edge id (u, v) instead of v
        // MODE 3 keeps the candidate's edge id; MODE 2 the owner of its
        // triangles when that is v (flipped), else -1 (owner u)
        if (MODE == 3) s_v[lane] = idx < dc ? g.ceid[(C - g.cand) + idx] : 0;
        else if (MODE == 2) s_v[lane] = idx < dc && flp ? v : -1;
        else s_v[lane] = v;
        if (MODE == 2) s_fc[lane] = 0;
        __syncwarp();
        const int T = s_pref[32];
        if (lane < T) {
            int a = 0, b = 32;   // candidate slot of pair `lane`
            while (b - a > 1) {
                int mid = (a + b) >> 1;
                if (s_pref[mid] <= lane) a = mid; else b = mid;
            }
            int end = s_pref[a + 1];
            const int32_t* base = g.fwd + (s_vb[a] - s_pref[a]);   // pair k's w: base[k]
            // kPairIlp pairs per lane per step (k, k+32, ...): their loads
            // of w are issued together, then probed.  FULL steps (every
            // lane's kPairIlp pairs exist; uniform in the warp) skip the
            // bounds checks; the last step of a group is partial.
            unsigned c32 = 0, c32u = 0;   // hits of this group; MODE 2: those owned by u
            auto step = [&](int k0, auto full_tag) {
                constexpr bool FULL = decltype(full_tag)::value;
                int wv[kPairIlp], va[kPairIlp];
#pragma unroll
                for (int j = 0; j < kPairIlp; j++) {
                    const int k = k0 + 32 * j;
                    wv[j] = -1;
                    va[j] = a;
                    if (FULL || k < T) {
                        if (k >= end) {   // the candidate holding pair k
                            a++;
                            if (s_pref[a + 1] <= k) {
                                // short lists: k skipped several candidates;
                                // search s_pref[a..32] (s_pref[32] = T > k)
                                int hi = 32;
                                while (hi - a > 1) {
                                    int mid = (a + hi) >> 1;
                                    if (s_pref[mid] <= k) a = mid; else hi = mid;
                                }
                            }
                            end = s_pref[a + 1];
                            base = g.fwd + (s_vb[a] - s_pref[a]);
                        }
                        wv[j] = base[k];
                        va[j] = a;
                    }
                }
                // a lane's first lookup that needs probing past its home
                // bucket waits until after the step (one divergent probe
                // loop per step instead of one per pair)
                int dw = -1, da = 0, dk = 0;
                // MODE 3: the edge (v, w) of pair k of candidate slot c
                auto e_vw = [&](int c, int k) { return g.feid[s_vb[c] - s_pref[c] + k]; };
#pragma unroll
                for (int j = 0; j < kPairIlp; j++) {
                    const int w = wv[j];
                    if (!FULL && w < 0) continue;
                    bool hit;
                    int e_uw = 0;   // MODE 3: edge (u, w)
                    if (TAB) {
                        const unsigned f = tc_fbit(w, bits);
                        bool more;
                        unsigned slot;
                        hit = tab_bucket(tab, bits, w, (filt[f >> 5] >> (f & 31)) & 1u, more, slot);
                        if (more) {
                            if (dw < 0) {
                                dw = w;
                                da = va[j];
                                dk = k0 + 32 * j;
                            } else {
                                const int sl = tab_rest(tab, bits, w);
                                hit = sl >= 0;
                                slot = (unsigned)sl;
                            }
                        }
                        if (MODE == 3 && hit) e_uw = teid[slot];
                    } else {
                        int lo = 0, hi = du;
                        while (lo < hi) {
                            int mid = (lo + hi) >> 1;
                            if (L[mid] < w) lo = mid + 1; else hi = mid;
                        }
                        hit = lo < du && L[lo] == w;
                        if (MODE == 3 && hit) e_uw = g.feid[(L - g.fwd) + lo];
                    }
                    c32 += hit ? 1u : 0u;
                    if (MODE == 1 && hit) {
                        atomicAdd(per_vertex + w, 1ull);
                        atomicAdd(per_vertex + u, 1ull);
                        atomicAdd(per_vertex + s_v[va[j]], 1ull);
                    }
                    if (MODE == 3 && hit)
                        tc_credit_edges(g.esup, s_v[va[j]], e_vw(va[j], k0 + 32 * j), e_uw);
                    if (MODE == 2 && hit) {
                        if (s_v[va[j]] >= 0) atomicAdd(s_fc + va[j], 1u);
                        else c32u++;
                    }
                }
                if (TAB && dw >= 0) {
                    const int sl = tab_rest(tab, bits, dw);
                    if (sl >= 0) {
                        c32++;
                        if (MODE == 1) {
                            atomicAdd(per_vertex + dw, 1ull);
                            atomicAdd(per_vertex + u, 1ull);
                            atomicAdd(per_vertex + s_v[da], 1ull);
                        }
                        if (MODE == 3) tc_credit_edges(g.esup, s_v[da], e_vw(da, dk), teid[sl]);
                        if (MODE == 2) {
                            if (s_v[da] >= 0) atomicAdd(s_fc + da, 1u);
                            else c32u++;
                        }
                    }
                }
            };
            int k0 = lane;
            for (; k0 - lane + 32 * kPairIlp <= T; k0 += 32 * kPairIlp)
                step(k0, std::integral_constant<bool, true>());
            if (k0 < T) step(k0, std::integral_constant<bool, false>());
            cnt += c32;
            cnt_u += c32u;
        }
        __syncwarp();
        if (MODE == 2) {   // flipped candidates own their triangles
            if (s_v[lane] >= 0 && s_fc[lane]) atomicAdd(per_vertex + s_v[lane], (unsigned long long)s_fc[lane]);
            __syncwarp();
        }
    }
    if (MODE == 2) tc_credit_owner(per_vertex, u, cnt_u);
    return cnt;
}

// Small vertices (d+(u) <= small_du, at most small_dc candidates; used with
// the smaller-side assignment, so every probed list is at most d+(u) long):
// a thread each, merging N+(u) with each candidate's list.  No table, no
// warp-wide steps: the per-vertex overhead that dominates tiny vertices in
// the warp kernel is gone.
template <int MODE>
__global__ void __launch_bounds__(256)
k_tc_thread(TcView g, int nV, int small_du, int small_dc,
            unsigned long long* __restrict__ per_vertex,
            unsigned long long* __restrict__ total_out) {
    __shared__ unsigned long long s_sum[8];
    unsigned long long mine = 0;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < nV;
         x += (long long)gridDim.x * blockDim.x) {
        const int u = (int)x;
        const long long ub = g.offp[u];
        const int du = (int)(g.offp[u + 1] - ub);
        const long long cb = g.coff[u];
        const int dc = (int)(g.coff[u + 1] - cb);
        if (du == 0 || dc == 0 || du > small_du || dc > small_dc) continue;
        const int32_t* A = g.fwd + ub;
        unsigned cu = 0;   // MODE 2: hits owned by u
        for (int c = 0; c < dc; c++) {
            int v = g.cand[cb + c];
            const bool flp = v < 0;
            if (flp) v = ~v;
            const long long vb = g.offp[v];
            const int dv = (int)(g.offp[v + 1] - vb);
            const int32_t* Bv = g.fwd + vb;
            unsigned hits = 0;
            for (int i = 0, j = 0; i < du && j < dv;) {
                const int a = A[i], b = Bv[j];
                if (a == b) {
                    hits++;
                    if (MODE == 1) {
                        atomicAdd(per_vertex + a, 1ull);
                        atomicAdd(per_vertex + u, 1ull);
                        atomicAdd(per_vertex + v, 1ull);
                    }
                    if (MODE == 3)
                        tc_credit_edges(g.esup, g.ceid[cb + c], g.feid[vb + j], g.feid[ub + i]);
                    i++;
                    j++;
                } else if (a < b) {
                    i++;
                } else {
                    j++;
                }
            }
            if (MODE == 2) {
                if (flp) { if (hits) atomicAdd(per_vertex + v, (unsigned long long)hits); }
                else cu += hits;
            }
            mine += hits;
        }
        if (MODE == 2 && cu) atomicAdd(per_vertex + u, (unsigned long long)cu);
    }
    for (int o = 16; o; o >>= 1) mine += __shfl_down_sync(0xFFFFFFFFu, mine, o);
    if ((threadIdx.x & 31) == 0) s_sum[threadIdx.x >> 5] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < 8; w++) t += s_sum[w];
        if (t) atomicAdd(total_out, t);
    }
}

// Five CTAs per SM for the plain count (48 registers, no spills); the
// modes that credit vertices or edges carry more state and get 64.
template <int MODE>
__global__ void __launch_bounds__(kTcWarps * 32, MODE == 0 ? 5 : 4)
k_tc_warp(TcView g, int nV, unsigned long long* __restrict__ per_vertex,
          unsigned long long* __restrict__ total_out,
          int* __restrict__ counters /*[0] next vertex, [1] mid, [2] huge list size*/,
          long long* __restrict__ big, long long big_cap, int warp_cap, int mid_cap,
          long long warp_work, long long item_work, int chunk, int narrow_min, int small_du,
          int small_dc) {
    __shared__ __align__(16) int s_tab[kTcWarps][kWarpTab];
    __shared__ unsigned s_filt[kTcWarps][kWarpTab / 4];
    // MODE 3: edge id (u, w) of each table slot, kWarpTab per warp (dynamic)
    extern __shared__ int s_teid[];
    __shared__ int s_pref[kTcWarps][33];
    __shared__ long long s_vb[kTcWarps][32];
    __shared__ int s_v[kTcWarps][32];
    __shared__ unsigned s_fc[kTcWarps][32];   // MODE 2: hits owned by each candidate
    __shared__ unsigned long long s_sum[kTcWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int* tab = s_tab[warp];
    unsigned long long mine = 0;
    while (true) {
        int u0 = 0;
        if (lane == 0) u0 = atomicAdd(counters, chunk);
        u0 = __shfl_sync(0xFFFFFFFFu, u0, 0);
        if (u0 >= nV) break;
        int u1 = u0 + chunk < nV ? u0 + chunk : nV;
        for (int u = u0; u < u1; u++) {
            long long ub = g.offp[u];
            int du = (int)(g.offp[u + 1] - ub);
            const long long cb = g.coff[u];
            const int dc = (int)(g.coff[u + 1] - cb);
            if (du == 0 || dc == 0) continue;
            if (du <= small_du && dc <= small_dc) continue;   // k_tc_thread's
            // every probed list of u is at most du long: dc * du bounds u's pairs
            if (du > warp_cap || (long long)dc * du > warp_work) {
                // listed: one work item (u, chunk) per item_cands candidates;
                // mid items from the front of `big`, huge items from the back
                if (lane == 0) {
                    const int ipc = item_cands(du, item_work);
                    const int nch = (dc + ipc - 1) / ipc;
                    if (du <= mid_cap) {
                        const int p = atomicAdd(counters + 1, nch);
                        for (int c = 0; c < nch; c++) big[p + c] = ((long long)u << 32) | c;
                    } else {
                        const int p = atomicAdd(counters + 2, nch);
                        for (int c = 0; c < nch; c++)
                            big[big_cap - 1 - (p + c)] = ((long long)u << 32) | c;
                    }
                }
                continue;
            }
            int bits = 32 - __clz(2 * du - 1);   // table of 2^bits >= 2*du slots
            if (bits < 5) bits = 5;
            unsigned* filt = s_filt[warp];
            for (int i = lane; i < (1 << bits); i += 32) tab[i] = -1;
            for (int i = lane; i < (1 << (bits - 2)); i += 32) filt[i] = 0u;
            __syncwarp();
            int* teid = MODE == 3 ? s_teid + warp * kWarpTab : nullptr;
            for (int i = lane; i < du; i += 32) {
                const unsigned h = tab_insert_f(tab, filt, bits, g.fwd[ub + i]);
                if (MODE == 3) teid[h] = g.feid[ub + i];
            }
            __syncwarp();
            const unsigned long long cu = tc_vertex_warp<MODE, true>(
                u, g.fwd + ub, du, g.cand + cb, dc, tab, filt, teid, bits, narrow_min, nullptr, g,
                s_pref[warp], s_vb[warp], s_v[warp], s_fc[warp], per_vertex);
            mine += cu;
            __syncwarp();
        }
    }
    for (int o = 16; o; o >>= 1) mine += __shfl_down_sync(0xFFFFFFFFu, mine, o);
    if (lane == 0) s_sum[warp] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kTcWarps; w++) t += s_sum[w];
        if (t) atomicAdd(total_out, t);
    }
}

// Listed vertices (d+(u) > warp_cap): one CTA each, its warps claiming
// groups of 32 candidates from a shared counter.  Two launches: the mid list
// (d+(u) <= tc.mid_cap, several CTAs per SM) and the huge list (d+(u) up to
// tc.cta_table_cap in a table, binary search of N+(u) beyond that).  A
// table of d entries takes the power of two >= 2*d slots, so the dynamic
// shared memory holds tc_table_slots(cap) slots and their filter.  The
// lists share `big` (items (u << 32) | chunk, each item_cands(d+(u))
// candidates of u): mid from the front (counters[1] entries), huge from the
// back (counters[2] entries).
template <int MODE>
__global__ void __launch_bounds__(kTcWarps * 32, 4)
k_tc_cta(TcView g, int nV, unsigned long long* __restrict__ per_vertex,
         unsigned long long* __restrict__ total_out, const int* __restrict__ counters,
         const long long* __restrict__ big, long long big_cap, long long item_work, int narrow_min,
         int huge, int cap) {
    extern __shared__ __align__(16) int s_dyn[];
    __shared__ int s_pref[kTcWarps][33];
    __shared__ long long s_vb[kTcWarps][32];
    __shared__ int s_v[kTcWarps][32];
    __shared__ unsigned s_fc[kTcWarps][32];   // MODE 2: hits owned by each candidate
    __shared__ unsigned long long s_sum[kTcWarps];
    __shared__ int s_next;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nbig = counters[huge ? 2 : 1];
    unsigned long long mine = 0;
    for (int i = blockIdx.x; i < nbig; i += gridDim.x) {
        const long long item = huge ? big[big_cap - 1 - i] : big[i];
        const int u = (int)(item >> 32);
        const int ch = (int)(item & 0xFFFFFFFF);
        long long ub = g.offp[u];
        int du = (int)(g.offp[u + 1] - ub);
        const int ipc = item_cands(du, item_work);
        const long long cb = g.coff[u] + (long long)ch * ipc;
        const int rest = (int)(g.coff[u + 1] - cb);
        const int dc = rest < ipc ? rest : ipc;
        const int* tab = nullptr;
        unsigned* filt = (unsigned*)(s_dyn + tc_table_slots(cap));
        int* teid = MODE == 3 ? (int*)(filt + tc_table_slots(cap) / 4) : nullptr;
        int bits = 0;
        if (threadIdx.x == 0) s_next = 0;
        if (du <= cap) {
            bits = 32 - __clz(2 * du - 1);
            if (bits < 5) bits = 5;
            for (int j = threadIdx.x; j < (1 << bits); j += blockDim.x) s_dyn[j] = -1;
            for (int j = threadIdx.x; j < (1 << (bits - 2)); j += blockDim.x) filt[j] = 0u;
            __syncthreads();
            for (int j = threadIdx.x; j < du; j += blockDim.x) {
                const unsigned h = tab_insert_f(s_dyn, filt, bits, g.fwd[ub + j]);
                if (MODE == 3) teid[h] = g.feid[ub + j];
            }
            tab = s_dyn;
        }
        __syncthreads();
        const unsigned long long cu =
            tab ? tc_vertex_warp<MODE, true>(u, g.fwd + ub, du, g.cand + cb, dc, tab, filt, teid,
                                             bits, narrow_min, &s_next, g, s_pref[warp],
                                             s_vb[warp], s_v[warp], s_fc[warp], per_vertex)
                : tc_vertex_warp<MODE, false>(u, g.fwd + ub, du, g.cand + cb, dc, tab, filt, teid,
                                              bits, narrow_min, &s_next, g, s_pref[warp],
                                              s_vb[warp], s_v[warp], s_fc[warp], per_vertex);
        mine += cu;
        __syncthreads();
    }
    for (int o = 16; o; o >>= 1) mine += __shfl_down_sync(0xFFFFFFFFu, mine, o);
    if (lane == 0) s_sum[warp] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kTcWarps; w++) t += s_sum[w];
        if (t) atomicAdd(total_out, t);
    }
}

}  // namespace

void build_oriented(hn_graph* g, Oriented& o, const int32_t* canon) {
    cudaStream_t s = g->stream;
    const int nV = g->nV;
    const long long m = g->nE;
    o.prefix.alloc((size_t)nV + 1, s);
    degree_prefix(g, nullptr, nV, o.prefix.get());
    DevBuf<int32_t> pos((size_t)m + 1, s);
    const long long grid = (long long)g->info.sms * 8;
    DevBuf<long long> splits;
    lb_splits(g, o.prefix.get(), nV, m, Tile::TILE, splits);
    HN_LAUNCH(k_orient_flags, grid, kB, 0, s, o.prefix.get(), nV, g->vtab, g->pool, pos.get(),
              splits.get(), (long long)splits.n - 1);
    exclusive_scan(g, (const int32_t*)pos.get(), pos.get(), m + 1, s);
    o.offp.alloc((size_t)nV + 1, s);
    o.fwd.alloc((size_t)(m + 4), s);
    if (canon) o.feid.alloc((size_t)(m + 4), s);
    HN_LAUNCH(k_orient_fill, grid, kB, 0, s, o.prefix.get(), nV, g->vtab, g->pool, pos.get(),
              o.fwd.get(), o.offp.get(), splits.get(), (long long)splits.n - 1, canon,
              canon ? o.feid.get() : (int32_t*)nullptr);
}

// C(z) for every vertex z: offsets coff (nV+1) and lists cand.
void build_candidates(hn_graph* g, const Oriented& o, DevBuf<long long>& coff,
                      DevBuf<int32_t>& cand, DevBuf<int32_t>* ceid) {
    cudaStream_t s = g->stream;
    const int nV = g->nV;
    const long long m = g->nE;   // bound on the oriented edge count (read on the device)
    DevBuf<int> cnt((size_t)nV + 1, s);
    HN_CUDA(cudaMemsetAsync(cnt.get(), 0, sizeof(int) * ((size_t)nV + 1), s));
    DevBuf<long long> splits;
    lb_splits(g, o.offp.get(), nV, m, Tile::TILE, splits);
    const long long grid = (long long)g->info.sms * 8;
    coff.alloc((size_t)nV + 1, s);
    cand.alloc((size_t)m + 4, s);
    HN_LAUNCH(k_cand<false>, grid, kB, 0, s, o.offp.get(), nV, o.fwd.get(), cnt.get(),
              (const long long*)nullptr, (int32_t*)nullptr, splits.get(), (long long)splits.n - 1,
              (const int32_t*)nullptr, (int32_t*)nullptr);
    exclusive_scan(g, (const int*)cnt.get(), coff.get(), (long long)nV + 1, s);
    HN_CUDA(cudaMemsetAsync(cnt.get(), 0, sizeof(int) * ((size_t)nV + 1), s));
    if (ceid) ceid->alloc((size_t)m + 4, s);
    HN_LAUNCH(k_cand<true>, grid, kB, 0, s, o.offp.get(), nV, o.fwd.get(), cnt.get(),
              (const long long*)coff.get(), cand.get(), splits.get(), (long long)splits.n - 1,
              ceid ? (const int32_t*)o.feid.get() : (const int32_t*)nullptr,
              ceid ? ceid->get() : (int32_t*)nullptr);
}

// mode 0: total only; 1: per-vertex counts (each triangle credited to its
// three vertices); 2: owner counts (each triangle credited once, to its
// lowest vertex in the degree orientation).
// Dynamic shared memory of a listed-vertex table of up to `cap` entries:
// its slots, their filter (8 bits per slot) and, for edge support, the edge
// id of each slot.
constexpr size_t tc_table_bytes(int cap, bool eid = false) {
    return (size_t)tc_table_slots(cap) * (sizeof(int) + 1 + (eid ? sizeof(int) : 0));
}
constexpr int kCtaCapEid = 8192;   // largest table with edge ids (147 KB)

template <int MODE>
void launch_counting(hn_graph* g, const TcView& view, unsigned long long* d_counts,
                     unsigned long long* d_total, int* counters, long long* big,
                     long long big_cap, bool flipped) {
    cudaStream_t s = g->stream;
    const long long gw = (long long)g->info.sms * knob(kKnobTcWarpCtasPerSm);
    const int warp_cap = (int)knob(kKnobTcWarpCap);
    const int chunk = (int)knob(kKnobTcChunk);
    const int narrow_min = (int)knob(kKnobTcNarrowMin);
    const long long warp_work = knob(kKnobTcWarpWork), item_work = knob(kKnobTcItemWork);
    constexpr bool eid = MODE == 3;
    const int cap_max = eid ? kCtaCapEid : kCtaCap;
    const int mid_cap = (int)knob(kKnobTcMidCap);
    const int cta_cap = (int)std::min<long long>(knob(kKnobTcCtaTableCap), cap_max);
    const size_t dyn_mid = tc_table_bytes(mid_cap, eid), dyn_huge = tc_table_bytes(cta_cap, eid);
    const size_t dyn_warp = eid ? (size_t)kTcWarps * kWarpTab * sizeof(int) : 0;
    static bool attr_set = false;   // one attribute per instantiation
    if (!attr_set) {
        HN_CUDA(cudaFuncSetAttribute(k_tc_cta<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)tc_table_bytes(cap_max, eid)));
        HN_CUDA(cudaFuncSetAttribute(k_tc_warp<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)dyn_warp));
        attr_set = true;
    }
    int mid_per_sm = 0;
    HN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&mid_per_sm, k_tc_cta<MODE>,
                                                          kTcWarps * 32, dyn_mid));
    if (mid_per_sm < 1) mid_per_sm = 1;
    // small vertices by thread (only with the smaller-side assignment, which
    // bounds every probed list by d+(u))
    const int small_du = flipped ? (int)knob(kKnobTcThreadDu) : 0;
    const int small_dc = (int)knob(kKnobTcThreadDc);
    if (small_du > 0)
        HN_LAUNCH(k_tc_thread<MODE>, (long long)g->info.sms * 8, 256, 0, s, view, g->nV, small_du,
                  small_dc, d_counts, d_total);
    HN_LAUNCH(k_tc_warp<MODE>, gw, kTcWarps * 32, dyn_warp, s, view, g->nV, d_counts, d_total,
              counters, big, big_cap, warp_cap, mid_cap, warp_work, item_work, chunk, narrow_min,
              small_du, small_dc);
    HN_LAUNCH(k_tc_cta<MODE>, (long long)g->info.sms * mid_per_sm, kTcWarps * 32, dyn_mid, s, view,
              g->nV, d_counts, d_total, counters, big, big_cap, item_work, narrow_min, 0, mid_cap);
    HN_LAUNCH(k_tc_cta<MODE>, (long long)g->info.sms, kTcWarps * 32, dyn_huge, s, view, g->nV,
              d_counts, d_total, counters, big, big_cap, item_work, narrow_min, 1, cta_cap);
}

namespace {

// mode 0: total; 1: per-vertex counts; 2: owner counts; 3: edge supports.
unsigned long long run_counting(hn_graph* g, const Oriented& o, int mode,
                                unsigned long long* d_counts, int* esup) {
    cudaStream_t s = g->stream;
    unsigned long long* d_total = (unsigned long long*)g->d_scalar;
    HN_CUDA(cudaMemsetAsync(d_total, 0, sizeof(unsigned long long), s));
    int* counters = (int*)(g->d_scalar + 1);  // next vertex, mid and huge list sizes
    HN_CUDA(cudaMemsetAsync(counters, 0, 3 * sizeof(int), s));
    // work items: at most one per vertex plus one per 32 candidates
    const long long big_cap = (long long)g->nV + g->nE / 32 + 2;
    DevBuf<long long> big((size_t)big_cap, s);
    // candidate lists: each oriented edge with the endpoint of the longer
    // out-list (owner counts credit the edge's tail, the lowest vertex of
    // the triangles it finds, which a flipped entry names)
    // (tc.flip = 0: every edge stays with its tail, C(u) = N+(u); edge
    // supports always use the lists)
    DevBuf<long long> coff;
    DevBuf<int32_t> cand, ceid;
    TcView view{o.offp.get(), o.fwd.get(), o.offp.get(), o.fwd.get(), nullptr, nullptr, nullptr};
    const bool flipped = mode == 3 || knob(kKnobTcFlip);
    if (flipped) {
        build_candidates(g, o, coff, cand, mode == 3 ? &ceid : nullptr);
        view.coff = coff.get();
        view.cand = cand.get();
    }
    if (mode == 3) {
        view.feid = o.feid.get();
        view.ceid = ceid.get();
        view.esup = esup;
    }
    if (d_counts) HN_CUDA(cudaMemsetAsync(d_counts, 0, sizeof(unsigned long long) * g->nV, s));
    long long* bp = big.get();
    switch (mode) {
        case 0: launch_counting<0>(g, view, nullptr, d_total, counters, bp, big_cap, flipped); break;
        case 1: launch_counting<1>(g, view, d_counts, d_total, counters, bp, big_cap, flipped); break;
        case 2: launch_counting<2>(g, view, d_counts, d_total, counters, bp, big_cap, flipped); break;
        default: launch_counting<3>(g, view, nullptr, d_total, counters, bp, big_cap, flipped);
    }
    read_scalars(g, 1);
    return (unsigned long long)g->h_scalar[0];
}

}  // namespace

unsigned long long count_triangles(hn_graph* g, const Oriented& o, unsigned long long* d_counts,
                                   int mode) {
    return run_counting(g, o, d_counts ? mode : 0, d_counts, nullptr);
}

unsigned long long edge_support(hn_graph* g, const Oriented& o, int32_t* sup) {
    HN_REQUIRE(o.feid.get() != nullptr, "edge support needs an orientation built with edge ids");
    return run_counting(g, o, 3, nullptr, sup);
}

}  // namespace hn

using namespace hn;

extern "C" int hn_tc(hn_graph_t* g, uint64_t* per_vertex, int mem, uint64_t* total) {
    HN_API_BEGIN
    HN_REQUIRE(g != nullptr, "graph is null");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    HandleUse use(g);
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    if (g->nV == 0) {
        if (total) *total = 0;
        return HN_OK;
    }
    Oriented o;
    build_oriented(g, o);
    DevBuf<unsigned long long> pv;
    unsigned long long* d_pv = nullptr;
    if (per_vertex) {
        if (mem == HN_MEM_HOST) {
            pv.alloc((size_t)g->nV, s);
            d_pv = pv.get();
        } else {
            d_pv = (unsigned long long*)per_vertex;
        }
    }
    unsigned long long t = count_triangles(g, o, d_pv);
    if (per_vertex && mem == HN_MEM_HOST)
        HN_CUDA(cudaMemcpyAsync(per_vertex, d_pv, sizeof(unsigned long long) * g->nV,
                                cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    if (total) *total = t;
    HN_API_END
}

extern "C" int hn_tc_owner(hn_graph_t* g, uint64_t* counts, int mem, uint64_t* total) {
    HN_API_BEGIN
    HN_REQUIRE(g && counts, "null argument");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    if (g->nV == 0) {
        if (total) *total = 0;
        return HN_OK;
    }
    Oriented o;
    build_oriented(g, o);
    DevBuf<unsigned long long> buf;
    unsigned long long* d_c = (unsigned long long*)counts;
    if (mem == HN_MEM_HOST) {
        buf.alloc((size_t)g->nV, s);
        d_c = buf.get();
    }
    unsigned long long t = count_triangles(g, o, d_c, 2);
    if (mem == HN_MEM_HOST)
        HN_CUDA(cudaMemcpyAsync(counts, d_c, sizeof(unsigned long long) * g->nV,
                                cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    if (total) *total = t;
    HN_API_END
}
