// Internal graph / batch objects behind the C ABI handles.
#pragma once

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "hn_internal.cuh"

namespace hn {

void count_launch(int n = 1);

// Optional per-kernel timing with CUDA events recorded on the launching
// stream (enabled by hn_profile_enable; off by default).
extern bool g_profiling;
void profile_begin(cudaStream_t s, cudaEvent_t* a);
void profile_end(const char* name, cudaStream_t s, cudaEvent_t a);

// Records the stream time of a region (library calls such as CUB sorts and
// scans, or a host round trip) under `name` when profiling is enabled.
struct ProfileScope {
    const char* name;
    cudaStream_t s;
    cudaEvent_t ev = nullptr;
    ProfileScope(const char* n, cudaStream_t st) : name(n), s(st) {
        if (g_profiling) profile_begin(s, &ev);
    }
    ~ProfileScope() {
        if (ev) profile_end(name, s, ev);
    }
    ProfileScope(const ProfileScope&) = delete;
    ProfileScope& operator=(const ProfileScope&) = delete;
};

// Launch a kernel on `stream` and count it.  Grids of size 0 are skipped.
#define HN_LAUNCH(kernel, grid, block, smem, stream, ...)                    \
    do {                                                                     \
        long long _g = (long long)(grid);                                    \
        if (_g > 0) {                                                        \
            cudaEvent_t _ev0 = nullptr;                                      \
            if (::hn::g_profiling) ::hn::profile_begin((stream), &_ev0);     \
            kernel<<<(unsigned)_g, (block), (smem), (stream)>>>(__VA_ARGS__);\
            if (_ev0) ::hn::profile_end(#kernel, (stream), _ev0);            \
            ::hn::count_launch();                                            \
            HN_CUDA(cudaGetLastError());                                     \
        }                                                                    \
    } while (0)

// Stream-ordered temporary device buffer (cudaMallocAsync on the graph's
// stream; the memory returns to the device pool, not to the driver).
template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    DevBuf() = default;
    DevBuf(size_t count, cudaStream_t st) { alloc(count, st); }
    void alloc(size_t count, cudaStream_t st) {
        release();
        s = st;
        n = count;
        if (count) HN_CUDA(cudaMallocAsync((void**)&p, count * sizeof(T), st));
    }
    void release() {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            n = o.n;
            s = o.s;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
    T* get() const { return p; }
};

// Grow-only persistent device buffer (kept across calls on one graph).
struct Persist {
    void* p = nullptr;
    size_t bytes = 0;
    template <typename T>
    T* ensure(size_t count, cudaStream_t st) {
        size_t need = count * sizeof(T);
        if (need > bytes) {
            if (p) HN_CUDA(cudaFreeAsync(p, st));
            size_t nb = need + need / 4 + 256;
            HN_CUDA(cudaMallocAsync(&p, nb, st));
            bytes = nb;
        }
        return (T*)p;
    }
    void release(cudaStream_t st) {
        if (p) cudaFreeAsync(p, st);
        p = nullptr;
        bytes = 0;
    }
};

struct DeviceInfo {
    int sms = 148;
    int max_threads_per_sm = 2048;
};

// Tuning knobs (hn_tune_set / hn_tune_get); read on the host at launch.
enum Knob {
    kKnobBfsCtasPerSm,
    kKnobBfsDoAlpha,
    kKnobBfsDoBeta,
    kKnobMsBlock,
    kKnobMsCtasPerSm,
    kKnobTcWarpCap,
    kKnobTcChunk,
    kKnobTcWarpCtasPerSm,
    kKnobBfsDynamicChunks,
    kKnobBfsWarpStrided,
    kKnobBfsHostLevels,
    kKnobTcNarrowMin,
    kKnobMsBottomUp,
    kKnobTcMidCap,
    kKnobTcCtaTableCap,
    kKnobTcItemWork,
    kKnobTcWarpWork,
    kKnobTcFlip,
    kKnobTcThreadDu,
    kKnobTcThreadDc,
    kKnobBfsKernel,
    kKnobBfsWarpCtasPerSm,
    kKnobKtDeviceRounds,
    kKnobUpdateBigMin,
    kKnobUpdateInPlace,
    kKnobUpdateOwnSort,
    kNumKnobs
};
long long knob(Knob k);

// A device array that grows in place: virtual address range reserved once,
// physical memory mapped onto its end as it grows (no copy, no second
// copy of the data during growth).  Defined in hn_graph.cu.
struct VmArray;
void vm_free(VmArray* a);

struct BfsGraph;
void free_bfs_graph(BfsGraph* bg);
struct MsGraph;
void free_ms_graph(MsGraph* mg);

}  // namespace hn

// C ABI bodies: exceptions become HN_ERR_* codes, never process exits.
// A stale error left by an unchecked call (e.g. a free in a destructor) is
// cleared on entry so it is never reported against this call.
#define HN_API_BEGIN try { (void)cudaGetLastError();
#define HN_API_END                                                   \
    }                                                                \
    catch (const hn::Error& e) {                                     \
        hn::set_last_error(e.what());                                \
        return e.code;                                               \
    }                                                                \
    catch (const std::bad_alloc&) {                                  \
        hn::set_last_error("host allocation failed");                \
        return HN_ERR_OOM;                                           \
    }                                                                \
    catch (const std::exception& e) {                                \
        hn::set_last_error(e.what());                                \
        return HN_ERR_CUDA;                                          \
    }                                                                \
    return HN_OK;
#define HN_REQUIRE(cond, msg) \
    do { if (!(cond)) throw hn::Error(HN_ERR_INVALID, msg); } while (0)

struct hn_graph {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    hn::DeviceInfo info;

    int32_t nV = 0;
    int64_t nE = 0;
    int key_bits = 1;              // bits needed for a vertex id

    hn::VRec* vtab = nullptr;      // nV records
    int32_t* pool = nullptr;       // edge pool
    unsigned long long pool_cap = 0;
    bool weighted = false;         // one 32-bit value per edge slot in wpool
    uint32_t* wpool = nullptr;     // edge weights, parallel to pool (weighted only)
    hn::VmArray* vm_pool = nullptr;    // backing of pool / wpool when the device
    hn::VmArray* vm_wpool = nullptr;   // supports virtual memory management

    hn::AllocState* alloc = nullptr;      // device
    hn::AllocState* h_alloc = nullptr;    // pinned host mirror
    long long* fl[hn::kNumClasses] = {};  // free lists (block offsets)
    int fl_cap[hn::kNumClasses] = {};
    long long** d_fl = nullptr;           // device copy of fl[]
    int fl_count[hn::kNumClasses] = {};   // free blocks per class (host-owned)
    unsigned long long bump_host = 0;     // first never-used pool slot

    long long* h_scalar = nullptr;        // pinned host scalars (16)
    long long* d_scalar = nullptr;        // device scalars (16)

    hn::Persist scratch[8];               // reusable device scratch
    hn::BfsGraph* bfs = nullptr;          // instantiated BFS CUDA graph
    hn::MsGraph* ms = nullptr;            // instantiated batched-BFS CUDA graph

    // a query view (hn_graph_view_create): shares the parent's vertex table
    // and edge pool read-only, owns its stream and scratch
    hn_graph* parent = nullptr;

    // set while a call that uses this handle's stream and scratch runs
    std::atomic<int> in_use{0};
};

namespace hn {
// Stable LSD radix sort of 64-bit keys by their low `bits` bits, carrying
// optional 32-bit values (vals may be null); the *_alt buffers are scratch
// of the same size, and on return keys / vals point at the sorted data.
// A bounded device wait that gave up stores HN_ERR_TIMEOUT in *err (device
// memory).  g may be null (the current device is used).  Defined in
// hn_sort.cu.
void radix_sort_u64(hn_graph* g, unsigned long long*& keys, unsigned long long*& keys_alt,
                    uint32_t*& vals, uint32_t*& vals_alt, long long n, int bits, int* err,
                    cudaStream_t s);

// out[i] = in[0] + ... + in[i-1] (out may be in), on stream s, in OutT.
// Defined in hn_scan.cu for (int, int), (int, long long), (long long,
// long long) and (unsigned long long, unsigned long long).
template <typename InT, typename OutT>
void exclusive_scan(hn_graph* g, const InT* in, OutT* out, long long n, cudaStream_t s);

// Update entry points call this: a query view never changes the graph.
inline void require_owner(const hn_graph* g) {
    if (g->parent) throw Error(HN_ERR_STATE, "a query view cannot update the graph");
}

// Held for the duration of a call that uses the handle's stream and scratch
// (traversals, counts, updates): one handle serves one host thread at a
// time, and a second thread's call on a busy handle is refused instead of
// sharing the scratch.  Concurrent queries use one view per thread.
class HandleUse {
public:
    explicit HandleUse(hn_graph* g) : g_(g) {
        int idle = 0;
        if (!g_->in_use.compare_exchange_strong(idle, 1, std::memory_order_acquire))
            throw Error(HN_ERR_STATE,
                        "graph handle in use by another host thread (use one view per thread)");
    }
    ~HandleUse() { g_->in_use.store(0, std::memory_order_release); }
    HandleUse(const HandleUse&) = delete;
    HandleUse& operator=(const HandleUse&) = delete;

private:
    hn_graph* g_;
};
}  // namespace hn

struct hn_batch {
    hn_graph* g = nullptr;
    int device = 0;          // kept so destroy never touches the graph
    int64_t n = 0;
    int32_t* src = nullptr;  // device copies (owned)
    int32_t* dst = nullptr;
    uint32_t* w = nullptr;   // edge weights (owned)
    bool has_w = false;      // the current contents carry weights
    size_t cap = 0;
    size_t wcap = 0;
};

namespace hn {

// Grid size for a grid-stride loop over n items.
inline long long grid_for(const hn_graph* g, long long n, int block, int per_sm = 8) {
    long long need = (n + block - 1) / block;
    long long lim = (long long)g->info.sms * per_sm;
    return need < lim ? need : lim;
}

// Read device scalars back to the host (synchronises the graph stream).
void read_scalars(hn_graph* g, int count);

// (Re)build the vertex table and pool from a device CSR with int64
// offsets; adjacency is sorted when `sorted` is false.
void build_from_csr(hn_graph* g, int32_t nV, int64_t nE, const long long* d_off,
                    const int32_t* d_adj, bool sorted, const uint32_t* d_w = nullptr);

// Device exclusive prefix of degrees over `verts` (or all vertices when
// verts == nullptr), n+1 entries written to `prefix`.
void degree_prefix(hn_graph* g, const int32_t* verts, int32_t n, long long* prefix);

// Check the device error word; throws on error (synchronises).
void check_device_error(hn_graph* g);

// Ensure the pool holds at least `slots` slots (grows by copy).
void ensure_pool(hn_graph* g, unsigned long long slots);
// Free the pool and weight pool (synchronises the graph's stream first
// when they are mapped memory).  Never throws.
void release_pool(hn_graph* g);
// Ensure free list c can hold `count` entries.
void ensure_free_list(hn_graph* g, int c, long long count);

// Tile splits for a merge-path LB kernel over `prefix` (nseg segments,
// at most max_total items, tiles of `tile` merged elements); see
// lb_partition.  Returns the device array (max_tiles + 1 entries).
void lb_splits(hn_graph* g, const long long* prefix, long long nseg, long long max_total,
               int tile, DevBuf<long long>& splits);

// Scratch export of the graph as a contiguous CSR (device, int64 offsets).
void export_csr64(hn_graph* g, long long* off /*nV+1*/, int32_t* adj /*nE*/);

}  // namespace hn
