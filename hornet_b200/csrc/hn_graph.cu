// Graph construction from CSR, queries, export and the C ABI plumbing.
//
// Construction replaces gpu::Hornet(HornetInit&) / initialize()
// (hornet/include/Core/HornetInitialize/HornetInitialize.i.cuh:99-146), whose
// host loop visits every vertex, asks the host BlockArrayManager for a block
// and stages edges in host mirrors.  Here everything runs on the device:
//   1. degrees and block classes (cap = next power of two, as Vertex::limit(),
//      hornet/include/Core/HornetDevice/impl/Vertex.i.cuh:95-104);
//   2. a class histogram and per-class bases with the LARGEST class first, so
//      every block starts on a multiple of its own size (16-byte aligned for
//      cap >= 4) and the initial pool has no holes;
//   3. warp-aggregated per-class ranks place each vertex's block;
//   4. a merge-path load-balanced copy moves the CSR into the pool.
#include <cub/cub.cuh>
#include <cuda.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <map>
#include <string>
#include <vector>

#include "hn_graph.cuh"

namespace hn {

static std::atomic<long long> g_launches{0};
static thread_local std::string g_last_error;

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

bool g_profiling = false;

namespace {
struct KnobDef {
    const char* name;
    long long def, lo, hi;
    bool pow2;   // value must be a power of two
};
const KnobDef kKnobs[kNumKnobs] = {
    {"bfs.ctas_per_sm", 9, 1, 16, false},
    {"bfs.do_alpha", 14, 1, 1 << 20, false},
    {"bfs.do_beta", 24, 1, 1 << 20, false},
    {"msbfs.block", 256, 128, 512, true},
    {"msbfs.ctas_per_sm", 4, 1, 8, false},
    {"tc.warp_cap", 512, 32, 512, false},
    {"tc.chunk", 16, 1, 256, false},
    {"tc.warp_ctas_per_sm", 8, 1, 16, false},
    {"bfs.dynamic_chunks", 0, 0, 1, false},
    {"bfs.warp_strided", 0, 0, 1, false},
    {"bfs.host_levels", 0, 0, 1, false},
    {"tc.narrow_min", 0, 0, 1024, false},
    {"msbfs.bottom_up", 1, 0, 1, false},
    {"tc.mid_cap", 4096, 32, 4096, false},
    {"tc.cta_table_cap", 16384, 32, 16384, false},
    {"tc.item_work", 1 << 18, 1024, 1 << 30, false},
    {"tc.warp_work", 1 << 16, 1024, 1 << 30, false},
    {"tc.flip", 1, 0, 1, false},
    {"tc.thread_du", 16, 0, 64, false},
    {"tc.thread_dc", 32, 1, 1024, false},
    {"bfs.kernel", 1, 0, 1, false},
    {"bfs.warp_ctas_per_sm", 4, 1, 8, false},
    {"ktruss.device_rounds", 1, 0, 1, false},
    {"update.big_min", 2048, 4, 1 << 30, false},
    {"update.in_place", 1, 0, 1, false},
    {"update.own_sort", 1, 0, 1, false},
};
std::atomic<long long> g_knob[kNumKnobs];
// every knob starts at its default (static initialisation, in definition
// order after kKnobs)
struct KnobDefaults {
    KnobDefaults() {
        for (int i = 0; i < kNumKnobs; i++) g_knob[i].store(kKnobs[i].def, std::memory_order_relaxed);
    }
} g_knob_defaults;

int knob_index(const char* name) {
    if (!name) return -1;
    for (int i = 0; i < kNumKnobs; i++)
        if (std::strcmp(name, kKnobs[i].name) == 0) return i;
    return -1;
}
}  // namespace

long long knob(Knob k) { return g_knob[k].load(std::memory_order_relaxed); }
struct ProfRec {
    std::string name;
    cudaEvent_t a, b;
};
static std::vector<ProfRec> g_prof;
static std::mutex g_prof_mu;

void profile_begin(cudaStream_t s, cudaEvent_t* a) {
    cudaEventCreate(a);
    cudaEventRecord(*a, s);
}

void profile_end(const char* name, cudaStream_t s, cudaEvent_t a) {
    cudaEvent_t b;
    cudaEventCreate(&b);
    cudaEventRecord(b, s);
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_prof.push_back({name, a, b});
}

void set_last_error(const std::string& s) { g_last_error = s; }

void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
    if (e == cudaSuccess) return;
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e),
                  file, line);
    cudaGetLastError();  // clear a non-sticky error
    throw Error(e == cudaErrorMemoryAllocation ? HN_ERR_OOM : HN_ERR_CUDA, buf);
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

__global__ void k_off32_to_64(const int32_t* __restrict__ in, long long* __restrict__ out,
                              long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = in[i];
}

// Offsets must start at 0, be non-decreasing and end at nE; ids in [0,nV).
__global__ void k_validate_csr(const long long* __restrict__ off,
                               const int32_t* __restrict__ adj, int nV, long long nE,
                               AllocState* st) {
    long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long stride = (long long)gridDim.x * blockDim.x;
    bool bad = false;
    if (tid == 0) bad |= (off[0] != 0) || (off[nV] != nE);
    for (long long v = tid; v < nV; v += stride) bad |= off[v + 1] < off[v];
    for (long long e = tid; e < nE; e += stride) {
        int x = adj[e];
        bad |= (x < 0) || (x >= nV);
    }
    if (bad) atomicExch(&st->error, HN_ERR_INVALID);
}

__device__ __forceinline__ int pow2_ceil_int(int d) {
    return d <= 1 ? d : (int)(1u << (32 - __clz(d - 1)));
}

// Degrees, capacities and the class histogram.
// Sorting an unsorted CSR's lists: the row of entry i is the number of
// vertices v >= 1 whose list starts at or before i, an inclusive scan of the
// row-start marks; entries become keys row << L | neighbour, which the
// batch radix sort orders (stably, weights carried), and the neighbours
// are read back out of the sorted keys.
__global__ void k_row_marks(const long long* __restrict__ off, int nV, long long nE,
                            int* __restrict__ mark) {
    for (long long v = 1 + blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x)
        if (off[v] < nE) atomicAdd(mark + off[v], 1);
}

__global__ void k_csr_keys(const int* __restrict__ mark, const int* __restrict__ rows_excl,
                           const int32_t* __restrict__ adj, long long nE, int L,
                           unsigned long long* __restrict__ keys) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nE;
         i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long row = (unsigned)(rows_excl[i] + mark[i]);
        keys[i] = (row << L) | (unsigned)adj[i];
    }
}

__global__ void k_keys_dst(const unsigned long long* __restrict__ keys, long long nE, int L,
                           int32_t* __restrict__ adj) {
    const unsigned long long mask = (1ull << L) - 1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nE;
         i += (long long)gridDim.x * blockDim.x)
        adj[i] = (int32_t)(keys[i] & mask);
}

__global__ void k_class_hist(const long long* __restrict__ off, int nV, VRec* vtab,
                             AllocState* st) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x) {
        int deg = (int)(off[v + 1] - off[v]);
        int cap = pow2_ceil_int(deg);
        VRec r;
        r.off = 0;
        r.deg = deg;
        r.cap = cap;
        vtab[v] = r;
        if (cap) atomicAdd(&st->need[cap_class(cap)], 1);
    }
}

// Single thread: class bases, largest class first; resets counters.
__global__ void k_class_base(AllocState* st) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    unsigned long long base = 0;
    for (int c = kNumClasses - 1; c >= 0; c--) {
        st->bump_base[c] = base;
        base += (unsigned long long)st->need[c] << c;
        st->rank[c] = 0;
    }
    st->bump = base;
    for (int c = 0; c < kNumClasses; c++) st->need[c] = 0;
}

// Place every block: off = base[class] + rank * cap, ranks warp-aggregated.
__global__ void k_class_place(int nV, VRec* vtab, AllocState* st) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x) {
        int cap = vtab[v].cap;
        int c = cap ? cap_class(cap) : -1;
        unsigned mask = __activemask();
        unsigned grp = __match_any_sync(mask, c);
        int leader = __ffs(grp) - 1;
        int lane = threadIdx.x & 31;
        int base = 0;
        if (c >= 0 && lane == leader) base = atomicAdd(&st->rank[c], __popc(grp));
        base = __shfl_sync(mask, base, leader);
        if (c >= 0) {
            int r = base + __popc(grp & ((1u << lane) - 1));
            vtab[v].off = (long long)(st->bump_base[c] + ((unsigned long long)r << c));
        }
    }
}

constexpr int kLbBlock = 256;
constexpr int kLbItems = 8;
using Tile = LbTile<kLbBlock, kLbItems>;

// CSR -> pool copy, merge-path balanced over (edges, vertex boundaries).
__global__ void __launch_bounds__(kLbBlock)
k_fill_pool(const long long* __restrict__ off, int nV, long long nE,
            const int32_t* __restrict__ adj, const VRec* __restrict__ vtab,
            int32_t* __restrict__ pool, const long long* __restrict__ splits, long long split_tiles,
            const uint32_t* __restrict__ w, uint32_t* __restrict__ wpool) {
    __shared__ Tile t;
    __shared__ long long dst_base[Tile::TILE + 1];
    long long ntiles = (nE + nV + Tile::TILE - 1) / Tile::TILE;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int n = lb_tile_load(t, off, (long long)nV, nE, tile, splits, split_tiles);
        for (int b = threadIdx.x; b <= t.nends; b += kLbBlock) {
            long long v = t.seg0 + b;
            dst_base[b] = v < nV ? vtab[v].off - (b == 0 ? t.start0 : t.ends[b - 1]) : 0;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += kLbBlock) {
            long long e = t.item0 + i;
            pool[dst_base[t.seg[i]] + e] = adj[e];
            if (wpool) wpool[dst_base[t.seg[i]] + e] = w[e];
        }
        __syncthreads();
    }
}

__global__ void k_degrees(const VRec* __restrict__ vtab, const int32_t* __restrict__ verts,
                          int n, long long* __restrict__ deg) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i <= n;
         i += (long long)gridDim.x * blockDim.x) {
        if (i == n) { deg[i] = 0; continue; }
        int v = verts ? verts[i] : (int)i;
        deg[i] = vtab[v].deg;
    }
}

// Graph -> (src,dst) or CSR adjacency, merge-path balanced.
__global__ void __launch_bounds__(kLbBlock)
k_export(const long long* __restrict__ prefix, int nV, long long nE,
         const VRec* __restrict__ vtab, const int32_t* __restrict__ pool,
         int32_t* __restrict__ src, int32_t* __restrict__ dst,
         const long long* __restrict__ splits, long long split_tiles,
         const uint32_t* __restrict__ wpool = nullptr, uint32_t* __restrict__ wout = nullptr) {
    __shared__ Tile t;
    __shared__ long long src_base[Tile::TILE + 1];
    long long ntiles = (nE + nV + Tile::TILE - 1) / Tile::TILE;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int n = lb_tile_load(t, prefix, (long long)nV, nE, tile, splits, split_tiles);
        for (int b = threadIdx.x; b <= t.nends; b += kLbBlock) {
            long long v = t.seg0 + b;
            src_base[b] = v < nV ? vtab[v].off - (b == 0 ? t.start0 : t.ends[b - 1]) : 0;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += kLbBlock) {
            long long e = t.item0 + i;
            int b = t.seg[i];
            if (src) src[e] = (int)(t.seg0 + b);
            dst[e] = pool[src_base[b] + e];
            if (wout) wout[e] = wpool[src_base[b] + e];
        }
        __syncthreads();
    }
}

__global__ void k_off64_to_32(const long long* __restrict__ in, int32_t* __restrict__ out,
                              long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = (int32_t)in[i];
}

// max degree, lowest id on ties: maximise (deg << 32) | (~id)
__global__ void k_max_degree(const VRec* __restrict__ vtab, int nV,
                             unsigned long long* out) {
    unsigned long long best = 0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x) {
        unsigned long long k = ((unsigned long long)(unsigned)vtab[v].deg << 32) |
                               (unsigned)(0xFFFFFFFFu - (unsigned)v);
        best = k > best ? k : best;
    }
    for (int o = 16; o; o >>= 1) {
        unsigned long long x = __shfl_down_sync(0xFFFFFFFFu, best, o);
        best = x > best ? x : best;
    }
    if ((threadIdx.x & 31) == 0 && best) atomicMax(out, best);
}

__global__ void k_degree_out(const VRec* __restrict__ vtab, int nV, int32_t* out) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
         v += (long long)gridDim.x * blockDim.x)
        out[v] = vtab[v].deg;
}

__global__ void k_copy_slots(const int32_t* __restrict__ a, int32_t* __restrict__ b,
                             unsigned long long n) {
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
         i < n; i += (unsigned long long)gridDim.x * blockDim.x)
        b[i] = a[i];
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------

void read_scalars(hn_graph* g, int count) {
    HN_CUDA(cudaMemcpyAsync(g->h_scalar, g->d_scalar, sizeof(long long) * count,
                            cudaMemcpyDeviceToHost, g->stream));
    HN_CUDA(cudaStreamSynchronize(g->stream));
}

void check_device_error(hn_graph* g) {
    int err = 0;
    HN_CUDA(cudaMemcpyAsync(&g->h_alloc->error, &g->alloc->error, sizeof(int),
                            cudaMemcpyDeviceToHost, g->stream));
    HN_CUDA(cudaStreamSynchronize(g->stream));
    err = g->h_alloc->error;
    if (err) {
        HN_CUDA(cudaMemsetAsync(&g->alloc->error, 0, sizeof(int), g->stream));
        throw Error(err, err == HN_ERR_INVALID ? "invalid input (offsets or ids out of range)"
                                               : "device-side error");
    }
}

// ---- growable device arrays (CUDA virtual memory management) -------------
// The driver entry points are fetched through the runtime
// (cudaGetDriverEntryPoint), so the library does not link the driver
// library itself.
struct VmArray {
    CUdeviceptr base = 0;
    size_t reserved = 0;   // bytes of address space
    size_t mapped = 0;     // bytes backed by device memory
    size_t gran = 0;
    int device = 0;
    std::vector<std::pair<CUmemGenericAllocationHandle, size_t>> chunks;
};

namespace {
typedef CUresult (*PfnGran)(size_t*, const CUmemAllocationProp*, CUmemAllocationGranularity_flags);
typedef CUresult (*PfnReserve)(CUdeviceptr*, size_t, size_t, CUdeviceptr, unsigned long long);
typedef CUresult (*PfnAddrFree)(CUdeviceptr, size_t);
typedef CUresult (*PfnCreate)(CUmemGenericAllocationHandle*, size_t, const CUmemAllocationProp*,
                              unsigned long long);
typedef CUresult (*PfnRelease)(CUmemGenericAllocationHandle);
typedef CUresult (*PfnMap)(CUdeviceptr, size_t, size_t, CUmemGenericAllocationHandle,
                           unsigned long long);
typedef CUresult (*PfnUnmap)(CUdeviceptr, size_t);
typedef CUresult (*PfnAccess)(CUdeviceptr, size_t, const CUmemAccessDesc*, size_t);
typedef CUresult (*PfnDeviceGet)(CUdevice*, int);
typedef CUresult (*PfnDevAttr)(int*, CUdevice_attribute, CUdevice);

struct VmApi {
    PfnGran gran = nullptr;
    PfnReserve reserve = nullptr;
    PfnAddrFree addr_free = nullptr;
    PfnCreate create = nullptr;
    PfnRelease release = nullptr;
    PfnMap map = nullptr;
    PfnUnmap unmap = nullptr;
    PfnAccess access = nullptr;
    PfnDeviceGet device_get = nullptr;
    PfnDevAttr dev_attr = nullptr;
    bool ok = false;
};

const VmApi& vm_api() {
    static VmApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        auto get = [](const char* name, void** fn) {
            cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
            return cudaGetDriverEntryPoint(name, fn, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess && *fn != nullptr;
        };
        api.ok = get("cuMemGetAllocationGranularity", (void**)&api.gran) &&
                 get("cuMemAddressReserve", (void**)&api.reserve) &&
                 get("cuMemAddressFree", (void**)&api.addr_free) &&
                 get("cuMemCreate", (void**)&api.create) &&
                 get("cuMemRelease", (void**)&api.release) &&
                 get("cuMemMap", (void**)&api.map) && get("cuMemUnmap", (void**)&api.unmap) &&
                 get("cuMemSetAccess", (void**)&api.access) &&
                 get("cuDeviceGet", (void**)&api.device_get) &&
                 get("cuDeviceGetAttribute", (void**)&api.dev_attr);
        (void)cudaGetLastError();
    });
    return api;
}

CUmemAllocationProp vm_prop(int device) {
    CUmemAllocationProp prop = {};
    prop.type = CU_MEM_ALLOCATION_TYPE_PINNED;
    prop.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
    prop.location.id = device;
    return prop;
}

// Whether this device's arrays can grow in place.
bool vm_usable(int device) {
    const VmApi& api = vm_api();
    if (!api.ok) return false;
    CUdevice dev;
    int v = 0;
    if (api.device_get(&dev, device) != CUDA_SUCCESS) return false;
    if (api.dev_attr(&v, CU_DEVICE_ATTRIBUTE_VIRTUAL_MEMORY_MANAGEMENT_SUPPORTED, dev) !=
        CUDA_SUCCESS)
        return false;
    return v != 0;
}

void vm_check(CUresult r, const char* what) {
    if (r == CUDA_SUCCESS) return;
    throw Error(r == CUDA_ERROR_OUT_OF_MEMORY ? HN_ERR_OOM : HN_ERR_CUDA,
                std::string(what) + " failed (CUresult " + std::to_string((int)r) + ")");
}

// Map more memory onto the end of `a` until `bytes` are backed.
void vm_grow(VmArray& a, size_t bytes) {
    const VmApi& api = vm_api();
    CUmemAllocationProp prop = vm_prop(a.device);
    if (!a.base) {
        vm_check(api.gran(&a.gran, &prop, CU_MEM_ALLOC_GRANULARITY_RECOMMENDED),
                 "cuMemGetAllocationGranularity");
        size_t free_b = 0, total_b = 0;
        HN_CUDA(cudaMemGetInfo(&free_b, &total_b));
        // address space for the whole device: growth never needs a move
        a.reserved = (total_b + a.gran - 1) / a.gran * a.gran;
        vm_check(api.reserve(&a.base, a.reserved, a.gran, 0, 0), "cuMemAddressReserve");
    }
    if (bytes > a.reserved) throw Error(HN_ERR_OOM, "edge pool larger than device memory");
    while (a.mapped < bytes) {
        size_t want = bytes - a.mapped;
        if (want < a.mapped / 4) want = a.mapped / 4;
        size_t size = (want + a.gran - 1) / a.gran * a.gran;
        if (size > a.reserved - a.mapped) size = a.reserved - a.mapped;
        CUmemGenericAllocationHandle h;
        vm_check(api.create(&h, size, &prop, 0), "cuMemCreate");
        CUresult r = api.map(a.base + a.mapped, size, 0, h, 0);
        if (r != CUDA_SUCCESS) {
            api.release(h);
            vm_check(r, "cuMemMap");
        }
        CUmemAccessDesc desc = {};
        desc.location = prop.location;
        desc.flags = CU_MEM_ACCESS_FLAGS_PROT_READWRITE;
        r = api.access(a.base + a.mapped, size, &desc, 1);
        a.chunks.push_back({h, size});
        a.mapped += size;
        vm_check(r, "cuMemSetAccess");
    }
}
}  // namespace

void vm_free(VmArray* a) {
    if (!a) return;
    const VmApi& api = vm_api();
    size_t at = 0;
    for (auto& c : a->chunks) {
        api.unmap(a->base + at, c.second);
        api.release(c.first);
        at += c.second;
    }
    if (a->base) api.addr_free(a->base, a->reserved);
    delete a;
}

// Pool (and weight pool) of at least `slots` entries.  With virtual memory
// management the arrays grow in place; otherwise by reallocation and copy.
void ensure_pool(hn_graph* g, unsigned long long slots) {
    if (slots <= g->pool_cap) return;
    unsigned long long ncap = slots + slots / 4 + (1ull << 20);
    if (!g->pool && !g->vm_pool && vm_usable(g->device)) {
        g->vm_pool = new VmArray();
        g->vm_pool->device = g->device;
        if (g->weighted) {
            g->vm_wpool = new VmArray();
            g->vm_wpool->device = g->device;
        }
    }
    if (g->vm_pool) {
        vm_grow(*g->vm_pool, ncap * sizeof(int32_t));
        ncap = g->vm_pool->mapped / sizeof(int32_t);
        g->pool = (int32_t*)g->vm_pool->base;
        if (g->vm_wpool) {
            vm_grow(*g->vm_wpool, ncap * sizeof(uint32_t));
            g->wpool = (uint32_t*)g->vm_wpool->base;
        }
        g->pool_cap = ncap;
        HN_CUDA(cudaMemcpyAsync(&g->alloc->pool_cap, &g->pool_cap, sizeof(unsigned long long),
                                cudaMemcpyHostToDevice, g->stream));
        return;
    }
    int32_t* np = nullptr;
    HN_CUDA(cudaMallocAsync((void**)&np, ncap * sizeof(int32_t), g->stream));
    if (g->pool) {
        unsigned long long used = g->pool_cap;
        HN_CUDA(cudaMemcpyAsync(np, g->pool, used * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                                g->stream));
        HN_CUDA(cudaFreeAsync(g->pool, g->stream));
    }
    if (g->weighted) {
        uint32_t* nw = nullptr;
        HN_CUDA(cudaMallocAsync((void**)&nw, ncap * sizeof(uint32_t), g->stream));
        if (g->wpool) {
            HN_CUDA(cudaMemcpyAsync(nw, g->wpool, g->pool_cap * sizeof(uint32_t),
                                    cudaMemcpyDeviceToDevice, g->stream));
            HN_CUDA(cudaFreeAsync(g->wpool, g->stream));
        }
        g->wpool = nw;
    }
    g->pool = np;
    g->pool_cap = ncap;
    HN_CUDA(cudaMemcpyAsync(&g->alloc->pool_cap, &g->pool_cap, sizeof(unsigned long long),
                            cudaMemcpyHostToDevice, g->stream));
}

void release_pool(hn_graph* g) {
    if (g->vm_pool || g->vm_wpool) {
        cudaStreamSynchronize(g->stream);   // no kernel still reads the pool
        vm_free(g->vm_pool);
        vm_free(g->vm_wpool);
        g->vm_pool = g->vm_wpool = nullptr;
    } else {
        if (g->pool) cudaFreeAsync(g->pool, g->stream);
        if (g->wpool) cudaFreeAsync(g->wpool, g->stream);
    }
    g->pool = nullptr;
    g->wpool = nullptr;
    g->pool_cap = 0;
}

void ensure_free_list(hn_graph* g, int c, long long count) {
    if (count <= g->fl_cap[c]) return;
    long long ncap = count + count / 2 + 1024;
    if (ncap > 0x7FFFFFFF) ncap = 0x7FFFFFFF;
    long long* nl = nullptr;
    HN_CUDA(cudaMallocAsync((void**)&nl, ncap * sizeof(long long), g->stream));
    if (g->fl[c]) {
        HN_CUDA(cudaMemcpyAsync(nl, g->fl[c], (size_t)g->fl_cap[c] * sizeof(long long),
                                cudaMemcpyDeviceToDevice, g->stream));
        HN_CUDA(cudaFreeAsync(g->fl[c], g->stream));
    }
    g->fl[c] = nl;
    g->fl_cap[c] = (int)ncap;
    HN_CUDA(cudaMemcpyAsync(g->d_fl + c, &g->fl[c], sizeof(long long*), cudaMemcpyHostToDevice,
                            g->stream));
    HN_CUDA(cudaStreamSynchronize(g->stream));  // &g->fl[c] is a host source
}

void degree_prefix(hn_graph* g, const int32_t* verts, int32_t n, long long* prefix) {
    HN_LAUNCH(k_degrees, grid_for(g, (long long)n + 1, 256), 256, 0, g->stream, g->vtab, verts,
              n, prefix);
    exclusive_scan(g, (const long long*)prefix, prefix, (long long)n + 1, g->stream);
}

void lb_splits(hn_graph* g, const long long* prefix, long long nseg, long long max_total,
               int tile, DevBuf<long long>& splits) {
    long long max_tiles = (max_total + nseg + tile - 1) / tile + 1;
    splits.alloc((size_t)max_tiles + 1, g->stream);
    HN_LAUNCH(lb_partition<long long>, grid_for(g, max_tiles + 1, 256), 256, 0, g->stream, prefix,
              nseg, tile, max_tiles, splits.get());
}

void export_csr64(hn_graph* g, long long* off, int32_t* adj) {
    degree_prefix(g, nullptr, g->nV, off);
    long long ntiles = (g->nE + g->nV + Tile::TILE - 1) / Tile::TILE;
    DevBuf<long long> splits;
    lb_splits(g, off, g->nV, g->nE, Tile::TILE, splits);
    HN_LAUNCH(k_export, grid_for(g, ntiles, 1, 16), kLbBlock, 0, g->stream, off, g->nV,
              g->nE, g->vtab, g->pool, (int32_t*)nullptr, adj, splits.get(), (long long)splits.n - 1);
}

void build_from_csr(hn_graph* g, int32_t nV, int64_t nE, const long long* d_off,
                    const int32_t* d_adj, bool sorted, const uint32_t* d_w) {
    cudaStream_t s = g->stream;
    // validation
    HN_CUDA(cudaMemsetAsync(g->alloc, 0, sizeof(AllocState), s));
    HN_LAUNCH(k_validate_csr, grid_for(g, nE > nV ? nE : nV + 1, 256), 256, 0, s, d_off, d_adj,
              nV, (long long)nE, g->alloc);
    check_device_error(g);

    // vertex table
    if (g->vtab) HN_CUDA(cudaFreeAsync(g->vtab, s));
    g->vtab = nullptr;
    if (nV) HN_CUDA(cudaMallocAsync((void**)&g->vtab, sizeof(VRec) * (size_t)nV, s));
    g->nV = nV;
    g->nE = nE;
    g->key_bits = nV > 1 ? ceil_log2_u64((unsigned long long)nV) : 1;

    // free lists start empty
    for (int c = 0; c < kNumClasses; c++) {
        if (g->fl[c]) HN_CUDA(cudaFreeAsync(g->fl[c], s));
        g->fl[c] = nullptr;
        g->fl_cap[c] = 0;
    }
    HN_CUDA(cudaMemsetAsync(g->d_fl, 0, sizeof(long long*) * kNumClasses, s));

    HN_LAUNCH(k_class_hist, grid_for(g, nV, 256), 256, 0, s, d_off, nV, g->vtab, g->alloc);
    HN_LAUNCH(k_class_base, 1, 32, 0, s, g->alloc);
    HN_LAUNCH(k_class_place, grid_for(g, nV, 256), 256, 0, s, nV, g->vtab, g->alloc);

    HN_CUDA(cudaMemcpyAsync(g->h_alloc, g->alloc, sizeof(AllocState), cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    unsigned long long used = g->h_alloc->bump;
    g->bump_host = used;
    for (int c = 0; c < kNumClasses; c++) g->fl_count[c] = 0;

    // pool: exact fit plus headroom for updates
    release_pool(g);
    g->weighted = d_w != nullptr;
    ensure_pool(g, used + used / 2 + 1024);

    // sort adjacency lists if needed, then copy into the pool
    const int32_t* src_adj = d_adj;
    const uint32_t* src_w = d_w;
    DevBuf<int32_t> sorted_adj;
    DevBuf<uint32_t> sorted_w;
    if (!sorted && nE > 0 && nE < (1ll << 32) && nV > 1) {
        // the library's radix sort over (row, neighbour) keys; weights carried
        const int L = g->key_bits;
        DevBuf<int> mark((size_t)nE, s), rows((size_t)nE, s);
        HN_CUDA(cudaMemsetAsync(mark.get(), 0, sizeof(int) * (size_t)nE, s));
        HN_LAUNCH(k_row_marks, grid_for(g, nV, 256), 256, 0, s, d_off, nV, (long long)nE,
                  mark.get());
        exclusive_scan(g, (const int*)mark.get(), rows.get(), (long long)nE, s);
        DevBuf<unsigned long long> keys((size_t)nE, s), keys2((size_t)nE, s);
        HN_LAUNCH(k_csr_keys, grid_for(g, nE, 256), 256, 0, s, (const int*)mark.get(),
                  (const int*)rows.get(), d_adj, (long long)nE, L, keys.get());
        mark.release();
        rows.release();
        DevBuf<uint32_t> w2;
        if (d_w) {
            sorted_w.alloc((size_t)nE, s);
            w2.alloc((size_t)nE, s);
            HN_CUDA(cudaMemcpyAsync(sorted_w.get(), d_w, sizeof(uint32_t) * (size_t)nE,
                                    cudaMemcpyDeviceToDevice, s));
        }
        unsigned long long* kc = keys.get();
        unsigned long long* ka = keys2.get();
        uint32_t* vc = d_w ? sorted_w.get() : nullptr;
        uint32_t* va = d_w ? w2.get() : nullptr;
        HN_CUDA(cudaMemsetAsync(&g->alloc->error, 0, sizeof(int), s));
        radix_sort_u64(g, kc, ka, vc, va, (long long)nE, 2 * L, &g->alloc->error, s);
        if (d_w && vc != sorted_w.get()) std::swap(sorted_w.p, w2.p);
        sorted_adj.alloc((size_t)nE, s);
        HN_LAUNCH(k_keys_dst, grid_for(g, nE, 256), 256, 0, s, (const unsigned long long*)kc,
                  (long long)nE, L, sorted_adj.get());
        HN_CUDA(cudaMemcpyAsync(&g->h_alloc->error, &g->alloc->error, sizeof(int),
                                cudaMemcpyDeviceToHost, s));
        HN_CUDA(cudaStreamSynchronize(s));
        if (g->h_alloc->error) {
            HN_CUDA(cudaMemsetAsync(&g->alloc->error, 0, sizeof(int), s));
            throw Error(HN_ERR_TIMEOUT, "adjacency sort: a bounded wait gave up");
        }
        src_adj = sorted_adj.get();
        if (d_w) src_w = sorted_w.get();
    } else if (!sorted && nE > 0 && d_w) {
        // weights follow their edges; equal neighbours keep their input order
        sorted_adj.alloc((size_t)nE, s);
        sorted_w.alloc((size_t)nE, s);
        size_t tb = 0;
        HN_CUDA(cub::DeviceSegmentedSort::StableSortPairs(nullptr, tb, d_adj, sorted_adj.get(), d_w,
                                                          sorted_w.get(), nE, nV, d_off, d_off + 1,
                                                          s));
        DevBuf<char> tmp(tb, s);
        HN_CUDA(cub::DeviceSegmentedSort::StableSortPairs(tmp.get(), tb, d_adj, sorted_adj.get(),
                                                          d_w, sorted_w.get(), nE, nV, d_off,
                                                          d_off + 1, s));
        count_launch();
        src_adj = sorted_adj.get();
        src_w = sorted_w.get();
    } else if (!sorted && nE > 0) {
        sorted_adj.alloc((size_t)nE, s);
        size_t tb = 0;
        HN_CUDA(cub::DeviceSegmentedSort::SortKeys(nullptr, tb, d_adj, sorted_adj.get(), nE, nV,
                                                   d_off, d_off + 1, s));
        DevBuf<char> tmp(tb, s);
        HN_CUDA(cub::DeviceSegmentedSort::SortKeys(tmp.get(), tb, d_adj, sorted_adj.get(), nE,
                                                   nV, d_off, d_off + 1, s));
        count_launch();
        src_adj = sorted_adj.get();
    }
    long long ntiles = ((long long)nE + nV + Tile::TILE - 1) / Tile::TILE;
    DevBuf<long long> splits;
    lb_splits(g, d_off, nV, nE, Tile::TILE, splits);
    HN_LAUNCH(k_fill_pool, grid_for(g, ntiles, 1, 16), kLbBlock, 0, s, d_off, nV,
              (long long)nE, src_adj, g->vtab, g->pool, splits.get(), (long long)splits.n - 1,
              src_w, g->weighted ? g->wpool : (uint32_t*)nullptr);
    HN_CUDA(cudaStreamSynchronize(s));
}

}  // namespace hn

using namespace hn;

namespace {

void init_graph_object(hn_graph* g, int device) {
    g->device = device;
    HN_CUDA(cudaSetDevice(device));
    HN_CUDA(cudaDeviceGetAttribute(&g->info.sms, cudaDevAttrMultiProcessorCount, device));
    HN_CUDA(cudaDeviceGetAttribute(&g->info.max_threads_per_sm,
                                   cudaDevAttrMaxThreadsPerMultiProcessor, device));
    // keep freed stream-ordered memory in the process's pool
    cudaMemPool_t mp;
    HN_CUDA(cudaDeviceGetDefaultMemPool(&mp, device));
    unsigned long long thr = ~0ull;
    HN_CUDA(cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &thr));
    HN_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    g->own_stream = true;
    HN_CUDA(cudaMalloc((void**)&g->alloc, sizeof(AllocState)));
    HN_CUDA(cudaMallocHost((void**)&g->h_alloc, sizeof(AllocState)));
    HN_CUDA(cudaMalloc((void**)&g->d_fl, sizeof(long long*) * kNumClasses));
    HN_CUDA(cudaMallocHost((void**)&g->h_scalar, sizeof(long long) * 16));
    HN_CUDA(cudaMalloc((void**)&g->d_scalar, sizeof(long long) * 16));
}

void free_graph_object(hn_graph* g) {
    if (!g) return;
    cudaSetDevice(g->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
    for (int c = 0; c < kNumClasses; c++)
        if (g->fl[c]) cudaFreeAsync(g->fl[c], g->stream);
    for (auto& p : g->scratch) p.release(g->stream);
    free_bfs_graph(g->bfs);
    g->bfs = nullptr;
    free_ms_graph(g->ms);
    g->ms = nullptr;
    if (g->parent) {
        // a view borrows the parent's vertex table and pool
        g->vtab = nullptr;
        g->pool = nullptr;
        g->wpool = nullptr;
        g->vm_pool = nullptr;
        g->vm_wpool = nullptr;
    }
    if (g->vtab) cudaFreeAsync(g->vtab, g->stream);
    release_pool(g);
    if (g->stream) cudaStreamSynchronize(g->stream);
    cudaFree(g->alloc);
    cudaFreeHost(g->h_alloc);
    cudaFree(g->d_fl);
    cudaFreeHost(g->h_scalar);
    cudaFree(g->d_scalar);
    if (g->own_stream && g->stream) cudaStreamDestroy(g->stream);
    delete g;
    (void)cudaGetLastError();
}

// Copy a CSR into device buffers with int64 offsets.
template <typename OffT>
void stage_csr(hn_graph* g, int32_t nV, int64_t nE, const OffT* off, const int32_t* adj,
               int mem, DevBuf<long long>& d_off, DevBuf<int32_t>& d_adj_own,
               const int32_t*& d_adj) {
    cudaStream_t s = g->stream;
    d_off.alloc((size_t)nV + 1, s);
    if (mem == HN_MEM_HOST) {
        if (sizeof(OffT) == 8) {
            HN_CUDA(cudaMemcpyAsync(d_off.get(), off, sizeof(long long) * ((size_t)nV + 1),
                                    cudaMemcpyHostToDevice, s));
        } else {
            DevBuf<int32_t> o32((size_t)nV + 1, s);
            HN_CUDA(cudaMemcpyAsync(o32.get(), off, sizeof(int32_t) * ((size_t)nV + 1),
                                    cudaMemcpyHostToDevice, s));
            HN_LAUNCH(k_off32_to_64, grid_for(g, (long long)nV + 1, 256), 256, 0, s, o32.get(),
                      d_off.get(), (long long)nV + 1);
        }
        d_adj_own.alloc((size_t)nE, s);
        if (nE)
            HN_CUDA(cudaMemcpyAsync(d_adj_own.get(), adj, sizeof(int32_t) * (size_t)nE,
                                    cudaMemcpyHostToDevice, s));
        d_adj = d_adj_own.get();
    } else {
        if (sizeof(OffT) == 8) {
            HN_CUDA(cudaMemcpyAsync(d_off.get(), off, sizeof(long long) * ((size_t)nV + 1),
                                    cudaMemcpyDeviceToDevice, s));
        } else {
            HN_LAUNCH(k_off32_to_64, grid_for(g, (long long)nV + 1, 256), 256, 0, s,
                      (const int32_t*)off, d_off.get(), (long long)nV + 1);
        }
        d_adj = adj;
    }
}

template <typename OffT>
int create_impl(int32_t nV, int64_t nE, const OffT* off, const int32_t* adj, unsigned flags,
                int mem, int device, hn_graph_t** out, const uint32_t* w = nullptr) {
    HN_API_BEGIN
    HN_REQUIRE(out != nullptr, "out is null");
    *out = nullptr;
    HN_REQUIRE(nV >= 0 && nE >= 0, "negative size");
    HN_REQUIRE(off != nullptr, "offsets are null");
    HN_REQUIRE(nE == 0 || adj != nullptr, "edges are null");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    HN_REQUIRE(sizeof(OffT) == 8 || nE <= 0x7FFFFFFF, "nE exceeds int32 offsets");
    hn_graph* g = new hn_graph();
    try {
        init_graph_object(g, device);
        DevBuf<long long> d_off;
        DevBuf<int32_t> d_adj_own;
        const int32_t* d_adj = nullptr;
        stage_csr(g, nV, nE, off, adj, mem, d_off, d_adj_own, d_adj);
        DevBuf<uint32_t> d_w_own;
        const uint32_t* d_w = w;
        if (w && mem == HN_MEM_HOST) {
            d_w_own.alloc((size_t)nE + 1, g->stream);
            if (nE)
                HN_CUDA(cudaMemcpyAsync(d_w_own.get(), w, sizeof(uint32_t) * (size_t)nE,
                                        cudaMemcpyHostToDevice, g->stream));
            d_w = d_w_own.get();
        } else if (w && nE == 0) {
            d_w_own.alloc(1, g->stream);
            d_w = d_w_own.get();
        }
        build_from_csr(g, nV, nE, d_off.get(), d_adj, (flags & HN_CSR_SORTED) != 0, d_w);
    } catch (...) {
        free_graph_object(g);
        throw;
    }
    *out = g;
    HN_API_END
}

}  // namespace

// The parent's current shape, copied into a view (host fields only).
static void view_copy(hn_graph* v) {
    const hn_graph* p = v->parent;
    v->nV = p->nV;
    v->nE = p->nE;
    v->key_bits = p->key_bits;
    v->vtab = p->vtab;
    v->pool = p->pool;
    v->pool_cap = p->pool_cap;
    v->weighted = p->weighted;
    v->wpool = p->wpool;
}

extern "C" {

const char* hn_last_error_string(void) { return g_last_error.c_str(); }

int hn_version(void) { return 10000; }

int hn_tune_set(const char* name, int64_t value) {
    HN_API_BEGIN
    int i = knob_index(name);
    HN_REQUIRE(i >= 0, "unknown tuning knob");
    const KnobDef& d = kKnobs[i];
    if (value < d.lo || value > d.hi || (d.pow2 && (value & (value - 1))))
        throw Error(HN_ERR_INVALID, std::string("value out of range for ") + d.name);
    g_knob[i].store(value, std::memory_order_relaxed);
    HN_API_END
}

int hn_tune_get(const char* name, int64_t* value) {
    HN_API_BEGIN
    int i = knob_index(name);
    HN_REQUIRE(i >= 0 && value, "unknown tuning knob");
    *value = g_knob[i].load(std::memory_order_relaxed);
    HN_API_END
}

int hn_tune_reset(void) {
    for (int i = 0; i < kNumKnobs; i++) g_knob[i].store(kKnobs[i].def, std::memory_order_relaxed);
    return HN_OK;
}

const char* hn_tune_name(int32_t i) { return i >= 0 && i < kNumKnobs ? kKnobs[i].name : nullptr; }

int64_t hn_kernel_launches(void) { return g_launches.load(); }

int hn_profile_enable(int on) {
    HN_API_BEGIN
    std::lock_guard<std::mutex> lk(g_prof_mu);
    for (auto& r : g_prof) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    g_prof.clear();
    g_profiling = on != 0;
    HN_API_END
}

int hn_profile_report(char* buf, int64_t len) {
    HN_API_BEGIN
    HN_REQUIRE(buf && len > 0, "null buffer");
    std::lock_guard<std::mutex> lk(g_prof_mu);
    std::map<std::string, std::pair<long long, double>> agg;
    for (auto& r : g_prof) {
        HN_CUDA(cudaEventSynchronize(r.b));
        float ms = 0;
        HN_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
        auto& x = agg[r.name];
        x.first++;
        x.second += ms;
    }
    std::string out = "{";
    bool first = true;
    for (auto& kv : agg) {
        char item[256];
        std::snprintf(item, sizeof(item), "%s\"%s\": {\"launches\": %lld, \"ms\": %.6f}",
                      first ? "" : ", ", kv.first.c_str(), kv.second.first, kv.second.second);
        out += item;
        first = false;
    }
    out += "}";
    std::snprintf(buf, (size_t)len, "%s", out.c_str());
    HN_REQUIRE((int64_t)out.size() < len, "report buffer too small");
    HN_API_END
}

int hn_graph_create_csr(int32_t nV, int64_t nE, const int32_t* off, const int32_t* adj,
                        unsigned flags, int mem, int device, hn_graph_t** out) {
    return create_impl<int32_t>(nV, nE, off, adj, flags, mem, device, out);
}

int hn_graph_create_csr_w(int32_t nV, int64_t nE, const int32_t* off, const int32_t* adj,
                          const uint32_t* weights, unsigned flags, int mem, int device,
                          hn_graph_t** out) {
    if (!weights) {
        set_last_error("weights are null");
        return HN_ERR_INVALID;
    }
    return create_impl<int32_t>(nV, nE, off, adj, flags, mem, device, out, weights);
}

int hn_graph_weighted(const hn_graph_t* g, int32_t* weighted) {
    HN_API_BEGIN
    HN_REQUIRE(g && weighted, "null argument");
    *weighted = g->weighted ? 1 : 0;
    HN_API_END
}

int hn_graph_create_csr64(int32_t nV, int64_t nE, const int64_t* off, const int32_t* adj,
                          unsigned flags, int mem, int device, hn_graph_t** out) {
    return create_impl<long long>(nV, nE, (const long long*)off, adj, flags, mem, device, out);
}

int hn_graph_reset_csr(hn_graph_t* g, int32_t nV, int64_t nE, const int32_t* off,
                       const int32_t* adj, unsigned flags, int mem) {
    HN_API_BEGIN
    HN_REQUIRE(g != nullptr, "graph is null");
    HN_REQUIRE(nV >= 0 && nE >= 0 && off != nullptr && (nE == 0 || adj != nullptr),
               "bad CSR");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    require_owner(g);
    HN_CUDA(cudaSetDevice(g->device));
    DevBuf<long long> d_off;
    DevBuf<int32_t> d_adj_own;
    const int32_t* d_adj = nullptr;
    stage_csr(g, nV, nE, off, adj, mem, d_off, d_adj_own, d_adj);
    build_from_csr(g, nV, nE, d_off.get(), d_adj, (flags & HN_CSR_SORTED) != 0);
    HN_API_END
}

int hn_graph_view_create(hn_graph_t* parent, void* stream, hn_graph_t** out) {
    HN_API_BEGIN
    HN_REQUIRE(parent && out, "null argument");
    HN_REQUIRE(!parent->parent, "a view of a view: create it from the graph itself");
    *out = nullptr;
    hn_graph* v = new hn_graph();
    try {
        init_graph_object(v, parent->device);
        v->parent = parent;
        view_copy(v);
        if (stream) {
            HN_CUDA(cudaStreamDestroy(v->stream));
            v->stream = (cudaStream_t)stream;
            v->own_stream = false;
        }
    } catch (...) {
        free_graph_object(v);
        throw;
    }
    *out = v;
    HN_API_END
}

int hn_graph_view_refresh(hn_graph_t* view) {
    HN_API_BEGIN
    HN_REQUIRE(view && view->parent, "not a query view");
    HN_CUDA(cudaSetDevice(view->device));
    // the parent's pending work (an update) finishes before the view reads
    HN_CUDA(cudaStreamSynchronize(view->parent->stream));
    view_copy(view);
    HN_API_END
}

int hn_graph_destroy(hn_graph_t* g) {
    HN_API_BEGIN
    free_graph_object(g);
    HN_API_END
}

int hn_graph_set_stream(hn_graph_t* g, void* stream) {
    HN_API_BEGIN
    HN_REQUIRE(g != nullptr, "graph is null");
    HN_CUDA(cudaSetDevice(g->device));
    HN_CUDA(cudaStreamSynchronize(g->stream));
    if (stream) {
        if (g->own_stream) HN_CUDA(cudaStreamDestroy(g->stream));
        g->stream = (cudaStream_t)stream;
        g->own_stream = false;
    } else if (!g->own_stream) {
        HN_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
        g->own_stream = true;
    }
    HN_API_END
}

int hn_graph_nv(const hn_graph_t* g, int32_t* nV) {
    HN_API_BEGIN
    HN_REQUIRE(g && nV, "null argument");
    *nV = g->nV;
    HN_API_END
}

int hn_graph_ne(const hn_graph_t* g, int64_t* nE) {
    HN_API_BEGIN
    HN_REQUIRE(g && nE, "null argument");
    *nE = g->nE;
    HN_API_END
}

int hn_graph_max_degree(hn_graph_t* g, int32_t* max_degree, int32_t* max_id) {
    HN_API_BEGIN
    HN_REQUIRE(g != nullptr, "graph is null");
    HN_CUDA(cudaSetDevice(g->device));
    HN_CUDA(cudaMemsetAsync(g->d_scalar, 0, sizeof(long long), g->stream));
    HN_LAUNCH(k_max_degree, grid_for(g, g->nV, 256), 256, 0, g->stream, g->vtab, g->nV,
              (unsigned long long*)g->d_scalar);
    read_scalars(g, 1);
    unsigned long long k = (unsigned long long)g->h_scalar[0];
    int deg = (int)(k >> 32);
    int id = k ? (int)(0xFFFFFFFFu - (unsigned)(k & 0xFFFFFFFFu)) : 0;
    if (max_degree) *max_degree = deg;
    if (max_id) *max_id = id;
    HN_API_END
}

int hn_graph_export_coo(hn_graph_t* g, int sorted, int32_t* src, int32_t* dst, int mem) {
    return hn_graph_export_coo_w(g, sorted, src, dst, nullptr, mem);
}

int hn_graph_export_coo_w(hn_graph_t* g, int sorted, int32_t* src, int32_t* dst,
                          uint32_t* weights, int mem) {
    (void)sorted;
    HN_API_BEGIN
    HN_REQUIRE(g && src && dst, "null argument");
    HN_REQUIRE(!weights || g->weighted, "the graph has no weights");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    DevBuf<long long> prefix((size_t)g->nV + 1, s);
    degree_prefix(g, nullptr, g->nV, prefix.get());
    DevBuf<int32_t> ds, dd;
    DevBuf<uint32_t> dw;
    int32_t *ps = src, *pd = dst;
    uint32_t* pw = weights;
    if (mem == HN_MEM_HOST) {
        ds.alloc((size_t)g->nE, s);
        dd.alloc((size_t)g->nE, s);
        ps = ds.get();
        pd = dd.get();
        if (weights) {
            dw.alloc((size_t)g->nE, s);
            pw = dw.get();
        }
    }
    long long ntiles = (g->nE + g->nV + Tile::TILE - 1) / Tile::TILE;
    DevBuf<long long> splits;
    lb_splits(g, prefix.get(), g->nV, g->nE, Tile::TILE, splits);
    HN_LAUNCH(k_export, grid_for(g, ntiles, 1, 16), kLbBlock, 0, s, prefix.get(), g->nV,
              g->nE, g->vtab, g->pool, ps, pd, splits.get(), (long long)splits.n - 1,
              (const uint32_t*)g->wpool, pw);
    if (mem == HN_MEM_HOST && g->nE) {
        HN_CUDA(cudaMemcpyAsync(src, ps, sizeof(int32_t) * g->nE, cudaMemcpyDeviceToHost, s));
        HN_CUDA(cudaMemcpyAsync(dst, pd, sizeof(int32_t) * g->nE, cudaMemcpyDeviceToHost, s));
        if (weights)
            HN_CUDA(cudaMemcpyAsync(weights, pw, sizeof(uint32_t) * g->nE,
                                    cudaMemcpyDeviceToHost, s));
    }
    HN_CUDA(cudaStreamSynchronize(s));
    HN_API_END
}

int hn_graph_export_csr(hn_graph_t* g, int32_t* off, int32_t* adj, int mem) {
    HN_API_BEGIN
    HN_REQUIRE(g && off && adj, "null argument");
    HN_REQUIRE(mem == HN_MEM_HOST || mem == HN_MEM_DEVICE, "bad memory kind");
    HN_REQUIRE(g->nE <= 0x7FFFFFFF, "nE exceeds int32 offsets");
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    DevBuf<long long> prefix((size_t)g->nV + 1, s);
    DevBuf<int32_t> d_off, d_adj;
    int32_t *po = off, *pa = adj;
    if (mem == HN_MEM_HOST) {
        d_off.alloc((size_t)g->nV + 1, s);
        d_adj.alloc((size_t)g->nE, s);
        po = d_off.get();
        pa = d_adj.get();
    }
    export_csr64(g, prefix.get(), pa);
    HN_LAUNCH(k_off64_to_32, grid_for(g, (long long)g->nV + 1, 256), 256, 0, s, prefix.get(),
              po, (long long)g->nV + 1);
    if (mem == HN_MEM_HOST) {
        HN_CUDA(cudaMemcpyAsync(off, po, sizeof(int32_t) * ((size_t)g->nV + 1),
                                cudaMemcpyDeviceToHost, s));
        if (g->nE)
            HN_CUDA(cudaMemcpyAsync(adj, pa, sizeof(int32_t) * g->nE, cudaMemcpyDeviceToHost, s));
    }
    HN_CUDA(cudaStreamSynchronize(s));
    HN_API_END
}

int hn_graph_degrees(hn_graph_t* g, int32_t* deg, int mem) {
    HN_API_BEGIN
    HN_REQUIRE(g && deg, "null argument");
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    DevBuf<int32_t> d;
    int32_t* p = deg;
    if (mem == HN_MEM_HOST) {
        d.alloc((size_t)g->nV, s);
        p = d.get();
    }
    HN_LAUNCH(k_degree_out, grid_for(g, g->nV, 256), 256, 0, s, g->vtab, g->nV, p);
    if (mem == HN_MEM_HOST && g->nV)
        HN_CUDA(cudaMemcpyAsync(deg, p, sizeof(int32_t) * g->nV, cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    HN_API_END
}

int hn_graph_device_view(hn_graph_t* g, hn_device_view_t* view) {
    HN_API_BEGIN
    HN_REQUIRE(g && view, "null argument");
    view->nV = g->nV;
    view->pad = 0;
    view->nE = g->nE;
    view->vtab = g->vtab;
    view->pool = g->pool;
    HN_API_END
}

int hn_graph_memory(hn_graph_t* g, int64_t* pool_slots, int64_t* used_slots,
                    int64_t* free_list_blocks) {
    HN_API_BEGIN
    HN_REQUIRE(g != nullptr, "graph is null");
    HN_CUDA(cudaSetDevice(g->device));
    HN_CUDA(cudaMemcpyAsync(g->h_alloc, g->alloc, sizeof(AllocState), cudaMemcpyDeviceToHost,
                            g->stream));
    HN_CUDA(cudaStreamSynchronize(g->stream));
    if (pool_slots) *pool_slots = (int64_t)g->pool_cap;
    if (used_slots) *used_slots = (int64_t)g->bump_host;
    if (free_list_blocks) {
        long long t = 0;
        for (int c = 0; c < kNumClasses; c++) t += g->fl_count[c];
        *free_list_blocks = t;
    }
    HN_API_END
}

int hn_free_device(void* p) {
    HN_API_BEGIN
    if (p) HN_CUDA(cudaFree(p));
    HN_API_END
}

}  // extern "C"
