// Built-in operators over the operator primitives, exported through the C
// ABI.  They run the same header templates that user operators compile
// against (<hornet_b200/LoadBalancing.cuh>), so the C-ABI tests exercise
// the BinarySearch and VertexBased<VW> balancers themselves.
#include "../../include/hornet_b200/LoadBalancing.cuh"
#include "hn_graph.cuh"

namespace hn {
namespace {

// forAllEdges operator: out[dst] += 1 for every visited edge.
struct CountDst {
    int32_t* out;
    __device__ __forceinline__ void operator()(hornet::Vertex&, hornet::Edge& e) const {
        atomicAdd(out + e.dst_id(), 1);
    }
};

__global__ void k_vertex_degree(hornet::HornetDevice hd, int32_t* out) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < hd.nV();
         v += (long long)gridDim.x * blockDim.x)
        out[v] = hd.vertex((int)v).degree();
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// Order-independent checksum of the edge multiset: sum over edges (u, v) of
// SplitMix64(u << 32 | v), a warp per vertex, one atomic per warp.
__global__ void k_adjacency_hash(const VRec* __restrict__ vtab, const int32_t* __restrict__ pool,
                                 int nV, unsigned long long* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    unsigned long long h = 0;
    for (long long v = w0; v < nV; v += nw) {
        const VRec r = vtab[v];
        const unsigned long long hi = (unsigned long long)(unsigned)v << 32;
        for (int i = lane; i < r.deg; i += 32) h += mix64(hi | (unsigned)pool[r.off + i]);
    }
    for (int o = 16; o; o >>= 1) h += __shfl_down_sync(0xFFFFFFFFu, h, o);
    if (lane == 0 && h) atomicAdd(out, h);
}

__global__ void k_gather_i32(const int32_t* __restrict__ src, const long long* __restrict__ idx,
                             long long n, int32_t* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = src[idx[i]];
}

hornet::HornetDevice view_of(hn_graph* g) {
    hn_device_view_t v;
    v.nV = g->nV;
    v.pad = 0;
    v.nE = g->nE;
    v.vtab = g->vtab;
    v.pool = g->pool;
    return hornet::HornetDevice(v);
}

template <unsigned VW>
void vertex_based(hn_graph* g, const int32_t* verts, long long n, int32_t* out) {
    hornets_nest::load_balancing::VertexBased<VW>::run(view_of(g), verts, n, CountDst{out},
                                                      g->stream);
    count_launch();
}

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" int hn_for_all_edges_count(hn_graph_t* g, const int32_t* vertices, int32_t n, int lb,
                                      int vw, int32_t* out) {
    HN_API_BEGIN
    HN_REQUIRE(g && out, "null argument");
    HN_REQUIRE(lb == HN_LB_BINARY_SEARCH || lb == HN_LB_VERTEX_BASED, "bad load balancer");
    HN_CUDA(cudaSetDevice(g->device));
    long long cnt = vertices ? n : g->nV;
    HN_REQUIRE(cnt >= 0, "negative vertex count");
    if (lb == HN_LB_BINARY_SEARCH) {
        hornets_nest::load_balancing::BinarySearch::run(view_of(g), vertices, cnt, CountDst{out},
                                                        g->stream);
        count_launch(2);
    } else {
        switch (vw) {
            case 1: vertex_based<1>(g, vertices, cnt, out); break;
            case 2: vertex_based<2>(g, vertices, cnt, out); break;
            case 4: vertex_based<4>(g, vertices, cnt, out); break;
            case 8: vertex_based<8>(g, vertices, cnt, out); break;
            case 16: vertex_based<16>(g, vertices, cnt, out); break;
            case 32: vertex_based<32>(g, vertices, cnt, out); break;
            default: throw Error(HN_ERR_INVALID, "vw must be a power of two in [1, 32]");
        }
    }
    HN_CUDA(cudaGetLastError());
    HN_CUDA(cudaStreamSynchronize(g->stream));
    HN_API_END
}

extern "C" int hn_for_all_vertices_degree(hn_graph_t* g, int32_t* out) {
    HN_API_BEGIN
    HN_REQUIRE(g && out, "null argument");
    HN_CUDA(cudaSetDevice(g->device));
    HN_LAUNCH(k_vertex_degree, grid_for(g, g->nV, 256), 256, 0, g->stream, view_of(g), out);
    HN_CUDA(cudaStreamSynchronize(g->stream));
    HN_API_END
}

extern "C" int hn_graph_adjacency_hash(hn_graph_t* g, uint64_t* hash) {
    HN_API_BEGIN
    HN_REQUIRE(g && hash, "null argument");
    HN_CUDA(cudaSetDevice(g->device));
    DevBuf<unsigned long long> acc;
    acc.alloc(1, g->stream);
    HN_CUDA(cudaMemsetAsync(acc.get(), 0, sizeof(unsigned long long), g->stream));
    if (g->nV > 0)
        HN_LAUNCH(k_adjacency_hash, grid_for(g, (long long)g->nV * 32, 256), 256, 0, g->stream,
                  g->vtab, g->pool, g->nV, acc.get());
    unsigned long long h = 0;
    HN_CUDA(cudaMemcpyAsync(&h, acc.get(), sizeof(h), cudaMemcpyDeviceToHost, g->stream));
    HN_CUDA(cudaStreamSynchronize(g->stream));
    *hash = h;
    HN_API_END
}

// out[i] = sum of values[off[i] .. off[i+1]), a CTA per range (per-graph
// sums of per-vertex counts over a batch of graphs laid out side by side).
__global__ void __launch_bounds__(256)
k_segment_sum_u64(const unsigned long long* __restrict__ values,
                  const long long* __restrict__ off, long long nseg,
                  unsigned long long* __restrict__ out) {
    __shared__ unsigned long long wsum[8];
    for (long long sg = blockIdx.x; sg < nseg; sg += gridDim.x) {
        unsigned long long acc = 0;
        for (long long i = off[sg] + threadIdx.x; i < off[sg + 1]; i += 256) acc += values[i];
#pragma unroll
        for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
        if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long t = 0;
            for (int w = 0; w < 8; w++) t += wsum[w];
            out[sg] = t;
        }
        __syncthreads();
    }
}

extern "C" int hn_segment_sum_u64(hn_graph_t* g, const uint64_t* values, const int64_t* off,
                                  int64_t nseg, uint64_t* out) {
    HN_API_BEGIN
    HN_REQUIRE(g && (nseg == 0 || (values && off && out)) && nseg >= 0, "null argument");
    if (nseg == 0) return HN_OK;
    for (int64_t i = 0; i < nseg; i++)
        HN_REQUIRE(off[i] >= 0 && off[i] <= off[i + 1], "ranges must be increasing");
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    DevBuf<long long> d_off((size_t)nseg + 1, s);
    HN_CUDA(cudaMemcpyAsync(d_off.get(), off, sizeof(long long) * (nseg + 1),
                            cudaMemcpyHostToDevice, s));
    HN_LAUNCH(k_segment_sum_u64, grid_for(g, nseg, 1, 16), 256, 0, s,
              (const unsigned long long*)values, (const long long*)d_off.get(), (long long)nseg,
              (unsigned long long*)out);
    HN_CUDA(cudaStreamSynchronize(s));
    HN_API_END
}

// Read bandwidth of a buffer that stays in L2: every CTA streams the whole
// buffer `reps` times with 16-byte loads (rotated by CTA so that CTAs do not
// walk in step); the XOR of everything read is kept so that no load is
// dropped.
__global__ void __launch_bounds__(256)
k_read_probe(const int4* __restrict__ buf, long long n16, int reps,
             unsigned* __restrict__ sink) {
    unsigned acc = 0;
    const long long per = n16 / gridDim.x;   // this CTA's share of one pass
    const long long first = (long long)blockIdx.x * per;
    for (int r = 0; r < reps; r++) {
        const long long start = (first + (long long)r * per) % n16;
        for (long long i = threadIdx.x; i < per; i += 256) {
            long long j = start + i;
            if (j >= n16) j -= n16;
            const int4 v = __ldcg(buf + j);
            acc ^= (unsigned)(v.x ^ v.y ^ v.z ^ v.w);
        }
    }
    if (acc == 0x9E3779B9u) atomicAdd(sink, 1u);
}

extern "C" int hn_read_bandwidth(hn_graph_t* g, const void* buf, int64_t bytes, int32_t reps,
                                 double* gbs) {
    HN_API_BEGIN
    HN_REQUIRE(g && buf && gbs && bytes >= 16 * 256 && reps >= 1, "bad argument");
    HN_REQUIRE(((uintptr_t)buf & 15) == 0, "buffer must be 16-byte aligned");
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    const long long n16 = bytes / 16;
    const long long grid = (long long)g->info.sms * 8;
    DevBuf<unsigned> sink(1, s);
    cudaEvent_t a, b;
    HN_CUDA(cudaEventCreate(&a));
    HN_CUDA(cudaEventCreate(&b));
    // one pass to bring the buffer into L2, then the timed passes
    HN_LAUNCH(k_read_probe, grid, 256, 0, s, (const int4*)buf, n16, 1, sink.get());
    HN_CUDA(cudaEventRecord(a, s));
    HN_LAUNCH(k_read_probe, grid, 256, 0, s, (const int4*)buf, n16, (int)reps, sink.get());
    HN_CUDA(cudaEventRecord(b, s));
    HN_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    HN_CUDA(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    // each CTA reads per * reps 16-byte words
    const double read = 16.0 * (double)(n16 / grid) * (double)grid * (double)reps;
    *gbs = ms > 0 ? read / (ms * 1e-3) / 1e9 : 0.0;
    HN_API_END
}

extern "C" int hn_gather_int32(hn_graph_t* g, const int32_t* src, const int64_t* idx, int64_t n,
                               int32_t* out) {
    HN_API_BEGIN
    HN_REQUIRE(g && src && (idx || n == 0) && (out || n == 0) && n >= 0, "null argument");
    if (n == 0) return HN_OK;
    HN_CUDA(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    DevBuf<long long> d_idx((size_t)n, s);
    DevBuf<int32_t> d_out((size_t)n, s);
    HN_CUDA(cudaMemcpyAsync(d_idx.get(), idx, sizeof(long long) * n, cudaMemcpyHostToDevice, s));
    HN_LAUNCH(k_gather_i32, grid_for(g, n, 256), 256, 0, s, src, (const long long*)d_idx.get(),
              (long long)n, d_out.get());
    HN_CUDA(cudaMemcpyAsync(out, d_out.get(), sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
    HN_CUDA(cudaStreamSynchronize(s));
    HN_API_END
}
