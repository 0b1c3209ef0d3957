// Load balancers for forAllEdges: the names and apply() signatures of the
// reference's hornets_nest::load_balancing::BinarySearch and
// VertexBased<VW> (primitives/LoadBalancing/BinarySearch.cuh:52-94,
// VertexBased.cuh:48-79), rebuilt for sm_100a.
//
// BinarySearch: the reference runs computeWorkKernel, a CUB scan, a
// synchronous D2H copy of the total work and then binarySearchKernel with
// a grid sized from that total (BinarySearch.i.cuh:58-107).  Here the degree
// prefix is scanned on the device and a persistent grid reads the total from
// device memory, so apply() never waits on the host; each CTA takes
// merge-path tiles over (edges, vertex boundaries) with the tile's segment
// ends staged in shared memory and calls the operator item-striped.
//
// VertexBased<VW>: VW lanes (a power of two <= 32) per vertex striding its
// adjacency, as VertexBasedKernel.cuh:45-108.
#pragma once

#include <cub/cub.cuh>

#include "HornetDevice.cuh"
#include "detail/MergePathLB.cuh"

namespace hornets_nest {
namespace load_balancing {
namespace kernels {

template <typename Unused = void>
__global__ void degreesOf(hornet::HornetDevice hd, const int* __restrict__ input, long long n,
                          long long* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i <= n;
         i += (long long)gridDim.x * blockDim.x) {
        if (i == n) {
            out[i] = 0;
        } else {
            int v = input ? input[i] : (int)i;
            out[i] = hd.vertex_records()[v].deg;
        }
    }
}

template <int BLOCK, int ITEMS, typename Operator>
__global__ void __launch_bounds__(BLOCK)
binarySearchLB(hornet::HornetDevice hd, const int* __restrict__ input, long long n,
               const long long* __restrict__ prefix, const long long* __restrict__ splits,
               long long max_tiles, Operator op) {
    using Tile = hornet_b200::detail::LbTile<BLOCK, ITEMS>;
    __shared__ Tile t;
    const long long total = prefix[n];
    const long long ntiles = (total + n + Tile::TILE - 1) / Tile::TILE;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int cnt = hornet_b200::detail::lb_tile_load(t, prefix, n, total, tile, splits, max_tiles);
        for (int i = threadIdx.x; i < cnt; i += BLOCK) {
            int b = t.seg[i];
            long long s = t.seg0 + b;
            int vid = input ? input[s] : (int)s;
            hornet::degree_t rank = (hornet::degree_t)(t.item0 + i - t.seg_start(b));
            auto vertex = hd.vertex(vid);
            auto edge = vertex.edge(rank);
            op(vertex, edge);
        }
        __syncthreads();
    }
}

template <int VW, typename Operator>
__global__ void vertexBased(hornet::HornetDevice hd, const int* __restrict__ input, long long n,
                            Operator op) {
    long long gid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long stride = (long long)gridDim.x * blockDim.x / VW;
    int lane = (int)(gid % VW);
    for (long long i = gid / VW; i < n; i += stride) {
        int vid = input ? input[i] : (int)i;
        auto vertex = hd.vertex(vid);
        for (int j = lane; j < vertex.degree(); j += VW) {
            auto edge = vertex.edge(j);
            op(vertex, edge);
        }
    }
}

inline int num_sms() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

}  // namespace kernels

class BinarySearch {
public:
    BinarySearch() = default;
    template <typename HornetClass>
    explicit BinarySearch(HornetClass&, const float work_factor = 2.0f) noexcept {
        (void)work_factor;
    }

    // Core: every edge of the n vertices in d_input (all vertices when
    // d_input == nullptr), on `stream`.  Asynchronous.
    // The tile partition is precomputed for a work size of max_total (the
    // edge count by default, which bounds any list without repeats); tiles
    // past that bound search for their own split, so any list is correct.
    template <typename Operator>
    static void run(const hornet::HornetDevice& hd, const int* d_input, long long n,
                    const Operator& op, cudaStream_t stream, long long max_total = -1) {
        if (n <= 0) return;
        const int tile = BLOCK_SIZE * ITEMS;
        if (max_total < 0) max_total = hd.nE();
        const long long max_tiles = (max_total + n + tile - 1) / tile + 1;
        long long* prefix = nullptr;
        long long* splits = nullptr;
        cudaMallocAsync((void**)&prefix, sizeof(long long) * (size_t)(n + 1), stream);
        cudaMallocAsync((void**)&splits, sizeof(long long) * (size_t)(max_tiles + 1), stream);
        const int sms = kernels::num_sms();
        long long g = (n + 256) / 256;
        if (g > sms * 8) g = sms * 8;
        kernels::degreesOf<><<<(unsigned)g, 256, 0, stream>>>(hd, d_input, n, prefix);
        size_t tb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb, prefix, prefix, n + 1, stream);
        void* tmp = nullptr;
        cudaMallocAsync(&tmp, tb, stream);
        cub::DeviceScan::ExclusiveSum(tmp, tb, prefix, prefix, n + 1, stream);
        long long gp = (max_tiles + 256) / 256;
        if (gp > sms * 8) gp = sms * 8;
        hornet_b200::detail::lb_partition<long long><<<(unsigned)gp, 256, 0, stream>>>(
            prefix, n, tile, max_tiles, splits);
        kernels::binarySearchLB<BLOCK_SIZE, ITEMS><<<(unsigned)(sms * 8), BLOCK_SIZE, 0, stream>>>(
            hd, d_input, n, prefix, splits, max_tiles, op);
        cudaFreeAsync(tmp, stream);
        cudaFreeAsync(splits, stream);
        cudaFreeAsync(prefix, stream);
    }

    template <typename HornetClass, typename Operator, typename vid_t>
    void apply(HornetClass& hornet, const vid_t* d_input, int num_vertices,
               const Operator& op) const noexcept {
        run(hornet.device(), (const int*)d_input, num_vertices, op, hornet.stream());
        hornet.sync();
    }

    template <typename HornetClass, typename Operator>
    void apply(HornetClass& hornet, const Operator& op) const noexcept {
        run(hornet.device(), nullptr, hornet.nV(), op, hornet.stream());
        hornet.sync();
    }

    static const unsigned BLOCK_SIZE = 256;
    static const unsigned ITEMS = 8;
};

template <unsigned VW_SIZE>
class VertexBased {
    static_assert(VW_SIZE >= 1 && VW_SIZE <= 32 && (VW_SIZE & (VW_SIZE - 1)) == 0,
                  "VW_SIZE must be a power of two in [1, 32]");

public:
    VertexBased() = default;
    template <typename T>
    VertexBased(const T&) {}

    template <typename Operator>
    static void run(const hornet::HornetDevice& hd, const int* d_input, long long n,
                    const Operator& op, cudaStream_t stream) {
        if (n <= 0) return;
        const int sms = kernels::num_sms();
        long long g = (n * VW_SIZE + BLOCK_SIZE - 1) / BLOCK_SIZE;
        if (g > sms * 16) g = sms * 16;
        kernels::vertexBased<VW_SIZE><<<(unsigned)g, BLOCK_SIZE, 0, stream>>>(hd, d_input, n, op);
    }

    template <typename HornetClass, typename Operator, typename vid_t>
    void apply(HornetClass& hornet, const vid_t* d_input, int num_vertices,
               const Operator& op) const noexcept {
        run(hornet.device(), (const int*)d_input, num_vertices, op, hornet.stream());
        hornet.sync();
    }

    template <typename HornetClass, typename Operator>
    void apply(HornetClass& hornet, const Operator& op) const noexcept {
        run(hornet.device(), nullptr, hornet.nV(), op, hornet.stream());
        hornet.sync();
    }

    static const unsigned BLOCK_SIZE = 128;
};

using VertexBased1 = VertexBased<1>;
using VertexBased2 = VertexBased<2>;
using VertexBased4 = VertexBased<4>;
using VertexBased8 = VertexBased<8>;
using VertexBased16 = VertexBased<16>;
using VertexBased32 = VertexBased<32>;

}  // namespace load_balancing
}  // namespace hornets_nest
