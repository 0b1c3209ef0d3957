// Operator primitives with the reference's names and call shapes
// (primitives/Operator++.cuh:68-215, Operator++.i.cuh:8-37,248-313,524-645):
// forAll, forAllnumV, forAllnumE, forAllVertices, forAllEdges.  Operators are
// functors (or __device__ lambdas) inlined into sm_100a kernels:
//   op(int i)                     forAll / forAllnumV / forAllnumE
//   op(T item)                    forAll(queue, op)
//   op(Vertex& v)                 forAllVertices
//   op(Vertex& v, Edge& e)        forAllEdges (BinarySearch or VertexBased<VW>)
// Every call synchronises before returning, as the reference's
// CHECK_CUDA_ERROR after each launch does.
#pragma once

#include "HornetDevice.cuh"
#include "LoadBalancing.cuh"
#include "TwoLevelQueue.cuh"

#define OPERATOR                                                    \
    template <typename Vertex = void, typename Edge = void>         \
    __device__ __forceinline__ void operator()

namespace hornets_nest {

const int BLOCK_SIZE_OP2 = 256;

namespace detail {

template <typename Operator>
__global__ void forAllKernel(int size, Operator op) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < size; i += gridDim.x * blockDim.x)
        op(i);
}

template <typename T, typename Operator>
__global__ void forAllArrayKernel(const T* __restrict__ array, int size, Operator op) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < size; i += gridDim.x * blockDim.x) {
        T value = array[i];
        op(value);
    }
}

template <typename Operator>
__global__ void forAllVerticesKernel(hornet::HornetDevice hd, const int* __restrict__ array,
                                     int size, Operator op) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < size; i += gridDim.x * blockDim.x) {
        auto v = hd.vertex(array ? array[i] : i);
        op(v);
    }
}

inline int grid_of(long long n) {
    long long g = (n + BLOCK_SIZE_OP2 - 1) / BLOCK_SIZE_OP2;
    long long lim = (long long)load_balancing::kernels::num_sms() * 16;
    return (int)(g < 1 ? 1 : (g > lim ? lim : g));
}

}  // namespace detail

template <typename Operator>
void forAll(int num_items, const Operator& op) {
    if (num_items <= 0) return;
    detail::forAllKernel<<<detail::grid_of(num_items), BLOCK_SIZE_OP2>>>(num_items, op);
    cudaDeviceSynchronize();
}

template <typename T, typename Operator>
void forAll(const TwoLevelQueue<T>& queue, const Operator& op) {
    int n = queue.size();
    if (n <= 0) return;
    detail::forAllArrayKernel<<<detail::grid_of(n), BLOCK_SIZE_OP2>>>(queue.device_input_ptr(), n,
                                                                     op);
    cudaDeviceSynchronize();
}

template <typename HornetClass, typename Operator>
void forAllnumV(HornetClass& hornet, const Operator& op) {
    forAll(hornet.nV(), op);
}

template <typename HornetClass, typename Operator>
void forAllnumE(HornetClass& hornet, const Operator& op) {
    forAll(hornet.nE(), op);
}

template <typename HornetClass, typename Operator>
void forAllVertices(HornetClass& hornet, const Operator& op) {
    int n = hornet.nV();
    if (n <= 0) return;
    detail::forAllVerticesKernel<<<detail::grid_of(n), BLOCK_SIZE_OP2, 0, hornet.stream()>>>(
        hornet.device(), nullptr, n, op);
    hornet.sync();
}

template <typename HornetClass, typename Operator>
void forAllVertices(HornetClass& hornet, const typename HornetClass::VertexType* vertex_array,
                    int size, const Operator& op) {
    if (size <= 0) return;
    detail::forAllVerticesKernel<<<detail::grid_of(size), BLOCK_SIZE_OP2, 0, hornet.stream()>>>(
        hornet.device(), vertex_array, size, op);
    hornet.sync();
}

template <typename HornetClass, typename Operator>
void forAllVertices(HornetClass& hornet,
                    const TwoLevelQueue<typename HornetClass::VertexType>& queue,
                    const Operator& op) {
    forAllVertices(hornet, queue.device_input_ptr(), queue.size(), op);
}

template <typename HornetClass, typename Operator, typename LoadBalancing>
void forAllEdges(HornetClass& hornet, const Operator& op, const LoadBalancing& load_balancing) {
    load_balancing.apply(hornet, op);
}

template <typename HornetClass, typename Operator>
void forAllEdges(HornetClass& hornet, const Operator& op) {
    load_balancing::BinarySearch lb(hornet);
    lb.apply(hornet, op);
}

template <typename HornetClass, typename Operator, typename LoadBalancing>
void forAllEdges(HornetClass& hornet, const typename HornetClass::VertexType* vertex_array,
                 int size, const Operator& op, const LoadBalancing& load_balancing) {
    load_balancing.apply(hornet, vertex_array, size, op);
}

template <typename HornetClass, typename Operator, typename LoadBalancing>
void forAllEdges(HornetClass& hornet,
                 const TwoLevelQueue<typename HornetClass::VertexType>& queue,
                 const Operator& op, const LoadBalancing& load_balancing) {
    load_balancing.apply(hornet, queue.device_input_ptr(), queue.size(), op);
}

}  // namespace hornets_nest
