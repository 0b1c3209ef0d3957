// hornets_nest::TwoLevelQueue<T> (primitives/Queue/TwoLevelQueue.cuh:62-204):
// a double-buffered device frontier.  Device insert() is a warp-aggregated
// append (one atomicAdd per warp via ballot/popc/shfl); swap() exchanges
// the input and output buffers.  The reference's swap launches a <<<1,1>>>
// kernel and copies the counters to the host (TwoLevelQueue.i.cuh:158-179);
// here swap() reads the output counter once with cudaMemcpy on the default
// stream and swaps on the host.  Copies made for kernels (pass-by-value into
// an operator) do not own the buffers, as in the reference
// (TwoLevelQueue.i.cuh:67-92).
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>

namespace hornets_nest {

template <typename T>
class TwoLevelQueue {
public:
    TwoLevelQueue() = default;

    template <typename HornetClass>
    explicit TwoLevelQueue(const HornetClass& hornet, const float work_factor = 2.0f) noexcept {
        initialize(hornet, work_factor);
    }

    explicit TwoLevelQueue(size_t max_allocated_items) noexcept { initialize(max_allocated_items); }

    template <typename HornetClass>
    void initialize(const HornetClass& hornet, const float work_factor = 2.0f) noexcept {
        initialize((size_t)(work_factor * (float)hornet.nV()) + 1);
    }

    void initialize(size_t max_allocated_items) noexcept {
        _max = max_allocated_items;
        if (cudaMalloc(&_in, sizeof(T) * _max) != cudaSuccess ||
            cudaMalloc(&_out, sizeof(T) * _max) != cudaSuccess ||
            cudaMalloc(&_counters, sizeof(int2)) != cudaSuccess) {
            std::fprintf(stderr, "TwoLevelQueue: allocation failed\n");
            std::abort();
        }
        cudaMemset(_counters, 0, sizeof(int2));
        _h = make_int2(0, 0);
        _kernel_copy = false;
    }

    __host__ __device__ TwoLevelQueue(const TwoLevelQueue<T>& o) noexcept
        : _in(o._in), _out(o._out), _max(o._max), _counters(o._counters), _h(o._h),
          _kernel_copy(true) {}

    __host__ __device__ ~TwoLevelQueue() noexcept {
#if !defined(__CUDA_ARCH__)
        if (!_kernel_copy) {
            cudaFree(_in);
            cudaFree(_out);
            cudaFree(_counters);
        }
#endif
    }

    // Device: append to the output buffer (warp-aggregated).
    // Host: append to the INPUT buffer (as the reference's host insert).
    __host__ __device__ __forceinline__ void insert(const T& item) noexcept {
#if defined(__CUDA_ARCH__)
        unsigned mask = __activemask();
        int leader = __ffs(mask) - 1;
        int lane = threadIdx.x & 31;
        int base = 0;
        if (lane == leader) base = atomicAdd(&_counters->y, __popc(mask));
        base = __shfl_sync(mask, base, leader);
        int pos = base + __popc(mask & ((1u << lane) - 1));
        if (pos < (int)_max) _out[pos] = item;
#else
        insert(&item, 1);
#endif
    }

    void insert(const T* items, int n) noexcept {
        sync();
        cudaMemcpy(_in + _h.x, items, sizeof(T) * n, cudaMemcpyHostToDevice);
        _h.x += n;
        cudaMemcpy(_counters, &_h, sizeof(int2), cudaMemcpyHostToDevice);
    }

    void swap() noexcept {
        sync();
        T* t = _in;
        _in = _out;
        _out = t;
        _h.x = _h.y < (int)_max ? _h.y : (int)_max;
        _h.y = 0;
        _enqueued += _h.x;
        cudaMemcpy(_counters, &_h, sizeof(int2), cudaMemcpyHostToDevice);
    }

    void clear() noexcept {
        _h = make_int2(0, 0);
        cudaMemcpy(_counters, &_h, sizeof(int2), cudaMemcpyHostToDevice);
    }

    void sync() const noexcept { cudaMemcpy(&_h, _counters, sizeof(int2), cudaMemcpyDeviceToHost); }

    int size() const noexcept { return _h.x; }
    int size_sync_in() const noexcept { sync(); return _h.x; }
    int size_sync_out() const noexcept { sync(); return _h.y; }
    int output_size() const noexcept { return _h.y; }
    __host__ __device__ const T* device_input_ptr() const noexcept { return _in; }
    __host__ __device__ const T* device_output_ptr() const noexcept { return _out; }
    int enqueue_items() const noexcept { return _enqueued; }
    // output overflowed max_allocated_items (items past the end were dropped)
    bool overflowed() const noexcept { sync(); return _h.y > (int)_max; }

private:
    T* _in = nullptr;
    T* _out = nullptr;
    size_t _max = 0;
    int2* _counters = nullptr;
    mutable int2 _h{0, 0};
    bool _kernel_copy = true;
    int _enqueued = 0;
};

}  // namespace hornets_nest
