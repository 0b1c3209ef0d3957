// Device view of a hornet_b200 graph for user operators: the same accessor
// names as the reference's hornet::HornetDevice / Vertex / Edge
// (hornet/include/Core/HornetDevice/HornetDevice.cuh:52-90,
//  impl/Vertex.i.cuh:59-146, impl/Edge.i.cuh:43-116), for the
// vid_t = degree_t = int, no-metadata instantiation.
//
// Storage differs from the reference: each vertex is one 16-byte record
// {int64 off; int32 degree; int32 capacity} and its neighbours are
// pool[off .. off+degree), always sorted ascending.  One 16-byte load per
// vertex replaces the reference's four SoA loads (Vertex.i.cuh:59-93).
#pragma once

#include <cuda_runtime.h>

#include "../hornet_b200.h"

#ifndef HOST_DEVICE
#define HOST_DEVICE __host__ __device__ __forceinline__
#endif

namespace hornet {

using vid_t = int;
using degree_t = int;

struct __align__(16) VertexRecord {
    long long off;
    int deg;
    int cap;
};

class HornetDevice;
class Vertex;

class Edge {
public:
    __device__ __forceinline__ Edge(const VertexRecord* vtab, const vid_t* pool, vid_t src,
                                    const vid_t* nbr, degree_t index)
        : _vtab(vtab), _pool(pool), _src(src), _nbr(nbr), _index(index) {}
    __device__ __forceinline__ vid_t src_id() const { return _src; }
    __device__ __forceinline__ vid_t dst_id() const { return _nbr[_index]; }
    __device__ __forceinline__ degree_t index() const { return _index; }
    __device__ __forceinline__ Vertex src() const;
    __device__ __forceinline__ Vertex dst() const;

private:
    const VertexRecord* _vtab;
    const vid_t* _pool;
    vid_t _src;
    const vid_t* _nbr;
    degree_t _index;
};

class Vertex {
public:
    __device__ __forceinline__ Vertex(const VertexRecord* vtab, const vid_t* pool, vid_t id)
        : _vtab(vtab), _pool(pool), _id(id) {
        VertexRecord r = vtab[id];
        _deg = r.deg;
        _cap = r.cap;
        _nbr = pool + r.off;
    }
    __device__ __forceinline__ vid_t id() const { return _id; }
    __device__ __forceinline__ degree_t degree() const { return _deg; }
    // block capacity (a power of two), Vertex::limit() in the reference
    __device__ __forceinline__ degree_t limit() const { return _cap; }
    __device__ __forceinline__ const vid_t* neighbor_ptr() const { return _nbr; }
    __device__ __forceinline__ Edge edge(degree_t index) const {
        return Edge(_vtab, _pool, _id, _nbr, index);
    }

private:
    const VertexRecord* _vtab;
    const vid_t* _pool;
    vid_t _id;
    degree_t _deg;
    degree_t _cap;
    const vid_t* _nbr;
};

__device__ __forceinline__ Vertex Edge::src() const { return Vertex(_vtab, _pool, _src); }
__device__ __forceinline__ Vertex Edge::dst() const { return Vertex(_vtab, _pool, dst_id()); }

class HornetDevice {
public:
    HornetDevice() = default;
    explicit HornetDevice(const hn_device_view_t& v)
        : _nV(v.nV), _nE(v.nE), _vtab((const VertexRecord*)v.vtab), _pool(v.pool) {}
    HOST_DEVICE vid_t nV() const { return _nV; }
    HOST_DEVICE long long nE() const { return _nE; }
    __device__ __forceinline__ Vertex vertex(vid_t id) const { return Vertex(_vtab, _pool, id); }
    HOST_DEVICE const VertexRecord* vertex_records() const { return _vtab; }
    HOST_DEVICE const vid_t* edge_pool() const { return _pool; }

private:
    vid_t _nV = 0;
    long long _nE = 0;
    const VertexRecord* _vtab = nullptr;
    const vid_t* _pool = nullptr;
};

}  // namespace hornet
