// Umbrella header of the C++ shim: the reference's Hornet / HornetsNest API
// (hornet::HornetInit, hornet::gpu::Hornet, BatchUpdate, forAllVertices /
// forAllEdges with BinarySearch and VertexBased<VW>, TwoLevelQueue,
// StaticAlgorithm, BfsTopDown, TriangleCounting2, CC, KTruss) on top of
// libhornet_b200.so.  Compile user code with nvcc for sm_100a and link
// -lhornet_b200.
#pragma once

#include "../hornet_b200.h"
#include "Algorithms.cuh"
#include "Hornet.cuh"
#include "HornetAlg.cuh"
#include "HornetDevice.cuh"
#include "LoadBalancing.cuh"
#include "Operator++.cuh"
#include "TwoLevelQueue.cuh"
