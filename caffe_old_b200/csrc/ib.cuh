// Immersed-boundary (ghost-cell) state on the device.
#pragma once
#include <functional>
#include "common.cuh"
#include "../../include/caffe_b200.h"

namespace cb {

struct IbState {
    int nGhost = 0;          // ghost rows (host copy of the device count)
    int nGhostHost = 0;
    long long nInactiveHost = 0;
    int* gCell = nullptr;    // ghost cells, ascending (k-j-i order)
    int* gCol = nullptr;     // 9 per ghost: own cell, then the 8 stencil cells (-1 = dropped)
    double* gValMom = nullptr;
    double* gValP = nullptr;
    uint32_t* bits = nullptr;
    int* chunkCount = nullptr;
    int* chunkOffset = nullptr;
    int* err = nullptr;      // device error flag of the stencil kernel
    long long nChunks = 0;
};

using Alloc = std::function<char*(size_t)>;

int ib_create(IbState& s, const Lat& L, uint8_t*& status, const Alloc& alloc, cudaStream_t st);
// Classify cells, list ghost cells and build their stencil rows (IbPiso.cpp:65-190).
int ib_setup(IbState& s, const Geo& g, const caffe_case& cs, const double* d_xyz, uint8_t* status, const Alloc& alloc,
             cudaStream_t st);
// Per step: cells inside the sphere (ghost and inactive) get u = 0, p = 0 (IbPiso.cpp:74-80).
int ib_compute_field(IbState& s, const Geo& g, const caffe_case& cs, double* u, double* p, const uint8_t* status, cudaStream_t st);
// Per inner iteration: ghost diagonals into both systems' diagonal arrays.
int ib_compute_coeffs(IbState& s, const Geo& g, const caffe_case& cs, const uint8_t* status, double* momDiag, double* pDiag,
                      cudaStream_t st);

}  // namespace cb
