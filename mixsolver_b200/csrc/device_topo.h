// device_topo.h -- the integer mesh pipeline and the RCM order on the device
// (device_topo.cu).
#pragma once

#include <cuda_runtime.h>

#include <functional>

#include "common.cuh"

namespace mgpu {

// 0-based device arrays, entry for entry those of build_topology (mesh_host.cpp)
struct DeviceTopo {
  int N = 0, F = 0, ncf = 0, ncc = 0, nnz = 0;
  int *cf_ptr = nullptr, *cf = nullptr, *c2c_ptr = nullptr, *c2c = nullptr;
  int *row_ptr = nullptr, *col = nullptr, *diag = nullptr, *cf_slot = nullptr, *mirror = nullptr;
  int nlev_lo = 0, nlev_up = 0;
  int *lo_ptr = nullptr, *lo_rows = nullptr, *up_ptr = nullptr, *up_rows = nullptr;
};

// allocation of the arrays that outlive the call (the caller owns them)
using TopoAlloc = std::function<int(int*&, size_t)>;

// From the device face arrays c0, c1 (0-based, c1 = -1 on the boundary).
// levels: build the triangular level sets too (only the FP64 form's ILU(0) /
// IC(0) sweeps read them; without them lo_ptr, up_ptr, ... stay null and
// nlev_lo = nlev_up = 0). Waits for stream s before returning.
int device_topology(int N, int F, const int* c0, const int* c1, DeviceTopo& t, const TopoAlloc& alloc,
                    cudaStream_t s, bool levels = true);
// Widest row W of the pattern and, when W <= max_width, its column-major ELL
// copy: entry t of row i at t * ld + i with ld = N rounded up to a multiple of
// 4 (every column starts 16-byte aligned), padding the row itself.
int device_ell(int N, const int* row_ptr, const int* col, int max_width, int& W, long& ld, int*& ell,
               const TopoAlloc& alloc, cudaStream_t s);
// Each cell's boundary faces that carry a group, in the order of its face list.
int device_boundary_lists(int N, const int* cf_ptr, const int* cf, const int* c1, const int* fgrp, int*& bf_ptr,
                          int*& bf, const TopoAlloc& alloc, cudaStream_t s);
// Reverse Cuthill-McKee on a device CSR pattern: new_of_old[c] = 1-based new
// number of cell c, the order of mgpu_rcm_order. Waits for stream s.
int device_rcm(int N, const int* row_ptr, const int* col, int* new_of_old, cudaStream_t s);

}  // namespace mgpu
