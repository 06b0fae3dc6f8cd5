// agpu_multi.h — one step of many independent instances in one launch per
// phase (FP32 split form, one running species).  Small grids make every
// per-instance kernel a few microseconds of mostly fixed cost; here each
// phase of the step is a single kernel over all instances' work: the tile
// kernel takes one block per tile of any instance (instance found from the
// tile offsets), the other phases take one row of blocks per instance
// (blockIdx.y = instance) running the same device bodies as the
// single-instance kernels.
#pragma once
#include <cuda_runtime.h>

#include "agpu_tile.h"

namespace agpu {

struct MultiInst {
  TileArgs32 ta;               // geometry, fields (read), currents, particles, binning arrays
  float* ebf;                  // fields (written by the field phases)
  YeeC yc;
  int* cursor;                 // scatter cursors (nkeys + 1)
  unsigned long long* pushed;  // the instance's device push counter
  unsigned long long* removed;
  double* fmax;
  long long np;                // stored particle records
};

struct MultiPlan {
  int n;              // instances
  int ndim;           // common to all instances
  int total_tiles;    // sum of ntiles
  int gx_cells;       // blocks per instance for cell-wide phases
  int gx_faces;       // blocks per instance for face-wide phases
  int gx_parts;       // blocks per instance for particle-wide phases
};

// pre: currents and cursors zeroed, next histogram seeded, push counter and
// step counters; then the x-face field extrapolation (field_xyzbd, x).
void multi_pre32(const MultiInst* d, const MultiPlan& pl, cudaStream_t st, int* launches);
// y (and z) face extrapolation
void multi_field_bd32(const MultiInst* d, const MultiPlan& pl, cudaStream_t st, int* launches);
// gather + push + deposit of every tile of every instance
void multi_tile32(const MultiInst* d, const int* tile_off, const MultiPlan& pl, cudaStream_t st, int* launches);
// scan of the next histogram and the permutation scatter
void multi_bin32(const MultiInst* d, const MultiPlan& pl, cudaStream_t st, int* launches);
// current fold (hi and lo) and the leapfrog Yee update with its boundaries
void multi_fields32(const MultiInst* d, const MultiPlan& pl, cudaStream_t st, int* launches);

}  // namespace agpu
