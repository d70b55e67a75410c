// Registry of the coarse grids built into this library: per grid and
// precision, function pointers into the templated pipeline.  Each grid is
// compiled in its own translation unit (grid_instance.cu, one object per line
// of grids.inc) and registers itself when the library is loaded.
#pragma once
#include <cuda_runtime.h>

#include "common.hpp"

namespace pwb {

using HpsiFn = int (*)(pw_ctx*, const void*, int, void*, int, int, int, int, int, cudaStream_t);
using ChunkFn = int (*)();
using BuildQFn = int (*)(pw_ctx*, const int*, const double*, const long*, const long*, const int*, int, cudaStream_t,
                         int, void*);
using DensFn = int (*)(pw_ctx*, const void*, int, int, int, int, const double*, double*, cudaStream_t);
using TeterScratchFn = int (*)(pw_ctx*, const void*, int, void*, int, int, int, int, int, cudaStream_t, void*);
using ExxFn = int (*)(pw_ctx*, const void*, int, int, void*, int, int, cudaStream_t);
using HpsiKFn = int (*)(pw_ctx*, const void*, int, void*, int, int, int, int, cudaStream_t);
using HpsiKBFn = int (*)(pw_ctx*, const void*, int, void*, int, int, int, int, cudaStream_t, int, const void*,
                         const void*);
using VpermFn = int (*)(pw_ctx*, cudaStream_t);
using BuildQKFn = int (*)(pw_ctx*, const int*, const double*, const double*, const long*, const long*, const int*, int,
                          const double*, void*, cudaStream_t);

struct GridEntry {
  int n0, n1, n2;
  HpsiFn hpsi[2];
  HpsiFn teter[2];
  ChunkFn cr[2];
  BuildQFn bq[2];
  DensFn dens[2];
  TeterScratchFn teter_scratch[2];
  ExxFn exx[2];
  ExxFn ace[2];
  HpsiKFn hpsik[2];
  BuildQKFn bqk[2];
  HpsiKBFn hpsikb[2];
  HpsiFn hpsigs[2];     // sphere-cut (G-space) contexts whose G-space grid is twice this grid
  DensFn densgs[2];
  VpermFn vperm[2];     // rebuild pw_ctx::vperm from pw_ctx::vtot
};

void register_grid(const GridEntry& e);
const GridEntry* find_grid(const int n[3]);

}  // namespace pwb
