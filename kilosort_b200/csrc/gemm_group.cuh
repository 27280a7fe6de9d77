// Parameters of a grouped split-BF16 contraction (gemm_bf16x3.cu).
#pragma once
#include <cuda.h>

#include "project.cuh"

namespace ks {

// One batch of a grouped contraction: output B (row-major with ldb, or tiled),
// K templates, L samples, its recording, the first row of its Y block in the
// recording's concatenated Y, its template tiles and its first global tile.
struct GemmBatch {
  float* B;
  long long ldb;
  int K, L, rec, row_off, tiles_m, tile_begin;
};

// Tensor maps of up to kGroupRecs recordings (Uhi, Ulo, Yhi, Ylo each) and the
// tile table of up to kGroupBatches batches; passed whole as a kernel
// parameter, so a grouped launch needs no host-to-device copy.
struct GemmGroup {
  CUtensorMap maps[kGroupRecs][4];
  int nk[kGroupRecs];
  GemmBatch batches[kGroupBatches];
  int n_batches, n_tiles, tiled;
  int* err;
};

}  // namespace ks
