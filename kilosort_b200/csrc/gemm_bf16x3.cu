// Split-BF16 score contraction on the 5th-generation tensor cores (tcgen05).
//
//   B[k, tau] = sum_q U[k, q] * Y[tau, q]
//             ~ Uhi.Yhi + Uhi.Ylo + Ulo.Yhi        (FP32 accumulate in TMEM)
// with x = hi + lo, hi = bf16(x), lo = bf16(x - hi): the dropped lo.lo term and
// the two roundings leave a relative error of about 2^-16 per product.
//
// Persistent kernel, one CTA per SM, 6 warps:
//   warp 0     TMA producer: per 64-wide slice of q, four tiles (Uhi, Ulo
//              128x64, Yhi, Ylo 256x64, bf16, 128-byte swizzle) into a 2-stage
//              shared-memory ring (96 KB per stage), completion on an mbarrier
//   warp 1     allocates 512 TMEM columns; one lane issues per slice 12 MMAs
//              (3 products x 4 steps of K=16, M=128, N=256) into a double-
//              buffered 128x256 FP32 accumulator and commits stage releases and
//              accumulator hand-offs to mbarriers
//   warps 2-5  epilogue: tcgen05.ld 32 columns at a time (one template row per
//              thread) and store 128-byte rows of the output (row-major B, or
//              the 32-column tiled layout of the peel, where a warp's 32 rows
//              are one contiguous 4 KB run)
// Tiles are (128 templates) x (256 samples), template tiles of one sample tile
// consecutive so concurrent CTAs share the Y tile through L2.  No TMA multicast.
// One launch can cover many batches of up to kGroupRecs recordings: the tile
// table (GemmGroup, a __grid_constant__ parameter with the tensor maps of each
// recording) maps a global tile number to (batch, template tile, sample tile);
// the Y operands of a recording's batches are stacked in one tensor and each
// batch reads its own row range.
// Every mbarrier wait is bounded by %globaltimer; a wait that runs out sets the
// error word, the CTA drains its own copies in flight (bounded), frees TMEM and
// returns.
#include "ks_common.cuh"
#include "gemm_group.cuh"
#include "tcgen05.cuh"

#include <cuda.h>
#include <cuda_bf16.h>

namespace {

constexpr int kBM = 128;              // templates per tile (TMEM lanes)
constexpr int kBN = 256;              // samples per tile (TMEM columns)
constexpr int kBK = 64;               // q per slice: one 128-byte swizzle row
constexpr int kStages = 2;
constexpr int kTileA = kBM * kBK * 2;             // 16 KB
constexpr int kTileB = kBN * kBK * 2;             // 32 KB
constexpr int kStageBytes = 2 * kTileA + 2 * kTileB;
constexpr int kThreads = 192;
constexpr int kTmemCols = 512;
constexpr unsigned long long kLimitNs = 2000000000ull;

// instruction descriptor: FP32 accumulate, BF16 A and B, both K-major,
// N = 256 (bits 17-22 hold N >> 3), M = 128 (bits 24-28 hold M >> 4)
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kBN >> 3) << 17) |
                            ((uint32_t)(kBM >> 4) << 24);

using namespace ks::tc;

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int* err) {
  return mbar_wait_bounded(bar, parity, err, kLimitNs);
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), version 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  return make_smem_desc(addr, 16, 1024, kSwizzle128B);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
  mma_f16(d_tmem, a, b, kIdesc, acc);
}

using ks::GemmBatch;
using ks::GemmGroup;

// Batch of global tile t (the batches' tile ranges are consecutive).
__device__ __forceinline__ int tile_batch(const GemmGroup& g, int t) {
  int lo = 0, hi = g.n_batches - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (g.batches[mid].tile_begin <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void __launch_bounds__(kThreads, 1)
ks_bf16x3_kernel(const __grid_constant__ GemmGroup g) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // 1024-byte alignment for the swizzled tiles
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char* gbase = smem_raw + (base - raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(gbase + kStages * kStageBytes);
  // bars: full[kStages], empty[kStages], tfull[2], tempty[2], drain[1]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 5);
  const uint32_t full0 = smem_u32(bars);
  const uint32_t empty0 = full0 + 8 * kStages;
  const uint32_t tfull0 = empty0 + 8 * kStages;
  const uint32_t tempty0 = tfull0 + 16;
  const uint32_t drain = tempty0 + 16;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(tfull0 + 8 * a, 1);
      mbar_init(tempty0 + 8 * a, 4);
    }
    mbar_init(drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tmem_slot);

  if (warp == 0) {
    // ---------------------------------------------------------- TMA producer
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      bool pending[kStages] = {};     // a load was issued into the stage ...
      uint32_t pend_ph[kStages] = {}; // ... completing this phase of full[stage]
      bool ok = true;
      for (int t = blockIdx.x; ok && t < g.n_tiles; t += gridDim.x) {
        const GemmBatch& bt = g.batches[tile_batch(g, t)];
        const int lt = t - bt.tile_begin;
        const int m0 = (lt % bt.tiles_m) * kBM;
        const int y0 = bt.row_off + (lt / bt.tiles_m) * kBN;
        const CUtensorMap* maps = g.maps[bt.rec];
        const int nk = g.nk[bt.rec];
        for (int kb = 0; kb < nk; ++kb) {
          if (!mbar_wait(empty0 + 8 * s, ph ^ 1u, g.err)) { ok = false; break; }
          const uint32_t st = base + s * kStageBytes;
          const uint32_t fb = full0 + 8 * s;
          mbar_expect_tx(fb, kStageBytes);
          tma_load_2d(st, &maps[0], kb * kBK, m0, fb);
          tma_load_2d(st + kTileA, &maps[1], kb * kBK, m0, fb);
          tma_load_2d(st + 2 * kTileA, &maps[2], kb * kBK, y0, fb);
          tma_load_2d(st + 2 * kTileA + kTileB, &maps[3], kb * kBK, y0, fb);
          pending[s] = true;
          pend_ph[s] = ph;
          if (++s == kStages) { s = 0; ph ^= 1u; }
        }
      }
      if (!ok) {
        // leave no copy in flight: wait (bounded) for the last load of each stage
        const unsigned long long t0 = ks_globaltimer();
        for (int si = 0; si < kStages; ++si) {
          if (!pending[si]) continue;
          while (!mbar_try_wait(full0 + 8 * si, pend_ph[si])) {
            if (ks_globaltimer() - t0 > kLimitNs) break;
          }
        }
      }
    }
  } else if (warp == 1) {
    // ---------------------------------------------------------- MMA issuer
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      int acc = 0;
      uint32_t acc_ph = 0;
      bool ok = true;
      for (int t = blockIdx.x; ok && t < g.n_tiles; t += gridDim.x) {
        if (!mbar_wait(tempty0 + 8 * acc, acc_ph ^ 1u, g.err)) { ok = false; break; }
        fence_after();
        const uint32_t d = tmem + (uint32_t)(acc * kBN);
        const int nk = g.nk[g.batches[tile_batch(g, t)].rec];
        for (int kb = 0; kb < nk; ++kb) {
          if (!mbar_wait(full0 + 8 * s, ph, g.err)) { ok = false; break; }
          fence_after();
          const uint32_t st = base + s * kStageBytes;
#pragma unroll
          for (int kk = 0; kk < kBK / 16; ++kk) {
            const uint64_t a_hi = smem_desc(st + kk * 32);
            const uint64_t a_lo = smem_desc(st + kTileA + kk * 32);
            const uint64_t b_hi = smem_desc(st + 2 * kTileA + kk * 32);
            const uint64_t b_lo = smem_desc(st + 2 * kTileA + kTileB + kk * 32);
            const uint32_t first = (kb == 0 && kk == 0) ? 0u : 1u;
            mma_bf16(d, a_hi, b_hi, first);
            mma_bf16(d, a_hi, b_lo, 1u);
            mma_bf16(d, a_lo, b_hi, 1u);
          }
          mma_commit(empty0 + 8 * s);   // stage free once these MMAs finish
          if (++s == kStages) { s = 0; ph ^= 1u; }
        }
        if (!ok) break;
        mma_commit(tfull0 + 8 * acc);   // accumulator complete
        acc ^= 1;
        if (acc == 0) acc_ph ^= 1u;
      }
      // every MMA issued by this thread has completed once this commit lands
      mma_commit(drain);
      const unsigned long long t0 = ks_globaltimer();
      while (!mbar_try_wait(drain, 0u)) {
        if (ks_globaltimer() - t0 > kLimitNs) break;
      }
    }
  } else {
    // ---------------------------------------------------------- epilogue
    const int q = warp & 3;                  // TMEM lane quadrant of this warp
    int acc = 0;
    uint32_t acc_ph = 0;
    for (int t = blockIdx.x; t < g.n_tiles; t += gridDim.x) {
      const GemmBatch& bt = g.batches[tile_batch(g, t)];
      const int lt = t - bt.tile_begin;
      const int m0 = (lt % bt.tiles_m) * kBM;
      const int n0 = (lt / bt.tiles_m) * kBN;
      // the warp leaves together (tcgen05.ld below needs every lane)
      if (!__all_sync(0xffffffffu, mbar_wait(tfull0 + 8 * acc, acc_ph, g.err))) break;
      fence_after();
      const int row = m0 + q * 32 + lane;    // template of this thread
      const uint32_t tl = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * kBN);
#pragma unroll 1
      for (int c = 0; c < kBN / 32; ++c) {
        uint32_t r[32];
        tmem_ld32(tl + (uint32_t)(c * 32), r);
        const int n = n0 + c * 32;
        if (row < bt.K && n < bt.L) {
          float* dst = g.tiled ? bt.B + ((size_t)(n >> 5) * bt.K + row) * 32
                               : bt.B + (size_t)row * bt.ldb + n;
          // the tiled layout's last block is written whole (zeros past L)
          const bool full = (g.tiled || n + 32 <= bt.L) &&
                            ((reinterpret_cast<uintptr_t>(dst) & 15) == 0);
          if (full) {
            const int nv = bt.L - n;   // valid columns of this block (>= 1)
#pragma unroll
            for (int e = 0; e < 32; ++e)
              if (e >= nv) r[e] = 0u;
#pragma unroll
            for (int v = 0; v < 8; ++v)
              reinterpret_cast<float4*>(dst)[v] =
                  make_float4(__uint_as_float(r[4 * v]), __uint_as_float(r[4 * v + 1]),
                              __uint_as_float(r[4 * v + 2]), __uint_as_float(r[4 * v + 3]));
          } else {
#pragma unroll
            for (int e = 0; e < 32; ++e)
              if (n + e < bt.L) dst[e] = __uint_as_float(r[e]);
          }
        }
      }
      fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(tempty0 + 8 * acc);
      acc ^= 1;
      if (acc == 0) acc_ph ^= 1u;
    }
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

// ------------------------------------------------------------------ host side
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static EncodeTiled fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return static_cast<EncodeTiled>(nullptr);
    return reinterpret_cast<EncodeTiled>(p);
  }();
  return fn;
}

// 2-D bf16 tensor [rows][cols] (cols contiguous), box [box_rows][64], 128B swizzle
int make_map(CUtensorMap* map, const __nv_bfloat16* ptr, int64_t rows, int64_t cols,
             int box_rows) {
  EncodeTiled fn = encode_fn();
  if (!fn) return ks::fail(KS_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(ptr), dims,
                  strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return ks::fail(KS_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  return KS_OK;
}

}  // namespace

namespace ks {

int make_bf16_map(CUtensorMap* map, const __nv_bfloat16* ptr, int64_t rows, int64_t cols,
                  int box_rows) {
  if (reinterpret_cast<uintptr_t>(ptr) & 15) return fail(KS_ERR_ARG, "bf16x3: operands must be 16-byte aligned");
  return make_map(map, ptr, rows, cols, box_rows);
}

int make_bf16_store_map(CUtensorMap* map, const __nv_bfloat16* ptr, int64_t rows, int64_t cols,
                        int64_t row_stride, int box_cols, int box_rows) {
  EncodeTiled fn = encode_fn();
  if (!fn) return fail(KS_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
  if ((reinterpret_cast<uintptr_t>(ptr) & 15) || (row_stride * 2) % 16 || (box_cols * 2) % 16)
    return fail(KS_ERR_ARG, "tensor map: 16-byte alignment needed");
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)row_stride * 2};
  const cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(ptr), dims,
                  strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(KS_ERR_CUDA, "cuTensorMapEncodeTiled failed (store map)");
  return KS_OK;
}

int gemm_tile_n() { return kBN; }
int gemm_tile_m() { return kBM; }

int launch_gemm_group(GemmGroup& g, cudaStream_t stream) {
  if (g.n_batches < 1 || g.n_batches > kGroupBatches) return fail(KS_ERR_ARG, "bf16x3: bad group size");
  if (!g.err) return fail(KS_ERR_ARG, "bf16x3: error word missing");
  DeviceInfo dev;
  int rc = device_info(&dev);
  if (rc) return rc;
  const size_t smem = (size_t)kStages * kStageBytes + 1024 + 256;
  static thread_local int attr_device = -1;
  if (attr_device != dev.device) {
    KS_CUDA(cudaFuncSetAttribute(ks_bf16x3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    attr_device = dev.device;
  }
  const int grid = std::min(dev.sm_count, g.n_tiles);
  if (grid < 1) return KS_OK;
  ks_bf16x3_kernel<<<grid, kThreads, smem, stream>>>(g);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

int gemm_bf16x3(const __nv_bfloat16* Uhi, const __nv_bfloat16* Ulo, const __nv_bfloat16* Yhi,
                const __nv_bfloat16* Ylo, float* B, int64_t K, int64_t L, int64_t Q,
                int64_t Kpad, int64_t Lpad, int64_t ldb, bool tiled, int* err,
                cudaStream_t stream) {
  if (!err) return fail(KS_ERR_ARG, "bf16x3: error word missing");
  if (Q % kBK) return fail(KS_ERR_ARG, "bf16x3: contraction length must be a multiple of 64");
  if (Kpad % kBM) return fail(KS_ERR_ARG, "bf16x3: template rows must be padded to 128");
  static thread_local GemmGroup g;   // about 14 KB: kept off the stack
  int rc;
  if ((rc = make_bf16_map(&g.maps[0][0], Uhi, Kpad, Q, kBM))) return rc;
  if ((rc = make_bf16_map(&g.maps[0][1], Ulo, Kpad, Q, kBM))) return rc;
  if ((rc = make_bf16_map(&g.maps[0][2], Yhi, Lpad, Q, kBN))) return rc;
  if ((rc = make_bf16_map(&g.maps[0][3], Ylo, Lpad, Q, kBN))) return rc;
  g.nk[0] = (int)(Q / kBK);
  GemmBatch& b = g.batches[0];
  b.B = B;
  b.ldb = ldb;
  b.K = (int)K;
  b.L = (int)L;
  b.rec = 0;
  b.row_off = 0;
  b.tiles_m = (int)(Kpad / kBM);
  b.tile_begin = 0;
  g.n_batches = 1;
  g.n_tiles = b.tiles_m * (int)((L + kBN - 1) / kBN);
  g.tiled = tiled ? 1 : 0;
  g.err = err;
  return launch_gemm_group(g, stream);
}

}  // namespace ks
