// High-pass FIR of the batch filter on the 5th-generation tensor cores.
//
// The circular correlation y[c, n] = sum_j taps[j] x[c, (n + j - h) mod L]
// (kilosort/io.py:1008-1010 in the time domain) of the 128 samples
// n0 .. n0+127 of every channel is one matrix product
//
//   Y[i, c] = sum_m H[i, m] * P[c, n0 + m],   H[i, m] = taps[m - i]  (0 <= m - i < ntaps)
//
// with H the banded Toeplitz matrix of the taps (128 x Kpad, Kpad = 127 +
// ntaps rounded up to 64: at most 1152) -- the same for every tile -- and P
// the batch padded circularly, P[c, j] = x[c, (j - h) mod L], so that the
// window of tile n0 is the plain column range [n0, n0 + Kpad) of P.  Both
// operands are split into bf16 hi + lo and the product is Hhi.Phi + Hhi.Plo +
// Hlo.Phi with FP32 accumulation in TMEM (about 2^-16 of sum |taps x| per
// sample; 7e-6 of the batch maximum on Neuropixels-like data).  The FP32 FIR
// spends 2 * ntaps flops per sample on the SIMT pipes; here the tensor cores
// spend 3 * 2 * Kpad per sample at their much higher rate.
//
// Persistent kernel, one CTA per SM, 6 warps (as the score contraction):
//   warp 0     TMA producer: per 64-wide slice of m, Hhi, Hlo (128x64) and
//              Phi, Plo (N x 64), 128-byte swizzle, into a 2-stage ring
//   warp 1     allocates TMEM; one lane issues 12 MMAs per slice (M = 128,
//              N = channels per tile, K = 16) into a double-buffered
//              accumulator and commits stage releases and hand-offs
//   warps 2-5  epilogue: tcgen05.ld 32 channels at a time (one sample row per
//              thread); flags artifacts (|y| >= threshold); writes the bf16
//              hi/lo [rows][Cq] operand of the whitening contraction (zeros
//              past L and C), or f32 rows X[c][n]
// Tiles are 128 samples x N channels, the channel tiles of one sample tile
// consecutive.  No TMA multicast.  Every mbarrier wait is bounded by
// %globaltimer; a wait that runs out sets the error word, the CTA drains its
// own copies in flight (bounded), frees TMEM and returns.
#include "ks_common.cuh"
#include "project.cuh"
#include "tcgen05.cuh"

#include <algorithm>
#include <cuda.h>
#include <cuda_bf16.h>

namespace {

constexpr int kTM = 128;              // samples per tile (TMEM lanes)
constexpr int kBK = 64;               // m per slice: one 128-byte swizzle row
constexpr int kMaxN = 256;            // channels per tile
constexpr int kStages = 2;
constexpr int kTileA = kTM * kBK * 2;             // 16 KB
constexpr int kThreads = 192;
constexpr unsigned long long kLimitNs = 2000000000ull;

using namespace ks::tc;

struct FirArgs {
  CUtensorMap a_hi, a_lo, p_hi, p_lo;
  int C, L, rows, Cq;                 // channels, samples, output rows, operand width
  int N, tiles_t, tiles_c, nk;        // channels per tile, tile counts, slices
  uint32_t idesc;
  int check;
  float thr;
  float* X;                           // f32 rows (split output absent)
  long long ldx;
  __nv_bfloat16* yhi;                 // bf16 hi/lo [rows][Cq] (or null)
  __nv_bfloat16* ylo;
  int* art;
  int* err;
};

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int* err) {
  return mbar_wait_bounded(bar, parity, err, kLimitNs);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  return make_smem_desc(addr, 16, 1024, kSwizzle128B);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&v);
}

__global__ void __launch_bounds__(kThreads, 1)
ks_fir_tc_kernel(const __grid_constant__ FirArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  const uint32_t tileB = (uint32_t)a.N * kBK * 2;
  const uint32_t stage_bytes = 2u * kTileA + 2u * tileB;
  unsigned char* gbase = smem_raw + (base - raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(gbase + kStages * stage_bytes);
  // bars: full[kStages], empty[kStages], tfull[2], tempty[2], drain[1]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 5);
  const uint32_t full0 = smem_u32(bars);
  const uint32_t empty0 = full0 + 8 * kStages;
  const uint32_t tfull0 = empty0 + 8 * kStages;
  const uint32_t tempty0 = tfull0 + 16;
  const uint32_t drain = tempty0 + 16;
  uint32_t tcols = 32;
  while (tcols < 2u * (uint32_t)a.N) tcols <<= 1;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_tiles = a.tiles_t * a.tiles_c;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(tfull0 + 8 * b, 1);
      mbar_init(tempty0 + 8 * b, 4);
    }
    mbar_init(drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(smem_u32(tmem_slot), tcols);
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tmem_slot);

  if (warp == 0) {
    // ---------------------------------------------------------- TMA producer
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      bool pending[kStages] = {};
      uint32_t pend_ph[kStages] = {};
      bool ok = true;
      for (int t = blockIdx.x; ok && t < n_tiles; t += gridDim.x) {
        const int n0 = (t / a.tiles_c) * kTM;
        const int c0 = (t % a.tiles_c) * a.N;
        for (int kb = 0; kb < a.nk; ++kb) {
          if (!mbar_wait(empty0 + 8 * s, ph ^ 1u, a.err)) { ok = false; break; }
          const uint32_t st = base + s * stage_bytes;
          const uint32_t fb = full0 + 8 * s;
          mbar_expect_tx(fb, stage_bytes);
          tma_load_2d(st, &a.a_hi, kb * kBK, 0, fb);
          tma_load_2d(st + kTileA, &a.a_lo, kb * kBK, 0, fb);
          tma_load_2d(st + 2 * kTileA, &a.p_hi, n0 + kb * kBK, c0, fb);
          tma_load_2d(st + 2 * kTileA + tileB, &a.p_lo, n0 + kb * kBK, c0, fb);
          pending[s] = true;
          pend_ph[s] = ph;
          if (++s == kStages) { s = 0; ph ^= 1u; }
        }
      }
      if (!ok) {
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
      for (int t = blockIdx.x; ok && t < n_tiles; t += gridDim.x) {
        if (!mbar_wait(tempty0 + 8 * acc, acc_ph ^ 1u, a.err)) { ok = false; break; }
        fence_after();
        const uint32_t d = tmem + (uint32_t)(acc * a.N);
        for (int kb = 0; kb < a.nk; ++kb) {
          if (!mbar_wait(full0 + 8 * s, ph, a.err)) { ok = false; break; }
          fence_after();
          const uint32_t st = base + s * stage_bytes;
#pragma unroll
          for (int kk = 0; kk < kBK / 16; ++kk) {
            const uint64_t a_hi = smem_desc(st + kk * 32);
            const uint64_t a_lo = smem_desc(st + kTileA + kk * 32);
            const uint64_t b_hi = smem_desc(st + 2 * kTileA + kk * 32);
            const uint64_t b_lo = smem_desc(st + 2 * kTileA + tileB + kk * 32);
            const uint32_t first = (kb == 0 && kk == 0) ? 0u : 1u;
            mma_f16(d, a_hi, b_hi, a.idesc, first);
            mma_f16(d, a_hi, b_lo, a.idesc, 1u);
            mma_f16(d, a_lo, b_hi, a.idesc, 1u);
          }
          mma_commit(empty0 + 8 * s);
          if (++s == kStages) { s = 0; ph ^= 1u; }
        }
        if (!ok) break;
        mma_commit(tfull0 + 8 * acc);
        acc ^= 1;
        if (acc == 0) acc_ph ^= 1u;
      }
      mma_commit(drain);
      const unsigned long long t0 = ks_globaltimer();
      while (!mbar_try_wait(drain, 0u)) {
        if (ks_globaltimer() - t0 > kLimitNs) break;
      }
    }
  } else {
    // ---------------------------------------------------------- epilogue
    const int q = warp & 3;
    int acc = 0;
    uint32_t acc_ph = 0;
    bool art = false;
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
      const int n0 = (t / a.tiles_c) * kTM;
      const int c0 = (t % a.tiles_c) * a.N;
      if (!__all_sync(0xffffffffu, mbar_wait(tfull0 + 8 * acc, acc_ph, a.err))) break;
      fence_after();
      const int n = n0 + q * 32 + lane;      // sample of this thread
      const uint32_t tl = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * a.N);
#pragma unroll 1
      for (int cc = 0; cc < a.N / 32; ++cc) {
        uint32_t r[32];
        tmem_ld32(tl + (uint32_t)(cc * 32), r);
        const int cb = c0 + cc * 32;
        if (a.check && n < a.L) {
#pragma unroll
          for (int e = 0; e < 32; ++e)
            if (cb + e < a.C && fabsf(__uint_as_float(r[e])) >= a.thr) art = true;
        }
        if (a.yhi) {
          if (n < a.rows && cb < a.Cq) {
            // zeros past L and past C: the contraction reads whole rows
            float v[32];
#pragma unroll
            for (int e = 0; e < 32; ++e)
              v[e] = (n < a.L && cb + e < a.C) ? __uint_as_float(r[e]) : 0.f;
            uint32_t hi[16], lo[16];
#pragma unroll
            for (int e = 0; e < 16; ++e) {
              const __nv_bfloat16 h0 = __float2bfloat16_rn(v[2 * e]);
              const __nv_bfloat16 h1 = __float2bfloat16_rn(v[2 * e + 1]);
              const __nv_bfloat162 hh = __halves2bfloat162(h0, h1);
              hi[e] = *reinterpret_cast<const uint32_t*>(&hh);
              lo[e] = pack_bf16(v[2 * e] - __bfloat162float(h0),
                                v[2 * e + 1] - __bfloat162float(h1));
            }
            // Cq is a multiple of 64 and cb of 32: the 32 channels are all inside
            uint4* dh = reinterpret_cast<uint4*>(a.yhi + (size_t)n * a.Cq + cb);
            uint4* dl = reinterpret_cast<uint4*>(a.ylo + (size_t)n * a.Cq + cb);
#pragma unroll
            for (int v4 = 0; v4 < 4; ++v4) {
              dh[v4] = make_uint4(hi[4 * v4], hi[4 * v4 + 1], hi[4 * v4 + 2], hi[4 * v4 + 3]);
              dl[v4] = make_uint4(lo[4 * v4], lo[4 * v4 + 1], lo[4 * v4 + 2], lo[4 * v4 + 3]);
            }
          }
        } else if (n < a.L) {
#pragma unroll
          for (int e = 0; e < 32; ++e)
            if (cb + e < a.C) a.X[(size_t)(cb + e) * a.ldx + n] = __uint_as_float(r[e]);
        }
      }
      fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(tempty0 + 8 * acc);
      acc ^= 1;
      if (acc == 0) acc_ph ^= 1u;
    }
    if (__any_sync(0xffffffffu, art) && lane == 0) atomicOr(a.art, 1);
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 1) tmem_dealloc(tmem, tcols);
}

// H[i][m] = taps[m - i] for 0 <= m - i < ntaps, else 0; bf16 hi and lo planes.
__global__ void ks_fir_toeplitz_kernel(const float* __restrict__ taps, int ntaps, int kpad,
                                       __nv_bfloat16* __restrict__ hi,
                                       __nv_bfloat16* __restrict__ lo) {
  const int n = kTM * kpad;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int i = e / kpad, m = e - i * kpad;
    const int j = m - i;
    const float v = (j >= 0 && j < ntaps) ? taps[j] : 0.f;
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    hi[e] = h;
    lo[e] = __float2bfloat16_rn(v - __bfloat162float(h));
  }
}

}  // namespace

namespace ks {

int64_t fir_tc_kpad(int ntaps) { return round_up((int64_t)kTM - 1 + ntaps, kBK); }

int64_t fir_tc_cols(int64_t rows, int ntaps) {
  const int64_t tiles = (rows + kTM - 1) / kTM;
  return kTM * (tiles - 1) + fir_tc_kpad(ntaps);
}

size_t fir_tc_toeplitz_bytes(int ntaps) { return 2 * (size_t)kTM * fir_tc_kpad(ntaps) * 2; }

int fir_tc(const float* taps, int ntaps, const __nv_bfloat16* p_hi, const __nv_bfloat16* p_lo,
           int64_t C, int64_t L, int64_t cols, int64_t rows, __nv_bfloat16* h_hi,
           __nv_bfloat16* h_lo, bool check, float thr, float* X, int64_t ldx,
           __nv_bfloat16* yhi, __nv_bfloat16* ylo, int64_t Cq, int* art, int* err,
           cudaStream_t stream) {
  if (!taps || ntaps < 1 || ntaps > 1023 || !p_hi || !p_lo || !h_hi || !h_lo || !art || !err)
    return fail(KS_ERR_ARG, "fir_tc: bad arguments");
  if (C < 1 || L < 1 || rows < L || cols != fir_tc_cols(rows, ntaps) || cols % 8)
    return fail(KS_ERR_ARG, "fir_tc: operand geometry");
  if (yhi ? (!ylo || Cq % 64 || Cq < C) : (!X || ldx < L))
    return fail(KS_ERR_ARG, "fir_tc: output");
  const int64_t kpad = fir_tc_kpad(ntaps);
  static thread_local FirArgs a;      // about 600 bytes of tensor maps: kept off the stack
  int rc;
  if ((rc = make_bf16_map(&a.a_hi, h_hi, kTM, kpad, kTM))) return rc;
  if ((rc = make_bf16_map(&a.a_lo, h_lo, kTM, kpad, kTM))) return rc;
  // channel tiles: as few as fit 256 columns, each a multiple of 32 wide,
  // covering the whole operand width (the zero channels past C included)
  const int64_t width = yhi ? Cq : C;
  const int tiles_c = (int)((width + kMaxN - 1) / kMaxN);
  const int N = (int)round_up((width + tiles_c - 1) / tiles_c, 32);
  if ((rc = make_bf16_map(&a.p_hi, p_hi, C, cols, N))) return rc;
  if ((rc = make_bf16_map(&a.p_lo, p_lo, C, cols, N))) return rc;
  a.C = (int)C;
  a.L = (int)L;
  a.rows = (int)rows;
  a.Cq = (int)Cq;
  a.N = N;
  a.tiles_t = (int)((rows + kTM - 1) / kTM);
  a.tiles_c = tiles_c;
  a.nk = (int)(kpad / kBK);
  a.idesc = idesc_bf16_f32(kTM, N);
  a.check = check ? 1 : 0;
  a.thr = thr;
  a.X = X;
  a.ldx = ldx;
  a.yhi = yhi;
  a.ylo = ylo;
  a.art = art;
  a.err = err;
  {
    const int n = kTM * (int)kpad;
    ks_fir_toeplitz_kernel<<<(n + 255) / 256, 256, 0, stream>>>(taps, ntaps, (int)kpad, h_hi, h_lo);
    KS_CUDA(cudaGetLastError());
  }
  DeviceInfo dev;
  if ((rc = device_info(&dev))) return rc;
  const size_t stage = 2 * (size_t)kTileA + 2 * (size_t)N * kBK * 2;
  const size_t smem = kStages * stage + 1024 + 256;
  KS_CUDA(cudaFuncSetAttribute(ks_fir_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
  const int grid = (int)std::min<int64_t>(dev.sm_count, (int64_t)a.tiles_t * tiles_c);
  ks_fir_tc_kernel<<<grid, kThreads, smem, stream>>>(a);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

}  // namespace ks
