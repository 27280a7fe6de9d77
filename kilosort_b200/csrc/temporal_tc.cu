// Temporal projection of the split form on the tensor cores (tcgen05):
//
//   Y[tau, c*P + p] = sum_t W[p, t] * X[c, tau - nt/2 + t]     (zero padding)
//
// written as the bf16 hi/lo planes the split-BF16 contraction reads
// (kilosort/template_matching.py:180, the conv1d of the batch with wPCA).
//
// The convolution of one channel is a product with a Toeplitz operand.  With
// the window x_w[u] = X[c, tau0 - nt/2 + u], MMA row r stands for the eight
// samples tau0 + 8r + phi (phi = 0..7) and the phases go to the N dimension:
//
//   D[r, phi*P + p] = sum_k x_w[8r + k] * Wsh[phi*P + p, k],
//   Wsh[phi*P + p, k] = W[p, k - phi]  (zero outside 0 <= k - phi < nt)
//
// A[r, k] = x_w[8r + k] is the canonical non-swizzled K-major layout read
// straight from the window: rows 16 bytes (8 samples) apart inside a core
// matrix, the next 8 taps 16 bytes on (LBO), the next 8 rows 128 bytes on
// (SBO); core matrices overlap in memory, which the tensor core does not
// mind.  So a tile is M = 128 rows = 1024 samples of one channel, N = 8P
// (rounded to 16), K = nt + 7 (rounded to 16); split-BF16 as the score
// contraction: x = hi + lo, Wsh = hi + lo, D = Ahi.Bhi + Ahi.Blo + Alo.Bhi with
// FP32 accumulation, then D is split again into the bf16 hi/lo planes of Y.
//
// Persistent, one CTA per SM, 8 warps; a tile is 1024 samples x 4 channels:
//   warps 4-7  producer: the 4 channel windows (f32 -> bf16 hi/lo) into a
//              double-buffered shared-memory slot (all of a tile's loads in
//              flight at once, in registers); one lane then issues the MMAs (4 channels x 3 products x K/16 steps) into a
//              double-buffered TMEM accumulator and commits them to an mbarrier
//   warps 0-3  epilogue: thread r reads its row (8 samples x P components of
//              each channel), splits it into hi/lo and stages it in shared
//              memory as the boxes of the output (phase, row) blocks; one
//              thread then writes the 16 blocks (2 planes x 8 phases, 128 rows
//              x 4P values each) with TMA stores (no multicast) through one
//              tensor map per phase whose rows are 8 samples apart
// Tiles of one time range are consecutive (channel groups fastest), so the
// partial 32-byte sectors at channel-group edges meet in L2.  Every mbarrier
// wait is bounded; a wait that runs out sets the error word and the CTA
// drains its MMAs, frees TMEM and returns.
#include "ks_common.cuh"
#include "project.cuh"
#include "tcgen05.cuh"

#include <algorithm>
#include <cuda_bf16.h>

namespace {

using namespace ks::tc;

constexpr int kRows = 128;                 // MMA rows (TMEM lanes)
constexpr int kSamples = 8 * kRows;        // samples per tile
constexpr int kG = 4;                      // channels per tile
constexpr int kEpiThreads = 128;       // warps 0-3: epilogue
constexpr int kThreads = kEpiThreads + 128;   // warps 4-7: producer
constexpr int kTmemCols = 512;
constexpr int kMaxK = 128;                 // taps + 7, rounded to 16
constexpr unsigned long long kLimitNs = 2000000000ull;
// sample pairs of a window per producer thread: window_len(kMaxK) / 2 / 128, rounded up
constexpr int kPairIters = (8 * (kRows - 1) + kMaxK + 255) / 256;

template <int PP>
struct Shape {
  static constexpr int NN = (8 * PP + 15) / 16 * 16;   // MMA N
  // staged output: [plane][phase][row][4*PP bf16], the boxes of the TMA stores
  static constexpr int kStageBytes = 2 * 8 * kRows * 8 * PP;
};

// TMA store maps of the output planes: m[plane][phi] covers the rows
// tau = 8*y + phi of Y (base Y + phi*Q, row stride 8*Q), boxes of 128 rows x
// 4*P columns.
struct TemporalMaps {
  CUtensorMap m[2][8];
};

__host__ __device__ constexpr int window_len(int kext) { return 8 * (kRows - 1) + kext; }

template <int PP>
struct Smem {
  int kext;
  __host__ __device__ size_t b_bytes() const { return (size_t)2 * Shape<PP>::NN * kext * 2; }
  __host__ __device__ size_t a_slot() const { return (size_t)window_len(kext) * 2; }
  __host__ __device__ size_t a_bytes() const { return 2 * kG * 2 * a_slot(); }
  __host__ __device__ size_t off_a() const { return b_bytes(); }
  __host__ __device__ size_t off_s() const { return (off_a() + a_bytes() + 127) & ~size_t(127); }
  __host__ __device__ size_t s_bytes() const { return (size_t)Shape<PP>::kStageBytes; }
  __host__ __device__ size_t off_bar() const { return (off_s() + s_bytes() + 15) & ~size_t(15); }
  __host__ __device__ size_t total() const { return off_bar() + 64 + 128; }
};

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr));
}
// TMA store of a 2-D box from shared memory (no multicast), bulk-group completion.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, uint32_t src, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
          reinterpret_cast<uint64_t>(map)),
      "r"(src), "r"(x), "r"(y)
      : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// the source shared memory of every committed store has been read
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// every committed store has completed
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Named barrier over `count` threads that also ANDs a predicate: every
// participant gets the same answer, so a group leaves its loop together.
__device__ __forceinline__ bool group_all(bool ok, int id, int count) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)ok), "r"(id), "r"(count)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void group_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

__device__ __forceinline__ uint32_t bf16x2_bits(__nv_bfloat162 v) {
  return *reinterpret_cast<uint32_t*>(&v);
}

template <int PP>
__global__ void __launch_bounds__(kThreads, 1)
ks_temporal_tc_kernel(const float* __restrict__ X, const float* __restrict__ W, int C, int L,
                      int nt, int kext, int n_cg, int n_tiles,
                      const __grid_constant__ TemporalMaps maps, int* err) {
  constexpr int NN = Shape<PP>::NN;
  extern __shared__ __align__(128) unsigned char smem[];
  const Smem<PP> lay{kext};
  unsigned char* sB = smem;
  unsigned char* sA = smem + lay.off_a();
  uint32_t* sS = reinterpret_cast<uint32_t*>(smem + lay.off_s());
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + lay.off_bar());
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 8);
  const uint32_t full0 = smem_u32(bars);        // full[2]: MMAs of a buffer done
  const uint32_t tfree0 = full0 + 16;           // tfree[2]: epilogue read the accumulator
  const uint32_t drain = full0 + 32;
  const int warp = threadIdx.x >> 5;
  const int half = nt / 2;
  const size_t aslot = lay.a_slot();
  const size_t bplane = (size_t)NN * kext * 2;

  // shifted, split basis Wsh (hi, lo) in the K-major core-matrix layout:
  // (n, k) at ((n/8)*(kext/8) + k/8)*128 + (n%8)*16 + (k%8)*2
  for (int e = threadIdx.x; e < NN * kext; e += kThreads) {
    const int n = e / kext, k = e - n * kext;
    const int phi = n / PP, p = n - phi * PP;
    const int t = k - phi;
    const float v = (phi < 8 && t >= 0 && t < nt) ? W[p * nt + t] : 0.f;
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
    const size_t o = ((size_t)(n >> 3) * (kext >> 3) + (k >> 3)) * 128 + (n & 7) * 16 + (k & 7) * 2;
    *reinterpret_cast<__nv_bfloat16*>(sB + o) = h;
    *reinterpret_cast<__nv_bfloat16*>(sB + bplane + o) = l;
  }
  if (threadIdx.x == 0) {
    for (int b = 0; b < 2; ++b) {
      mbar_init(full0 + 8 * b, 1);
      mbar_init(tfree0 + 8 * b, kEpiThreads);
    }
    mbar_init(drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(smem_u32(tmem_slot), kTmemCols);
  fence_proxy_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tmem_slot);
  constexpr uint32_t idesc = idesc_bf16_f32(kRows, NN);
  const int nk = kext / 16;

  if (warp >= kEpiThreads / 32) {
    // ------------------------------------------------------------ producer
    const int pt = threadIdx.x - kEpiThreads;
    const int wl = window_len(kext);
    // thread pt owns the sample pairs u = 2*(pt + 128*i) of the four windows;
    // all of them are loaded before the first is converted (zero outside the
    // recording and for channels past C)
    float2 xv[kG][kPairIters];
    auto load_windows = [&](int tile) {
      const int tau0 = (tile / n_cg) * kSamples;
      const int c0 = (tile % n_cg) * kG;
#pragma unroll
      for (int g = 0; g < kG; ++g) {
        const int c = c0 + g;
        const float* xr = X + (size_t)(c < C ? c : 0) * L;
#pragma unroll
        for (int i = 0; i < kPairIters; ++i) {
          const int u = 2 * (pt + 128 * i);
          const int s0 = tau0 - half + u;
          const bool in = c < C && u < wl;
          xv[g][i].x = (in && s0 >= 0 && s0 < L) ? __ldg(xr + s0) : 0.f;
          xv[g][i].y = (in && s0 + 1 >= 0 && s0 + 1 < L) ? __ldg(xr + s0 + 1) : 0.f;
        }
      }
    };
    bool ok = true;
    int j = 0;
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++j) {
      const int b = j & 1;
      const uint32_t use = (uint32_t)(j >> 1);
      // the slot's previous MMAs have read it
      if (use > 0) ok = mbar_wait_bounded(full0 + 8 * b, (use - 1) & 1u, err, kLimitNs);
      if (!group_all(ok, 2, 128)) { ok = false; break; }
      unsigned char* slot = sA + (size_t)b * kG * 2 * aslot;
      load_windows(t);
#pragma unroll
      for (int g = 0; g < kG; ++g) {
        uint32_t* hi = reinterpret_cast<uint32_t*>(slot + (size_t)(2 * g) * aslot);
        uint32_t* lo = reinterpret_cast<uint32_t*>(slot + (size_t)(2 * g + 1) * aslot);
#pragma unroll
        for (int i = 0; i < kPairIters; ++i) {
          const int u2 = pt + 128 * i;
          if (2 * u2 < wl) {
            const __nv_bfloat162 h = __floats2bfloat162_rn(xv[g][i].x, xv[g][i].y);
            const float2 hf = __bfloat1622float2(h);
            hi[u2] = bf16x2_bits(h);
            lo[u2] = bf16x2_bits(__floats2bfloat162_rn(xv[g][i].x - hf.x, xv[g][i].y - hf.y));
          }
        }
      }
      fence_proxy_async_smem();
      group_sync(2, 128);
      if (pt == 0) {
        // the accumulator's previous contents have been read
        if (use > 0 && !mbar_wait_bounded(tfree0 + 8 * b, (use - 1) & 1u, err, kLimitNs)) {
          ok = false;
        } else {
          fence_after();
          const uint32_t a0 = smem_u32(slot), b0 = smem_u32(sB);
          for (int g = 0; g < kG; ++g) {
            const uint32_t d = tmem + (uint32_t)(b * 256 + g * NN);
            const uint32_t ahi = a0 + (uint32_t)((2 * g) * aslot);
            const uint32_t alo = a0 + (uint32_t)((2 * g + 1) * aslot);
            for (int kk = 0; kk < nk; ++kk) {
              const uint64_t dah = make_smem_desc(ahi + 32 * kk, 16, 128, kSwizzleNone);
              const uint64_t dal = make_smem_desc(alo + 32 * kk, 16, 128, kSwizzleNone);
              const uint32_t sbo = (uint32_t)(kext / 8) * 128;
              const uint64_t dbh = make_smem_desc(b0 + 256 * kk, 128, sbo, kSwizzleNone);
              const uint64_t dbl = make_smem_desc(b0 + (uint32_t)bplane + 256 * kk, 128, sbo,
                                                  kSwizzleNone);
              mma_f16(d, dah, dbh, idesc, kk > 0 ? 1u : 0u);
              mma_f16(d, dah, dbl, idesc, 1u);
              mma_f16(d, dal, dbh, idesc, 1u);
            }
          }
          mma_commit(full0 + 8 * b);
        }
      }
      // the issuing lane's decision reaches every producer before the next tile
      if (!group_all(ok, 2, 128)) { ok = false; break; }
    }
    if (pt == 0) {
      // every MMA issued by this thread has completed once this commit lands
      mma_commit(drain);
      const unsigned long long t0 = ks_globaltimer();
      while (!mbar_try_wait(drain, 0u)) {
        if (ks_globaltimer() - t0 > kLimitNs) break;
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    // Thread r holds MMA row r: samples tau0 + 8r + phi of the tile.  Per half
    // h of the phases it reads 4P columns of each channel, splits them and
    // writes the staged rows (plane, phi, r): 4P bf16 (all four channels) as
    // P/2 16-byte stores (48-byte pitch for P = 6: the 8 lanes of a quarter
    // warp hit 8 distinct 16-byte bank groups).
    constexpr int HV = 4 * PP;               // columns of a channel per half
    constexpr int RB = 8 * PP;               // bytes of a staged row (one plane)
    const int r = threadIdx.x;               // TMEM lane = MMA row
    unsigned char* stage = reinterpret_cast<unsigned char*>(sS);
    int j = 0;
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++j) {
      const int b = j & 1;
      const uint32_t use = (uint32_t)(j >> 1);
      const bool ok = mbar_wait_bounded(full0 + 8 * b, use & 1u, err, kLimitNs);
      if (!group_all(ok, 1, kEpiThreads)) break;
      fence_after();
      const int tau0 = (t / n_cg) * kSamples;
      const int c0 = (t % n_cg) * kG;
      const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(b * 256);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        uint32_t v[kG][HV];
#pragma unroll
        for (int g = 0; g < kG; ++g)
#pragma unroll
          for (int i = 0; i < HV / 8; ++i)
            tmem_ld8(trow + (uint32_t)(g * NN + h * HV + 8 * i), &v[g][8 * i]);
        tmem_wait_ld();
        if (h == 1) {
          // the accumulator may be overwritten now
          fence_before();
          mbar_arrive(tfree0 + 8 * b);
        } else {
          // the staging area is free once the last tile's stores have read it
          if (r == 0) bulk_wait_read();
          group_sync(1, kEpiThreads);
        }
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          const int phi = 4 * h + f;
          uint32_t hw[2 * PP], lw[2 * PP];
#pragma unroll
          for (int g = 0; g < kG; ++g)
#pragma unroll
            for (int i = 0; i < PP / 2; ++i) {
              const float a = __uint_as_float(v[g][f * PP + 2 * i]);
              const float c = __uint_as_float(v[g][f * PP + 2 * i + 1]);
              const __nv_bfloat162 hv = __floats2bfloat162_rn(a, c);
              const float2 hf = __bfloat1622float2(hv);
              hw[g * (PP / 2) + i] = bf16x2_bits(hv);
              lw[g * (PP / 2) + i] = bf16x2_bits(__floats2bfloat162_rn(a - hf.x, c - hf.y));
            }
          uint4* dh = reinterpret_cast<uint4*>(stage + ((size_t)(phi * kRows + r)) * RB);
          uint4* dl = reinterpret_cast<uint4*>(stage + ((size_t)((8 + phi) * kRows + r)) * RB);
#pragma unroll
          for (int q = 0; q < PP / 2; ++q) {
            dh[q] = make_uint4(hw[4 * q], hw[4 * q + 1], hw[4 * q + 2], hw[4 * q + 3]);
            dl[q] = make_uint4(lw[4 * q], lw[4 * q + 1], lw[4 * q + 2], lw[4 * q + 3]);
          }
        }
      }
      fence_proxy_async_smem();
      group_sync(1, kEpiThreads);
      if (threadIdx.x == 0) {
        const uint32_t s0 = smem_u32(stage);
        for (int pl = 0; pl < 2; ++pl)
          for (int phi = 0; phi < 8; ++phi)
            tma_store_2d(&maps.m[pl][phi], s0 + (uint32_t)((pl * 8 + phi) * kRows * RB), c0 * PP,
                         tau0 / 8);
        bulk_commit();
      }
    }
    // the stores in flight are complete before the CTA exits
    if (threadIdx.x == 0) bulk_wait_all();
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

template <int PP>
int launch_pp(const float* X, const float* W, int64_t C, int64_t L, int64_t nt, int64_t Q,
              int64_t Lpad, __nv_bfloat16* Yhi, __nv_bfloat16* Ylo, int* err,
              cudaStream_t stream) {
  using namespace ks;
  const int kext = (int)round_up(nt + 7, 16);
  const Smem<PP> lay{kext};
  const size_t smem = lay.total();
  DeviceInfo dev;
  int rc = device_info(&dev);
  if (rc) return rc;
  if (smem > (size_t)dev.smem_optin) return KS_ERR_UNSUPPORTED;
  const int n_cg = (int)(round_up(C, 16) / kG);
  const long long n_tiles = ((Lpad + kSamples - 1) / kSamples) * (long long)n_cg;
  if (n_tiles > 0x7fffffffLL) return fail(KS_ERR_UNSUPPORTED, "temporal: too many tiles");
  static thread_local int attr_device = -1;
  if (attr_device != dev.device) {
    KS_CUDA(cudaFuncSetAttribute(ks_temporal_tc_kernel<PP>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_device = dev.device;
  }
  const int grid = (int)std::min<long long>(n_tiles, dev.sm_count);
  if (grid < 1) return KS_OK;
  static thread_local TemporalMaps maps;
  for (int pl = 0; pl < 2; ++pl)
    for (int phi = 0; phi < 8; ++phi) {
      rc = make_bf16_store_map(&maps.m[pl][phi], (pl ? Ylo : Yhi) + phi * Q, Lpad / 8, Q, 8 * Q,
                               4 * PP, kRows);
      if (rc) return rc;
    }
  ks_temporal_tc_kernel<PP><<<grid, kThreads, smem, stream>>>(X, W, (int)C, (int)L, (int)nt, kext,
                                                              n_cg, (int)n_tiles, maps, err);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

}  // namespace

namespace ks {

int launch_temporal_split_tc(const float* X, const float* W, int64_t C, int64_t L, int64_t P,
                             int64_t nt, int64_t Q, int64_t Lpad, __nv_bfloat16* Yhi,
                             __nv_bfloat16* Ylo, int* err, cudaStream_t stream) {
  if (!err || nt + 7 > kMaxK || Lpad > 0x7fffffffLL - kSamples ||
      (reinterpret_cast<uintptr_t>(Yhi) & 15) || (reinterpret_cast<uintptr_t>(Ylo) & 15) ||
      (Q % 8) || (Lpad % 8))
    return KS_ERR_UNSUPPORTED;
  switch (P) {
    case 2: return launch_pp<2>(X, W, C, L, nt, Q, Lpad, Yhi, Ylo, err, stream);
    case 4: return launch_pp<4>(X, W, C, L, nt, Q, Lpad, Yhi, Ylo, err, stream);
    case 6: return launch_pp<6>(X, W, C, L, nt, Q, Lpad, Yhi, Ylo, err, stream);
    case 8: return launch_pp<8>(X, W, C, L, nt, Q, Lpad, Yhi, Ylo, err, stream);
    default: return KS_ERR_UNSUPPORTED;
  }
}

}  // namespace ks
