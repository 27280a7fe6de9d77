// Preprocessing of a raw int16 batch on the device, as kilosort/io.py:994-1026
// (BinaryFiltered.filter) does it:
//
//   X = raw[:, chan_map] (channels x samples), * -1 when inverting the sign
//   X = X - mean_t(X)                          per channel
//   X = X - median_c(X)                        per sample (common average, lower median)
//   X = highpass(X)                            circular correlation over the batch
//   X = 0 when any |X| >= artifact_threshold   (the whole batch)
//   X = whiten @ X                             (whiten may include the drift matrix)
//
// The high-pass of the reference, real(ifft(fft(X) * conj(fft(h_pad)))) shifted
// by L/2, is the circular correlation X'[c, n] = sum_d h[d] X[c, (n + d + o) mod L]
// with the filter centred at d = 0 and o the offset of its centre from L/2
// after padding or cropping to L (0 for even L); the caller passes the centre
// taps and the index of the centre tap minus o (the Butterworth filtfilt
// response is below 1e-9 of its peak 504 samples out).
//
// Kernels (C = selected channels, L = batch samples):
//   ks_pre_sum_kernel   per-channel sums in double (int16 values: exact)
//   ks_pre_car_kernel   32-sample tiles: centred values into shared memory,
//                       per-sample lower median by one warp: counts in 256
//                       buckets over mean -/+ 4 sd, then an exact rank among the
//                       few values of the median's bucket (a radix select on the
//                       order-preserving integer keys when that bucket is
//                       crowded); coalesced [C][L] rows out
//                       (with a high-pass: the bf16 hi/lo samples of the
//                       circularly padded batch P[c][j] = x[c][(j - h) mod L]
//                       instead, the operand of the tensor-core FIR)
//   fir_tc              with a high-pass: the FIR as a split-BF16 tcgen05
//                       product with the Toeplitz matrix of the taps
//                       (fir_tc.cu); writes f32 rows or the whitening operand,
//                       flags artifacts
//   ks_pre_fir_kernel   without one: the identity in the same output forms
//                       (an FP32 circular FIR, tiles of 128 samples x 16
//                       channels, 8 samples per thread, taps in groups of 8
//                       over a 16-sample register window)
//   whitening           the split-BF16 tcgen05 contraction (gemm_bf16x3)
#include "ks_common.cuh"
#include "project.cuh"

#include <algorithm>
#include <cmath>
#include <cuda_bf16.h>

namespace {

constexpr int kCarTile = 32;          // samples per CAR block
constexpr int kCarThreads = 256;
constexpr int kMaxC = 1024;           // channels (CAR tile in shared memory)
constexpr int kFirT = 128;            // samples per FIR tile
constexpr int kFirC = 16;             // channels per FIR tile
constexpr int kFirThreads = 256;      // 8 samples x 1 channel per thread
constexpr int kMaxTaps = 1023;

__global__ void ks_pre_sum_kernel(const int16_t* __restrict__ raw, int L, long long ldr,
                                  const long long* __restrict__ map, int C, int chunk,
                                  double* __restrict__ sums, int* err) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  const long long m = map ? map[c] : c;
  if (m < 0 || m >= ldr) {
    atomicCAS(err, 0, KS_ERR_ARG);
    return;
  }
  const int t0 = blockIdx.y * chunk, t1 = min(L, t0 + chunk);
  long long s = 0;                    // |int16| * chunk fits easily
  for (int t = t0; t < t1; ++t) s += raw[(long long)t * ldr + m];
  atomicAdd(sums + c, (double)s);
}

__device__ __forceinline__ uint32_t order_key(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_value(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Rank-k value (0-based, ascending) of column s of the tile, by one warp:
// four passes of an 8-bit radix select on the order keys.
__device__ float warp_select(const float* tile, int pitch, int C, int s, int k, int* hist) {
  const int lane = threadIdx.x & 31;
  uint32_t prefix = 0, mask = 0;
#pragma unroll 1
  for (int shift = 24; shift >= 0; shift -= 8) {
#pragma unroll
    for (int b = 0; b < 8; ++b) hist[lane * 8 + b] = 0;
    __syncwarp();
    for (int c = lane; c < C; c += 32) {
      const uint32_t key = order_key(tile[c * pitch + s]);
      if ((key & mask) == prefix) atomicAdd(hist + ((key >> shift) & 255u), 1);
    }
    __syncwarp();
    int cnt[8], local = 0;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      cnt[b] = hist[lane * 8 + b];
      local += cnt[b];
    }
    int incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const int excl = incl - local;
    const unsigned hit = __ballot_sync(0xffffffffu, excl <= k && k < incl);
    const int src = __ffs(hit) - 1;
    int sel = 0, before = 0;
    if (lane == src) {
      int acc = excl;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        if (k < acc + cnt[b]) {
          sel = lane * 8 + b;
          before = acc;
          break;
        }
        acc += cnt[b];
      }
    }
    sel = __shfl_sync(0xffffffffu, sel, src);
    before = __shfl_sync(0xffffffffu, before, src);
    k -= before;
    prefix |= (uint32_t)sel << shift;
    mask |= 255u << shift;
    __syncwarp();
  }
  return key_value(prefix);
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Bucket of v among 256 over [lo, lo + 256 / inv): a non-decreasing function of
// v (a rounded difference, a rounded product by inv > 0, truncation, clamping).
__device__ __forceinline__ int median_bucket(float v, float lo, float inv) {
  const float t = __fmul_rn(__fsub_rn(v, lo), inv);
  return t < 0.f ? 0 : (t >= 255.f ? 255 : (int)t);
}

// Rank-k value (0-based, ascending) of column s of the tile, by one warp.
// The values are counted into 256 buckets over mean -/+ 4 sd of the column
// (outliers clamp to the end buckets); the bucket that holds rank k is found
// from the counts, and since the bucket is a non-decreasing function of the
// value, the rank-k value is the (k - values below the bucket)-th smallest of
// that bucket's values, ranked exactly by comparisons.  Near the median the
// buckets hold a few values each, so the shared-memory counts hardly collide.
// A bucket of more than 32 values, or a zero or non-finite spread, goes to the
// radix select.
__device__ float warp_median(const float* tile, int pitch, int C, int s, int k, int* hist,
                             float* cand, int* ncand) {
  const int lane = threadIdx.x & 31;
  float sum = 0.f, sq = 0.f;
  for (int c = lane; c < C; c += 32) {
    const float v = tile[c * pitch + s];
    sum += v;
    sq = fmaf(v, v, sq);
  }
  sum = warp_sum(sum);
  sq = warp_sum(sq);
  const float mean = sum / (float)C;
  const float sd = sqrtf(fmaxf(sq / (float)C - mean * mean, 0.f));
  const float lo = mean - 4.f * sd;
  const float inv = 32.f / sd;                 // 256 buckets over 8 sd
  if (!(sd > 0.f) || !isfinite(inv) || !isfinite(lo))
    return warp_select(tile, pitch, C, s, k, hist);
#pragma unroll
  for (int b = 0; b < 8; ++b) hist[lane * 8 + b] = 0;
  if (lane == 0) *ncand = 0;
  __syncwarp();
  for (int c = lane; c < C; c += 32)
    atomicAdd(hist + median_bucket(tile[c * pitch + s], lo, inv), 1);
  __syncwarp();
  int cnt[8], local = 0;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    cnt[b] = hist[lane * 8 + b];
    local += cnt[b];
  }
  int incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const int excl = incl - local;
  const unsigned hit = __ballot_sync(0xffffffffu, excl <= k && k < incl);
  const int src = __ffs(hit) - 1;
  int sel = 0, before = 0, m = 0;
  if (lane == src) {
    int acc = excl;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      if (k < acc + cnt[b]) {
        sel = lane * 8 + b;
        before = acc;
        m = cnt[b];
        break;
      }
      acc += cnt[b];
    }
  }
  sel = __shfl_sync(0xffffffffu, sel, src);
  before = __shfl_sync(0xffffffffu, before, src);
  m = __shfl_sync(0xffffffffu, m, src);
  if (m > 32) {
    __syncwarp();
    return warp_select(tile, pitch, C, s, k, hist);
  }
  for (int c = lane; c < C; c += 32) {
    const float v = tile[c * pitch + s];
    if (median_bucket(v, lo, inv) == sel) cand[atomicAdd(ncand, 1)] = v;
  }
  __syncwarp();
  const int kk = k - before;
  const float mine = lane < m ? cand[lane] : 0.f;
  int less = 0, leq = 0;
  for (int j = 0; j < m; ++j) {
    const float o = cand[j];
    less += o < mine ? 1 : 0;
    leq += o <= mine ? 1 : 0;
  }
  const unsigned win = __ballot_sync(0xffffffffu, lane < m && less <= kk && kk < leq);
  const float r = cand[__ffs(win) - 1];
  __syncwarp();
  return r;
}

// Centred (and common-average-referenced) samples: Xc[c][t], t < L; with kPad
// instead the bf16 hi/lo planes of the circularly padded batch
// P[c][j] = x[c][(j - h) mod L], j < cols (sample t at every j = t + h mod L).
template <bool kCar, bool kPad>
__global__ void __launch_bounds__(kCarThreads)
ks_pre_car_kernel(const int16_t* __restrict__ raw, int L, long long ldr,
                  const long long* __restrict__ map, int C, float sign,
                  const double* __restrict__ sums, float* __restrict__ Xc,
                  __nv_bfloat16* __restrict__ Phi, __nv_bfloat16* __restrict__ Plo, int h,
                  long long cols, int* err) {
  extern __shared__ __align__(16) float sm[];
  constexpr int pitch = kCarTile + 1;
  float* tile = sm;                                        // [C][pitch]
  int* hist = reinterpret_cast<int*>(tile + (size_t)C * pitch);   // [8 warps][256]
  float* med = reinterpret_cast<float*>(hist + 8 * 256);   // [kCarTile]
  float* cand = med + kCarTile;                            // [8 warps][32]
  int* ncand = reinterpret_cast<int*>(cand + 8 * 32);      // [8 warps]
  const int t0 = blockIdx.x * kCarTile;
  const int nt = min(kCarTile, L - t0);
  for (int c = threadIdx.x; c < C; c += kCarThreads) {
    const long long m = map ? map[c] : c;
    if (m < 0 || m >= ldr) {
      atomicCAS(err, 0, KS_ERR_ARG);
      for (int s = 0; s < nt; ++s) tile[c * pitch + s] = 0.f;
      continue;
    }
    // the mean of the (sign-inverted) samples: negation commutes with the
    // rounded mean and difference, so this is fl(sign * raw - mean(sign * raw))
    const float mean = sign * (float)(sums[c] / (double)L);
    const int16_t* src = raw + (long long)t0 * ldr + m;
    for (int s = 0; s < nt; ++s)
      tile[c * pitch + s] = __fsub_rn(sign * (float)src[(long long)s * ldr], mean);
  }
  __syncthreads();
  if (kCar) {
    const int warp = threadIdx.x >> 5;
    for (int s = warp; s < nt; s += kCarThreads / 32) {
      const float m = warp_median(tile, pitch, C, s, (C - 1) / 2, hist + warp * 256,
                                  cand + warp * 32, ncand + warp);
      if ((threadIdx.x & 31) == 0) med[s] = m;
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < C * kCarTile; e += kCarThreads) {
    const int c = e / kCarTile, s = e - c * kCarTile;
    if (s < nt) {
      const float v = tile[c * pitch + s];
      const float y = kCar ? __fsub_rn(v, med[s]) : v;
      if (kPad) {
        const __nv_bfloat16 hv = __float2bfloat16_rn(y);
        const __nv_bfloat16 lv = __float2bfloat16_rn(y - __bfloat162float(hv));
        // t0 + s < L and h < L: the first position is one subtraction away
        long long j = t0 + s + h;
        if (j >= L) j -= L;
        for (; j < cols; j += L) {
          Phi[(size_t)c * cols + j] = hv;
          Plo[(size_t)c * cols + j] = lv;
        }
      } else {
        Xc[(size_t)c * L + t0 + s] = y;
      }
    }
  }
}

__host__ __device__ inline int fir_taps_rounded(int ntaps) { return (ntaps + 7) & ~7; }
__host__ __device__ inline int fir_window(int ntaps) {
  return (kFirT + fir_taps_rounded(ntaps) + 8 + 3) & ~3;
}

// Circular FIR: y[c, n] = sum_j taps[j] * Xc[c, (n + j - h) mod L], h = the
// centre tap, taps accumulated in increasing j (taps == nullptr: the identity).  kSplit:
// write the bf16 hi/lo operand [rows][Cq] (row = sample, zero past L and C);
// otherwise f32 rows X[c][ldx].  With check, |y| >= thr flags an artifact.
template <bool kSplit>
__global__ void __launch_bounds__(kFirThreads)
ks_pre_fir_kernel(const float* __restrict__ Xc, int C, int L, const float* __restrict__ taps,
                  int ntaps, int h, int tiles_t, bool check, float thr, float* __restrict__ X,
                  long long ldx,
                  __nv_bfloat16* __restrict__ Yhi, __nv_bfloat16* __restrict__ Ylo, int Cq,
                  int rows, int* artifact) {
  extern __shared__ __align__(16) float sm[];
  const int ntr = fir_taps_rounded(ntaps);
  const int xw = fir_window(ntaps);
  float* sT = sm;                          // taps, zero past ntaps
  float* sX = sT + ntr;                    // [kFirC][xw]
  const int tt = blockIdx.x % tiles_t, cg = blockIdx.x / tiles_t;
  const int t0 = tt * kFirT, c0 = cg * kFirC;
  // no filter: one unit tap
  for (int i = threadIdx.x; i < ntr; i += kFirThreads)
    sT[i] = i < ntaps ? (taps ? taps[i] : 1.f) : 0.f;
  for (int e = threadIdx.x; e < kFirC * xw; e += kFirThreads) {
    const int cl = e / xw, u = e - cl * xw;
    const int c = c0 + cl;
    int t = t0 - h + u;
    t %= L;
    if (t < 0) t += L;
    sX[e] = c < C ? Xc[(size_t)c * L + t] : 0.f;
  }
  __syncthreads();
  constexpr int kS = 8;
  const int cl = threadIdx.x & (kFirC - 1);
  const int g = threadIdx.x / kFirC;      // 16 groups of 8 samples
  const float4* xs4 = reinterpret_cast<const float4*>(sX + cl * xw + g * kS);
  const float4* t4 = reinterpret_cast<const float4*>(sT);
  float acc[kS];
#pragma unroll
  for (int i = 0; i < kS; ++i) acc[i] = 0.f;
  float win[2 * kS];
  {
    const float4 a = xs4[0], b = xs4[1];
    win[0] = a.x; win[1] = a.y; win[2] = a.z; win[3] = a.w;
    win[4] = b.x; win[5] = b.y; win[6] = b.z; win[7] = b.w;
  }
  for (int j0 = 0; j0 < ntr; j0 += 8) {
    {
      const float4 a = xs4[(j0 + kS) / 4], b = xs4[(j0 + kS) / 4 + 1];
      win[8] = a.x; win[9] = a.y; win[10] = a.z; win[11] = a.w;
      win[12] = b.x; win[13] = b.y; win[14] = b.z; win[15] = b.w;
    }
    const float4 ta = t4[j0 / 4], tb = t4[j0 / 4 + 1];
    const float w[8] = {ta.x, ta.y, ta.z, ta.w, tb.x, tb.y, tb.z, tb.w};
#pragma unroll
    for (int jj = 0; jj < 8; ++jj)
#pragma unroll
      for (int i = 0; i < kS; ++i) acc[i] = fmaf(w[jj], win[i + jj], acc[i]);
#pragma unroll
    for (int i = 0; i < kS; ++i) win[i] = win[i + 8];
  }
  const int c = c0 + cl;
  const int n0 = t0 + g * kS;
  bool art = false;
#pragma unroll
  for (int i = 0; i < kS; ++i)
    if (check && c < C && n0 + i < L && fabsf(acc[i]) >= thr) art = true;
  if (art) atomicOr(artifact, 1);
  if (!kSplit) {
    if (c < C) {
#pragma unroll
      for (int i = 0; i < kS; ++i)
        if (n0 + i < L) X[(size_t)c * ldx + n0 + i] = acc[i];
    }
    return;
  }
  // bf16 hi/lo operand: stage the tile as [sample][channel] and write 32-byte
  // rows (16 channels) per sample and plane
  __syncthreads();                         // the window is no longer read
  __nv_bfloat16* st = reinterpret_cast<__nv_bfloat16*>(sX);   // [2][kFirT][kFirC]
#pragma unroll
  for (int i = 0; i < kS; ++i) {
    const float v = c < C && n0 + i < L ? acc[i] : 0.f;
    const __nv_bfloat16 hv = __float2bfloat16_rn(v);
    st[(g * kS + i) * kFirC + cl] = hv;
    st[kFirT * kFirC + (g * kS + i) * kFirC + cl] = __float2bfloat16_rn(v - __bfloat162float(hv));
  }
  __syncthreads();
  // 2 planes x 128 samples x 2 chunks of 16 bytes
  for (int e = threadIdx.x; e < 2 * kFirT * 2; e += kFirThreads) {
    const int pl = e / (2 * kFirT), r = (e / 2) % kFirT, q = e & 1;
    const int row = t0 + r;
    if (row < rows && c0 + 8 * q < Cq) {
      const uint4 v = reinterpret_cast<const uint4*>(st + pl * kFirT * kFirC + r * kFirC)[q];
      __nv_bfloat16* dst = (pl ? Ylo : Yhi) + (size_t)row * Cq + c0 + 8 * q;
      *reinterpret_cast<uint4*>(dst) = v;
    }
  }
}

// The whole batch is zeroed when the artifact flag is set.
__global__ void ks_pre_zero_kernel(float* X, int C, int L, long long ldx, const int* artifact) {
  if (*reinterpret_cast<const volatile int*>(artifact) == 0) return;
  const long long n = (long long)C * L;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const long long c = e / L;
    X[c * ldx + (e - c * L)] = 0.f;
  }
}

struct PreLayout {
  int64_t Cq, Cpad, Tpad, pcols;
  size_t flags, sums, xc, phi, plo, thi, tlo, whi, wlo, yhi, ylo, bytes;
};

PreLayout pre_layout(int64_t L, int64_t C, bool whiten) {
  PreLayout p{};
  p.Cq = ks::round_up(C, 64);
  p.Cpad = ks::round_up(C, 128);
  p.Tpad = ks::round_up(L, 256);
  // the padded FIR operand for the most taps and the longest output
  p.pcols = ks::fir_tc_cols(whiten ? p.Tpad : L, kMaxTaps);
  size_t o = 0;
  auto take = [&](size_t b) {
    const size_t at = o;
    o = ks::align256(o + b);
    return at;
  };
  p.flags = take(256);                     // [0] device error, [1] artifact
  p.sums = take(sizeof(double) * (size_t)C);
  p.xc = take(sizeof(float) * (size_t)C * L);
  p.phi = take(2 * (size_t)C * p.pcols);
  p.plo = take(2 * (size_t)C * p.pcols);
  p.thi = take(ks::fir_tc_toeplitz_bytes(kMaxTaps) / 2);
  p.tlo = take(ks::fir_tc_toeplitz_bytes(kMaxTaps) / 2);
  if (whiten) {
    p.whi = take(2 * (size_t)p.Cpad * p.Cq);
    p.wlo = take(2 * (size_t)p.Cpad * p.Cq);
    p.yhi = take(2 * (size_t)p.Tpad * p.Cq);
    p.ylo = take(2 * (size_t)p.Tpad * p.Cq);
  }
  p.bytes = o;
  return p;
}

}  // namespace

extern "C" KS_API size_t ks_preprocess_workspace_size(int64_t L, int64_t C, int whiten) {
  if (L < 1 || C < 1) return 0;
  return pre_layout(L, C, whiten != 0).bytes;
}

extern "C" KS_API int ks_preprocess_int16(const int16_t* raw, int64_t L, int64_t ld_raw,
                                          const int64_t* chan_map, int64_t C, int invert_sign,
                                          int do_car, const float* hp_taps, int64_t ntaps,
                                          int64_t hp_centre, float artifact_threshold, const float* whiten,
                                          float* X, int64_t ldx, int* flags, void* workspace,
                                          size_t workspace_bytes, void* stream) {
  using namespace ks;
  if (!raw || !X || !flags) return fail(KS_ERR_ARG, "ks_preprocess_int16: null pointer");
  if (L < 1 || C < 1 || ld_raw < 1 || ldx < L || (!chan_map && C > ld_raw))
    return fail(KS_ERR_ARG, "ks_preprocess_int16: need L, C >= 1, ldx >= L, C <= ld_raw without a map");
  if (C > kMaxC) return fail(KS_ERR_UNSUPPORTED, "ks_preprocess_int16: more than 1024 channels");
  if (L > 0x7fffffffLL / 2) return fail(KS_ERR_UNSUPPORTED, "ks_preprocess_int16: batch too long");
  if (hp_taps && (ntaps < 1 || ntaps > kMaxTaps || ntaps > L || hp_centre < 0 || hp_centre >= L))
    return fail(KS_ERR_ARG, "ks_preprocess_int16: need 1 <= ntaps <= min(1023, L), 0 <= centre < L");
  if (!(artifact_threshold > 0.f)) return fail(KS_ERR_ARG, "ks_preprocess_int16: threshold must be > 0");
  const PreLayout p = pre_layout(L, C, whiten != nullptr);
  if (!workspace || workspace_bytes < p.bytes)
    return fail(KS_ERR_WORKSPACE, "ks_preprocess_int16: workspace too small");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  char* base = static_cast<char*>(workspace);
  int* err = reinterpret_cast<int*>(base + p.flags);
  int* art = err + 1;
  double* sums = reinterpret_cast<double*>(base + p.sums);
  float* Xc = reinterpret_cast<float*>(base + p.xc);
  KS_CUDA(cudaMemsetAsync(err, 0, 2 * sizeof(int), s));
  KS_CUDA(cudaMemsetAsync(sums, 0, sizeof(double) * C, s));
  const long long* map = reinterpret_cast<const long long*>(chan_map);

  // 1. per-channel sums
  {
    const int chunk = 512;
    const dim3 grid((unsigned)((C + 255) / 256), (unsigned)((L + chunk - 1) / chunk));
    ks_pre_sum_kernel<<<grid, 256, 0, s>>>(raw, (int)L, ld_raw, map, (int)C, chunk, sums, err);
    KS_CUDA(cudaGetLastError());
  }
  // 2. centring and common average reference (with a high-pass: into the
  //    padded bf16 operand of the tensor-core FIR)
  const bool split = whiten != nullptr;
  const int64_t rows = split ? p.Tpad : L;
  const int64_t pcols = hp_taps ? ks::fir_tc_cols(rows, (int)ntaps) : 0;
  __nv_bfloat16* phi = reinterpret_cast<__nv_bfloat16*>(base + p.phi);
  __nv_bfloat16* plo = reinterpret_cast<__nv_bfloat16*>(base + p.plo);
  {
    const size_t smem = sizeof(float) * (size_t)C * (kCarTile + 1) + sizeof(int) * 8 * 256 +
                        sizeof(float) * kCarTile + sizeof(float) * 8 * 32 + sizeof(int) * 8;
    const unsigned grid = (unsigned)((L + kCarTile - 1) / kCarTile);
    const float sign = invert_sign ? -1.f : 1.f;
    auto run = [&](auto kernel) -> int {
      KS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      kernel<<<grid, kCarThreads, smem, s>>>(raw, (int)L, ld_raw, map, (int)C, sign, sums, Xc,
                                             phi, plo, (int)hp_centre, (long long)pcols, err);
      KS_CUDA(cudaGetLastError());
      return KS_OK;
    };
    int rc;
    if (hp_taps)
      rc = do_car ? run(ks_pre_car_kernel<true, true>) : run(ks_pre_car_kernel<false, true>);
    else
      rc = do_car ? run(ks_pre_car_kernel<true, false>) : run(ks_pre_car_kernel<false, false>);
    if (rc) return rc;
  }
  // 3. high-pass (the identity when there is no filter), artifact flag
  const bool check = artifact_threshold < INFINITY;
  {
    __nv_bfloat16* yhi = split ? reinterpret_cast<__nv_bfloat16*>(base + p.yhi) : nullptr;
    __nv_bfloat16* ylo = split ? reinterpret_cast<__nv_bfloat16*>(base + p.ylo) : nullptr;
    if (hp_taps) {
      int rc = ks::fir_tc(hp_taps, (int)ntaps, phi, plo, C, L, pcols, rows,
                          reinterpret_cast<__nv_bfloat16*>(base + p.thi),
                          reinterpret_cast<__nv_bfloat16*>(base + p.tlo), check,
                          artifact_threshold, X, ldx, yhi, ylo, p.Cq, art, err, s);
      if (rc) return rc;
    } else {
      // the split operand is written whole (Tpad rows, zeros past L)
      const int nt = 1, centre = 0;
      const int tiles_t = (int)((rows + kFirT - 1) / kFirT);
      const int cgroups = (int)((split ? p.Cq : C) + kFirC - 1) / kFirC;
      const long long blocks = (long long)tiles_t * cgroups;
      if (blocks > 0x7fffffffLL) return fail(KS_ERR_UNSUPPORTED, "ks_preprocess_int16: too many tiles");
      const size_t smem = sizeof(float) * ((size_t)fir_taps_rounded(nt) + (size_t)kFirC * fir_window(nt));
      if (split) {
        KS_CUDA(cudaFuncSetAttribute(ks_pre_fir_kernel<true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        ks_pre_fir_kernel<true><<<(unsigned)blocks, kFirThreads, smem, s>>>(
            Xc, (int)C, (int)L, nullptr, nt, centre, tiles_t, check, artifact_threshold, nullptr,
            0, yhi, ylo, (int)p.Cq, (int)p.Tpad, art);
      } else {
        KS_CUDA(cudaFuncSetAttribute(ks_pre_fir_kernel<false>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        ks_pre_fir_kernel<false><<<(unsigned)blocks, kFirThreads, smem, s>>>(
            Xc, (int)C, (int)L, nullptr, nt, centre, tiles_t, check, artifact_threshold, X, ldx,
            nullptr, nullptr, (int)p.Cq, 0, art);
      }
      KS_CUDA(cudaGetLastError());
    }
    // 4. whitening on the tensor cores
    if (split) {
      __nv_bfloat16* whi = reinterpret_cast<__nv_bfloat16*>(base + p.whi);
      __nv_bfloat16* wlo = reinterpret_cast<__nv_bfloat16*>(base + p.wlo);
      int rc = launch_matrix_split(whiten, C, 1.f, p.Cpad, p.Cq, whi, wlo, s);
      if (rc) return rc;
      // the FIR tiles cover channels up to Cq and rows up to Tpad (zeros)
      rc = gemm_bf16x3(whi, wlo, yhi, ylo, X, C, L, p.Cq, p.Cpad, p.Tpad, ldx, false, err, s);
      if (rc) return rc;
    }
  }
  // 5. artifact: the whole batch becomes zeros
  {
    const int blocks = (int)std::min<long long>(4096, ((long long)C * L + 255) / 256);
    ks_pre_zero_kernel<<<blocks, 256, 0, s>>>(X, (int)C, (int)L, ldx, art);
    KS_CUDA(cudaGetLastError());
  }
  KS_CUDA(cudaMemcpyAsync(flags, err, 2 * sizeof(int), cudaMemcpyDeviceToDevice, s));
  return KS_OK;
}
