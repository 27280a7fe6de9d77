// Score projection B[k, tau] = sum_{p,c} U[k,p,c] * Y[c,p,tau],
// Y[c,p,tau] = sum_t W[p,t] X[c, tau - nt/2 + t] (zero padding),
// i.e. kilosort/template_matching.py:180-181 (conv1d then einsum).
//
// Layout in HBM (per call, carved from the caller's workspace)
//   Yt  [Lpad, Q] temporal projection, q = c*P + p contiguous ("K-major" for
//       the contraction), Lpad = roundup(L, 128), Q = roundup(roundup(C,16)*P, 64)
//       float32 (FP32 form) or two bf16 planes hi/lo (split form)
//   Uq  [Kpad, Q] templates in the same q order, zero padded; float32 or bf16 hi/lo
//   B   [K, ldb] float32 output
//
// Kernels
//   ks_prep_templates  nm[k] and Uq (both precisions)
//   ks_temporal        X -> Yt: each thread owns 8 consecutive samples of one
//                      channel and all P components (8*P FMA per tap, one
//                      shared-memory load of X per tap); output staged in
//                      shared memory and written as contiguous rows
//   ks_sgemm_tn        FP32 SIMT contraction, 128x128x16 tiles, 8x8 per thread,
//                      register double buffering; tile order puts the template
//                      tiles of one time tile next to each other so each Yt tile
//                      is read from HBM once
#include "ks_common.cuh"
#include "project.cuh"

#include <cuda_bf16.h>

namespace ks {

// ------------------------------------------------------------------ prep
__global__ void ks_template_energy_kernel(const float* __restrict__ U, int K,
                                          int P, int C, float* __restrict__ nm) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= K) return;
  const float* u = U + (long long)warp * P * C;
  float tot = 0.f;
  for (int p = 0; p < P; ++p) {
    float s = 0.f;
    for (int c = lane; c < C; c += 32) s = __fadd_rn(s, __fmul_rn(u[p * C + c], u[p * C + c]));
    for (int o = 16; o; o >>= 1) s = __fadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
    tot = __fadd_rn(tot, s);
  }
  if (lane == 0) nm[warp] = tot;
}

__global__ void ks_reorder_templates_kernel(const float* __restrict__ U, int K,
                                            int P, int C, int Kpad, int Q,
                                            float* __restrict__ Uf,
                                            __nv_bfloat16* __restrict__ Uhi,
                                            __nv_bfloat16* __restrict__ Ulo) {
  const long long n = (long long)Kpad * Q;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(e / Q);
    const int q = (int)(e - (long long)k * Q);
    const int c = q / P, p = q - (q / P) * P;
    float v = 0.f;
    if (k < K && c < C) v = U[((long long)k * P + p) * C + c];
    if (Uf) Uf[e] = v;
    if (Uhi) {
      const __nv_bfloat16 h = __float2bfloat16_rn(v);
      Uhi[e] = h;
      Ulo[e] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
  }
}

// ------------------------------------------------------------------ temporal
constexpr int kTT = 128;   // samples per tile
constexpr int kCG = 16;    // channels per tile
constexpr int kTemporalThreads = 256;
constexpr int kPMax = 8;

// X window per channel: samples tau0 - nt/2 .. tau0 + kTT + nt + 7, padded so
// every row starts on a 16-byte boundary.
__host__ __device__ inline int temporal_xw(int nt) { return (kTT + nt + 8 + 3) & ~3; }

// Asynchronous 4-byte global -> shared copy; src_bytes 0 fills zeros.
__device__ __forceinline__ void cp_async4(float* dst, const float* src, int src_bytes) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() {
  asm volatile("cp.async.wait_group 1;" ::: "memory");
}

// Persistent: block b takes tiles b, b + grid, ... (a tile is kTT samples x
// kCG channels).  The X window of the next tile is copied (cp.async) while the
// current one is computed.  Each thread owns 8 consecutive samples of one
// channel and all PP components; taps run in groups of 8 over a 16-sample
// register window (every operand index a compile-time constant) and each
// tap's components come from the transposed basis Wt[t][8] as two broadcast
// 16-byte loads.  acc[i][p] accumulates taps t = 0 .. nt-1 in increasing
// order.  Results go straight from registers to Y: the PP values of one
// (sample, channel) are contiguous there.
template <int PP>
__global__ void __launch_bounds__(kTemporalThreads)
ks_temporal_kernel(const float* __restrict__ X, const float* __restrict__ W,
                   int C, int L, int nt, int Q, int tiles_t, int n_tiles,
                   float* __restrict__ Yf, __nv_bfloat16* __restrict__ Yhi,
                   __nv_bfloat16* __restrict__ Ylo, float* __restrict__ YT, long long ldyt) {
  extern __shared__ __align__(16) float sm[];
  constexpr int kS = kTT / (kTemporalThreads / kCG);   // samples per thread (8)
  const int xw = temporal_xw(nt);
  const int ntr = (nt + 7) & ~7;            // taps rounded to the group of 8
  float* sW = sm;                           // Wt[ntr][8] (zero past nt and PP)
  float* sX[2] = {sW + 8 * ntr, sW + 8 * ntr + kCG * xw};   // [kCG][xw] each
  const int half = nt / 2;
  for (int i = threadIdx.x; i < 8 * ntr; i += kTemporalThreads) {
    const int t = i >> 3, p = i & 7;
    sW[i] = (p < PP && t < nt) ? W[p * nt + t] : 0.f;
  }
  auto fetch = [&](int tile, float* dst) {
    const int tau0 = (tile % tiles_t) * kTT, cg0 = (tile / tiles_t) * kCG;
    for (int cl = 0; cl < kCG; ++cl) {
      const int c = cg0 + cl;
      const float* xrow = X + (long long)(c < C ? c : 0) * L;
      for (int u = threadIdx.x; u < xw; u += kTemporalThreads) {
        const int t = tau0 - half + u;
        const bool ok = c < C && t >= 0 && t < L;
        cp_async4(dst + cl * xw + u, ok ? xrow + t : X, ok ? 4 : 0);
      }
    }
    cp_async_commit();
  };
  const int cl = threadIdx.x & (kCG - 1);
  const int g = threadIdx.x / kCG;          // groups of kS samples
  int buf = 0;
  if (blockIdx.x < n_tiles) fetch(blockIdx.x, sX[0]);
  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int next = tile + gridDim.x;
    if (next < n_tiles) fetch(next, sX[buf ^ 1]);
    else cp_async_commit();                 // keep the group count in step
    cp_async_wait_prev();                   // this tile's window has landed
    __syncthreads();
    const int tau0 = (tile % tiles_t) * kTT, cg0 = (tile / tiles_t) * kCG;
    const float4* xs4 = reinterpret_cast<const float4*>(sX[buf] + cl * xw + g * kS);
    float acc[kS][PP];
#pragma unroll
    for (int i = 0; i < kS; ++i)
#pragma unroll
      for (int p = 0; p < PP; ++p) acc[i][p] = 0.f;
    float win[kS + 8];
#pragma unroll
    for (int k = 0; k < kS / 4; ++k) {
      const float4 a = xs4[k];
      win[4 * k] = a.x; win[4 * k + 1] = a.y; win[4 * k + 2] = a.z; win[4 * k + 3] = a.w;
    }
    const float4* w4 = reinterpret_cast<const float4*>(sW);
    for (int t0 = 0; t0 < nt; t0 += 8) {
      {
        const float4 a = xs4[(t0 + kS) / 4], b = xs4[(t0 + kS) / 4 + 1];
        win[kS + 0] = a.x; win[kS + 1] = a.y; win[kS + 2] = a.z; win[kS + 3] = a.w;
        win[kS + 4] = b.x; win[kS + 5] = b.y; win[kS + 6] = b.z; win[kS + 7] = b.w;
      }
#pragma unroll
      for (int tt = 0; tt < 8; ++tt) {
        if (t0 + tt < nt) {
          const float4 wa = w4[2 * (t0 + tt)], wb = w4[2 * (t0 + tt) + 1];
          const float w[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
#pragma unroll
          for (int i = 0; i < kS; ++i)
#pragma unroll
            for (int p = 0; p < PP; ++p) acc[i][p] = fmaf(w[p], win[i + tt], acc[i][p]);
        }
      }
#pragma unroll
      for (int i = 0; i < kS; ++i) win[i] = win[i + 8];
    }
    // the window is no longer read: the next fetch may overwrite this buffer
    __syncthreads();
    const long long q0 = (long long)(cg0 + cl) * PP;
    if (YT) {
      // rows (channel, component), samples contiguous: 8 samples per store pair
      if (cg0 + cl < C) {
#pragma unroll
        for (int p = 0; p < PP; ++p) {
          float4* dst = reinterpret_cast<float4*>(YT + (q0 + p) * ldyt + tau0 + g * kS);
          dst[0] = make_float4(acc[0][p], acc[1][p], acc[2][p], acc[3][p]);
          dst[1] = make_float4(acc[4][p], acc[5][p], acc[6][p], acc[7][p]);
        }
      }
      buf ^= 1;
      continue;
    }
#pragma unroll
    for (int i = 0; i < kS; ++i) {
      const long long o = (long long)(tau0 + g * kS + i) * Q + q0;
      // pairs of components as one 8-byte (f32) or 4-byte (bf16) store: with
      // PP even, o + p is even for even p
      if (Yf) {
#pragma unroll
        for (int p = 0; p < PP; p += 2) {
          if (PP % 2 == 0)
            *reinterpret_cast<float2*>(Yf + o + p) = make_float2(acc[i][p], acc[i][p + 1]);
          else {
            Yf[o + p] = acc[i][p];
            if (p + 1 < PP) Yf[o + p + 1] = acc[i][p + 1];
          }
        }
      }
      if (Yhi) {
#pragma unroll
        for (int p = 0; p < PP; p += 2) {
          const float v0 = acc[i][p], v1 = p + 1 < PP ? acc[i][p + 1] : 0.f;
          const __nv_bfloat162 h = __floats2bfloat162_rn(v0, v1);
          const float2 hf = __bfloat1622float2(h);
          const __nv_bfloat162 l = __floats2bfloat162_rn(v0 - hf.x, v1 - hf.y);
          if (PP % 2 == 0) {
            *reinterpret_cast<__nv_bfloat162*>(Yhi + o + p) = h;
            *reinterpret_cast<__nv_bfloat162*>(Ylo + o + p) = l;
          } else {
            Yhi[o + p] = h.x;
            Ylo[o + p] = l.x;
            if (p + 1 < PP) {
              Yhi[o + p + 1] = h.y;
              Ylo[o + p + 1] = l.y;
            }
          }
        }
      }
    }
    buf ^= 1;
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}

size_t temporal_smem(int nt, int P) {
  (void)P;
  const int ntr = (nt + 7) & ~7;
  return sizeof(float) * (8 * (size_t)ntr + 2 * (size_t)kCG * temporal_xw(nt));
}

// ------------------------------------------------------------------ FP32 GEMM
constexpr int kBM = 128, kBN = 128, kBK = 16;

// C[m, n] = sum_q A[m, q] * Bt[n, q]; A is [>= tiles_m*128, Kd], Bt is
// [>= tiles_n*128, Kd] (both zero padded), Kd % 16 == 0.  Stores m < M, n < N,
// row-major with leading dimension ldc, or (kTiled) in 32-column blocks
// C[((n/32)*M + m)*32 + n%32].
template <bool kTiled>
__global__ void __launch_bounds__(256, 2)
ks_sgemm_tn_kernel(const float* __restrict__ A, const float* __restrict__ Bt,
                   float* __restrict__ Cm, int M, int N, int Kd, long long ldc,
                   int tiles_m) {
  __shared__ __align__(16) float As[2][kBK][kBM + 4];
  __shared__ __align__(16) float Bs[2][kBK][kBN + 4];
  const int tid = threadIdx.x;
  const int tm = blockIdx.x % tiles_m;
  const int tn = blockIdx.x / tiles_m;
  const long long m0 = (long long)tm * kBM, n0 = (long long)tn * kBN;
  const int tx = tid & 15, ty = tid >> 4;
  // loader mapping: two float4 per operand per thread
  int lrow[2], lc4[2];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int idx = tid + i * 256;
    lrow[i] = idx >> 2;
    lc4[i] = idx & 3;
  }
  float4 ra[2], rb[2];
  auto gload = [&](int k0) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      ra[i] = *reinterpret_cast<const float4*>(A + (m0 + lrow[i]) * Kd + k0 + lc4[i] * 4);
      rb[i] = *reinterpret_cast<const float4*>(Bt + (n0 + lrow[i]) * Kd + k0 + lc4[i] * 4);
    }
  };
  auto sstore = [&](int buf) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int kk = lc4[i] * 4;
      As[buf][kk + 0][lrow[i]] = ra[i].x;
      As[buf][kk + 1][lrow[i]] = ra[i].y;
      As[buf][kk + 2][lrow[i]] = ra[i].z;
      As[buf][kk + 3][lrow[i]] = ra[i].w;
      Bs[buf][kk + 0][lrow[i]] = rb[i].x;
      Bs[buf][kk + 1][lrow[i]] = rb[i].y;
      Bs[buf][kk + 2][lrow[i]] = rb[i].z;
      Bs[buf][kk + 3][lrow[i]] = rb[i].w;
    }
  };
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

  gload(0);
  sstore(0);
  __syncthreads();
  const int nk = Kd / kBK;
  for (int kt = 0; kt < nk; ++kt) {
    const int buf = kt & 1;
    if (kt + 1 < nk) gload((kt + 1) * kBK);
#pragma unroll
    for (int kk = 0; kk < kBK; ++kk) {
      const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 4]);
      const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][kk][64 + ty * 4]);
      const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][kk][tx * 4]);
      const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][kk][64 + tx * 4]);
      const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
    if (kt + 1 < nk) sstore(buf ^ 1);
    __syncthreads();
  }
  // the tiled layout's last block is written whole: columns past N get zeros
  const long long nw = kTiled ? (((long long)N + 31) & ~31LL) : N;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const long long m = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
    if (m >= M) continue;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const long long n = n0 + h * 64 + tx * 4;
      float* dst = kTiled ? Cm + (((n >> 5) * M + m) << 5) + (n & 31) : Cm + m * ldc + n;
      float v[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) v[e] = n + e < N ? acc[i][h * 4 + e] : 0.f;
      if (n + 3 < nw && ((reinterpret_cast<uintptr_t>(dst) & 15) == 0)) {
        *reinterpret_cast<float4*>(dst) = make_float4(v[0], v[1], v[2], v[3]);
      } else {
        for (int e = 0; e < 4; ++e)
          if (n + e < nw) dst[e] = v[e];
      }
    }
  }
}

int sgemm_tn(const float* A, const float* Bt, float* Cm, int64_t M, int64_t N,
             int64_t Kd, int64_t ldc, cudaStream_t stream, bool tiled) {
  if (Kd % kBK) return fail(KS_ERR_ARG, "sgemm_tn: Kd must be a multiple of 16");
  const int tiles_m = (int)((M + kBM - 1) / kBM);
  const int tiles_n = (int)((N + kBN - 1) / kBN);
  const long long nblocks = (long long)tiles_m * tiles_n;
  if (nblocks > 0x7fffffffLL) return fail(KS_ERR_UNSUPPORTED, "sgemm_tn: too many tiles");
  if (tiled)
    ks_sgemm_tn_kernel<true><<<(unsigned)nblocks, 256, 0, stream>>>(A, Bt, Cm, (int)M, (int)N,
                                                                  (int)Kd, ldc, tiles_m);
  else
    ks_sgemm_tn_kernel<false><<<(unsigned)nblocks, 256, 0, stream>>>(A, Bt, Cm, (int)M, (int)N,
                                                                   (int)Kd, ldc, tiles_m);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

// ------------------------------------------------------------------ driver
ProjLayout proj_layout(int64_t C, int64_t L, int64_t K, int64_t P, int precision) {
  ProjLayout l;
  l.Q = round_up(round_up(C, kCG) * P, 64);
  l.Lpad = round_up(L, 128);
  l.Kpad = round_up(K, 128);
  Carve cv(nullptr);
  cv.take<int>(64);   // error word
  if (precision == KS_PROJ_FP32) {
    cv.take<float>((size_t)l.Kpad * l.Q);
    cv.take<float>((size_t)l.Lpad * l.Q);
  } else {
    cv.take<__nv_bfloat16>((size_t)l.Kpad * l.Q * 2);
    cv.take<__nv_bfloat16>((size_t)l.Lpad * l.Q * 2);
  }
  l.bytes = cv.used;
  return l;
}

int launch_template_energy(const float* U, int64_t K, int64_t P, int64_t C,
                           float* nm, cudaStream_t stream) {
  if (!U || !nm || K < 1 || P < 1 || C < 1) return fail(KS_ERR_ARG, "template_energy: bad args");
  const int threads = 256;
  const long long blocks = (K * 32 + threads - 1) / threads;
  ks_template_energy_kernel<<<(unsigned)blocks, threads, 0, stream>>>(U, (int)K, (int)P, (int)C, nm);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

int launch_reorder_templates(const float* U, int64_t K, int64_t P, int64_t C, int64_t Kpad,
                             int64_t Q, float* Uf, __nv_bfloat16* Uhi, __nv_bfloat16* Ulo,
                             cudaStream_t stream) {
  const int blocks = (int)std::min<int64_t>(4096, (Kpad * Q + 255) / 256);
  ks_reorder_templates_kernel<<<blocks, 256, 0, stream>>>(U, (int)K, (int)P, (int)C, (int)Kpad,
                                                          (int)Q, Uf, Uhi, Ulo);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

static int launch_temporal_simt(const float* X, const float* W, int64_t C, int64_t L,
                                int64_t P, int64_t nt, int64_t Q, int64_t Lpad, float* Yf,
                                __nv_bfloat16* Yhi, __nv_bfloat16* Ylo, float* YT,
                                int64_t ldyt, cudaStream_t stream) {
  const size_t smem = temporal_smem((int)nt, (int)P);
  const int tiles_t = (int)(Lpad / kTT);
  const long long n_tiles = (long long)tiles_t * ((C + kCG - 1) / kCG);
  if (n_tiles > 0x7fffffffLL) return fail(KS_ERR_UNSUPPORTED, "project: too many temporal tiles");
  DeviceInfo dev;
  int drc = device_info(&dev);
  if (drc) return drc;
  // persistent: as many blocks as are resident at once
  int occ = 0;
#define KS_TEMPORAL_CASE(PPV)                                                              \
  case PPV: {                                                                              \
    KS_CUDA(cudaFuncSetAttribute(ks_temporal_kernel<PPV>,                                  \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    KS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ks_temporal_kernel<PPV>,   \
                                                          kTemporalThreads, smem));        \
    const unsigned grid =                                                                  \
        (unsigned)std::min<long long>(n_tiles, (long long)std::max(occ, 1) * dev.sm_count); \
    ks_temporal_kernel<PPV><<<grid, kTemporalThreads, smem, stream>>>(                     \
        X, W, (int)C, (int)L, (int)nt,                                                     \
                                                         (int)Q, tiles_t, (int)n_tiles,    \
                                                         Yf, Yhi, Ylo, YT, ldyt);          \
    break;                                                                                 \
  }
  switch (P) {
    KS_TEMPORAL_CASE(1)
    KS_TEMPORAL_CASE(2)
    KS_TEMPORAL_CASE(3)
    KS_TEMPORAL_CASE(4)
    KS_TEMPORAL_CASE(5)
    KS_TEMPORAL_CASE(6)
    KS_TEMPORAL_CASE(7)
    KS_TEMPORAL_CASE(8)
    default:
      return fail(KS_ERR_UNSUPPORTED, "project: n_pcs must be 1..8");
  }
#undef KS_TEMPORAL_CASE
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

int launch_temporal_rows(const float* X, const float* W, int64_t C, int64_t L, int64_t P,
                         int64_t nt, int64_t Lpad, float* YT, int64_t ldyt,
                         cudaStream_t stream) {
  if (Lpad % kTT || ldyt < Lpad || ldyt % 4 || (reinterpret_cast<uintptr_t>(YT) & 15))
    return fail(KS_ERR_ARG, "temporal rows: Lpad % 128, ldyt >= Lpad, 16-byte rows");
  return launch_temporal_simt(X, W, C, L, P, nt, round_up(round_up(C, kCG) * P, 64), Lpad,
                              nullptr, nullptr, nullptr, YT, ldyt, stream);
}

int launch_temporal(const float* X, const float* W, int64_t C, int64_t L,
                    int64_t P, int64_t nt, int64_t Q, int64_t Lpad, float* Yf,
                    __nv_bfloat16* Yhi, __nv_bfloat16* Ylo, int* err, cudaStream_t stream) {
  if (Yhi && Ylo && !Yf && err) {
    const int rc = launch_temporal_split_tc(X, W, C, L, P, nt, Q, Lpad, Yhi, Ylo, err, stream);
    if (rc == KS_OK) return zero_q_padding(C, P, Q, Lpad, Yf, Yhi, Ylo, stream);
    if (rc != KS_ERR_UNSUPPORTED) return rc;
  }
  const int rc = launch_temporal_simt(X, W, C, L, P, nt, Q, Lpad, Yf, Yhi, Ylo, nullptr, 0,
                                      stream);
  if (rc) return rc;
  return zero_q_padding(C, P, Q, Lpad, Yf, Yhi, Ylo, stream);
}

// q columns past the last group of 16 channels are padding: zero them.
int zero_q_padding(int64_t C, int64_t P, int64_t Q, int64_t Lpad, float* Yf, __nv_bfloat16* Yhi,
                   __nv_bfloat16* Ylo, cudaStream_t stream) {
  const int64_t qused = round_up(C, kCG) * P;
  if (qused < Q) {
    if (Yf) KS_CUDA(cudaMemset2DAsync(Yf + qused, Q * sizeof(float), 0, (Q - qused) * sizeof(float), Lpad, stream));
    if (Yhi) {
      KS_CUDA(cudaMemset2DAsync(Yhi + qused, Q * 2, 0, (Q - qused) * 2, Lpad, stream));
      KS_CUDA(cudaMemset2DAsync(Ylo + qused, Q * 2, 0, (Q - qused) * 2, Lpad, stream));
    }
  }
  return KS_OK;
}


int launch_project(const float* X, const float* U, const float* W, int64_t C,
                   int64_t L, int64_t K, int64_t P, int64_t nt, int precision,
                   float* B, int64_t ldb, bool tiled, void* ws, size_t ws_bytes,
                   int* err_out, cudaStream_t stream) {
  if (!X || !U || !W || !B) return fail(KS_ERR_ARG, "ks_project: null pointer");
  if (C < 1 || L < 1 || K < 1 || P < 1 || nt < 1 || (nt % 2) == 0)
    return fail(KS_ERR_ARG, "ks_project: need C,L,K,P >= 1 and odd nt");
  if (P > kPMax) return fail(KS_ERR_UNSUPPORTED, "ks_project: n_pcs must be <= 8");
  if (nt > 1023) return fail(KS_ERR_UNSUPPORTED, "ks_project: nt must be <= 1023");
  if (!tiled && ldb < L) return fail(KS_ERR_ARG, "ks_project: ldb < L");
  if (precision != KS_PROJ_FP32 && precision != KS_PROJ_BF16X3)
    return fail(KS_ERR_ARG, "ks_project: unknown precision");
  const ProjLayout lay = proj_layout(C, L, K, P, precision);
  if (!ws || ws_bytes < lay.bytes) return fail(KS_ERR_WORKSPACE, "ks_project: workspace too small");
  Carve cv(ws);
  int* err = cv.take<int>(64);
  KS_CUDA(cudaMemsetAsync(err, 0, sizeof(int), stream));
  const int reorder_blocks = (int)std::min<int64_t>(4096, (lay.Kpad * lay.Q + 255) / 256);
  if (precision == KS_PROJ_FP32) {
    float* Uq = cv.take<float>((size_t)lay.Kpad * lay.Q);
    float* Yt = cv.take<float>((size_t)lay.Lpad * lay.Q);
    ks_reorder_templates_kernel<<<reorder_blocks, 256, 0, stream>>>(
        U, (int)K, (int)P, (int)C, (int)lay.Kpad, (int)lay.Q, Uq, nullptr, nullptr);
    KS_CUDA(cudaGetLastError());
    int rc = launch_temporal(X, W, C, L, P, nt, lay.Q, lay.Lpad, Yt, nullptr, nullptr, nullptr, stream);
    if (rc) return rc;
    rc = sgemm_tn(Uq, Yt, B, K, L, lay.Q, ldb, stream, tiled);
    if (rc) return rc;
    if (err_out) KS_CUDA(cudaMemcpyAsync(err_out, err, sizeof(int), cudaMemcpyDeviceToDevice, stream));
    return KS_OK;
  }
  __nv_bfloat16* Uhl = cv.take<__nv_bfloat16>((size_t)lay.Kpad * lay.Q * 2);
  __nv_bfloat16* Yhl = cv.take<__nv_bfloat16>((size_t)lay.Lpad * lay.Q * 2);
  __nv_bfloat16* Uhi = Uhl;
  __nv_bfloat16* Ulo = Uhl + (size_t)lay.Kpad * lay.Q;
  __nv_bfloat16* Yhi = Yhl;
  __nv_bfloat16* Ylo = Yhl + (size_t)lay.Lpad * lay.Q;
  ks_reorder_templates_kernel<<<reorder_blocks, 256, 0, stream>>>(
      U, (int)K, (int)P, (int)C, (int)lay.Kpad, (int)lay.Q, nullptr, Uhi, Ulo);
  KS_CUDA(cudaGetLastError());
  int rc = launch_temporal(X, W, C, L, P, nt, lay.Q, lay.Lpad, nullptr, Yhi, Ylo, err, stream);
  if (rc) return rc;
  rc = gemm_bf16x3(Uhi, Ulo, Yhi, Ylo, B, K, L, lay.Q, lay.Kpad, lay.Lpad, ldb, tiled, err, stream);
  if (rc) return rc;
  if (err_out) KS_CUDA(cudaMemcpyAsync(err_out, err, sizeof(int), cudaMemcpyDeviceToDevice, stream));
  return KS_OK;
}

}  // namespace ks
