// Fixed-assignment reconstruction loss and its adjoint.
//
// Given spikes s = (tau_s, k_s) with amplitudes a_s, templates U [K,P,C] and the
// temporal basis W [P,nt], the reconstruction is
//   R[c, tau] = sum_s a_s * wave_{k_s}[c, tau - tau_s + nt/2],
//   wave_k[c, t] = sum_p U[k,p,c] * W[p,t]          (0 <= t < nt, 0 <= tau < L)
// -- the subtraction kilosort/template_matching.py:237 applies spike by spike --
// and the loss is  loss = sum_{c,tau} (X - R)^2.  With G = dloss * dLoss/dR =
// -2 * dloss * Xres (Xres = X - R):
//   d a_s      = sum_{c,t} G[c, tau_s - nt/2 + t] * wave_{k_s}[c, t]
//   d U[k,p,c] = sum_t W[p,t] * H_k[c,t]
//   d W[p,t]   = sum_k sum_c U[k,p,c] * H_k[c,t]
// where H_k[c,t] = sum_{s: k_s = k} a_s * G[c, tau_s - nt/2 + t] is the
// amplitude-weighted sum of the residual windows of template k's spikes.  The
// adjoint never stores the K x C x nt waveforms: each block recomputes the
// slice of wave_k it needs in shared memory.
//
// Determinism: every sum runs in a fixed order (spikes in index order per
// template, per-block partials reduced in block order in double precision), so
// repeated calls give identical bits.
//
// Forward kernels: count spikes per time sample, scan, bucket them by time,
// then one warp per (32-column block, 32 channels) applies the spikes whose
// window meets the block in (time, index) order, writes Xres and a double
// partial of sum Xres^2.  Adjoint kernels: group spikes by template (CSR in
// index order), one block per (template, 32-channel chunk) accumulates H in
// shared memory and the per-spike dot products, then fixed-order reductions.
#include "ks_common.cuh"

#include <algorithm>

namespace {

constexpr int kCol = 32;
constexpr int kChunkC = 32;        // channels per adjoint block
constexpr int kAdjThreads = 256;
constexpr int kRecThreads = 256;
constexpr int kScanThreads = 1024;

struct ReconLayout {
  size_t status, cnt, off, idx, part, cntk, offk, list, dwpart, dapart, bytes;
  int64_t nblk, ngrp, nchunk, nwarps;
};

ReconLayout recon_layout(int64_t C, int64_t L, int64_t K, int64_t P, int64_t nt, int64_t N) {
  ReconLayout r;
  r.nblk = (L + kCol - 1) / kCol;
  r.ngrp = (C + 31) / 32;
  r.nchunk = (C + kChunkC - 1) / kChunkC;
  r.nwarps = r.nblk * r.ngrp;
  size_t o = 0;
  auto take = [&](size_t b) {
    const size_t at = o;
    o = ks::align256(o + b);
    return at;
  };
  r.status = take(256);
  r.cnt = take(4 * (size_t)(L + 1));
  r.off = take(4 * (size_t)(L + 1));
  r.idx = take(4 * (size_t)std::max<int64_t>(N, 1));
  r.part = take(8 * (size_t)r.nwarps);
  r.cntk = take(4 * (size_t)(K + 1));
  r.offk = take(4 * (size_t)(K + 1));
  r.list = take(4 * (size_t)std::max<int64_t>(N, 1));
  r.dwpart = take(4 * (size_t)K * r.nchunk * P * nt);
  r.dapart = take(4 * (size_t)r.nchunk * std::max<int64_t>(N, 1));
  r.bytes = o;
  return r;
}

// ------------------------------------------------------------------ helpers
// Exclusive scan of n ints into out[0..n] (out[n] = total), one block.
__global__ void __launch_bounds__(kScanThreads) ks_scan_kernel(const int* __restrict__ in, int n,
                                                               int* __restrict__ out) {
  __shared__ int part[kScanThreads];
  const int per = (n + kScanThreads - 1) / kScanThreads;
  const int b = threadIdx.x * per, e = min(n, b + per);
  int s = 0;
  for (int i = b; i < e; ++i) s += in[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int d = 1; d < kScanThreads; d <<= 1) {
    const int v = threadIdx.x >= d ? part[threadIdx.x - d] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = part[threadIdx.x] - s;   // exclusive prefix of this segment
  for (int i = b; i < e; ++i) {
    out[i] = run;
    run += in[i];
  }
  if (threadIdx.x == kScanThreads - 1) out[n] = part[kScanThreads - 1];
}

// Spikes per time sample; an out-of-range time or template marks the call
// invalid (the spike is skipped everywhere).
__global__ void ks_recon_count_kernel(const long long* __restrict__ st, int N, int L, int K,
                                      int* __restrict__ cnt, int* __restrict__ cntk,
                                      int* __restrict__ status) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < N; s += gridDim.x * blockDim.x) {
    const long long tau = st[2 * (long long)s], k = st[2 * (long long)s + 1];
    if (tau < 0 || tau >= L || k < 0 || k >= K) {
      atomicCAS(status, 0, KS_ERR_ARG);
      continue;
    }
    atomicAdd(&cnt[tau], 1);
    atomicAdd(&cntk[k], 1);
  }
}

__global__ void ks_recon_fill_kernel(const long long* __restrict__ st, int N, int L, int K,
                                     const int* __restrict__ off, int* __restrict__ fill,
                                     int* __restrict__ idx) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < N; s += gridDim.x * blockDim.x) {
    const long long tau = st[2 * (long long)s], k = st[2 * (long long)s + 1];
    if (tau < 0 || tau >= L || k < 0 || k >= K) continue;
    idx[off[tau] + atomicAdd(&fill[tau], 1)] = s;
  }
}

// ------------------------------------------------------------------ forward
// One warp per (32-column block, 32 channels): lanes own channels and keep the
// block's 32 values in registers; spikes whose window meets the block are
// applied in (time, index) order.
__global__ void __launch_bounds__(kRecThreads)
ks_recon_kernel(const float* __restrict__ X, const long long* __restrict__ st,
                const float* __restrict__ amps, const float* __restrict__ U,
                const float* __restrict__ W, const int* __restrict__ off,
                const int* __restrict__ idx, int C, int L, int K, int P, int nt, int nblk,
                int ngrp, float* __restrict__ Xres, double* __restrict__ part) {
  extern __shared__ __align__(16) float sW[];   // Wt[t][8], components padded to 8
  for (int i = threadIdx.x; i < 8 * nt; i += blockDim.x) {
    const int t = i >> 3, p = i & 7;
    sW[i] = p < P ? W[p * nt + t] : 0.f;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long long w = (long long)blockIdx.x * (kRecThreads / 32) + (threadIdx.x >> 5);
  if (w >= (long long)nblk * ngrp) return;
  const int blk = (int)(w / ngrp), cg = (int)(w % ngrp);
  const int c0 = blk * kCol, c = cg * 32 + lane, half = nt / 2;
  const bool chok = c < C;
  const int ncol = min(kCol, L - c0);
  const float* xrow = X + (long long)(chok ? c : 0) * L + c0;
  float x[kCol];
#pragma unroll
  for (int j = 0; j < kCol; ++j) x[j] = (chok && j < ncol) ? xrow[j] : 0.f;
  // spike times whose window [tau - half, tau + half] meets [c0, c0 + 31]
  const int lo = max(0, c0 - half), hi = min(L - 1, c0 + kCol - 1 + half);
  for (int t0 = lo; t0 <= hi; t0 += 32) {
    const int tau_l = t0 + lane;
    const int n_l = tau_l <= hi ? off[tau_l + 1] - off[tau_l] : 0;
    unsigned busy = __ballot_sync(0xffffffffu, n_l > 0);
    while (busy) {
      const int src = __ffs(busy) - 1;
      busy &= busy - 1;
      const int tau = t0 + src;
      const int n = __shfl_sync(0xffffffffu, n_l, src);
      const int base = off[tau];
      // the bucket's spikes in increasing index order (buckets hold a few)
      int last = -1;
      for (int r = 0; r < n; ++r) {
        int best = 0x7fffffff;
        for (int i = 0; i < n; ++i) {
          const int v = idx[base + i];
          if (v > last && v < best) best = v;
        }
        last = best;
        const int k = (int)st[2 * (long long)best + 1];
        const float amp = amps[best];
        float u[8];
#pragma unroll
        for (int pp = 0; pp < 8; ++pp)
          u[pp] = (chok && pp < P) ? __ldg(U + ((long long)k * P + pp) * C + c) : 0.f;
        const int tt0 = c0 - tau + half;
        const float4* W4 = reinterpret_cast<const float4*>(sW);
#pragma unroll
        for (int j = 0; j < kCol; ++j) {
          const int t = tt0 + j;
          if (t >= 0 && t < nt) {
            const float4 wa = W4[2 * t], wb = W4[2 * t + 1];
            const float wt[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
            float wv = 0.f;
#pragma unroll
            for (int pp = 0; pp < 8; ++pp)
              if (pp < P) wv = fmaf(u[pp], wt[pp], wv);
            x[j] = __fsub_rn(x[j], __fmul_rn(amp, wv));
          }
        }
      }
    }
  }
  double sq = 0.0;
  float* orow = Xres + (long long)(chok ? c : 0) * L + c0;
#pragma unroll
  for (int j = 0; j < kCol; ++j)
    if (chok && j < ncol) {
      orow[j] = x[j];
      sq += (double)x[j] * (double)x[j];
    }
  for (int o = 16; o; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
  if (lane == 0) part[w] = sq;
}

// Fixed-order sum of the per-warp partials.
__global__ void __launch_bounds__(1024) ks_sum_double_kernel(const double* __restrict__ part,
                                                             long long n, double* __restrict__ out) {
  __shared__ double red[1024];
  double s = 0.0;
  for (long long i = threadIdx.x; i < n; i += 1024) s += part[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int d = 512; d; d >>= 1) {
    if (threadIdx.x < d) red[threadIdx.x] += red[threadIdx.x + d];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// ------------------------------------------------------------------ adjoint
// Spikes of each template, in index order: block b handles templates b, b+G...
__global__ void __launch_bounds__(256) ks_group_by_template_kernel(
    const long long* __restrict__ st, int N, int L, int K, const int* __restrict__ offk,
    int* __restrict__ list) {
  __shared__ int wsum[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = blockIdx.x; k < K; k += gridDim.x) {
    int pos = offk[k];
    for (int s0 = 0; s0 < N; s0 += 256) {
      const int s = s0 + threadIdx.x;
      bool m = false;
      if (s < N) {
        const long long tau = st[2 * (long long)s], kk = st[2 * (long long)s + 1];
        m = kk == k && tau >= 0 && tau < L;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, m);
      if (lane == 0) wsum[warp] = __popc(bal);
      __syncthreads();
      int before = 0, total = 0;
      for (int i = 0; i < 8; ++i) {
        if (i < warp) before += wsum[i];
        total += wsum[i];
      }
      if (m) list[pos + before + __popc(bal & ((1u << lane) - 1u))] = s;
      pos += total;
      __syncthreads();
    }
  }
}

// Block (k, chunk): H_k and wave_k over 32 channels in shared memory.
__global__ void __launch_bounds__(kAdjThreads) ks_adjoint_kernel(
    const float* __restrict__ Xres, const long long* __restrict__ st,
    const float* __restrict__ amps, const float* __restrict__ U, const float* __restrict__ W,
    const int* __restrict__ offk, const int* __restrict__ list, const float* __restrict__ dloss,
    int C, int L, int K, int P, int nt, int nchunk, float* __restrict__ dU,
    float* __restrict__ dwpart, float* __restrict__ dapart) {
  extern __shared__ float sm[];
  const int k = blockIdx.x, ch = blockIdx.y;
  const int c0 = ch * kChunkC;
  const int ncl = min(kChunkC, C - c0);
  const int ne = kChunkC * nt;
  float* sW = sm;                     // [P][nt]
  float* wave = sW + P * nt;          // [kChunkC][nt]
  float* H = wave + ne;                // [kChunkC][nt]
  float* red = H + ne;                // [kAdjThreads / 32]
  for (int i = threadIdx.x; i < P * nt; i += kAdjThreads) sW[i] = W[i];
  __syncthreads();
  for (int e = threadIdx.x; e < ne; e += kAdjThreads) {
    const int cl = e / nt, t = e - cl * nt;
    float v = 0.f;
    if (cl < ncl) {
      for (int p = 0; p < P; ++p) v = fmaf(U[((long long)k * P + p) * C + c0 + cl], sW[p * nt + t], v);
    }
    wave[e] = v;
    H[e] = 0.f;
  }
  const float scale = -2.f * dloss[0];
  const int half = nt / 2;
  const int b = offk[k], n = offk[k + 1] - b;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = 0; i < n; ++i) {
    const int s = list[b + i];
    const int tau = (int)st[2 * (long long)s];
    const float a = amps[s];
    float dot = 0.f;
    for (int e = threadIdx.x; e < ne; e += kAdjThreads) {
      const int cl = e / nt, t = e - cl * nt;
      const int col = tau - half + t;
      float g = 0.f;
      if (cl < ncl && col >= 0 && col < L) g = Xres[(long long)(c0 + cl) * L + col];
      H[e] = fmaf(a, g, H[e]);
      dot = fmaf(g, wave[e], dot);
    }
    for (int o = 16; o; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
    if (lane == 0) red[warp] = dot;
    __syncthreads();
    if (threadIdx.x == 0) {
      float tot = 0.f;
      for (int w = 0; w < kAdjThreads / 32; ++w) tot += red[w];
      dapart[(long long)s * nchunk + ch] = tot;
    }
    __syncthreads();
  }
  // H is complete (each element was written by one thread): publish it
  __syncthreads();
  // dU[k, p, c0 + cl] = scale * sum_t W[p,t] H[cl,t]
  for (int o = threadIdx.x; o < P * ncl; o += kAdjThreads) {
    const int p = o / ncl, cl = o - p * ncl;
    float v = 0.f;
    for (int t = 0; t < nt; ++t) v = fmaf(sW[p * nt + t], H[cl * nt + t], v);
    dU[((long long)k * P + p) * C + c0 + cl] = scale * v;
  }
  // partial dW of this block: sum_cl U[k,p,c0+cl] H[cl,t] (unscaled)
  float* dst = dwpart + ((long long)k * nchunk + ch) * P * nt;
  for (int o = threadIdx.x; o < P * nt; o += kAdjThreads) {
    const int p = o / nt, t = o - p * nt;
    float v = 0.f;
    for (int cl = 0; cl < ncl; ++cl) v = fmaf(U[((long long)k * P + p) * C + c0 + cl], H[cl * nt + t], v);
    dst[o] = v;
  }
}

// dW[o] = scale * sum over (template, chunk) blocks of the partials, in block
// order, accumulated in double.
__global__ void ks_adjoint_dw_kernel(const float* __restrict__ dwpart, int nblocks, int PN,
                                     const float* __restrict__ dloss, float* __restrict__ dW) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= PN) return;
  double s = 0.0;
  for (int b = 0; b < nblocks; ++b) s += (double)dwpart[(long long)b * PN + o];
  dW[o] = (float)((double)(-2.f * dloss[0]) * s);
}

// damps[s] = scale * sum over chunks of the per-chunk dot products.
__global__ void ks_adjoint_da_kernel(const float* __restrict__ dapart, const long long* __restrict__ st,
                                     int N, int L, int K, int nchunk,
                                     const float* __restrict__ dloss, float* __restrict__ damps) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < N; s += gridDim.x * blockDim.x) {
    const long long tau = st[2 * (long long)s], k = st[2 * (long long)s + 1];
    if (tau < 0 || tau >= L || k < 0 || k >= K) {
      damps[s] = 0.f;
      continue;
    }
    double v = 0.0;
    for (int ch = 0; ch < nchunk; ++ch) v += (double)dapart[(long long)s * nchunk + ch];
    damps[s] = (float)((double)(-2.f * dloss[0]) * v);
  }
}

int check_recon(int64_t C, int64_t L, int64_t K, int64_t P, int64_t nt, int64_t N) {
  if (C < 1 || L < 1 || K < 1 || P < 1 || nt < 1 || (nt % 2) == 0 || N < 0)
    return ks::fail(KS_ERR_ARG, "ks_recon: need C,L,K,P >= 1, N >= 0 and odd nt");
  if (P > 8 || nt > 1023 || L >= (1LL << 31) - 1 || N >= (1LL << 31) || C > (1 << 24))
    return ks::fail(KS_ERR_UNSUPPORTED, "ks_recon: shape beyond supported limits");
  return KS_OK;
}

}  // namespace

extern "C" KS_API size_t ks_recon_workspace_size(int64_t C, int64_t L, int64_t K, int64_t P,
                                                int64_t nt, int64_t n_spikes) {
  if (check_recon(C, L, K, P, nt, n_spikes)) return 0;
  return recon_layout(C, L, K, P, nt, n_spikes).bytes;
}

extern "C" KS_API int ks_recon_loss(const float* X, const int64_t* st, const float* amps,
                                    int64_t n_spikes, const float* U, const float* W, int64_t C,
                                    int64_t L, int64_t K, int64_t P, int64_t nt, float* Xres,
                                    double* loss, int* status, void* workspace,
                                    size_t workspace_bytes, void* stream) {
  using namespace ks;
  int rc = check_recon(C, L, K, P, nt, n_spikes);
  if (rc) return rc;
  if (!X || !U || !W || !Xres || !loss || !status || (n_spikes > 0 && (!st || !amps)))
    return fail(KS_ERR_ARG, "ks_recon_loss: null pointer");
  const ReconLayout r = recon_layout(C, L, K, P, nt, n_spikes);
  if (!workspace || workspace_bytes < r.bytes) return fail(KS_ERR_WORKSPACE, "ks_recon_loss: workspace too small");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  char* base = static_cast<char*>(workspace);
  int* cnt = reinterpret_cast<int*>(base + r.cnt);
  int* off = reinterpret_cast<int*>(base + r.off);
  int* idx = reinterpret_cast<int*>(base + r.idx);
  int* cntk = reinterpret_cast<int*>(base + r.cntk);
  double* part = reinterpret_cast<double*>(base + r.part);
  const long long* stp = reinterpret_cast<const long long*>(st);
  const int N = (int)n_spikes;
  KS_CUDA(cudaMemsetAsync(status, 0, sizeof(int), s));
  KS_CUDA(cudaMemsetAsync(cnt, 0, 4 * (size_t)(L + 1), s));
  KS_CUDA(cudaMemsetAsync(cntk, 0, 4 * (size_t)(K + 1), s));
  const int gb = (int)std::min<int64_t>(4096, std::max<int64_t>(1, (N + 255) / 256));
  if (N > 0) {
    ks_recon_count_kernel<<<gb, 256, 0, s>>>(stp, N, (int)L, (int)K, cnt, cntk, status);
    KS_CUDA(cudaGetLastError());
  }
  ks_scan_kernel<<<1, kScanThreads, 0, s>>>(cnt, (int)L, off);
  KS_CUDA(cudaGetLastError());
  if (N > 0) {
    KS_CUDA(cudaMemsetAsync(cnt, 0, 4 * (size_t)L, s));   // reused as fill counters
    ks_recon_fill_kernel<<<gb, 256, 0, s>>>(stp, N, (int)L, (int)K, off, cnt, idx);
    KS_CUDA(cudaGetLastError());
  }
  const unsigned grid = (unsigned)((r.nwarps + kRecThreads / 32 - 1) / (kRecThreads / 32));
  ks_recon_kernel<<<grid, kRecThreads, sizeof(float) * 8 * nt, s>>>(
      X, stp, amps, U, W, off, idx, (int)C, (int)L, (int)K, (int)P, (int)nt, (int)r.nblk,
      (int)r.ngrp, Xres, part);
  KS_CUDA(cudaGetLastError());
  ks_sum_double_kernel<<<1, 1024, 0, s>>>(part, r.nwarps, loss);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

extern "C" KS_API int ks_recon_adjoint(const float* Xres, const int64_t* st, const float* amps,
                                       int64_t n_spikes, const float* U, const float* W,
                                       int64_t C, int64_t L, int64_t K, int64_t P, int64_t nt,
                                       const float* dloss, float* dU, float* dW, float* damps,
                                       int* status, void* workspace, size_t workspace_bytes,
                                       void* stream) {
  using namespace ks;
  int rc = check_recon(C, L, K, P, nt, n_spikes);
  if (rc) return rc;
  if (!Xres || !U || !W || !dloss || !dU || !dW || !status ||
      (n_spikes > 0 && (!st || !amps || !damps)))
    return fail(KS_ERR_ARG, "ks_recon_adjoint: null pointer");
  const ReconLayout r = recon_layout(C, L, K, P, nt, n_spikes);
  if (!workspace || workspace_bytes < r.bytes)
    return fail(KS_ERR_WORKSPACE, "ks_recon_adjoint: workspace too small");
  DeviceInfo dev;
  rc = device_info(&dev);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  char* base = static_cast<char*>(workspace);
  int* cnt = reinterpret_cast<int*>(base + r.cnt);
  int* cntk = reinterpret_cast<int*>(base + r.cntk);
  int* offk = reinterpret_cast<int*>(base + r.offk);
  int* list = reinterpret_cast<int*>(base + r.list);
  float* dwpart = reinterpret_cast<float*>(base + r.dwpart);
  float* dapart = reinterpret_cast<float*>(base + r.dapart);
  const long long* stp = reinterpret_cast<const long long*>(st);
  const int N = (int)n_spikes;
  KS_CUDA(cudaMemsetAsync(status, 0, sizeof(int), s));
  KS_CUDA(cudaMemsetAsync(cnt, 0, 4 * (size_t)(L + 1), s));
  KS_CUDA(cudaMemsetAsync(cntk, 0, 4 * (size_t)(K + 1), s));
  const int gb = (int)std::min<int64_t>(4096, std::max<int64_t>(1, (N + 255) / 256));
  if (N > 0) {
    ks_recon_count_kernel<<<gb, 256, 0, s>>>(stp, N, (int)L, (int)K, cnt, cntk, status);
    KS_CUDA(cudaGetLastError());
  }
  ks_scan_kernel<<<1, kScanThreads, 0, s>>>(cntk, (int)K, offk);
  KS_CUDA(cudaGetLastError());
  if (N > 0) {
    ks_group_by_template_kernel<<<(unsigned)std::min<int64_t>(K, 4 * dev.sm_count), 256, 0, s>>>(
        stp, N, (int)L, (int)K, offk, list);
    KS_CUDA(cudaGetLastError());
  }
  const size_t smem = sizeof(float) * ((size_t)P * nt + 2 * (size_t)kChunkC * nt + kAdjThreads / 32);
  if (smem > dev.smem_optin) return fail(KS_ERR_UNSUPPORTED, "ks_recon_adjoint: nt too long");
  KS_CUDA(cudaFuncSetAttribute(ks_adjoint_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const dim3 grid((unsigned)K, (unsigned)r.nchunk);
  ks_adjoint_kernel<<<grid, kAdjThreads, smem, s>>>(Xres, stp, amps, U, W, offk, list, dloss,
                                                    (int)C, (int)L, (int)K, (int)P, (int)nt,
                                                    (int)r.nchunk, dU, dwpart, dapart);
  KS_CUDA(cudaGetLastError());
  const int PN = (int)(P * nt);
  ks_adjoint_dw_kernel<<<(PN + 127) / 128, 128, 0, s>>>(dwpart, (int)(K * r.nchunk), PN, dloss, dW);
  KS_CUDA(cudaGetLastError());
  if (N > 0) {
    ks_adjoint_da_kernel<<<gb, 256, 0, s>>>(dapart, stp, N, (int)L, (int)K, (int)r.nchunk, dloss,
                                            damps);
    KS_CUDA(cudaGetLastError());
  }
  return KS_OK;
}
