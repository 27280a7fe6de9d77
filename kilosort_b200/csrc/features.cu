// Per-spike PC features (kilosort/template_matching.py:85-86) and the
// per-template channel selection of prepare_extract (:50-51).
//
// ks_features_kernel: one warp per spike.  For each of the nC channels nearest
// to the template's peak channel the warp gathers the nt-sample residual
// window around the spike (lanes over taps), projects it on the P basis rows
// with warp-shuffle reductions and adds amp * Ucc, rounding the product and
// the sum separately as the reference does.  Output [N, nC, P] (the layout
// `extract` stores, :108).
#include "ks_common.cuh"
#include "project.cuh"

namespace ks {

constexpr int kFeatWarps = 8;

__global__ void __launch_bounds__(kFeatWarps * 32)
ks_features_kernel(const float* __restrict__ Xres, const long long* __restrict__ st,
                   const float* __restrict__ amps, const float* __restrict__ W,
                   const long long* __restrict__ iCC, const long long* __restrict__ iU,
                   const float* __restrict__ Ucc, int C, int L, int K, int P,
                   int nt, int nC, long long N, const long long* __restrict__ n_dev,
                   float* __restrict__ tF) {
  // with n_dev, the spikes to process are min(N, *n_dev) (a count the peel wrote)
  const long long n = n_dev ? min(N, max(*n_dev, 0LL)) : N;
  if ((long long)blockIdx.x * kFeatWarps >= n) return;
  extern __shared__ float sW[];  // [P][nt]
  for (int i = threadIdx.x; i < P * nt; i += blockDim.x) sW[i] = W[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long long s = (long long)blockIdx.x * kFeatWarps + (threadIdx.x >> 5);
  if (s >= n) return;
  const long long tau = st[2 * s];
  const long long kk = st[2 * s + 1];
  const long long t0 = tau - nt / 2;
  if (kk < 0 || kk >= K || t0 < 0 || t0 + nt > L) {
    // not a spike of this batch: mark the row instead of reading out of bounds
    for (int e = lane; e < nC * P; e += 32) tF[s * nC * P + e] = __int_as_float(0x7fc00000);
    return;
  }
  const int k = (int)kk;
  const float amp = amps[s];
  const int peak = (int)iU[k];
  for (int i = 0; i < nC; ++i) {
    int c = (int)iCC[(long long)i * C + peak];
    if (c < 0 || c >= C) c = 0;
    const float* x = Xres + (long long)c * L + t0;
    float part[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) part[p] = 0.f;
    for (int t = lane; t < nt; t += 32) {
      const float xv = x[t];
#pragma unroll
      for (int p = 0; p < 8; ++p)
        if (p < P) part[p] = fmaf(xv, sW[p * nt + t], part[p]);
    }
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      if (p < P) {
        float v = part[p];
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == p) {
          const float u = Ucc[((long long)i * K + k) * P + p];
          tF[(s * nC + i) * P + p] = __fadd_rn(v, __fmul_rn(amp, u));
        }
      }
    }
  }
}

// iU[k] = argmax_c sum_p U[k,p,c]^2 (first index on ties);
// Ucc[i,k,p] = U[k,p,iCC[i,iU[k]]].  One warp per template.
__global__ void ks_template_channels_kernel(const float* __restrict__ U,
                                            const long long* __restrict__ iCC,
                                            int K, int P, int C, int nC,
                                            long long* __restrict__ iU,
                                            float* __restrict__ Ucc) {
  const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (k >= K) return;
  const float* u = U + (long long)k * P * C;
  float best = -1.f;
  int arg = 0;
  for (int c = lane; c < C; c += 32) {
    float v = 0.f;
    for (int p = 0; p < P; ++p) v = __fadd_rn(v, __fmul_rn(u[p * C + c], u[p * C + c]));
    if (v > best) {
      best = v;
      arg = c;
    }
  }
  for (int o = 16; o; o >>= 1) {
    const float ov = __shfl_xor_sync(0xffffffffu, best, o);
    const int oa = __shfl_xor_sync(0xffffffffu, arg, o);
    if (ov > best || (ov == best && oa < arg)) {
      best = ov;
      arg = oa;
    }
  }
  if (lane == 0) iU[k] = arg;
  for (int e = lane; e < nC * P; e += 32) {
    const int i = e / P, p = e - (e / P) * P;
    const int c = (int)iCC[(long long)i * C + arg];
    Ucc[((long long)i * K + k) * P + p] = u[p * C + c];
  }
}

int launch_features(const float* Xres, const int64_t* st, const float* amps,
                    const float* W, const int64_t* iCC, const int64_t* iU,
                    const float* Ucc, int64_t C, int64_t L, int64_t K, int64_t P,
                    int64_t nt, int64_t nC, int64_t N, float* tF,
                    cudaStream_t stream, const int64_t* n_dev) {
  if (N == 0) return KS_OK;
  if (!Xres || !st || !amps || !W || !iCC || !iU || !Ucc || !tF)
    return fail(KS_ERR_ARG, "ks_features: null pointer");
  if (P < 1 || P > 8 || nt < 1 || nC < 1 || nC > C || N < 0)
    return fail(KS_ERR_ARG, "ks_features: bad sizes (need 1 <= P <= 8, 1 <= nC <= C)");
  const long long blocks = (N + kFeatWarps - 1) / kFeatWarps;
  const size_t smem = sizeof(float) * P * nt;
  ks_features_kernel<<<(unsigned)blocks, kFeatWarps * 32, smem, stream>>>(
      Xres, reinterpret_cast<const long long*>(st), amps, W,
      reinterpret_cast<const long long*>(iCC), reinterpret_cast<const long long*>(iU), Ucc,
      (int)C, (int)L, (int)K, (int)P, (int)nt, (int)nC, N,
      reinterpret_cast<const long long*>(n_dev), tF);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

int launch_template_channels(const float* U, const int64_t* iCC, int64_t K,
                             int64_t P, int64_t C, int64_t nC, int64_t* iU,
                             float* Ucc, cudaStream_t stream) {
  if (!U || !iCC || !iU || !Ucc || K < 1 || P < 1 || C < 1 || nC < 1 || nC > C)
    return fail(KS_ERR_ARG, "ks_template_channels: bad args");
  const long long blocks = (K * 32 + 255) / 256;
  ks_template_channels_kernel<<<(unsigned)blocks, 256, 0, stream>>>(
      U, reinterpret_cast<const long long*>(iCC), (int)K, (int)P, (int)C, (int)nC,
      reinterpret_cast<long long*>(iU), Ucc);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

}  // namespace ks
