// Template cross-correlations (kilosort/template_matching.py:155-167):
//   WtW[k, m, l] = sum_t W[m, t] * W[k, t + nt - l]      (flipped full xcorr)
//   G[(i,k), (j,m)] = sum_c U[i,k,c] * U[j,m,c]            (Gram of U rows)
//   ctc[i, j, l] = sum_{k,m} G[(i,k), (j,m)] * WtW[k, m, l]
// G is one FP32 contraction over channels (the TN SIMT GEMM of the
// projection); the lag contraction is a small per-(i, j-tile) kernel.
#include "ks_common.cuh"
#include "project.cuh"

#include <cmath>

namespace ks {

__global__ void ks_wtw_kernel(const float* __restrict__ W, int P, int nt,
                              float* __restrict__ WtW) {
  const int nlag = 2 * nt + 1;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= P * P * nlag) return;
  const int l = e % nlag;
  const int km = e / nlag;
  const int k = km / P, m = km % P;
  const int t_lo = max(0, l - nt), t_hi = min(nt - 1, l - 1);
  float s = 0.f;
  for (int t = t_lo; t <= t_hi; ++t) s = fmaf(W[m * nt + t], W[k * nt + t + nt - l], s);
  WtW[e] = s;
}

constexpr int kCtcJ = 16;

__global__ void __launch_bounds__(256)
ks_ctc_lag_kernel(const float* __restrict__ G, long long ldg,
                  const float* __restrict__ WtW, int K, int P, int nt,
                  float* __restrict__ ctc) {
  extern __shared__ float sm[];
  const int nlag = 2 * nt + 1;
  float* sWtW = sm;                   // [P*P][nlag]
  float* sG = sm + P * P * nlag;      // [kCtcJ][P][P]  (j, k, m)
  const int i = blockIdx.y;
  const int j0 = blockIdx.x * kCtcJ;
  for (int e = threadIdx.x; e < P * P * nlag; e += blockDim.x) sWtW[e] = WtW[e];
  for (int e = threadIdx.x; e < kCtcJ * P * P; e += blockDim.x) {
    const int jj = e / (P * P), km = e % (P * P);
    const int k = km / P, m = km % P;
    const int j = j0 + jj;
    sG[e] = (j < K) ? G[(long long)(i * P + k) * ldg + (long long)j * P + m] : 0.f;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < kCtcJ * nlag; e += blockDim.x) {
    const int jj = e / nlag, l = e % nlag;
    const int j = j0 + jj;
    if (j >= K) continue;
    float s = 0.f;
    for (int km = 0; km < P * P; ++km) s = fmaf(sG[jj * P * P + km], sWtW[km * nlag + l], s);
    ctc[((long long)i * K + j) * nlag + l] = s;
  }
}

// Template similarity (kilosort/CCG.py:94-102): the ctc contraction on the
// templates scaled to unit norm, maximised over lags without storing the lags.
// 16 threads per template j of the tile, each over lags l = part, part + 16, ...
__global__ void __launch_bounds__(256)
ks_sim_lag_kernel(const float* __restrict__ G, long long ldg,
                  const float* __restrict__ WtW, int K, int P, int nt,
                  float* __restrict__ sim) {
  extern __shared__ float sm[];
  const int nlag = 2 * nt + 1;
  float* sWtW = sm;                   // [P*P][nlag]
  float* sG = sm + P * P * nlag;      // [kCtcJ][P][P]
  const int i = blockIdx.y;
  const int j0 = blockIdx.x * kCtcJ;
  for (int e = threadIdx.x; e < P * P * nlag; e += blockDim.x) sWtW[e] = WtW[e];
  for (int e = threadIdx.x; e < kCtcJ * P * P; e += blockDim.x) {
    const int jj = e / (P * P), km = e % (P * P);
    const int k = km / P, m = km % P;
    const int j = j0 + jj;
    sG[e] = (j < K) ? G[(long long)(i * P + k) * ldg + (long long)j * P + m] : 0.f;
  }
  __syncthreads();
  const int jj = threadIdx.x >> 4, part = threadIdx.x & 15;
  float best = -INFINITY;
  for (int l = part; l < nlag; l += 16) {
    float s = 0.f;
    for (int km = 0; km < P * P; ++km) s = fmaf(sG[jj * P * P + km], sWtW[km * nlag + l], s);
    best = fmaxf(best, s);
  }
  for (int o = 8; o; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o, 16));
  const int j = j0 + jj;
  if (part == 0 && j < K) sim[(long long)i * K + j] = best;
}

// Wall [K, C, P] -> rows (i*P + k) of the Gram operand, column c:
// Wall[i, c, k] / (1e-6 + ||Wall[i]||), one block per template.
__global__ void __launch_bounds__(256)
ks_unit_templates_kernel(const float* __restrict__ Wall, int C, int P, float* __restrict__ Upad,
                         long long ldu) {
  __shared__ float red[256];
  const int i = blockIdx.x;
  const float* w = Wall + (long long)i * C * P;
  float s = 0.f;
  for (int e = threadIdx.x; e < C * P; e += blockDim.x) s = fmaf(w[e], w[e], s);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  const float den = __fadd_rn(1e-6f, __fsqrt_rn(red[0]));
  for (int e = threadIdx.x; e < C * P; e += blockDim.x) {
    const int c = e / P, k = e - c * P;
    Upad[((long long)i * P + k) * ldu + c] = __fdiv_rn(w[e], den);
  }
}

struct CtcLayout {
  int64_t rows, cols, ldg;
  size_t bytes;
};

static CtcLayout ctc_layout(int64_t K, int64_t P, int64_t C, int64_t nt) {
  CtcLayout l;
  l.rows = round_up(K * P, 128);
  l.cols = round_up(C, 16);
  l.ldg = round_up(K * P, 4);
  Carve cv(nullptr);
  cv.take<float>((size_t)l.rows * l.cols);
  cv.take<float>((size_t)K * P * l.ldg);
  cv.take<float>((size_t)P * P * (2 * nt + 1));
  l.bytes = cv.used;
  return l;
}

size_t ctc_workspace_size(int64_t K, int64_t P, int64_t C, int64_t nt) {
  return ctc_layout(K, P, C, nt).bytes;
}

int launch_ctc(const float* U, const float* W, int64_t K, int64_t P, int64_t C,
               int64_t nt, float* ctc, void* ws, size_t ws_bytes,
               cudaStream_t stream) {
  if (!U || !W || !ctc || K < 1 || P < 1 || C < 1 || nt < 1 || (nt % 2) == 0)
    return fail(KS_ERR_ARG, "ks_ctc: bad args (need odd nt)");
  if (P > 16 || nt > 1023) return fail(KS_ERR_UNSUPPORTED, "ks_ctc: P <= 16 and nt <= 1023");
  const CtcLayout lay = ctc_layout(K, P, C, nt);
  if (!ws || ws_bytes < lay.bytes) return fail(KS_ERR_WORKSPACE, "ks_ctc: workspace too small");
  Carve cv(ws);
  float* Upad = cv.take<float>((size_t)lay.rows * lay.cols);
  float* G = cv.take<float>((size_t)K * P * lay.ldg);
  float* WtW = cv.take<float>((size_t)P * P * (2 * nt + 1));
  KS_CUDA(cudaMemsetAsync(Upad, 0, sizeof(float) * lay.rows * lay.cols, stream));
  KS_CUDA(cudaMemcpy2DAsync(Upad, lay.cols * sizeof(float), U, C * sizeof(float),
                            C * sizeof(float), K * P, cudaMemcpyDeviceToDevice, stream));
  const int nw = (int)(P * P * (2 * nt + 1));
  ks_wtw_kernel<<<(nw + 255) / 256, 256, 0, stream>>>(W, (int)P, (int)nt, WtW);
  KS_CUDA(cudaGetLastError());
  int rc = sgemm_tn(Upad, Upad, G, K * P, K * P, lay.cols, lay.ldg, stream, false);
  if (rc) return rc;
  const size_t smem = sizeof(float) * (P * P * (2 * nt + 1) + kCtcJ * P * P);
  KS_CUDA(cudaFuncSetAttribute(ks_ctc_lag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((unsigned)((K + kCtcJ - 1) / kCtcJ), (unsigned)K);
  ks_ctc_lag_kernel<<<grid, 256, smem, stream>>>(G, lay.ldg, WtW, (int)K, (int)P, (int)nt, ctc);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

int launch_similarity(const float* Wall, const float* W, int64_t K, int64_t C, int64_t P,
                      int64_t nt, float* sim, void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (!Wall || !W || !sim || K < 1 || P < 1 || C < 1 || nt < 1 || (nt % 2) == 0)
    return fail(KS_ERR_ARG, "ks_similarity: bad args (need odd nt)");
  if (P > 16 || nt > 1023) return fail(KS_ERR_UNSUPPORTED, "ks_similarity: P <= 16 and nt <= 1023");
  if (K > 65535) return fail(KS_ERR_UNSUPPORTED, "ks_similarity: K <= 65535");
  const CtcLayout lay = ctc_layout(K, P, C, nt);
  if (!ws || ws_bytes < lay.bytes) return fail(KS_ERR_WORKSPACE, "ks_similarity: workspace too small");
  Carve cv(ws);
  float* Upad = cv.take<float>((size_t)lay.rows * lay.cols);
  float* G = cv.take<float>((size_t)K * P * lay.ldg);
  float* WtW = cv.take<float>((size_t)P * P * (2 * nt + 1));
  KS_CUDA(cudaMemsetAsync(Upad, 0, sizeof(float) * lay.rows * lay.cols, stream));
  ks_unit_templates_kernel<<<(unsigned)K, 256, 0, stream>>>(Wall, (int)C, (int)P, Upad, lay.cols);
  KS_CUDA(cudaGetLastError());
  const int nw = (int)(P * P * (2 * nt + 1));
  ks_wtw_kernel<<<(nw + 255) / 256, 256, 0, stream>>>(W, (int)P, (int)nt, WtW);
  KS_CUDA(cudaGetLastError());
  int rc = sgemm_tn(Upad, Upad, G, K * P, K * P, lay.cols, lay.ldg, stream, false);
  if (rc) return rc;
  const size_t smem = sizeof(float) * (P * P * (2 * nt + 1) + kCtcJ * P * P);
  KS_CUDA(cudaFuncSetAttribute(ks_sim_lag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((unsigned)((K + kCtcJ - 1) / kCtcJ), (unsigned)K);
  ks_sim_lag_kernel<<<grid, 256, smem, stream>>>(G, lay.ldg, WtW, (int)K, (int)P, (int)nt, sim);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

}  // namespace ks

extern "C" KS_API size_t ks_similarity_workspace_size(int64_t K, int64_t C, int64_t P,
                                                      int64_t nt) {
  return ks::ctc_workspace_size(K, P, C, nt);
}

extern "C" KS_API int ks_similarity(const float* Wall, const float* W, int64_t K, int64_t C,
                                    int64_t P, int64_t nt, float* sim, void* workspace,
                                    size_t workspace_bytes, void* stream) {
  return ks::launch_similarity(Wall, W, K, C, P, nt, sim, workspace, workspace_bytes,
                               static_cast<cudaStream_t>(stream));
}
