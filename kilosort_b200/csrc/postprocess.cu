// Output consumers of extract on the device: spike positions and amplitudes.
//
//   w_i  = m_i * ||tF[s, i, :]|| / sum_j m_j * ||tF[s, j, :]||,
//          m_i = iCC_mask[i, iU[k_s]]                     (f32)
//   x_s  = sum_i xc[iCC[i, iU[k_s]]] * w_i,  y_s likewise  (f64)
//   a_s  = ||tF[s, :, :]||                                  (f32)
// -- kilosort/postprocessing.py:33-62 and kilosort/io.py:353.  One thread per
// spike; the nC x P features of a spike are contiguous and read as a run.
#include "ks_common.cuh"

namespace {

__global__ void ks_spike_positions_kernel(const float* __restrict__ tF,
                                          const int64_t* __restrict__ templ,
                                          const int64_t* __restrict__ iCC,
                                          const uint8_t* __restrict__ mask,
                                          const int64_t* __restrict__ iU,
                                          const double* __restrict__ xc,
                                          const double* __restrict__ yc, int N, int nC, int P,
                                          int C, int K, double* __restrict__ xs,
                                          double* __restrict__ ys, float* __restrict__ amps,
                                          int* __restrict__ status) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < N; s += gridDim.x * blockDim.x) {
    const int64_t k = templ[s];
    if (k < 0 || k >= K) {
      atomicCAS(status, 0, KS_ERR_ARG);
      xs[s] = ys[s] = 0.0;
      amps[s] = 0.f;
      continue;
    }
    const int64_t u = iU[k];
    const float* f = tF + (size_t)s * nC * P;
    float tm[32];
    float tot = 0.f, all = 0.f;
    for (int i = 0; i < nC; ++i) {
      float q = 0.f;
      for (int p = 0; p < P; ++p) q = fmaf(f[i * P + p], f[i * P + p], q);
      all += q;
      const float m = mask[(size_t)i * C + u] ? 1.f : 0.f;
      tm[i] = sqrtf(q) * m;
      tot += tm[i];
    }
    double x = 0.0, y = 0.0;
    for (int i = 0; i < nC; ++i) {
      const int64_t ch = iCC[(size_t)i * C + u];
      const double w = (double)(tm[i] / tot);
      x += xc[ch] * w;
      y += yc[ch] * w;
    }
    xs[s] = x;
    ys[s] = y;
    amps[s] = sqrtf(all);
  }
}

}  // namespace

extern "C" KS_API int ks_spike_positions(const float* tF, const int64_t* templ,
                                         const int64_t* iCC, const uint8_t* iCC_mask,
                                         const int64_t* iU, const double* xc, const double* yc,
                                         int64_t N, int64_t nC, int64_t P, int64_t C, int64_t K,
                                         double* xs, double* ys, float* amps, int* status,
                                         void* stream) {
  using namespace ks;
  if (N < 0 || nC < 1 || nC > 32 || P < 1 || C < 1 || K < 1)
    return fail(KS_ERR_ARG, "ks_spike_positions: need N >= 0, 1 <= nC <= 32, P, C, K >= 1");
  if (!status || (N > 0 && (!tF || !templ || !iCC || !iCC_mask || !iU || !xc || !yc || !xs ||
                            !ys || !amps)))
    return fail(KS_ERR_ARG, "ks_spike_positions: null pointer");
  if (N >= (1LL << 31)) return fail(KS_ERR_UNSUPPORTED, "ks_spike_positions: too many spikes");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  KS_CUDA(cudaMemsetAsync(status, 0, sizeof(int), s));
  if (N == 0) return KS_OK;
  const unsigned grid = (unsigned)std::min<int64_t>((N + 127) / 128, 65535);
  ks_spike_positions_kernel<<<grid, 128, 0, s>>>(tF, templ, iCC, iCC_mask, iU, xc, yc, (int)N,
                                                 (int)nC, (int)P, (int)C, (int)K, xs, ys, amps,
                                                 status);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}
