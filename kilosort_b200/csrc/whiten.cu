// Whitening of raw int16 samples on the tensor cores (the streaming front end).
//
//   X[c, t] = sum_c' Wrot[c, c'] * scale * raw[t, c']        (t < T, c < C)
//
// raw is the recording's own layout, samples x channels (channels of a sample
// contiguous), which is the K-major operand of the split-BF16 contraction
// kernel: int16 values are exact as bf16 hi + lo (|x| < 2^15 leaves at most 8
// significant bits in x - bf16(x)), so the only rounding is that of the
// whitening matrix, split into hi/lo as in the score contraction.  The scale
// is folded into the matrix.  The whitening of kilosort/io.py:1019-1025
// (X = whiten_mat @ X) on a batch of raw samples.
#include "ks_common.cuh"
#include "project.cuh"

#include <algorithm>

namespace {

// raw [T][ldr] int16 -> Y hi/lo [Tpad][Cq] bf16 (zero for t >= T or c >= C).
__global__ void ks_raw_split_kernel(const int16_t* __restrict__ raw, long long T, int C,
                                    long long ldr, int Cq, long long Tpad,
                                    __nv_bfloat16* __restrict__ Yhi,
                                    __nv_bfloat16* __restrict__ Ylo) {
  const long long n = Tpad * Cq;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const long long t = e / Cq;
    const int c = (int)(e - t * Cq);
    const float v = (t < T && c < C) ? (float)raw[t * ldr + c] : 0.f;
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    Yhi[e] = h;
    Ylo[e] = __float2bfloat16_rn(v - __bfloat162float(h));
  }
}

// scale * Wrot [C][C] -> hi/lo [Cpad][Cq] (zero padded).
__global__ void ks_wrot_split_kernel(const float* __restrict__ Wrot, int C, float scale,
                                     int Cpad, int Cq, __nv_bfloat16* __restrict__ Uhi,
                                     __nv_bfloat16* __restrict__ Ulo) {
  const long long n = (long long)Cpad * Cq;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e / Cq), c = (int)(e - (long long)r * Cq);
    const float v = (r < C && c < C) ? __fmul_rn(scale, Wrot[(long long)r * C + c]) : 0.f;
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    Uhi[e] = h;
    Ulo[e] = __float2bfloat16_rn(v - __bfloat162float(h));
  }
}

struct WhitenLayout {
  int64_t Cq, Cpad, Tpad;
  size_t err, uhi, ulo, yhi, ylo, bytes;
};

WhitenLayout whiten_layout(int64_t T, int64_t C) {
  WhitenLayout w;
  w.Cq = (C + 63) / 64 * 64;
  w.Cpad = (C + 127) / 128 * 128;
  w.Tpad = (T + 255) / 256 * 256;
  size_t o = 0;
  auto take = [&](size_t b) {
    const size_t at = o;
    o = ks::align256(o + b);
    return at;
  };
  w.err = take(256);
  w.uhi = take(2 * (size_t)w.Cpad * w.Cq);
  w.ulo = take(2 * (size_t)w.Cpad * w.Cq);
  w.yhi = take(2 * (size_t)w.Tpad * w.Cq);
  w.ylo = take(2 * (size_t)w.Tpad * w.Cq);
  w.bytes = o;
  return w;
}

}  // namespace

namespace ks {

int launch_matrix_split(const float* W, int64_t C, float scale, int64_t Cpad, int64_t Cq,
                        __nv_bfloat16* hi, __nv_bfloat16* lo, cudaStream_t stream) {
  const int g = (int)std::min<int64_t>(4096, (Cpad * Cq + 255) / 256);
  ks_wrot_split_kernel<<<g, 256, 0, stream>>>(W, (int)C, scale, (int)Cpad, (int)Cq, hi, lo);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

}  // namespace ks

extern "C" KS_API size_t ks_whiten_int16_workspace_size(int64_t T, int64_t C) {
  if (T < 1 || C < 1) return 0;
  return whiten_layout(T, C).bytes;
}

extern "C" KS_API int ks_whiten_int16(const int16_t* raw, int64_t T, int64_t C, int64_t ld_raw,
                                      const float* Wrot, float scale, float* X, int64_t ldx,
                                      int* status, void* workspace, size_t workspace_bytes,
                                      void* stream) {
  using namespace ks;
  if (!raw || !Wrot || !X || !status) return fail(KS_ERR_ARG, "ks_whiten_int16: null pointer");
  if (T < 1 || C < 1 || ld_raw < C || ldx < T)
    return fail(KS_ERR_ARG, "ks_whiten_int16: need T, C >= 1, ld_raw >= C, ldx >= T");
  if (T > 0x7fffffffLL || C > 65536) return fail(KS_ERR_UNSUPPORTED, "ks_whiten_int16: shape too large");
  const WhitenLayout w = whiten_layout(T, C);
  if (!workspace || workspace_bytes < w.bytes)
    return fail(KS_ERR_WORKSPACE, "ks_whiten_int16: workspace too small");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  char* base = static_cast<char*>(workspace);
  int* err = reinterpret_cast<int*>(base + w.err);
  __nv_bfloat16* uhi = reinterpret_cast<__nv_bfloat16*>(base + w.uhi);
  __nv_bfloat16* ulo = reinterpret_cast<__nv_bfloat16*>(base + w.ulo);
  __nv_bfloat16* yhi = reinterpret_cast<__nv_bfloat16*>(base + w.yhi);
  __nv_bfloat16* ylo = reinterpret_cast<__nv_bfloat16*>(base + w.ylo);
  KS_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  int rc = launch_matrix_split(Wrot, C, scale, w.Cpad, w.Cq, uhi, ulo, s);
  if (rc) return rc;
  const int gy = (int)std::min<int64_t>(8192, (w.Tpad * w.Cq + 255) / 256);
  ks_raw_split_kernel<<<gy, 256, 0, s>>>(raw, T, (int)C, ld_raw, (int)w.Cq, w.Tpad, yhi, ylo);
  KS_CUDA(cudaGetLastError());
  rc = gemm_bf16x3(uhi, ulo, yhi, ylo, X, C, T, w.Cq, w.Cpad, w.Tpad, ldx, false, err, s);
  if (rc) return rc;
  KS_CUDA(cudaMemcpyAsync(status, err, sizeof(int), cudaMemcpyDeviceToDevice, s));
  return KS_OK;
}
