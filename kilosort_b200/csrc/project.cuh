// Internal interfaces of the projection kernels.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ks {

struct ProjLayout {
  int64_t Q;      // contraction length, q = c*P + p, padded to 64
  int64_t Lpad;   // rows of the temporal projection (time), padded to 128
  int64_t Kpad;   // template rows, padded to 128
  size_t bytes;   // workspace bytes
};
ProjLayout proj_layout(int64_t C, int64_t L, int64_t K, int64_t P, int precision);

int launch_template_energy(const float* U, int64_t K, int64_t P, int64_t C,
                           float* nm, cudaStream_t stream);
int launch_project(const float* X, const float* U, const float* W, int64_t C,
                   int64_t L, int64_t K, int64_t P, int64_t nt, int precision,
                   float* B, int64_t ldb, void* ws, size_t ws_bytes,
                   cudaStream_t stream);
int sgemm_tn(const float* A, const float* Bt, float* Cm, int64_t M, int64_t N,
             int64_t Kd, int64_t ldc, cudaStream_t stream);
// Split-BF16 contraction on tcgen05: B = Uhi*Yhi^T + Uhi*Ylo^T + Ulo*Yhi^T.
int gemm_bf16x3(const __nv_bfloat16* Uhi, const __nv_bfloat16* Ulo,
                const __nv_bfloat16* Yhi, const __nv_bfloat16* Ylo, float* B,
                int64_t K, int64_t L, int64_t Q, int64_t Kpad, int64_t Lpad,
                int64_t ldb, cudaStream_t stream);

size_t peel_workspace_size(int64_t L);
int launch_peel(float* B, int64_t ldb, float* Xres, const float* U,
                const float* W, const float* ctc, const float* nm, int64_t C,
                int64_t L, int64_t K, int64_t P, int64_t nt, float th2,
                int64_t max_peels, int64_t capacity, int64_t* st, float* amps,
                float* th_amps, int64_t* info, void* ws, size_t ws_bytes,
                cudaStream_t stream, unsigned long long limit_ns);

}  // namespace ks
