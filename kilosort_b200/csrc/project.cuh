// Internal interfaces of the projection kernels.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ks {

constexpr int kGroupRecs = 8;       // recordings in one grouped contraction
constexpr int kGroupBatches = 256;  // batches in one grouped contraction
struct GemmGroup;
// Grouped split-BF16 contraction over the tiles of several batches/recordings
// (gemm_bf16x3.cu); the caller fills maps, nk, batches, n_batches, n_tiles, tiled, err.
int launch_gemm_group(GemmGroup& g, cudaStream_t stream);
// Tensor map of a bf16 [rows][cols] operand, boxes of box_rows x 64.
int make_bf16_map(CUtensorMap* map, const __nv_bfloat16* ptr, int64_t rows, int64_t cols,
                  int box_rows);
// Tensor map of a bf16 [rows][cols] array with a row stride (elements), no
// swizzle, boxes of box_rows x box_cols: the destination of TMA stores.
int make_bf16_store_map(CUtensorMap* map, const __nv_bfloat16* ptr, int64_t rows, int64_t cols,
                        int64_t row_stride, int box_cols, int box_rows);
int gemm_tile_n();
int gemm_tile_m();

struct ProjLayout {
  int64_t Q;      // contraction length, q = c*P + p, padded to 64
  int64_t Lpad;   // rows of the temporal projection (time), padded to 128
  int64_t Kpad;   // template rows, padded to 128
  size_t bytes;   // workspace bytes
};
ProjLayout proj_layout(int64_t C, int64_t L, int64_t K, int64_t P, int precision);

int launch_template_energy(const float* U, int64_t K, int64_t P, int64_t C,
                           float* nm, cudaStream_t stream);
// U [K,P,C] -> [Kpad][Q] (q = c*P + p, zero padded): f32 (Uf) and/or bf16 hi/lo.
int launch_reorder_templates(const float* U, int64_t K, int64_t P, int64_t C, int64_t Kpad,
                             int64_t Q, float* Uf, __nv_bfloat16* Uhi, __nv_bfloat16* Ulo,
                             cudaStream_t stream);
// X [C,L] -> Y [Lpad][Q] rows (f32 and/or bf16 hi/lo); Y is written for rows < Lpad.
// The split form alone (Yhi/Ylo without Yf) runs on the tensor cores when the
// shape allows it and err (the device error word of its bounded waits) is given.
int launch_temporal(const float* X, const float* W, int64_t C, int64_t L, int64_t P,
                    int64_t nt, int64_t Q, int64_t Lpad, float* Yf, __nv_bfloat16* Yhi,
                    __nv_bfloat16* Ylo, int* err, cudaStream_t stream);
// FP32 temporal projection with rows (channel, component) and samples
// contiguous: YT[(c * P + p) * ldyt + tau], tau < Lpad (a multiple of 128).
int launch_temporal_rows(const float* X, const float* W, int64_t C, int64_t L, int64_t P,
                         int64_t nt, int64_t Lpad, float* YT, int64_t ldyt,
                         cudaStream_t stream);
// Split-BF16 temporal projection on tcgen05 (temporal_tc.cu); KS_ERR_UNSUPPORTED
// (nothing launched) for shapes it does not cover (odd P, P > 8, nt > 121).
int launch_temporal_split_tc(const float* X, const float* W, int64_t C, int64_t L, int64_t P,
                             int64_t nt, int64_t Q, int64_t Lpad, __nv_bfloat16* Yhi,
                             __nv_bfloat16* Ylo, int* err, cudaStream_t stream);
// scale * W [C][C] -> bf16 hi/lo [Cpad][Cq] (zero padded): the A operand of a
// split-BF16 contraction over channels (whiten.cu).
int launch_matrix_split(const float* W, int64_t C, float scale, int64_t Cpad, int64_t Cq,
                        __nv_bfloat16* hi, __nv_bfloat16* lo, cudaStream_t stream);
int zero_q_padding(int64_t C, int64_t P, int64_t Q, int64_t Lpad, float* Yf, __nv_bfloat16* Yhi,
                   __nv_bfloat16* Ylo, cudaStream_t stream);
// B is written row-major [K, ldb] or, when tiled, in 32-column blocks
// [ceil(L/32)][K][32] (the layout of the peel).
// The first 256 bytes of the workspace hold the device error word of the
// tensor-core contraction (zeroed here); with err_out the word is also copied
// there after the contraction.
int launch_project(const float* X, const float* U, const float* W, int64_t C,
                   int64_t L, int64_t K, int64_t P, int64_t nt, int precision,
                   float* B, int64_t ldb, bool tiled, void* ws, size_t ws_bytes,
                   int* err_out, cudaStream_t stream);
int sgemm_tn(const float* A, const float* Bt, float* Cm, int64_t M, int64_t N,
             int64_t Kd, int64_t ldc, cudaStream_t stream, bool tiled);
// High-pass FIR as a split-BF16 tcgen05 product with the Toeplitz matrix of
// the taps (fir_tc.cu).  P hi/lo [C][cols] is the batch padded circularly
// (P[c][j] = x[c][(j - h) mod L]) with cols = fir_tc_cols(rows, ntaps); the
// output is rows x Cq bf16 hi/lo (yhi non-null; zeros past L and C) or f32
// X[c][ldx]; |y| >= thr sets *art when check.  H hi/lo: scratch of
// fir_tc_toeplitz_bytes(ntaps) / 2 bytes each.
int64_t fir_tc_kpad(int ntaps);
int64_t fir_tc_cols(int64_t rows, int ntaps);
size_t fir_tc_toeplitz_bytes(int ntaps);
int fir_tc(const float* taps, int ntaps, const __nv_bfloat16* p_hi, const __nv_bfloat16* p_lo,
           int64_t C, int64_t L, int64_t cols, int64_t rows, __nv_bfloat16* h_hi,
           __nv_bfloat16* h_lo, bool check, float thr, float* X, int64_t ldx,
           __nv_bfloat16* yhi, __nv_bfloat16* ylo, int64_t Cq, int* art, int* err,
           cudaStream_t stream);
// Split-BF16 contraction on tcgen05: B = Uhi*Yhi^T + Uhi*Ylo^T + Ulo*Yhi^T.
int gemm_bf16x3(const __nv_bfloat16* Uhi, const __nv_bfloat16* Ulo,
                const __nv_bfloat16* Yhi, const __nv_bfloat16* Ylo, float* B,
                int64_t K, int64_t L, int64_t Q, int64_t Kpad, int64_t Lpad,
                int64_t ldb, bool tiled, int* err, cudaStream_t stream);

// Peel on a tiled score matrix Bt [ceil(L/32)][K][32] and a transposed
// cross-correlation ctcT[k][j][lag] = ctc[j][k][lag].
// grouped: the update that skips exact no-op (column, template group) pairs
// (scratch for its metadata and tables); otherwise every row of a touched
// column is rewritten.
size_t peel_scratch_size(int64_t L, int64_t K, bool grouped);
// Tables of the grouped update for one template set (group order, bounds,
// {nm, 1/nm} in group order), built on the stream by launch_group_setup.
size_t group_tables_bytes(int64_t K);
int launch_group_setup(const float* U, const float* ctcT, const float2* nmi, int64_t K,
                       int64_t P, int64_t C, int64_t nt, void* tables, cudaStream_t stream);
void group_tables(void* tables, int64_t K, const int** rperm, const float** mg,
                  const float2** nmip);
int64_t tiled_rows_floats(int64_t L, int64_t K);
int launch_tile_rows(const float* B, int64_t ldb, int64_t K, int64_t L, float* Bt,
                     cudaStream_t stream);
int launch_untile_rows(const float* Bt, int64_t K, int64_t L, float* B, int64_t ldb,
                       cudaStream_t stream);
int launch_ctc_transpose(const float* ctc, int64_t K, int64_t nt, float* ctcT,
                         cudaStream_t stream);
int check_peel_shape(int64_t C, int64_t L, int64_t K, int64_t P, int64_t nt, float th2,
                     int64_t max_peels, int64_t capacity);
int launch_nm_pairs(const float* nm, int64_t K, float2* nmi, cudaStream_t stream);
int launch_peel_tiled(float* Bt, float* Xres, const float* U, const float* W,
                      const float* ctcT, const float* nm, int64_t C, int64_t L, int64_t K,
                      int64_t P, int64_t nt, float th2, int64_t max_peels,
                      int64_t capacity, int64_t* st, float* amps, float* th_amps,
                      int64_t* info, void* ws, size_t ws_bytes, cudaStream_t stream,
                      unsigned long long limit_ns, const int* upstream_err, bool grouped);

}  // namespace ks
