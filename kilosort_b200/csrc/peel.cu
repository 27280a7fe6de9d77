// Single-batch launch of the greedy peel (device code in peel_core.cuh):
// one team made of the whole cooperative grid, then the residual pass.
#include "peel_core.cuh"

namespace ks {

size_t peel_scratch_size(int64_t L, int64_t K) {
  return al256(team_layout(L).bytes) + al256(list_layout(L).bytes) + al256(8 * (size_t)K);
}

int64_t tiled_rows_floats(int64_t L, int64_t K) { return ((L + kCol - 1) / kCol) * K * kCol; }

int launch_tile_rows(const float* B, int64_t ldb, int64_t K, int64_t L, float* Bt,
                     cudaStream_t stream) {
  const int nblk = (int)((L + kCol - 1) / kCol);
  ks_tile_rows_kernel<<<2048, 256, 0, stream>>>(B, ldb, (int)K, (int)L, nblk, Bt);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

int launch_untile_rows(const float* Bt, int64_t K, int64_t L, float* B, int64_t ldb,
                       cudaStream_t stream) {
  ks_untile_rows_kernel<<<2048, 256, 0, stream>>>(Bt, (int)K, (int)L, B, ldb);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

int launch_ctc_transpose(const float* ctc, int64_t K, int64_t nt, float* ctcT,
                         cudaStream_t stream) {
  if (!ctc || !ctcT || K < 1 || nt < 1) return fail(KS_ERR_ARG, "ks_ctc_transpose: bad args");
  if (ctc == ctcT) return fail(KS_ERR_ARG, "ks_ctc_transpose: in-place transpose is not supported");
  const long long rows = K * K;
  const int grid = (int)std::min<long long>(rows, 65535LL * 4);
  ks_ctc_transpose_kernel<<<grid, 128, 0, stream>>>(ctc, (int)K, (int)(2 * nt + 1), ctcT);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

int check_peel_shape(int64_t C, int64_t L, int64_t K, int64_t P, int64_t nt, float th2,
                     int64_t max_peels, int64_t capacity) {
  if (C < 1 || L < 1 || K < 1 || P < 1 || nt < 1 || (nt % 2) == 0)
    return fail(KS_ERR_ARG, "ks_peel: need C,L,K,P >= 1 and odd nt");
  if (L > (int64_t)kMaxChunks * kChunk || K > kMaxTemplates || C > (1 << 24) || nt > 1023 ||
      P > 8)
    return fail(KS_ERR_UNSUPPORTED, "ks_peel: shape beyond supported limits");
  if (capacity < 0 || max_peels < 0) return fail(KS_ERR_ARG, "ks_peel: negative capacity/max_peels");
  if (max_peels > kMaxIters) return fail(KS_ERR_UNSUPPORTED, "ks_peel: max_peels above 4096");
  if (capacity > 0x7fffffffLL) return fail(KS_ERR_UNSUPPORTED, "ks_peel: capacity above 2^31-1");
  if (!(th2 >= 0.f)) return fail(KS_ERR_ARG, "ks_peel: th2 must be a non-negative number");
  return KS_OK;
}

int launch_nm_pairs(const float* nm, int64_t K, float2* nmi, cudaStream_t stream) {
  ks_nm_pair_kernel<<<(unsigned)((K + 255) / 256), 256, 0, stream>>>(nm, (int)K, nmi);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

// Blocks per SM of the peel kernel for a given dynamic shared-memory size.
int peel_occupancy(const DeviceInfo& dev, size_t smem, const void* kernel, int* occ_out) {
  static thread_local int cached_dev = -1;
  static thread_local size_t cached_smem = 0;
  static thread_local const void* cached_kernel = nullptr;
  static thread_local int cached_occ = 0;
  if (cached_dev != dev.device || cached_smem != smem || cached_kernel != kernel) {
    KS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    KS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kThreads, smem));
    if (occ < 1) return fail(KS_ERR_UNSUPPORTED, "ks_peel: kernel does not fit on an SM");
    cached_dev = dev.device; cached_smem = smem; cached_kernel = kernel; cached_occ = occ;
  }
  *occ_out = cached_occ;
  return KS_OK;
}

int launch_peel_tiled(float* Bt, float* Xres, const float* U, const float* W,
                      const float* ctcT, const float* nm, int64_t C, int64_t L, int64_t K,
                      int64_t P, int64_t nt, float th2, int64_t max_peels,
                      int64_t capacity, int64_t* st, float* amps, float* th_amps,
                      int64_t* info, void* ws, size_t ws_bytes, cudaStream_t stream,
                      unsigned long long limit_ns, const int* upstream_err) {
  if (!Bt || !Xres || !U || !W || !ctcT || !nm || !st || !amps || !th_amps || !info)
    return fail(KS_ERR_ARG, "ks_peel: null pointer");
  int rc = check_peel_shape(C, L, K, P, nt, th2, max_peels, capacity);
  if (rc) return rc;
  if (ws_bytes < peel_scratch_size(L, K) || !ws)
    return fail(KS_ERR_WORKSPACE, "ks_peel: workspace too small");

  DeviceInfo dev;
  rc = device_info(&dev);
  if (rc) return rc;

  PeelArgs a{};
  a.Bt = Bt; a.Xres = Xres; a.U = U; a.W = W; a.ctcT = ctcT; a.nm = nm;
  a.C = (int)C; a.L = (int)L; a.K = (int)K; a.P = (int)P; a.nt = (int)nt;
  a.th2 = th2;
  a.max_peels = (int)max_peels;
  a.capacity = capacity;
  a.st = reinterpret_cast<long long*>(st); a.amps = amps; a.th_amps = th_amps;
  a.info = reinterpret_cast<long long*>(info);
  char* base = static_cast<char*>(ws);
  const size_t team_bytes = al256(team_layout(L).bytes);
  const size_t list_bytes = al256(list_layout(L).bytes);
  bind_scratch(a, base, base + team_bytes);
  float2* nmi = reinterpret_cast<float2*>(base + team_bytes + list_bytes);
  a.nmi = nmi;
  a.limit_ns = limit_ns;
  a.upstream_err = upstream_err;
#ifdef KS_PEEL_TRACE
  a.trace = 1;
#endif

  const size_t smem = smem_bytes(a.P, a.nt, a.nchunks, a.nwords);
  if (smem > dev.smem_optin) return fail(KS_ERR_UNSUPPORTED, "ks_peel: batch too long for shared memory");
  int occ = 0;
  rc = peel_occupancy(dev, smem, (const void*)peel_kernel, &occ);
  if (rc) return rc;
  const int grid = dev.sm_count * occ;
  KS_CUDA(cudaMemsetAsync(base, 0, 256, stream));       // barrier count and error word
  rc = launch_nm_pairs(nm, K, nmi, stream);
  if (rc) return rc;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  trace_mark(2, stream);
  KS_CUDA(cudaLaunchKernelEx(&cfg, peel_kernel, a));
  trace_mark(3, stream);
  // residual updates of all recorded spikes
  const long long n_res = (long long)a.nblk * ((C + 31) / 32);
  const unsigned rgrid = (unsigned)((n_res + kResWarps - 1) / kResWarps);
  ks_residual_kernel<<<rgrid, kResThreads, residual_smem_bytes(a.P, a.nt), stream>>>(a);
  KS_CUDA(cudaGetLastError());
  trace_mark(4, stream);
  return KS_OK;
}

}  // namespace ks
