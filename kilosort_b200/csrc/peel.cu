// Single-batch launch of the greedy peel (device code in peel_core.cuh):
// one team made of the whole cooperative grid, then the residual pass.
#include "peel_core.cuh"

namespace ks {

// Scratch of one single-batch peel: [team region] [lists] [nmi 8K], and for
// the grouped update its tables (group_tables_bytes).
// Tables of the grouped update: [rperm 4K] [key 4K] [mg 4*K*ng] [nmip 8K].
static size_t group_setup_bytes(int64_t K) {
  return al256(4 * (size_t)K) + al256(4 * (size_t)K) + al256(4 * (size_t)K * n_groups(K)) +
         al256(8 * (size_t)K);
}

size_t peel_scratch_size(int64_t L, int64_t K, bool grouped) {
  return al256(team_layout(L, grouped ? K : 0).bytes) + al256(list_layout(L).bytes) +
         al256(8 * (size_t)K) + (grouped ? group_setup_bytes(K) : 0);
}

size_t group_tables_bytes(int64_t K) { return group_setup_bytes(K); }

struct GroupTables {
  int* rperm;
  float* key;
  float* mg;
  float2* nmip;
};

static GroupTables group_tables_at(void* tables, int64_t K) {
  char* base = static_cast<char*>(tables);
  const size_t k4 = al256(4 * (size_t)K);
  GroupTables t;
  t.rperm = reinterpret_cast<int*>(base);
  t.key = reinterpret_cast<float*>(base + k4);
  t.mg = reinterpret_cast<float*>(base + 2 * k4);
  t.nmip = reinterpret_cast<float2*>(base + 2 * k4 + al256(4 * (size_t)K * n_groups(K)));
  return t;
}

// Group order, product bounds and permuted {nm, 1/nm} of the grouped update
// for one template set (ctcT in the transposed layout, nmi from
// launch_nm_pairs), written into tables (group_tables_bytes(K)).
int launch_group_setup(const float* U, const float* ctcT, const float2* nmi, int64_t K,
                       int64_t P, int64_t C, int64_t nt, void* tables, cudaStream_t stream) {
  const GroupTables t = group_tables_at(tables, K);
  const int ng = n_groups(K);
  ks_template_key_kernel<<<(unsigned)((K * 32 + 255) / 256), 256, 0, stream>>>(U, (int)K, (int)P,
                                                                              (int)C, t.key);
  KS_CUDA(cudaGetLastError());
  ks_group_order_kernel<<<(unsigned)((K + 255) / 256), 256, 0, stream>>>(t.key, (int)K, t.rperm);
  KS_CUDA(cudaGetLastError());
  const long long items = K * (long long)ng;
  ks_group_bound_kernel<<<(unsigned)std::min<long long>(items, 1 << 20), 256, 0, stream>>>(
      ctcT, t.rperm, (int)K, (int)(2 * nt + 1), ng, t.mg);
  KS_CUDA(cudaGetLastError());
  ks_group_nmi_kernel<<<(unsigned)((K + 255) / 256), 256, 0, stream>>>(nmi, t.rperm, (int)K,
                                                                      t.nmip);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

void group_tables(void* tables, int64_t K, const int** rperm, const float** mg,
                  const float2** nmip) {
  const GroupTables t = group_tables_at(tables, K);
  *rperm = t.rperm;
  *mg = t.mg;
  *nmip = t.nmip;
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
                      unsigned long long limit_ns, const int* upstream_err, bool grouped) {
  if (!Bt || !Xres || !U || !W || !ctcT || !nm || !st || !amps || !th_amps || !info)
    return fail(KS_ERR_ARG, "ks_peel: null pointer");
  int rc = check_peel_shape(C, L, K, P, nt, th2, max_peels, capacity);
  if (rc) return rc;
  if (ws_bytes < peel_scratch_size(L, K, grouped) || !ws)
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
  const size_t team_bytes = al256(team_layout(L, grouped ? K : 0).bytes);
  const size_t list_bytes = al256(list_layout(L).bytes);
  bind_scratch(a, base, base + team_bytes, grouped);
  float2* nmi = reinterpret_cast<float2*>(base + team_bytes + list_bytes);
  a.nmi = nmi;
  void* tables = base + team_bytes + list_bytes + al256(8 * (size_t)K);
  if (grouped) group_tables(tables, K, &a.rperm, &a.mg, &a.nmip);
  a.limit_ns = limit_ns;
  a.upstream_err = upstream_err;
#ifdef KS_PEEL_TRACE
  a.trace = 1;
#endif

  const size_t smem = smem_bytes(a.P, a.nt, a.nchunks, a.nwords, grouped);
  if (smem > dev.smem_optin) return fail(KS_ERR_UNSUPPORTED, "ks_peel: batch too long for shared memory");
  void (*kernel)(PeelArgs) = grouped ? peel_kernel<true> : peel_kernel<false>;
  int occ = 0;
  rc = peel_occupancy(dev, smem, (const void*)kernel, &occ);
  if (rc) return rc;
  const int grid = dev.sm_count * occ;
  KS_CUDA(cudaMemsetAsync(base, 0, 256, stream));       // barrier count and error word
  rc = launch_nm_pairs(nm, K, nmi, stream);
  if (rc) return rc;
  if (grouped) {
    rc = launch_group_setup(U, ctcT, nmi, K, P, C, nt, tables, stream);
    if (rc) return rc;
  }
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
  KS_CUDA(cudaLaunchKernelEx(&cfg, kernel, a));
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
