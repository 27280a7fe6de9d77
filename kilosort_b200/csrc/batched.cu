// Many batches, several recordings, few persistent launches (ks_match_batches).
//
// Per call:
//   per recording   template energy nm, {nm, 1/nm} pairs, U reordered to
//                   [Kpad][Q] (bf16 hi/lo, or f32)
//   per batch       Xres <- X; temporal projection into the recording's
//                   stacked Y (split-BF16) or a shared Y buffer (FP32)
//   contraction     split-BF16: ONE grouped tcgen05 launch over the tiles of
//                   every batch of every recording (tensor maps per recording,
//                   tile table per batch, all in the kernel parameter);
//                   FP32: one SIMT contraction per batch, interleaved with its
//                   temporal projection so one Y buffer serves all batches
//   peel            ONE cooperative launch: the grid is split into teams of
//                   co-resident blocks; team t peels batches t, t+T, ... of a
//                   longest-first order with team-wide barriers; every loop ends
//                   on the device (no host round trip between iterations or
//                   batches)
//   residual        ONE launch over (batch, block, 32 channels)
// Nothing is copied from host memory and nothing synchronises the host, so the
// sequence can be captured in a CUDA graph and replayed.
#include "peel_core.cuh"
#include "gemm_group.cuh"

#include <algorithm>
#include <numeric>
#include <vector>

namespace {

constexpr int kMaxRecs = KS_MAX_RECORDINGS;
constexpr int kMaxBatches = KS_MAX_BATCHES;
static_assert(kMaxRecs <= ks::kGroupRecs && kMaxBatches <= ks::kGroupBatches,
              "grouped contraction tables too small");

struct MultiRec {
  const float* U;
  const float* W;
  const float* ctcT;
  const float* nm;
  const float2* nmi;
  const int* rperm;             // group order of the grouped update
  const float* mg;              // its product bounds [K][ng]
  const float2* nmip;           // {nm, 1/nm} in group order
  int C, K, P, nt;
  float th2;
  int max_peels;
  long long capacity;
};

struct MultiBatch {
  float* Bt;
  float* Xres;
  long long* st;
  float* amps;
  float* th_amps;
  long long* info;
  char* lists;
  int L;
  int rec;
};

struct MultiParams {
  MultiRec recs[kMaxRecs];
  MultiBatch batches[kMaxBatches];
  int order[kMaxBatches];       // batches, longest first
  int n_batches;
  int team_size;
  char* teams;                  // team scratch regions, team_bytes apart
  size_t team_bytes;
  unsigned long long limit_ns;
  const int* upstream_err;
  size_t peel_smem;             // dynamic shared bytes of the peel
};

__device__ void fill_args(const MultiParams& p, int b, char* team, PeelArgs& a) {
  const MultiBatch& mb = p.batches[b];
  const MultiRec& r = p.recs[mb.rec];
  a = PeelArgs{};
  a.Bt = mb.Bt;
  a.Xres = mb.Xres;
  a.U = r.U;
  a.W = r.W;
  a.ctcT = r.ctcT;
  a.nm = r.nm;
  a.nmi = r.nmi;
  a.C = r.C;
  a.L = mb.L;
  a.K = r.K;
  a.P = r.P;
  a.nt = r.nt;
  a.th2 = r.th2;
  a.max_peels = r.max_peels;
  a.capacity = r.capacity;
  a.st = mb.st;
  a.amps = mb.amps;
  a.th_amps = mb.th_amps;
  a.info = mb.info;
  bind_scratch(a, team, mb.lists, true);
  a.rperm = r.rperm;
  a.mg = r.mg;
  a.nmip = r.nmip;
  a.limit_ns = p.limit_ns;
  a.upstream_err = p.upstream_err;
#ifdef KS_PEEL_TRACE
  a.trace = 1;
#endif
}

// Team blockIdx.x / team_size peels its batches one after the other; the
// team's barrier count carries over from batch to batch.  After a batch's
// peel the same team applies its residual pass (record order per element, as
// ks_residual_kernel does), so one team's residual work fills the barrier
// waits of the others.  A team stops at its first error (info of its later
// batches keeps the "not run" value).
template <int kRows, bool kLean>
__device__ __forceinline__ void peel_multi_body(const MultiParams& p, char* smem_raw,
                                                PeelArgs& sa);

// Alone on the device: 2 blocks per SM (64 registers per thread).
__global__ void __launch_bounds__(kThreads, 2) peel_multi_kernel(const __grid_constant__ MultiParams p) {
  extern __shared__ __align__(16) char smem_raw[];
  __shared__ PeelArgs sa;
  peel_multi_body<kRowsPerWarp, false>(p, smem_raw, sa);
}

// The same with the lean group fold (group_tile<true>), for small teams: a
// team of at most kLeanTeamBlocks blocks works through tens of tiles per warp
// and phase, where fewer instructions per row pay; larger teams (few tiles
// per warp, phases bound by their barriers) measured faster with the other
// fold.  Results are identical.
constexpr int kLeanTeamBlocks = 16;
__global__ void __launch_bounds__(kThreads, 2)
peel_multi_kernel_lean(const __grid_constant__ MultiParams p) {
  extern __shared__ __align__(16) char smem_raw[];
  __shared__ PeelArgs sa;
  peel_multi_body<kRowsPerWarp, true>(p, smem_raw, sa);
}

// Beside the projection kernels of the next group: 1 block per SM capped at
// 80 registers per thread (40960 of the SM's 65536), which leaves room for a
// tensor-core contraction CTA (192 x 64) or a temporal-projection block
// (256 x 80) on the same SM.
__global__ void __maxnreg__(80) peel_multi_kernel_shared(const __grid_constant__ MultiParams p) {
  extern __shared__ __align__(16) char smem_raw[];
  __shared__ PeelArgs sa;
  peel_multi_body<kRowsPerWarp, false>(p, smem_raw, sa);
}

template <int kRows, bool kLean>
__device__ __forceinline__ void peel_multi_body(const MultiParams& p, char* smem_raw,
                                                PeelArgs& sa) {
  const int team = blockIdx.x / p.team_size;
  const int rank = blockIdx.x % p.team_size;
  const int n_teams = gridDim.x / p.team_size;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  char* tbase = p.teams + (size_t)team * p.team_bytes;
  unsigned epoch = 0;
  for (int i = team; i < p.n_batches; i += n_teams) {
    __syncthreads();
    if (threadIdx.x == 0) fill_args(p, p.order[i], tbase, sa);
    __syncthreads();
    const Smem s = carve_smem(sa, smem_raw, true);
    const PeelOutcome o = run_peel<kRows, true, kLean>(sa, s, rank, (unsigned)p.team_size, epoch);
    if (o.status != KS_OK) {
      if (o.status == KS_ERR_OVERFLOW) continue;   // that batch only
      break;
    }
    if (o.n_out > 0) {
      // the residual's per-warp lists and transpose tiles use the update's
      // stage tiles, which the peel of this batch no longer needs
      int* xl = reinterpret_cast<int*>(s.stage);
      ResSmem rs;
      rs.W = s.W;
      rs.xl_tau = xl;
      rs.xl_k = xl + kWarps * kXList;
      rs.xl_amp = reinterpret_cast<float*>(xl + 2 * kWarps * kXList);
      rs.xt = reinterpret_cast<float*>(xl + 3 * kWarps * kXList);
      const int xg = (sa.C + 31) / 32;
      const long long n_items = (long long)sa.nblk * xg;
      for (long long w = (long long)rank * kWarps + warp; w < n_items;
           w += (long long)p.team_size * kWarps)
        residual_item<true>(sa, rs, o.iters, o.n_out, (int)(w / xg), (int)(w % xg), lane, warp);
    }
  }
}

// -------------------------------------------------------------- host layout
struct RecPlan {
  int64_t Q, Kpad, rows;          // rows: stacked Lpad of its batches (split form)
  size_t nm, nmi, groups, uhi, ulo, uf, yhi, ylo;
};

struct BatchPlan {
  int64_t Lpad, row_off;
  size_t bt, lists;
};

struct Plan {
  std::vector<RecPlan> rec;
  std::vector<BatchPlan> bat;
  size_t ctl, yf, teams, team_bytes, bytes;
  int64_t maxL, maxK, maxYf;
  int n_teams;
};

int make_plan(const ks_rec_desc* recs, int64_t n_recs, const ks_batch_desc* batches,
              int64_t n_batches, int precision, int64_t teams, Plan& pl) {
  using namespace ks;
  if (n_recs < 1 || n_recs > kMaxRecs)
    return fail(KS_ERR_ARG, "ks_match_batches: 1.." + std::to_string(kMaxRecs) + " recordings");
  if (n_batches < 1 || n_batches > kMaxBatches)
    return fail(KS_ERR_ARG, "ks_match_batches: 1.." + std::to_string(kMaxBatches) + " batches per call");
  if (precision != KS_PROJ_FP32 && precision != KS_PROJ_BF16X3)
    return fail(KS_ERR_ARG, "ks_match_batches: unknown precision");
  pl.rec.assign(n_recs, RecPlan{});
  pl.bat.assign(n_batches, BatchPlan{});
  pl.maxL = 0;
  pl.maxK = 0;
  pl.maxYf = 0;
  for (int64_t r = 0; r < n_recs; ++r) {
    const ks_rec_desc& d = recs[r];
    if (!d.U || !d.W || !d.ctcT) return fail(KS_ERR_ARG, "ks_match_batches: null recording pointer");
    int rc = check_peel_shape(d.C, 1, d.K, d.P, d.nt, d.th2, d.max_peels, d.capacity);
    if (rc) return rc;
    const ProjLayout pj = proj_layout(d.C, 128, d.K, d.P, precision);
    pl.rec[r].Q = pj.Q;
    pl.rec[r].Kpad = pj.Kpad;
    pl.rec[r].rows = 0;
  }
  for (int64_t b = 0; b < n_batches; ++b) {
    const ks_batch_desc& d = batches[b];
    if (d.rec < 0 || d.rec >= n_recs) return fail(KS_ERR_ARG, "ks_match_batches: batch recording index");
    if (!d.X || !d.Xres || !d.st || !d.amps || !d.th_amps || !d.info)
      return fail(KS_ERR_ARG, "ks_match_batches: null batch pointer");
    const ks_rec_desc& r = recs[d.rec];
    int rc = check_peel_shape(r.C, d.L, r.K, r.P, r.nt, r.th2, r.max_peels, r.capacity);
    if (rc) return rc;
    pl.bat[b].Lpad = round_up(d.L, 128);
    pl.bat[b].row_off = pl.rec[d.rec].rows;
    pl.rec[d.rec].rows += pl.bat[b].Lpad;
    if (pl.rec[d.rec].rows > 0x7fffffffLL)
      return fail(KS_ERR_UNSUPPORTED, "ks_match_batches: too many samples for one recording");
    pl.maxL = std::max(pl.maxL, d.L);
    pl.maxK = std::max(pl.maxK, r.K);
    pl.maxYf = std::max(pl.maxYf, pl.bat[b].Lpad * pl.rec[d.rec].Q);
  }
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o = align256(o + bytes);
    return at;
  };
  pl.ctl = take(256);
  for (int64_t r = 0; r < n_recs; ++r) {
    RecPlan& rp = pl.rec[r];
    const ks_rec_desc& d = recs[r];
    rp.nm = take(sizeof(float) * d.K);
    rp.nmi = take(sizeof(float2) * d.K);
    rp.groups = take(group_tables_bytes(d.K));
    if (precision == KS_PROJ_BF16X3) {
      rp.uhi = take(2 * (size_t)rp.Kpad * rp.Q);
      rp.ulo = take(2 * (size_t)rp.Kpad * rp.Q);
      rp.yhi = take(2 * (size_t)rp.rows * rp.Q);
      rp.ylo = take(2 * (size_t)rp.rows * rp.Q);
    } else {
      rp.uf = take(4 * (size_t)rp.Kpad * rp.Q);
    }
  }
  pl.yf = precision == KS_PROJ_FP32 ? take(4 * (size_t)pl.maxYf) : 0;
  for (int64_t b = 0; b < n_batches; ++b) {
    const ks_batch_desc& d = batches[b];
    pl.bat[b].bt = take(sizeof(float) * (size_t)tiled_rows_floats(d.L, recs[d.rec].K));
    pl.bat[b].lists = take(list_layout(d.L).bytes);
  }
  int64_t t = teams;
  if (t <= 0) t = std::min<int64_t>(8, std::max<int64_t>(1, n_batches / 4));
  t = std::min<int64_t>(t, n_batches);
  pl.n_teams = (int)t;
  pl.team_bytes = al256(team_layout(pl.maxL, pl.maxK).bytes);
  pl.teams = take(pl.team_bytes * (size_t)t);
  pl.bytes = o;
  return KS_OK;
}

}  // namespace

extern "C" KS_API size_t ks_match_batches_workspace_size(const ks_rec_desc* recs, int64_t n_recs,
                                                        const ks_batch_desc* batches,
                                                        int64_t n_batches, int precision,
                                                        int64_t teams) {
  Plan pl;
  if (!recs || !batches || make_plan(recs, n_recs, batches, n_batches, precision, teams, pl))
    return 0;
  return pl.bytes;
}

namespace {

// Events that order the projection stream and the peel stream of a pipelined
// call (per host thread, created once, reused by every call).
cudaEvent_t pipeline_event(int i) {
  static thread_local std::vector<cudaEvent_t> ev;
  while ((int)ev.size() <= i) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
    ev.push_back(e);
  }
  return ev[i];
}

// Kernel and resident blocks per SM of the peel: alone on the device 2 blocks
// per SM; pipelined 1 block per SM, which leaves room on every SM for a block
// of the projection kernels of the next group.
struct PeelVariant {
  void (*kernel)(MultiParams);
  int blocks_per_sm;
};

PeelVariant peel_variant(bool pipelined) {
  if (pipelined) return PeelVariant{peel_multi_kernel_shared, 1};
  return PeelVariant{peel_multi_kernel, 2};
}

}  // namespace

extern "C" KS_API int ks_match_batches(const ks_rec_desc* recs, int64_t n_recs,
                                       const ks_batch_desc* batches, int64_t n_batches,
                                       int precision, int64_t teams, int64_t groups,
                                       void* workspace, size_t workspace_bytes, void* stream,
                                       void* aux_stream) {
  using namespace ks;
  if (!recs || !batches) return fail(KS_ERR_ARG, "ks_match_batches: null descriptor array");
  Plan pl;
  int rc = make_plan(recs, n_recs, batches, n_batches, precision, teams, pl);
  if (rc) return rc;
  if (!workspace || workspace_bytes < pl.bytes)
    return fail(KS_ERR_WORKSPACE, "ks_match_batches: workspace too small");
  if (reinterpret_cast<uintptr_t>(workspace) & 255)
    return fail(KS_ERR_ARG, "ks_match_batches: workspace must be 256-byte aligned");
  DeviceInfo dev;
  rc = device_info(&dev);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaStream_t ps = aux_stream ? static_cast<cudaStream_t>(aux_stream) : s;
  const int G = (aux_stream && aux_stream != stream)
                    ? (int)std::max<int64_t>(1, std::min<int64_t>(groups, n_batches)) : 1;
  const bool pipelined = G > 1;
  char* base = static_cast<char*>(workspace);
  int* gemm_err = reinterpret_cast<int*>(base + pl.ctl);
  trace_mark(0, s);
  KS_CUDA(cudaMemsetAsync(gemm_err, 0, sizeof(int), s));

  // per recording: nm, {nm, 1/nm}, reordered templates
  for (int64_t r = 0; r < n_recs; ++r) {
    const ks_rec_desc& d = recs[r];
    const RecPlan& rp = pl.rec[r];
    float* nm = reinterpret_cast<float*>(base + rp.nm);
    if ((rc = launch_template_energy(d.U, d.K, d.P, d.C, nm, s))) return rc;
    if ((rc = launch_nm_pairs(nm, d.K, reinterpret_cast<float2*>(base + rp.nmi), s))) return rc;
    if ((rc = launch_group_setup(d.U, d.ctcT, reinterpret_cast<const float2*>(base + rp.nmi), d.K,
                                 d.P, d.C, d.nt, base + rp.groups, s)))
      return rc;
    if (precision == KS_PROJ_BF16X3)
      rc = launch_reorder_templates(d.U, d.K, d.P, d.C, rp.Kpad, rp.Q, nullptr,
                                    reinterpret_cast<__nv_bfloat16*>(base + rp.uhi),
                                    reinterpret_cast<__nv_bfloat16*>(base + rp.ulo), s);
    else
      rc = launch_reorder_templates(d.U, d.K, d.P, d.C, rp.Kpad, rp.Q,
                                    reinterpret_cast<float*>(base + rp.uf), nullptr, nullptr, s);
    if (rc) return rc;
  }
  trace_mark(1, s);
  if (pipelined) {
    cudaEvent_t e = pipeline_event(0);
    if (!e) return fail(KS_ERR_CUDA, "ks_match_batches: cudaEventCreate failed");
    KS_CUDA(cudaEventRecord(e, s));
    KS_CUDA(cudaStreamWaitEvent(ps, e, 0));
  }

  // batches longest first; groups are consecutive runs of that order
  std::vector<int> order(n_batches);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    return batches[x].L * recs[batches[x].rec].K > batches[y].L * recs[batches[y].rec].K;
  });

  // batch table of the peel, shared by every group's launch
  static thread_local MultiParams mp;   // about 19 KB: kept off the stack
  for (int64_t r = 0; r < n_recs; ++r) {
    const ks_rec_desc& d = recs[r];
    MultiRec& m = mp.recs[r];
    m.U = d.U;
    m.W = d.W;
    m.ctcT = d.ctcT;
    m.nm = reinterpret_cast<const float*>(base + pl.rec[r].nm);
    m.nmi = reinterpret_cast<const float2*>(base + pl.rec[r].nmi);
    group_tables(base + pl.rec[r].groups, d.K, &m.rperm, &m.mg, &m.nmip);
    m.C = (int)d.C;
    m.K = (int)d.K;
    m.P = (int)d.P;
    m.nt = (int)d.nt;
    m.th2 = d.th2;
    m.max_peels = (int)d.max_peels;
    m.capacity = d.capacity;
  }
  size_t smem = 0;
  for (int64_t b = 0; b < n_batches; ++b) {
    const ks_batch_desc& d = batches[b];
    const ks_rec_desc& r = recs[d.rec];
    MultiBatch& m = mp.batches[b];
    m.Bt = reinterpret_cast<float*>(base + pl.bat[b].bt);
    m.Xres = d.Xres;
    m.st = reinterpret_cast<long long*>(d.st);
    m.amps = d.amps;
    m.th_amps = d.th_amps;
    m.info = reinterpret_cast<long long*>(d.info);
    m.lists = base + pl.bat[b].lists;
    m.L = (int)d.L;
    m.rec = (int)d.rec;
    const int nchunks = (int)((d.L + kChunk - 1) / kChunk);
    const int nblk = (int)((d.L + kCol - 1) / kCol);
    const int nwords = (nblk + 31) / 32;
    smem = std::max(smem, smem_bytes((int)r.P, (int)r.nt, nchunks, nwords, true));
  }
  mp.teams = base + pl.teams;
  mp.team_bytes = pl.team_bytes;
  mp.limit_ns = wait_limit_ns();
  mp.upstream_err = precision == KS_PROJ_BF16X3 ? gemm_err : nullptr;
  smem = (smem + 15) & ~size_t(15);
  mp.peel_smem = smem;
  const PeelVariant pv = peel_variant(pipelined);
  cudaFuncAttributes fa;
  KS_CUDA(cudaFuncGetAttributes(&fa, pv.kernel));
  if (smem + fa.sharedSizeBytes > dev.smem_optin)
    return fail(KS_ERR_UNSUPPORTED, "ks_match_batches: batch too long for shared memory");
  KS_CUDA(cudaFuncSetAttribute(pv.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  KS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, pv.kernel, kThreads, smem));
  if (occ < 1) return fail(KS_ERR_UNSUPPORTED, "ks_match_batches: peel does not fit on an SM");
  const int max_blocks = dev.sm_count * std::min(occ, pv.blocks_per_sm);

  static thread_local GemmGroup g;      // about 14 KB: kept off the stack
  if (precision == KS_PROJ_BF16X3) {
    for (int64_t r = 0; r < n_recs; ++r) {
      const RecPlan& rp = pl.rec[r];
      g.nk[r] = (int)(rp.Q / 64);
      if (rp.rows == 0) continue;
      const __nv_bfloat16* uhi = reinterpret_cast<const __nv_bfloat16*>(base + rp.uhi);
      const __nv_bfloat16* ulo = reinterpret_cast<const __nv_bfloat16*>(base + rp.ulo);
      const __nv_bfloat16* yhi = reinterpret_cast<const __nv_bfloat16*>(base + rp.yhi);
      const __nv_bfloat16* ylo = reinterpret_cast<const __nv_bfloat16*>(base + rp.ylo);
      if ((rc = make_bf16_map(&g.maps[r][0], uhi, rp.Kpad, rp.Q, gemm_tile_m()))) return rc;
      if ((rc = make_bf16_map(&g.maps[r][1], ulo, rp.Kpad, rp.Q, gemm_tile_m()))) return rc;
      if ((rc = make_bf16_map(&g.maps[r][2], yhi, rp.rows, rp.Q, gemm_tile_n()))) return rc;
      if ((rc = make_bf16_map(&g.maps[r][3], ylo, rp.rows, rp.Q, gemm_tile_n()))) return rc;
    }
    g.tiled = 1;
    g.err = gemm_err;
  }

  for (int gi = 0; gi < G; ++gi) {
    const int i0 = (int)(n_batches * gi / G), i1 = (int)(n_batches * (gi + 1) / G);
    // projections of the group's batches (on the projection stream)
    for (int i = i0; i < i1; ++i) {
      const int b = order[i];
      const ks_batch_desc& d = batches[b];
      const ks_rec_desc& r = recs[d.rec];
      const RecPlan& rp = pl.rec[d.rec];
      const BatchPlan& bp = pl.bat[b];
      if (d.Xres != d.X)
        KS_CUDA(cudaMemcpyAsync(d.Xres, d.X, sizeof(float) * r.C * d.L, cudaMemcpyDeviceToDevice, ps));
      KS_CUDA(cudaMemsetAsync(d.info, 0xff, 4 * sizeof(int64_t), ps));   // "not run" until the peel writes it
      float* Bt = reinterpret_cast<float*>(base + bp.bt);
      if (precision == KS_PROJ_BF16X3) {
        __nv_bfloat16* yhi = reinterpret_cast<__nv_bfloat16*>(base + rp.yhi) + (size_t)bp.row_off * rp.Q;
        __nv_bfloat16* ylo = reinterpret_cast<__nv_bfloat16*>(base + rp.ylo) + (size_t)bp.row_off * rp.Q;
        if ((rc = launch_temporal(d.X, r.W, r.C, d.L, r.P, r.nt, rp.Q, bp.Lpad, nullptr, yhi, ylo, gemm_err,
                                   ps)))
          return rc;
      } else {
        float* yf = reinterpret_cast<float*>(base + pl.yf);
        if ((rc = launch_temporal(d.X, r.W, r.C, d.L, r.P, r.nt, rp.Q, bp.Lpad, yf, nullptr, nullptr,
                                   nullptr, ps)))
          return rc;
        if ((rc = sgemm_tn(reinterpret_cast<const float*>(base + rp.uf), yf, Bt, r.K, d.L, rp.Q, 0, ps,
                           true)))
          return rc;
      }
    }
    if (precision == KS_PROJ_BF16X3) {
      long long tiles = 0;
      for (int i = i0; i < i1; ++i) {
        const int b = order[i];
        const ks_batch_desc& d = batches[b];
        GemmBatch& gb = g.batches[i - i0];
        gb.B = reinterpret_cast<float*>(base + pl.bat[b].bt);
        gb.ldb = 0;
        gb.K = (int)recs[d.rec].K;
        gb.L = (int)d.L;
        gb.rec = (int)d.rec;
        gb.row_off = (int)pl.bat[b].row_off;
        gb.tiles_m = (int)(pl.rec[d.rec].Kpad / gemm_tile_m());
        gb.tile_begin = (int)tiles;
        tiles += (long long)gb.tiles_m * ((d.L + gemm_tile_n() - 1) / gemm_tile_n());
      }
      if (tiles > 0x7fffffffLL) return fail(KS_ERR_UNSUPPORTED, "ks_match_batches: too many tiles");
      g.n_batches = i1 - i0;
      g.n_tiles = (int)tiles;
      if ((rc = launch_gemm_group(g, ps))) return rc;
    }
    if (pipelined) {
      cudaEvent_t e = pipeline_event(gi + 1);
      if (!e) return fail(KS_ERR_CUDA, "ks_match_batches: cudaEventCreate failed");
      KS_CUDA(cudaEventRecord(e, ps));
      KS_CUDA(cudaStreamWaitEvent(s, e, 0));
    }
    if (gi == 0) trace_mark(2, s);
    // the group's peels and residual passes: one cooperative launch of teams
    const int nb = i1 - i0;
    const int n_teams = std::min(pl.n_teams, nb);
    if (n_teams > max_blocks) return fail(KS_ERR_UNSUPPORTED, "ks_match_batches: more teams than resident blocks");
    for (int i = i0; i < i1; ++i) mp.order[i - i0] = order[i];
    mp.n_batches = nb;
    mp.team_size = max_blocks / n_teams;
    for (int t = 0; t < n_teams; ++t)
      KS_CUDA(cudaMemsetAsync(base + pl.teams + (size_t)t * pl.team_bytes, 0, 256, s));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.gridDim = dim3(mp.team_size * n_teams);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void (*kernel)(MultiParams) = pv.kernel;
    if (pv.kernel == peel_multi_kernel && mp.team_size <= kLeanTeamBlocks) {
      // small teams: the lean fold, if it is as resident as the other form
      KS_CUDA(cudaFuncSetAttribute(peel_multi_kernel_lean,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      int occ_lean = 0;
      KS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_lean, peel_multi_kernel_lean,
                                                            kThreads, smem));
      if (dev.sm_count * std::min(occ_lean, pv.blocks_per_sm) >= max_blocks)
        kernel = peel_multi_kernel_lean;
    }
    KS_CUDA(cudaLaunchKernelEx(&cfg, kernel, mp));
  }
  // the residual passes ran inside the peel launches
  trace_mark(3, s);
  trace_mark(4, s);
  return KS_OK;
}
