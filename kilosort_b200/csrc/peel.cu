// Greedy peel (matching pursuit) of one batch as a single persistent,
// cooperative kernel.  Semantics follow kilosort/template_matching.py:183-244.
//
// Layout in HBM
//   B      [K, ldb]  float32 score matrix, updated in place
//   Xres   [C, L]    float32 residual, updated in place
//   ctc    [K, K, 2nt+1] float32, read as ctc[j, k_spike, lag]
//   cfmax  [L] float32 / imax [L] int32: best score relu(B)^2/nm over templates
//                                        and its template, per column
//   chunk buffers: peaks found per 512-column chunk in one iteration
//
// One iteration = two phases separated by device-wide barriers:
//   DETECT  per chunk: pooled = max of cfmax over +-nt; a column is a peak iff
//           pooled > th2 and |pooled - cfmax| < 1e-9 (kilosort :206-212).
//           Peaks are compacted in time order; amplitude B[k,tau]/nm[k] and
//           sqrt(pooled) are taken from the pre-subtraction B (:225-229);
//           32-column blocks within +-nt of a peak are flagged dirty.
//   UPDATE  every block computes the exclusive prefix of the chunk counts, so
//           the global (iteration-local) index of each peak is known; records
//           are written in (iteration, tau) order; each dirty 32-column block
//           applies, column by column, the subtractions B[j,c] -= amp*ctc[j,k,
//           c-tau+nt] of the peaks that touch it -- even-indexed peaks first,
//           then odd-indexed ones, exactly the order of the reference's two
//           interleaved groups (:235-238), with separately rounded product and
//           difference -- and recomputes cfmax/imax of its columns from the
//           updated values.  Xres windows are updated per peak (:237).
// The loop ends when no peak is found or after max_peels iterations, decided
// identically by every block from the same counts.
#include "ks_common.cuh"

#include <cooperative_groups.h>

namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kChunk = 512;     // detection chunk, one column per thread
constexpr int kCol = 32;        // update block, one column per lane
constexpr int kMaxTouch = 64;   // peaks touching one update block (ties incl.)
constexpr int kMaxChunks = 8192;
constexpr int kRows = 4;        // rows in flight per warp in the update loop

struct PeelArgs {
  float* B;
  long long ldb;
  float* Xres;
  const float* U;
  const float* W;
  const float* ctc;
  const float* nm;
  int C, L, K, P, nt;
  float th2;
  int max_peels;
  long long capacity;
  long long* st;
  float* amps;
  float* th_amps;
  long long* info;
  // scratch
  float* cfmax;
  int* imax;
  int* chunk_cnt;
  int* chunk_tau;
  int* chunk_k;
  float* chunk_amp;
  float* chunk_th;
  unsigned* dirty;  // two bitmaps of nwords each
  unsigned* bar;    // barrier {count, generation}
  int* err;
  int nchunks, nblk, nwords, xpieces;
  unsigned long long limit_ns;
};

struct Smem {
  float* W;        // P*nt
  int* prefix;     // nchunks+1
  float* win;      // kChunk + 2*nt
  float* red_v;    // kWarps*32
  int* red_i;      // kWarps*32
  int* sp_tau;     // kMaxTouch
  int* sp_k;
  float* sp_amp;
  int* sp_par;
  int* ord;        // kMaxTouch
  int* wcnt;       // kWarps+1
  int* misc;       // 4
};

__device__ __forceinline__ Smem carve_smem(const PeelArgs& a, char* base) {
  Smem s;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* p = base + off;
    off = (off + bytes + 15) & ~size_t(15);
    return p;
  };
  s.W = reinterpret_cast<float*>(take(sizeof(float) * a.P * a.nt));
  s.prefix = reinterpret_cast<int*>(take(sizeof(int) * (a.nchunks + 1)));
  s.win = reinterpret_cast<float*>(take(sizeof(float) * (kChunk + 2 * a.nt)));
  s.red_v = reinterpret_cast<float*>(take(sizeof(float) * kWarps * 32));
  s.red_i = reinterpret_cast<int*>(take(sizeof(int) * kWarps * 32));
  s.sp_tau = reinterpret_cast<int*>(take(sizeof(int) * kMaxTouch));
  s.sp_k = reinterpret_cast<int*>(take(sizeof(int) * kMaxTouch));
  s.sp_amp = reinterpret_cast<float*>(take(sizeof(float) * kMaxTouch));
  s.sp_par = reinterpret_cast<int*>(take(sizeof(int) * kMaxTouch));
  s.ord = reinterpret_cast<int*>(take(sizeof(int) * kMaxTouch));
  s.wcnt = reinterpret_cast<int*>(take(sizeof(int) * (kWarps + 1)));
  s.misc = reinterpret_cast<int*>(take(sizeof(int) * 4));
  return s;
}

size_t smem_bytes(int P, int nt, int nchunks) {
  auto r = [](size_t b) { return (b + 15) & ~size_t(15); };
  return r(sizeof(float) * P * nt) + r(sizeof(int) * (nchunks + 1)) +
         r(sizeof(float) * (kChunk + 2 * nt)) + 2 * r(sizeof(float) * kWarps * 32) +
         5 * r(sizeof(int) * kMaxTouch) + r(sizeof(int) * (kWarps + 1)) +
         r(sizeof(int) * 4);
}

// ---------------------------------------------------------------- DETECT
__device__ void detect_chunk(const PeelArgs& a, const Smem& s, int ch,
                             unsigned* bm) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nt = a.nt, L = a.L;
  const int a0 = ch * kChunk;
  const int a1 = min(a0 + kChunk, L);
  for (int i = tid; i < kChunk + 2 * nt; i += kThreads) {
    int col = a0 - nt + i;
    s.win[i] = (col >= 0 && col < L) ? a.cfmax[col] : -INFINITY;
  }
  __syncthreads();
  const int tau = a0 + tid;
  bool pk = false;
  float pooled = 0.f;
  if (tau < a1 && tau >= nt && tau < L - nt) {
    float m = -INFINITY;
    for (int d = 0; d <= 2 * nt; ++d) m = fmaxf(m, s.win[tid + d]);
    const float best = s.win[tid + nt];
    pk = (m > a.th2) && (fabsf(__fsub_rn(m, best)) < 1e-9f);
    pooled = m;
  }
  const unsigned bal = __ballot_sync(0xffffffffu, pk);
  if (lane == 0) s.wcnt[warp] = __popc(bal);
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int w = 0; w < kWarps; ++w) {
      int c = s.wcnt[w];
      s.wcnt[w] = acc;
      acc += c;
    }
    s.wcnt[kWarps] = acc;
  }
  __syncthreads();
  if (pk) {
    const int idx = s.wcnt[warp] + __popc(bal & ((1u << lane) - 1u));
    const int k = a.imax[tau];
    const float amp = __fdiv_rn(a.B[(long long)k * a.ldb + tau], a.nm[k]);
    const float th = __fsqrt_rn(pooled);
    const long long slot = (long long)ch * kChunk + idx;
    a.chunk_tau[slot] = tau;
    a.chunk_k[slot] = k;
    a.chunk_amp[slot] = amp;
    a.chunk_th[slot] = th;
    // peaks satisfy nt <= tau < L - nt (edge scores are zero)
    const int b0 = max(tau - nt, 0) / kCol;
    const int b1 = min(tau + nt, L - 1) / kCol;
    for (int b = b0; b <= b1; ++b) atomicOr(&bm[b >> 5], 1u << (b & 31));
  }
  if (tid == 0) a.chunk_cnt[ch] = s.wcnt[kWarps];
  __syncthreads();
}

// Exclusive prefix of chunk counts into s.prefix[0..nchunks]; returns total.
__device__ int chunk_prefix(const PeelArgs& a, const Smem& s) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int per = (a.nchunks + kThreads - 1) / kThreads;
  const int c0 = tid * per;
  int local = 0;
  for (int i = 0; i < per; ++i) {
    int c = c0 + i;
    if (c < a.nchunks) local += a.chunk_cnt[c];
  }
  int incl = local;
  for (int o = 1; o < 32; o <<= 1) {
    int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) s.wcnt[warp] = incl;
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int w = 0; w < kWarps; ++w) {
      int c = s.wcnt[w];
      s.wcnt[w] = acc;
      acc += c;
    }
    s.wcnt[kWarps] = acc;
  }
  __syncthreads();
  int run = s.wcnt[warp] + incl - local;
  for (int i = 0; i < per; ++i) {
    int c = c0 + i;
    if (c < a.nchunks) {
      s.prefix[c] = run;
      run += a.chunk_cnt[c];
    }
  }
  if (tid == 0) s.prefix[a.nchunks] = s.wcnt[kWarps];
  __syncthreads();
  return s.prefix[a.nchunks];
}

// ---------------------------------------------------------------- UPDATE
// Gather the peaks of this iteration that touch columns [c0, c0+32) into
// shared memory, ordered even global index first, then odd (each ascending).
__device__ int gather_touching(const PeelArgs& a, const Smem& s, int c0) {
  const int tid = threadIdx.x, lane = tid & 31;
  if (tid < 32) {
    const int lo = c0 - a.nt, hi = c0 + kCol - 1 + a.nt;
    const int ch_lo = max(lo, 0) / kChunk;
    const int ch_hi = min(hi, a.L - 1) / kChunk;
    int n = 0;
    for (int ch = ch_lo; ch <= ch_hi; ++ch) {
      const int cnt = a.chunk_cnt[ch];
      const int base = s.prefix[ch];
      for (int i0 = 0; i0 < cnt; i0 += 32) {
        const int i = i0 + lane;
        const bool ok = i < cnt;
        const long long slot = (long long)ch * kChunk + i;
        const int t = ok ? a.chunk_tau[slot] : -1;
        const bool in = ok && t >= lo && t <= hi;
        const unsigned bal = __ballot_sync(0xffffffffu, in);
        if (in) {
          const int pos = n + __popc(bal & ((1u << lane) - 1u));
          if (pos < kMaxTouch) {
            s.sp_tau[pos] = t;
            s.sp_k[pos] = a.chunk_k[slot];
            s.sp_amp[pos] = a.chunk_amp[slot];
            s.sp_par[pos] = (base + i) & 1;
          }
        }
        n += __popc(bal);
      }
    }
    if (n > kMaxTouch) {
      if (lane == 0) atomicCAS(a.err, 0, KS_ERR_DEGENERATE);
      n = kMaxTouch;
    }
    __syncwarp();
    if (lane == 0) {
      int m = 0;
      for (int par = 0; par < 2; ++par)
        for (int e = 0; e < n; ++e)
          if (s.sp_par[e] == par) s.ord[m++] = e;
      s.misc[0] = n;
    }
  }
  __syncthreads();
  return s.misc[0];
}

// Apply the gathered subtractions to columns [c0, c0+32) of B and rescore
// them (n_touch == 0: rescore only).
__device__ void update_block(const PeelArgs& a, const Smem& s, int c0,
                             int n_touch) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int c = c0 + lane;
  const bool colok = c < a.L;
  const int nt = a.nt, K = a.K, nlag = 2 * nt + 1;
  // which gathered peaks touch this lane's column (bit e of ord position)
  unsigned long long mine = 0ull;
  for (int e = 0; e < n_touch; ++e) {
    const int d = c - s.sp_tau[s.ord[e]];
    if (colok && d >= -nt && d <= nt) mine |= 1ull << e;
  }
  const bool touched = mine != 0ull;
  float best = -1.f;
  int arg = 0;
  for (int j0 = warp; j0 < K; j0 += kWarps * kRows) {
    float bv[kRows];
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const int j = j0 + r * kWarps;
      bv[r] = (colok && j < K) ? a.B[(long long)j * a.ldb + c] : 0.f;
    }
    for (int e = 0; e < n_touch; ++e) {
      const int q = s.ord[e];
      if ((mine >> e) & 1ull) {
        const int kk = s.sp_k[q];
        const float amp = s.sp_amp[q];
        const int lag = c - s.sp_tau[q] + nt;
#pragma unroll
        for (int r = 0; r < kRows; ++r) {
          const int j = j0 + r * kWarps;
          if (j < K) {
            const float w = a.ctc[((long long)j * K + kk) * nlag + lag];
            bv[r] = __fsub_rn(bv[r], __fmul_rn(amp, w));
          }
        }
      }
    }
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const int j = j0 + r * kWarps;
      if (j < K) {
        if (touched) a.B[(long long)j * a.ldb + c] = bv[r];
        const float rl = bv[r] > 0.f ? bv[r] : 0.f;
        const float cf = __fdiv_rn(__fmul_rn(rl, rl), a.nm[j]);
        if (cf > best) {
          best = cf;
          arg = j;
        }
      }
    }
  }
  s.red_v[warp * 32 + lane] = best;
  s.red_i[warp * 32 + lane] = arg;
  __syncthreads();
  if (warp == 0 && colok) {
    float bv = s.red_v[lane];
    int bi = s.red_i[lane];
    for (int w = 1; w < kWarps; ++w) {
      const float v = s.red_v[w * 32 + lane];
      const int i = s.red_i[w * 32 + lane];
      if (v > bv || (v == bv && i < bi)) {
        bv = v;
        bi = i;
      }
    }
    if (c < nt || c >= a.L - nt) {
      bv = 0.f;
      bi = 0;
    }
    a.cfmax[c] = bv;
    a.imax[c] = bi;
  }
  __syncthreads();
}

// Subtract amp * sum_p U[k,p,c] W[p,t] from Xres[c, tau - nt/2 + t] for the
// channels of one piece of one peak.
__device__ void xres_piece(const PeelArgs& a, const Smem& s, int sp, int piece) {
  // locate peak sp: largest chunk with prefix <= sp
  int lo = 0, hi = a.nchunks - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (s.prefix[mid] <= sp) lo = mid; else hi = mid - 1;
  }
  const long long slot = (long long)lo * kChunk + (sp - s.prefix[lo]);
  const int tau = a.chunk_tau[slot];
  const int k = a.chunk_k[slot];
  const float amp = a.chunk_amp[slot];
  const int per = (a.C + a.xpieces - 1) / a.xpieces;
  const int c_lo = piece * per;
  const int c_hi = min(a.C, c_lo + per);
  const int nt = a.nt;
  const int t0 = tau - nt / 2;
  const float* Uk = a.U + (long long)k * a.P * a.C;
  for (int e = threadIdx.x; e < (c_hi - c_lo) * nt; e += kThreads) {
    const int c = c_lo + e / nt;
    const int t = e - (e / nt) * nt;
    float wv = 0.f;
    for (int p = 0; p < a.P; ++p) wv = fmaf(Uk[(long long)p * a.C + c], s.W[p * nt + t], wv);
    float* x = a.Xres + (long long)c * a.L + t0 + t;
    *x = __fsub_rn(*x, __fmul_rn(amp, wv));
  }
}

__global__ void __launch_bounds__(kThreads) peel_kernel(PeelArgs a) {
  extern __shared__ __align__(16) char smem_raw[];
  const Smem s = carve_smem(a, smem_raw);
  const int tid = threadIdx.x;
  const unsigned G = gridDim.x;
  for (int i = tid; i < a.P * a.nt; i += kThreads) s.W[i] = a.W[i];
  for (int w = blockIdx.x * kThreads + tid; w < 2 * a.nwords; w += G * kThreads)
    a.dirty[w] = 0u;
  __syncthreads();

  // initial scores of every column
  for (int m = blockIdx.x; m < a.nblk; m += G) update_block(a, s, m * kCol, 0);

  long long n_out = 0;
  int it = 0;
  int status = KS_OK;
  bool ok = ks_grid_sync(a.bar, G, a.err, a.limit_ns);
  for (; ok && it < a.max_peels; ++it) {
    unsigned* bm = a.dirty + (it & 1) * a.nwords;
    unsigned* bm_next = a.dirty + ((it + 1) & 1) * a.nwords;
    for (int ch = blockIdx.x; ch < a.nchunks; ch += G) detect_chunk(a, s, ch, bm);
    if (!ks_grid_sync(a.bar, G, a.err, a.limit_ns)) break;

    const int total = chunk_prefix(a, s);
    if (total == 0) break;
    if (n_out + total > a.capacity) {
      status = KS_ERR_OVERFLOW;
      if (blockIdx.x == 0 && tid == 0) a.info[3] = n_out + total;
      break;
    }
    // records, in (iteration, tau) order
    for (int ch = blockIdx.x; ch < a.nchunks; ch += G) {
      const int cnt = a.chunk_cnt[ch];
      for (int i = tid; i < cnt; i += kThreads) {
        const long long slot = (long long)ch * kChunk + i;
        const long long o = n_out + s.prefix[ch] + i;
        a.st[2 * o] = a.chunk_tau[slot];
        a.st[2 * o + 1] = a.chunk_k[slot];
        a.amps[o] = a.chunk_amp[slot];
        a.th_amps[o] = a.chunk_th[slot];
      }
    }
    for (int w = blockIdx.x * kThreads + tid; w < a.nwords; w += G * kThreads)
      bm_next[w] = 0u;
    // subtract and rescore dirty blocks
    for (int m = blockIdx.x; m < a.nblk; m += G) {
      if ((bm[m >> 5] >> (m & 31)) & 1u) {
        const int n_touch = gather_touching(a, s, m * kCol);
        update_block(a, s, m * kCol, n_touch);
      }
    }
    // residual
    const long long nx = (long long)total * a.xpieces;
    for (long long w = blockIdx.x; w < nx; w += G) {
      xres_piece(a, s, (int)(w / a.xpieces), (int)(w % a.xpieces));
    }
    n_out += total;
    ok = ks_grid_sync(a.bar, G, a.err, a.limit_ns);
  }
  if (blockIdx.x == 0 && tid == 0) {
    const int e = ks_ld_volatile(a.err);
    a.info[0] = n_out;
    a.info[1] = e ? e : status;
    a.info[2] = it;
    if (status != KS_ERR_OVERFLOW) a.info[3] = n_out;
  }
}

struct PeelLayout {
  int nchunks, nblk, nwords;
  size_t bytes;
};

PeelLayout peel_layout(int64_t L) {
  PeelLayout l;
  l.nchunks = (int)((L + kChunk - 1) / kChunk);
  l.nblk = (int)((L + kCol - 1) / kCol);
  l.nwords = (l.nblk + 31) / 32;
  ks::Carve cv(nullptr);
  cv.take<float>(L);
  cv.take<int>(L);
  cv.take<int>(l.nchunks);
  for (int i = 0; i < 4; ++i) cv.take<int>((size_t)l.nchunks * kChunk);
  cv.take<unsigned>(2 * l.nwords);
  cv.take<unsigned>(4);
  l.bytes = cv.used;
  return l;
}

}  // namespace

namespace ks {

size_t peel_workspace_size(int64_t L) { return peel_layout(L).bytes; }

int launch_peel(float* B, int64_t ldb, float* Xres, const float* U,
                const float* W, const float* ctc, const float* nm, int64_t C,
                int64_t L, int64_t K, int64_t P, int64_t nt, float th2,
                int64_t max_peels, int64_t capacity, int64_t* st, float* amps,
                float* th_amps, int64_t* info, void* ws, size_t ws_bytes,
                cudaStream_t stream, unsigned long long limit_ns) {
  if (!B || !Xres || !U || !W || !ctc || !nm || !st || !amps || !th_amps || !info)
    return fail(KS_ERR_ARG, "ks_peel: null pointer");
  if (C < 1 || L < 1 || K < 1 || P < 1 || nt < 1 || (nt % 2) == 0)
    return fail(KS_ERR_ARG, "ks_peel: need C,L,K,P >= 1 and odd nt");
  if (ldb < L) return fail(KS_ERR_ARG, "ks_peel: ldb < L");
  if (L > (int64_t)kMaxChunks * kChunk || K > (1 << 24) || C > (1 << 24) ||
      nt > 1023 || P > 64)
    return fail(KS_ERR_UNSUPPORTED, "ks_peel: shape beyond supported limits");
  if (capacity < 0 || max_peels < 0) return fail(KS_ERR_ARG, "ks_peel: negative capacity/max_peels");
  if (!(th2 >= 0.f)) return fail(KS_ERR_ARG, "ks_peel: th2 must be a non-negative number");
  const PeelLayout lay = peel_layout(L);
  if (ws_bytes < lay.bytes || !ws) return fail(KS_ERR_WORKSPACE, "ks_peel: workspace too small");

  DeviceInfo dev;
  int rc = device_info(&dev);
  if (rc) return rc;

  PeelArgs a{};
  a.B = B; a.ldb = ldb; a.Xres = Xres; a.U = U; a.W = W; a.ctc = ctc; a.nm = nm;
  a.C = (int)C; a.L = (int)L; a.K = (int)K; a.P = (int)P; a.nt = (int)nt;
  a.th2 = th2;
  a.max_peels = (int)std::min<int64_t>(max_peels, 1 << 30);
  a.capacity = capacity;
  a.st = reinterpret_cast<long long*>(st); a.amps = amps; a.th_amps = th_amps;
  a.info = reinterpret_cast<long long*>(info);
  Carve cv(ws);
  a.cfmax = cv.take<float>(L);
  a.imax = cv.take<int>(L);
  a.chunk_cnt = cv.take<int>(lay.nchunks);
  a.chunk_tau = cv.take<int>((size_t)lay.nchunks * kChunk);
  a.chunk_k = cv.take<int>((size_t)lay.nchunks * kChunk);
  a.chunk_amp = cv.take<float>((size_t)lay.nchunks * kChunk);
  a.chunk_th = cv.take<float>((size_t)lay.nchunks * kChunk);
  a.dirty = cv.take<unsigned>(2 * lay.nwords);
  unsigned* ctl = cv.take<unsigned>(4);
  a.bar = ctl;
  a.err = reinterpret_cast<int*>(ctl + 2);
  a.nchunks = lay.nchunks; a.nblk = lay.nblk; a.nwords = lay.nwords;
  a.xpieces = (int)std::max<int64_t>(1, std::min<int64_t>(8, (C * nt + 2047) / 2048));
  a.limit_ns = limit_ns;

  const size_t smem = smem_bytes(a.P, a.nt, a.nchunks);
  static thread_local int cached_dev = -1;
  static thread_local size_t cached_smem = 0;
  static thread_local int cached_occ = 0;
  if (cached_dev != dev.device || cached_smem != smem) {
    if (smem > 48 * 1024)
      KS_CUDA(cudaFuncSetAttribute(peel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    KS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, peel_kernel, kThreads, smem));
    if (occ < 1) return fail(KS_ERR_UNSUPPORTED, "ks_peel: kernel does not fit on an SM");
    cached_dev = dev.device; cached_smem = smem; cached_occ = occ;
  }
  const int grid = dev.sm_count * cached_occ;
  KS_CUDA(cudaMemsetAsync(ctl, 0, 4 * sizeof(unsigned), stream));
  void* args[] = {&a};
  KS_CUDA(cudaLaunchCooperativeKernel((void*)peel_kernel, dim3(grid), dim3(kThreads), args, smem, stream));
  return KS_OK;
}

}  // namespace ks
