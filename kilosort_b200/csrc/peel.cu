// Greedy peel (matching pursuit) of one batch as a single persistent,
// cooperative kernel.  Semantics follow kilosort/template_matching.py:183-244.
//
// Layout in HBM
//   B      [K, ldb]  float32 score matrix, updated in place
//   Xres   [C, L]    float32 residual, updated in place
//   ctc    [K, K, 2nt+1] float32, read as ctc[j, k_spike, lag]
//   cfmax  [L] f32 / imax [L] i32   best score relu(B)^2/nm over templates and
//                                   its template, per column (settled values)
//   pack   [2][L] u64               per-iteration rescoring of dirty columns:
//                                   (score bits << 32) | ~template, combined
//                                   with atomicMax so that the larger score and,
//                                   on ties, the smaller template index win
//   chunk buffers                   peaks found per 512-column chunk
//   tcount/touch/dlist [2][...]     per-iteration dirty 32-column blocks and
//                                   the peaks touching each of them
//
// Iteration it (p = it & 1, q = p ^ 1), two phases between device-wide barriers:
//   DETECT  per chunk whose +-nt neighbourhood changed in iteration it-1:
//           settle the rescored columns (pack[q] -> cfmax/imax), then
//           pooled = max of cfmax over +-nt; a column is a peak iff pooled > th2
//           and |pooled - cfmax| < 1e-9 (kilosort :206-212).  Peaks are
//           compacted in time order; amplitude B[k,tau]/nm[k] and sqrt(pooled)
//           come from the pre-subtraction B (:225-229).  Each peak registers in
//           the touch list of the 32-column blocks within +-nt of it; the first
//           registration of a block appends it to dlist[p] and clears pack[p].
//   UPDATE  every block computes the exclusive prefix of the chunk counts (the
//           peak's global index in the iteration).  Records are written in
//           (iteration, tau) order.  Work items (dirty block, 128-row group):
//           for every column apply B[j,c] -= amp*ctc[j,k,c-tau+nt] of the peaks
//           touching it, even-indexed peaks first, then odd-indexed ones -- the
//           order of the reference's two interleaved groups (:235-238) -- with
//           separately rounded product and difference, then fold the rescored
//           rows into pack[p] with atomicMax.  Residual windows of every peak
//           are updated in place (:237).
// The loop ends when no peak is found or after max_peels iterations, decided
// identically by every block from the same counts.  Every device-wide wait is
// bounded; a wait that runs out records KS_ERR_TIMEOUT and all blocks leave.
#include "ks_common.cuh"

namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kChunk = 512;          // detection chunk, one column per thread
constexpr int kCol = 32;             // update block, one column per lane
constexpr int kRowsPerWarp = 8;      // template rows in flight per lane
constexpr int kTouch = 8;            // peaks touching one block (more: ties)
constexpr int kMaxChunks = 8192;

// Phase timeline for profiling builds (-DKS_PEEL_TRACE): block 0 writes
// %globaltimer stamps to info[8 + 8*it + slot]; the caller sizes info.
#ifdef KS_PEEL_TRACE
#define KS_TRACE(it, slot, value)                                        \
  do {                                                                   \
    if (blockIdx.x == 0 && threadIdx.x == 0 && (it) < 200)               \
      a.info[8 + 8 * (it) + (slot)] = (long long)(value);                \
  } while (0)
#else
#define KS_TRACE(it, slot, value) \
  do {                           \
  } while (0)
#endif

struct Touch {
  int tau;
  int k;
  float amp;
  int slot;  // chunk * kChunk + index in chunk
};

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
  unsigned long long* pack;   // [2][L]
  int* chunk_cnt;
  int* chunk_tau;
  int* chunk_k;
  float* chunk_amp;
  float* chunk_th;
  int* tcount;                // [2][nblk]
  Touch* touch;               // [2][nblk * kTouch]
  int* dlist;                 // [2][nblk]
  int* dcount;                // [2]
  unsigned* bar;              // {count, generation}
  int* err;
  int nchunks, nblk;
  unsigned long long limit_ns;
};

struct Smem {
  float* W;        // P*nt
  int* prefix;     // nchunks+1
  float* win;      // kChunk + 2*nt   column scores around the chunk
  float* mx0;      // kChunk + 2*nt   sliding-max doubling levels (ping-pong)
  float* mx1;      // kChunk + 2*nt
  int* kidx;       // kChunk          best template of the chunk's own columns
  int* wcnt;       // kWarps+1
  int* tl_tau;     // kWarps*kTouch   ordered touch list of each warp's item
  int* tl_k;       // kWarps*kTouch
  float* tl_amp;   // kWarps*kTouch
  float* xu;       // kWarps*64       U values of a residual item
};

__device__ __forceinline__ Smem carve_smem(const PeelArgs& a, char* base) {
  Smem s;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* p = base + off;
    off = (off + bytes + 15) & ~size_t(15);
    return p;
  };
  const int wn = kChunk + 2 * a.nt;
  s.W = reinterpret_cast<float*>(take(sizeof(float) * a.P * a.nt));
  s.prefix = reinterpret_cast<int*>(take(sizeof(int) * (a.nchunks + 1)));
  s.win = reinterpret_cast<float*>(take(sizeof(float) * wn));
  s.mx0 = reinterpret_cast<float*>(take(sizeof(float) * wn));
  s.mx1 = reinterpret_cast<float*>(take(sizeof(float) * wn));
  s.kidx = reinterpret_cast<int*>(take(sizeof(int) * kChunk));
  s.wcnt = reinterpret_cast<int*>(take(sizeof(int) * (kWarps + 1)));
  s.tl_tau = reinterpret_cast<int*>(take(sizeof(int) * kWarps * kTouch));
  s.tl_k = reinterpret_cast<int*>(take(sizeof(int) * kWarps * kTouch));
  s.tl_amp = reinterpret_cast<float*>(take(sizeof(float) * kWarps * kTouch));
  s.xu = reinterpret_cast<float*>(take(sizeof(float) * kWarps * 64));
  return s;
}

size_t smem_bytes(int P, int nt, int nchunks) {
  auto r = [](size_t b) { return (b + 15) & ~size_t(15); };
  const size_t wn = kChunk + 2 * (size_t)nt;
  return r(sizeof(float) * P * nt) + r(sizeof(int) * (nchunks + 1)) +
         3 * r(sizeof(float) * wn) + r(sizeof(int) * kChunk) + r(sizeof(int) * (kWarps + 1)) +
         3 * r(sizeof(int) * kWarps * kTouch) + r(sizeof(float) * kWarps * 64);
}

__device__ __forceinline__ unsigned long long pack_score(float cf, int j) {
  return ((unsigned long long)__float_as_uint(cf) << 32) | (unsigned)(~(unsigned)j);
}
__device__ __forceinline__ float pack_value(unsigned long long v) {
  return __uint_as_float((unsigned)(v >> 32));
}
__device__ __forceinline__ int pack_index(unsigned long long v) {
  return (int)(~(unsigned)(v & 0xffffffffull));
}

// ---------------------------------------------------------------- DETECT
__device__ void detect_chunk(const PeelArgs& a, const Smem& s, int ch, int it) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nt = a.nt, L = a.L;
  const int p = it & 1, q = p ^ 1;
  const int a0 = ch * kChunk;
  const int a1 = min(a0 + kChunk, L);
  const int wn = kChunk + 2 * nt;
  const int* tprev = a.tcount + (size_t)q * a.nblk;
  const unsigned long long* pprev = a.pack + (size_t)q * L;
  if (it > 0) {
    // nothing within +-nt of this chunk changed: its peak test cannot change
    const int b_lo = max(a0 - nt, 0) / kCol, b_hi = min(a1 - 1 + nt, L - 1) / kCol;
    int any = 0;
    for (int b = b_lo + tid; b <= b_hi; b += kThreads) any |= tprev[b] > 0;
    if (!__syncthreads_or(any)) {
      if (tid == 0) a.chunk_cnt[ch] = 0;
      return;
    }
  }
  // Column scores: rescored columns of the last iteration come from pack[q]
  // (and are settled into cfmax/imax by the chunk that owns them), the others
  // from cfmax.  The candidate loads are independent and issued together.
  for (int i = tid; i < wn; i += kThreads) {
    const int col = a0 - nt + i;
    float v;
    if (col < 0 || col >= L) {
      v = -INFINITY;
    } else if (col < nt || col >= L - nt) {
      v = 0.f;
    } else {
      const bool fresh = it == 0 || tprev[col / kCol] > 0;
      const unsigned long long pv = pprev[col];
      const float cv = a.cfmax[col];
      const bool own = i >= nt && i < nt + kChunk && col < a1;
      const int iv = own ? a.imax[col] : 0;
      v = fresh ? pack_value(pv) : cv;
      if (own) {
        const int kb = fresh ? pack_index(pv) : iv;
        s.kidx[i - nt] = kb;
        if (fresh) {
          a.cfmax[col] = v;
          a.imax[col] = kb;
        }
      }
    }
    s.win[i] = v;
  }
  __syncthreads();
  // sliding max over 2nt+1 columns: doubling levels up to the largest power
  // of two m <= 2nt+1, then the union of two overlapping m-windows
  const int len = 2 * nt + 1;
  int m = 1;
  const float* src = s.win;
  float* dst = s.mx0;
  while (2 * m <= len) {
    for (int i = tid; i + 2 * m <= wn; i += kThreads) dst[i] = fmaxf(src[i], src[i + m]);
    __syncthreads();
    m *= 2;
    src = dst;
    dst = (dst == s.mx0) ? s.mx1 : s.mx0;
  }
  const int tau = a0 + tid;
  bool pk = false;
  float pooled = 0.f;
  if (tau < a1 && tau >= nt && tau < L - nt) {
    pooled = fmaxf(src[tid], src[tid + len - m]);
    const float best = s.win[tid + nt];
    pk = (pooled > a.th2) && (fabsf(__fsub_rn(pooled, best)) < 1e-9f);
  }
  const unsigned bal = __ballot_sync(0xffffffffu, pk);
  if (lane == 0) s.wcnt[warp] = __popc(bal);
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int w = 0; w < kWarps; ++w) {
      const int c = s.wcnt[w];
      s.wcnt[w] = acc;
      acc += c;
    }
    s.wcnt[kWarps] = acc;
  }
  __syncthreads();
  if (pk) {
    const int idx = s.wcnt[warp] + __popc(bal & ((1u << lane) - 1u));
    const int k = s.kidx[tid];
    const float amp = __fdiv_rn(a.B[(long long)k * a.ldb + tau], a.nm[k]);
    const float th = __fsqrt_rn(pooled);
    const int slot = ch * kChunk + idx;
    a.chunk_tau[slot] = tau;
    a.chunk_k[slot] = k;
    a.chunk_amp[slot] = amp;
    a.chunk_th[slot] = th;
    int* tcur = a.tcount + (size_t)p * a.nblk;
    Touch* tch = a.touch + (size_t)p * a.nblk * kTouch;
    unsigned long long* pcur = a.pack + (size_t)p * L;
    const int b0 = (tau - nt) / kCol, b1 = (tau + nt) / kCol;
    for (int bb = b0; bb <= b1; bb += 8) {
      int pos[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) pos[i] = (bb + i <= b1) ? atomicAdd(&tcur[bb + i], 1) : -1;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int b = bb + i;
        if (pos[i] < 0) continue;
        if (pos[i] == 0) {
          const int d = atomicAdd(&a.dcount[p], 1);
          a.dlist[(size_t)p * a.nblk + d] = b;
          const int c_hi = min(L, (b + 1) * kCol);
          for (int c = b * kCol; c < c_hi; ++c) pcur[c] = 0ull;
        }
        if (pos[i] < kTouch) tch[(size_t)b * kTouch + pos[i]] = Touch{tau, k, amp, slot};
        else atomicCAS(a.err, 0, KS_ERR_DEGENERATE);
      }
    }
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
    const int c = c0 + i;
    if (c < a.nchunks) local += a.chunk_cnt[c];
  }
  int incl = local;
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) s.wcnt[warp] = incl;
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int w = 0; w < kWarps; ++w) {
      const int c = s.wcnt[w];
      s.wcnt[w] = acc;
      acc += c;
    }
    s.wcnt[kWarps] = acc;
  }
  __syncthreads();
  int run = s.wcnt[warp] + incl - local;
  for (int i = 0; i < per; ++i) {
    const int c = c0 + i;
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
// Work items are per warp (no block-wide synchronisation), so thousands run
// concurrently and the latency of one item hides behind the others.

// Ordered touch list of one 32-column block in the warp's shared-memory
// slot: entry e (application order: even global index first, then odd, each
// ascending) has peak time tau[e], template k[e], amplitude amp[e].
struct TouchList {
  int n;
  const int* tau;
  const int* k;
  const float* amp;
};

__device__ __forceinline__ TouchList load_touch_warp(const PeelArgs& a, const Smem& s,
                                                     int p, int blk, int lane, int warp) {
  Touch t{0, 0, 0.f, 0};
  if (lane < kTouch) t = a.touch[((size_t)p * a.nblk + blk) * kTouch + lane];
  int n = a.tcount[(size_t)p * a.nblk + blk];
  n = min(n, kTouch);
  int key = 0x7fffffff;
  if (lane < n) {
    const int ch = t.slot / kChunk;
    const int g = s.prefix[ch] + (t.slot - ch * kChunk);
    key = ((g & 1) << 30) | g;
  }
  int rank = 0;
  for (int j = 0; j < n; ++j) {
    const int kj = __shfl_sync(0xffffffffu, key, j);
    rank += (kj < key) ? 1 : 0;
  }
  int* tau = s.tl_tau + warp * kTouch;
  int* kk = s.tl_k + warp * kTouch;
  float* amp = s.tl_amp + warp * kTouch;
  __syncwarp();
  if (lane < n) {
    tau[rank] = t.tau;
    kk[rank] = t.k;
    amp[rank] = t.amp;
  }
  __syncwarp();
  return TouchList{n, tau, kk, amp};
}

// Columns [blk*32, blk*32+32) x template rows [j_lo, j_hi): subtract the
// touching peaks, store the changed rows, fold the rescored rows into pack_out.
// A column is touched by at most two peaks unless scores tie exactly; the two
// are preloaded with the rows of B so each group of rows costs one round trip.
__device__ void update_warp_item(const PeelArgs& a, const TouchList& tl, int blk,
                                 int j_lo, int j_hi, unsigned long long* pack_out,
                                 int lane) {
  const int c = blk * kCol + lane;
  const bool colok = c < a.L;
  const int nt = a.nt, K = a.K, nlag = 2 * nt + 1;
  const long long rstride = (long long)K * nlag;     // ctc row stride (j)
  int e0 = -1, e1 = -1;
  unsigned rest = 0u;                                 // further touching entries
  for (int e = 0; e < tl.n; ++e) {
    const int d = c - tl.tau[e];
    if (colok && d >= -nt && d <= nt) {
      if (e0 < 0) e0 = e;
      else if (e1 < 0) e1 = e;
      else rest |= 1u << e;
    }
  }
  const bool touched = e0 >= 0;
  const float* cp0 = a.ctc;
  const float* cp1 = a.ctc;
  float amp0 = 0.f, amp1 = 0.f;
  if (e0 >= 0) { cp0 = a.ctc + (long long)tl.k[e0] * nlag + (c - tl.tau[e0] + nt); amp0 = tl.amp[e0]; }
  if (e1 >= 0) { cp1 = a.ctc + (long long)tl.k[e1] * nlag + (c - tl.tau[e1] + nt); amp1 = tl.amp[e1]; }
  float best = -1.f;
  int arg = 0;
  for (int j0 = j_lo; j0 < j_hi; j0 += kRowsPerWarp) {
    float bv[kRowsPerWarp], w0[kRowsPerWarp], w1[kRowsPerWarp];
#pragma unroll
    for (int r = 0; r < kRowsPerWarp; ++r) {
      const int j = j0 + r;
      const bool ok = colok && j < j_hi;
      bv[r] = ok ? a.B[(long long)j * a.ldb + c] : 0.f;
      w0[r] = (ok && e0 >= 0) ? __ldg(cp0 + j * rstride) : 0.f;
      w1[r] = (ok && e1 >= 0) ? __ldg(cp1 + j * rstride) : 0.f;
    }
#pragma unroll
    for (int r = 0; r < kRowsPerWarp; ++r) {
      if (e0 >= 0) bv[r] = __fsub_rn(bv[r], __fmul_rn(amp0, w0[r]));
      if (e1 >= 0) bv[r] = __fsub_rn(bv[r], __fmul_rn(amp1, w1[r]));
    }
    if (rest) {
      for (int e = 0; e < tl.n; ++e) {
        if ((rest >> e) & 1u) {
          const float amp = tl.amp[e];
          const float* cp = a.ctc + (long long)tl.k[e] * nlag + (c - tl.tau[e] + nt);
#pragma unroll
          for (int r = 0; r < kRowsPerWarp; ++r) {
            const int j = j0 + r;
            if (j < j_hi) bv[r] = __fsub_rn(bv[r], __fmul_rn(amp, __ldg(cp + j * rstride)));
          }
        }
      }
    }
#pragma unroll
    for (int r = 0; r < kRowsPerWarp; ++r) {
      const int j = j0 + r;
      if (colok && j < j_hi) {
        if (touched) a.B[(long long)j * a.ldb + c] = bv[r];
        const float rl = bv[r] > 0.f ? bv[r] : 0.f;
        const float cf = __fdiv_rn(__fmul_rn(rl, rl), __ldg(a.nm + j));
        if (cf > best) {
          best = cf;
          arg = j;
        }
      }
    }
  }
  if (colok && best >= 0.f) atomicMax(&pack_out[c], pack_score(best, arg));
}

// Subtract amp * sum_p U[k,p,c] W[p,t] from Xres[c, tau - nt/2 + t] for 8
// channels of one peak; lanes run along t.  The U values of the 8 channels go
// through the warp's shared-memory slot and all residual values of a 64-tap
// span are loaded before any is written, so one item costs two round trips.
constexpr int kXresChans = 8;
__device__ void xres_warp_item(const PeelArgs& a, const Smem& s, int sp, int cg,
                               int lane, int warp) {
  int lo = 0, hi = a.nchunks - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (s.prefix[mid] <= sp) lo = mid; else hi = mid - 1;
  }
  const long long slot = (long long)lo * kChunk + (sp - s.prefix[lo]);
  const int tau = a.chunk_tau[slot];
  const int k = a.chunk_k[slot];
  const float amp = a.chunk_amp[slot];
  const int nt = a.nt, P = a.P;
  const int t0 = tau - nt / 2;
  const int cbase = cg * kXresChans;
  const int nch = min(kXresChans, a.C - cbase);
  float* su = s.xu + warp * kXresChans * 8;       // [channel][component]
  __syncwarp();
  for (int e = lane; e < kXresChans * 8; e += 32) {
    const int ci = e >> 3, pp = e & 7;
    su[e] = (ci < nch && pp < P) ? __ldg(a.U + ((long long)k * P + pp) * a.C + cbase + ci) : 0.f;
  }
  __syncwarp();
  for (int tb = 0; tb < nt; tb += 64) {
    float xv[kXresChans][2];
#pragma unroll
    for (int ci = 0; ci < kXresChans; ++ci)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int t = tb + lane + 32 * h;
        xv[ci][h] = (ci < nch && t < nt) ? a.Xres[(long long)(cbase + ci) * a.L + t0 + t] : 0.f;
      }
#pragma unroll
    for (int ci = 0; ci < kXresChans; ++ci)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int t = tb + lane + 32 * h;
        if (ci < nch && t < nt) {
          float wv = 0.f;
#pragma unroll
          for (int pp = 0; pp < 8; ++pp)
            if (pp < P) wv = fmaf(su[ci * 8 + pp], s.W[pp * nt + t], wv);
          a.Xres[(long long)(cbase + ci) * a.L + t0 + t] = __fsub_rn(xv[ci][h], __fmul_rn(amp, wv));
        }
      }
  }
}

__global__ void __launch_bounds__(kThreads, 2) peel_kernel(PeelArgs a) {
  extern __shared__ __align__(16) char smem_raw[];
  const Smem s = carve_smem(a, smem_raw);
  const int tid = threadIdx.x;
  const unsigned G = gridDim.x;
  for (int i = tid; i < a.P * a.nt; i += kThreads) s.W[i] = a.W[i];
  __syncthreads();

  // initial scores of every column, folded into pack[1] (zeroed by the host)
  const int lane = tid & 31;
  const long long gwarp = (long long)blockIdx.x * kWarps + (tid >> 5);
  const long long nwarps = (long long)G * kWarps;
  {
    unsigned long long* pinit = a.pack + (size_t)a.L;
    const int rg = (int)((a.K + 63) / 64);
    const TouchList none{0, nullptr, nullptr, nullptr};
    const long long n_items = (long long)a.nblk * rg;
    for (long long w = gwarp; w < n_items; w += nwarps) {
      const int blk = (int)(w / rg), r = (int)(w % rg);
      update_warp_item(a, none, blk, r * 64, min(a.K, (r + 1) * 64), pinit, lane);
    }
  }

  long long n_out = 0;
  int it = 0;
  int status = KS_OK;
  KS_TRACE(0, 7, ks_globaltimer());
  bool ok = ks_grid_sync(a.bar, G, a.err, a.limit_ns);
  for (; ok && it < a.max_peels; ++it) {
    const int p = it & 1, q = p ^ 1;
    KS_TRACE(it, 0, ks_globaltimer());
    for (int ch = blockIdx.x; ch < a.nchunks; ch += G) detect_chunk(a, s, ch, it);
    KS_TRACE(it, 1, ks_globaltimer());
    if (!ks_grid_sync(a.bar, G, a.err, a.limit_ns)) break;
    KS_TRACE(it, 2, ks_globaltimer());

    const int total = chunk_prefix(a, s);
    if (total == 0) break;
    if (n_out + total > a.capacity) {
      status = KS_ERR_OVERFLOW;
      if (blockIdx.x == 0 && tid == 0) a.info[3] = n_out + total;
      break;
    }
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
    // registration lists of the next iteration start empty
    for (int w = blockIdx.x * kThreads + tid; w < a.nblk; w += G * kThreads)
      a.tcount[(size_t)q * a.nblk + w] = 0;
    if (blockIdx.x == 0 && tid == 0) a.dcount[q] = 0;
    // subtract and rescore dirty blocks; residual windows -- one work list of
    // warp items, row ranges sized so that every warp gets about two items
    const int ndirty = a.dcount[p];
    int rgroups = 1;
    if (ndirty > 0) {
      const long long want = (2 * nwarps + ndirty - 1) / ndirty;
      const long long cap = (a.K + kRowsPerWarp - 1) / kRowsPerWarp;
      rgroups = (int)(want < 1 ? 1 : (want > cap ? cap : want));
    }
    const int rows = (a.K + rgroups - 1) / rgroups;
    const long long n_upd = (long long)ndirty * rgroups;
    const int xgroups = (a.C + kXresChans - 1) / kXresChans;
    const long long n_x = (long long)total * xgroups;
    unsigned long long* pcur = a.pack + (size_t)p * a.L;
    KS_TRACE(it, 3, ks_globaltimer());
    for (long long w = gwarp; w < n_upd + n_x; w += nwarps) {
      if (w < n_upd) {
        const int blk = a.dlist[(size_t)p * a.nblk + (int)(w / rgroups)];
        const int r = (int)(w % rgroups);
        const TouchList tl = load_touch_warp(a, s, p, blk, lane, tid >> 5);
        update_warp_item(a, tl, blk, r * rows, min(a.K, (r + 1) * rows), pcur, lane);
      } else {
        const long long x = w - n_upd;
        xres_warp_item(a, s, (int)(x / xgroups), (int)(x % xgroups), lane, tid >> 5);
      }
    }
    KS_TRACE(it, 4, ks_globaltimer());
    KS_TRACE(it, 5, total);
    KS_TRACE(it, 6, ndirty);
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
  int nchunks, nblk;
  size_t zero_bytes;   // leading bytes that must start at zero
  size_t bytes;
};

// Workspace order: [ctl: bar(2) err(1) pad(1) dcount(2) pad(2)] [tcount 2*nblk]
// [pack 2*L] -- the leading part up to and including pack[1] is zeroed per launch.
PeelLayout peel_layout(int64_t L) {
  PeelLayout l;
  l.nchunks = (int)((L + kChunk - 1) / kChunk);
  l.nblk = (int)((L + kCol - 1) / kCol);
  ks::Carve cv(nullptr);
  cv.take<unsigned>(8);
  cv.take<int>(2 * (size_t)l.nblk);
  cv.take<unsigned long long>(2 * (size_t)L);
  l.zero_bytes = cv.used;
  cv.take<float>(L);
  cv.take<int>(L);
  cv.take<int>(l.nchunks);
  for (int i = 0; i < 4; ++i) cv.take<int>((size_t)l.nchunks * kChunk);
  cv.take<Touch>(2 * (size_t)l.nblk * kTouch);
  cv.take<int>(2 * (size_t)l.nblk);
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
      nt > 1023 || P > 8)
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
  unsigned* ctl = cv.take<unsigned>(8);
  a.bar = ctl;
  a.err = reinterpret_cast<int*>(ctl + 2);
  a.dcount = reinterpret_cast<int*>(ctl + 4);
  a.tcount = cv.take<int>(2 * (size_t)lay.nblk);
  a.pack = cv.take<unsigned long long>(2 * (size_t)L);
  a.cfmax = cv.take<float>(L);
  a.imax = cv.take<int>(L);
  a.chunk_cnt = cv.take<int>(lay.nchunks);
  a.chunk_tau = cv.take<int>((size_t)lay.nchunks * kChunk);
  a.chunk_k = cv.take<int>((size_t)lay.nchunks * kChunk);
  a.chunk_amp = cv.take<float>((size_t)lay.nchunks * kChunk);
  a.chunk_th = cv.take<float>((size_t)lay.nchunks * kChunk);
  a.touch = cv.take<Touch>(2 * (size_t)lay.nblk * kTouch);
  a.dlist = cv.take<int>(2 * (size_t)lay.nblk);
  a.nchunks = lay.nchunks; a.nblk = lay.nblk;
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
  KS_CUDA(cudaMemsetAsync(ws, 0, lay.zero_bytes, stream));
  void* args[] = {&a};
  KS_CUDA(cudaLaunchCooperativeKernel((void*)peel_kernel, dim3(grid), dim3(kThreads), args, smem, stream));
  return KS_OK;
}

}  // namespace ks
