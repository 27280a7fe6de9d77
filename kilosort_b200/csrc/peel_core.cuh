// Device code of the greedy peel, shared by the single-batch launch
// (peel.cu) and the multi-batch launch (batched.cu).
// Greedy peel (matching pursuit) of one batch as a single persistent,
// cooperative kernel.  Semantics follow kilosort/template_matching.py:183-244.
//
// Layout in HBM
//   Bt     [nblk][K][32] f32   score matrix B[k, tau] tiled by 32-column blocks
//                              (nblk = ceil(L/32)): a block's K rows are one
//                              contiguous 128*K-byte run, so rescoring a block
//                              streams it instead of touching K scattered lines
//   ctcT   [K][K][2nt+1] f32   ctcT[k][j][l] = ctc[j][k][l]: the cross-
//                              correlations a peak of template k subtracts are
//                              one contiguous slab
//   Xres   [C][L] f32          residual, updated in place
//   cfmax [L] f32 / imax [L] i32  settled best score relu(B)^2/nm over
//                              templates, and its template, per column
//   pack   [2][L] u64          rescoring of dirty columns per iteration:
//                              (score bits << 32) | ~template under atomicMax,
//                              so the larger score and, on ties, the smaller
//                              template index win
//   per-iteration (double buffered by parity): dirty-block bitmap, touch
//   lists (peaks within +-nt of each dirty block) and a work counter
//
// Iteration it (p = it & 1, q = p ^ 1), two phases between device-wide barriers:
//   DETECT  per 256-column chunk whose +-nt neighbourhood changed in it-1:
//           settle the rescored columns (pack[q] -> cfmax/imax); pooled =
//           max of cfmax over +-nt (doubling levels of a sliding max); a column
//           is a peak iff pooled > th2 and |pooled - cfmax| < 1e-9 (kilosort
//           :206-212).  Peaks are compacted in time order; amplitude
//           B[k,tau]/nm[k] and sqrt(pooled) come from the pre-subtraction B
//           (:225-229).  Each peak registers in the touch lists of the blocks
//           within +-nt of it; the first registration sets the block's dirty bit
//           and clears its pack[p] entries.
//   UPDATE  every block computes the exclusive prefix of the chunk counts (a
//           peak's global index in the iteration) and of the dirty bitmap.
//           Records are written in (iteration, tau) order.  Warps take work
//           items (dirty block in column order, row range) from a counter
//           (large teams: round-robin, the last round from the counter):
//           B[j,c] -= amp*ctc[j,k,c-tau+nt] for the peaks touching column c,
//           even-indexed peaks first, then odd-indexed -- the order of the
//           reference's two interleaved groups (:235-238) -- product and
//           difference rounded separately; rescored rows fold into pack[p].
// The loop ends when no peak is found or after max_peels iterations, decided
// identically by every block from the same counts.  The residual (:237) is not
// read inside the loop, so its updates run once afterwards: per 32-column
// block the spikes whose windows cover it are gathered from the time-sorted
// records of each iteration and subtracted element by element in record order,
// the order of the reference's iterations; every element of Xres is read and
// written once instead of once per touching spike.  Every device-wide wait is
// bounded; a wait that runs out records KS_ERR_TIMEOUT and all blocks leave.
#pragma once
#include "ks_common.cuh"
#include "project.cuh"

namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kChunk = 256;          // detection chunk, one column per thread
constexpr int kCol = 32;             // update block, one column per lane
constexpr int kRowsPerWarp = 16;     // template rows in flight per lane (2 blocks per SM)
constexpr int kItemRows = 64;        // template rows per update item, large teams (at most)
constexpr int kItemRowsSmall = 640;  // the same, small teams: a whole block's rows per
                                     // item (one fold per column instead of ten)
constexpr int kStaticWarps = 1024;   // teams of at least this many warps deal items statically
constexpr int kTouch = 8;            // peaks touching one block (more: ties)
constexpr int kMaxChunks = 16384;
constexpr int kMaxIters = 4096;      // iterations whose record offsets are kept
constexpr int kMaxTemplates = 65536; // templates of one batch
constexpr int kXList = 64;           // residual list entries per warp and epoch
constexpr int kXCap = 32;            // spikes recorded per block for the residual

// Phase timeline for profiling builds (-DKS_PEEL_TRACE): block 0 writes
// %globaltimer stamps to info[8 + 8*it + slot]; the caller sizes info.
#ifdef KS_PEEL_TRACE
#define KS_TRACE(it, slot, value)                                        \
  do {                                                                   \
    if (a.trace && blockIdx.x == 0 && threadIdx.x == 0 && (it) < 200)    \
      a.info[8 + 8 * (it) + (slot)] = (long long)(value);                \
  } while (0)
// every block's end-of-work stamp of iterations < 8 at info[1608 + it*G + block]
#define KS_TRACE_CTA(it, value)                                                  \
  do {                                                                           \
    if (a.trace && threadIdx.x == 0 && (it) < 8)                                 \
      a.info[1608 + (it) * gridDim.x + blockIdx.x] = (long long)(value);          \
  } while (0)
#else
#define KS_TRACE(it, slot, value) \
  do {                           \
  } while (0)
#define KS_TRACE_CTA(it, value) \
  do {                          \
  } while (0)
#endif

struct Touch {
  int tau;
  int k;
  float amp;
  int slot;  // chunk * kChunk + index in chunk
};

struct PeelArgs {
  float* Bt;
  float* Xres;
  const float* U;
  const float* W;
  const float* ctcT;
  const float* nm;
  const float2* nmi;          // {nm[j], 1/nm[j]} (1/nm NaN when nm is not a positive normal)
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
  unsigned* dbits;            // [2][nwords]
  unsigned* wctr;             // [2] work counters
  int* itoff;                 // [kMaxIters] first record of each iteration
  int* xcount;                // [nblk] spikes whose residual window meets the block
  int* xlist;                 // [nblk * kXCap] their record indices (unordered)
  unsigned* bar;              // barrier arrival count (monotonic)
  int* err;
  const int* upstream_err;    // error word of the producer of Bt (may be null)
  int nchunks, nblk, nwords;
  int trace;                  // profiling builds: 1 where info has room for the timeline
  unsigned long long limit_ns;
};

struct Smem {
  float* W;        // Wt[nt][8] (the fused residual's basis)
  int* prefix;     // nchunks+1   exclusive prefix of chunk peak counts
  int* wprefix;    // nwords+1    exclusive prefix of dirty-bitmap popcounts
  float* win;      // kChunk + 2*nt   column scores around the chunk
  float* mx0;      // kChunk + 2*nt   sliding-max doubling levels (ping-pong)
  float* mx1;      // kChunk + 2*nt
  int* kidx;       // kChunk          best template of the chunk's own columns
  int* wcnt;       // kWarps+1
  int* tl_tau;     // kWarps*kTouch   ordered touch list of each warp's item
  int* tl_k;       // kWarps*kTouch
  float* tl_amp;   // kWarps*kTouch
};

// Wt[t][p] = W[p][t] for p < P, 0 for P <= p < 8: each tap's components are
// two aligned float4 in shared memory.
__device__ __forceinline__ void stage_basis_t8(const float* W, int P, int nt, float* sWt,
                                               int nthreads) {
  for (int i = threadIdx.x; i < 8 * nt; i += nthreads) {
    const int t = i >> 3, p = i & 7;
    sWt[i] = p < P ? W[p * nt + t] : 0.f;
  }
}

__device__ __forceinline__ Smem carve_smem(const PeelArgs& a, char* base) {
  Smem s;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* p = base + off;
    off = (off + bytes + 15) & ~size_t(15);
    return p;
  };
  const int wn = kChunk + 2 * a.nt;
  s.W = reinterpret_cast<float*>(take(sizeof(float) * 8 * a.nt));
  s.prefix = reinterpret_cast<int*>(take(sizeof(int) * (a.nchunks + 1)));
  s.wprefix = reinterpret_cast<int*>(take(sizeof(int) * (a.nwords + 1)));
  s.win = reinterpret_cast<float*>(take(sizeof(float) * wn));
  s.mx0 = reinterpret_cast<float*>(take(sizeof(float) * wn));
  s.mx1 = reinterpret_cast<float*>(take(sizeof(float) * wn));
  s.kidx = reinterpret_cast<int*>(take(sizeof(int) * kChunk));
  s.wcnt = reinterpret_cast<int*>(take(sizeof(int) * (kWarps + 1)));
  s.tl_tau = reinterpret_cast<int*>(take(sizeof(int) * kWarps * kTouch));
  s.tl_k = reinterpret_cast<int*>(take(sizeof(int) * kWarps * kTouch));
  s.tl_amp = reinterpret_cast<float*>(take(sizeof(float) * kWarps * kTouch));
  return s;
}

size_t smem_bytes(int P, int nt, int nchunks, int nwords) {
  auto r = [](size_t b) { return (b + 15) & ~size_t(15); };
  const size_t wn = kChunk + 2 * (size_t)nt;
  (void)P;
  return r(sizeof(float) * 8 * nt) + r(sizeof(int) * (nchunks + 1)) +
         r(sizeof(int) * (nwords + 1)) + 3 * r(sizeof(float) * wn) +
         r(sizeof(int) * kChunk) + r(sizeof(int) * (kWarps + 1)) +
         3 * r(sizeof(int) * kWarps * kTouch);
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
// Fold row j's score relu(b)^2/nm[j] into (best, arg) -- larger score wins,
// the earlier (smaller) row on ties -- computing the IEEE quotient only where
// it can matter: sq*(1/nm) is within a relative 2^-22 of sq/nm, so a row whose
// quotient could reach best has sq*(1/nm) >= best*(1 - 2^-20).  Rows failing
// that test cannot change (best, arg).  The quotient itself is the exactly
// rounded division, as in the reference.
__device__ __forceinline__ void fold_score(float b, float2 nmi, int j, float& best, int& arg) {
  const float rl = b > 0.f ? b : 0.f;
  const float sq = __fmul_rn(rl, rl);
  const float approx = __fmul_rn(sq, nmi.y);
  const bool maybe = best < 0.f || !(approx < best * 0.99999905f) || approx != approx;
  if (maybe) {
    const float cf = __fdiv_rn(sq, nmi.x);
    if (cf > best) {
      best = cf;
      arg = j;
    }
  }
}

__device__ __forceinline__ const float* bt_row(const PeelArgs& a, int blk, int j) {
  return a.Bt + ((size_t)blk * a.K + j) * kCol;
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
  // Column scores: rescored columns of the last iteration come from pack[q]
  // (and are settled into cfmax/imax by the chunk that owns them), the others
  // from cfmax.  The candidate loads are independent and issued together; if
  // nothing within +-nt of the chunk changed, its peak test cannot change and
  // the chunk is skipped.
  int any_fresh = 0;
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
      any_fresh |= fresh;
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
  if (!__syncthreads_or(any_fresh)) {
    if (tid == 0) a.chunk_cnt[ch] = 0;
    return;
  }
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
  if (tid < kChunk && tau < a1 && tau >= nt && tau < L - nt) {
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
    const float amp = __fdiv_rn(bt_row(a, tau / kCol, k)[tau % kCol], a.nm[k]);
    const float th = __fsqrt_rn(pooled);
    const int slot = ch * kChunk + idx;
    a.chunk_tau[slot] = tau;
    a.chunk_k[slot] = k;
    a.chunk_amp[slot] = amp;
    a.chunk_th[slot] = th;
    int* tcur = a.tcount + (size_t)p * a.nblk;
    Touch* tch = a.touch + (size_t)p * a.nblk * kTouch;
    unsigned* bits = a.dbits + (size_t)p * a.nwords;
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
          atomicOr(&bits[b >> 5], 1u << (b & 31));
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

// Both exclusive prefixes an iteration needs, in one pass: of the chunk peak
// counts into s.prefix[0..nchunks] and of the dirty-bitmap word popcounts into
// s.wprefix[0..nwords].  All threads of the block take part.
__device__ void two_prefix(const int* cnt, int nchunks, const unsigned* bits, int nwords,
                           const Smem& s, int& total, int& ndirty) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int pc = (nchunks + kThreads - 1) / kThreads;
  const int pw = (nwords + kThreads - 1) / kThreads;
  int lc = 0, lw = 0;
  for (int i = 0; i < pc; ++i) {
    const int c = tid * pc + i;
    if (c < nchunks) lc += cnt[c];
  }
  for (int i = 0; i < pw; ++i) {
    const int w = tid * pw + i;
    if (w < nwords) lw += __popc(bits[w]);
  }
  int ic = lc, iw = lw;
  for (int o = 1; o < 32; o <<= 1) {
    const int vc = __shfl_up_sync(0xffffffffu, ic, o);
    const int vw = __shfl_up_sync(0xffffffffu, iw, o);
    if (lane >= o) { ic += vc; iw += vw; }
  }
  int* wc = s.wcnt;                 // [kWarps+1] chunk totals per warp
  int* ww = s.kidx;                 // [kWarps+1] word totals per warp (kidx is free here)
  if (lane == 31) { wc[warp] = ic; ww[warp] = iw; }
  __syncthreads();
  if (tid == 0) {
    int ac = 0, aw = 0;
    for (int w = 0; w < kWarps; ++w) {
      const int c = wc[w], x = ww[w];
      wc[w] = ac; ww[w] = aw;
      ac += c; aw += x;
    }
    wc[kWarps] = ac; ww[kWarps] = aw;
  }
  __syncthreads();
  int rc = wc[warp] + ic - lc, rw = ww[warp] + iw - lw;
  for (int i = 0; i < pc; ++i) {
    const int c = tid * pc + i;
    if (c < nchunks) { s.prefix[c] = rc; rc += cnt[c]; }
  }
  for (int i = 0; i < pw; ++i) {
    const int w = tid * pw + i;
    if (w < nwords) { s.wprefix[w] = rw; rw += __popc(bits[w]); }
  }
  if (tid == 0) { s.prefix[nchunks] = wc[kWarps]; s.wprefix[nwords] = ww[kWarps]; }
  __syncthreads();
  total = s.prefix[nchunks];
  ndirty = s.wprefix[nwords];
}

// ---------------------------------------------------------------- UPDATE
// Ordered touch list of one block in the warp's shared-memory slot: entry e
// (application order: even global index first, then odd, each ascending) has
// peak time tau[e], template k[e], amplitude amp[e].
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

// Columns of block blk x template rows [j_lo, j_hi): subtract the touching
// peaks, store the changed rows, fold the rescored rows into pack_out.  Most
// columns are touched by one peak; its cross-correlations are loaded with the
// rows of B (16 rows per round trip).  Later peaks of the same column (at
// most one more unless scores tie exactly) are applied in a second round, in
// the same order.  A column no peak touches keeps its rows, so its score is
// its settled one (cfmax/imax): the item holding row 0 passes that on instead
// of re-reading the rows (all columns are scored from B when init is set).
template <int kRows>
__device__ void update_warp_item(const PeelArgs& a, const TouchList& tl, int blk,
                                 int j_lo, int j_hi, unsigned long long* pack_out,
                                 int lane, bool init = false) {
  const int c = blk * kCol + lane;
  const bool colok = c < a.L;
  const int nt = a.nt, K = a.K, nlag = 2 * nt + 1;
  int e0 = -1;
  unsigned rest = 0u;                                 // further touching entries
  for (int e = 0; e < tl.n; ++e) {
    const int d = c - tl.tau[e];
    if (colok && d >= -nt && d <= nt) {
      if (e0 < 0) e0 = e;
      else rest |= 1u << e;
    }
  }
  const bool touched = e0 >= 0;
  const bool score = init || touched;
  const bool any_rest = __any_sync(0xffffffffu, rest != 0u);
  const float* cp0 = a.ctcT;
  float amp0 = 0.f;
  if (e0 >= 0) { cp0 = a.ctcT + (size_t)tl.k[e0] * K * nlag + (c - tl.tau[e0] + nt); amp0 = tl.amp[e0]; }
  float* bcol = a.Bt + (size_t)blk * K * kCol + lane;
  float best = -1.f;
  int arg = 0;
  for (int j0 = j_lo; j0 < j_hi; j0 += kRows) {
    float bv[kRows], w0[kRows];
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const int j = j0 + r;
      const bool ok = score && colok && j < j_hi;
      bv[r] = ok ? bcol[(size_t)j * kCol] : 0.f;
      w0[r] = (ok && e0 >= 0) ? __ldg(cp0 + (size_t)j * nlag) : 0.f;
    }
    if (e0 >= 0) {
#pragma unroll
      for (int r = 0; r < kRows; ++r) bv[r] = __fsub_rn(bv[r], __fmul_rn(amp0, w0[r]));
    }
    if (any_rest) {
      for (int e = 0; e < tl.n; ++e) {
        if ((rest >> e) & 1u) {
          const float amp = tl.amp[e];
          const float* cp = a.ctcT + (size_t)tl.k[e] * K * nlag + (c - tl.tau[e] + nt);
#pragma unroll
          for (int r = 0; r < kRows; ++r) {
            const int j = j0 + r;
            w0[r] = (j < j_hi) ? __ldg(cp + (size_t)j * nlag) : 0.f;
          }
#pragma unroll
          for (int r = 0; r < kRows; ++r) bv[r] = __fsub_rn(bv[r], __fmul_rn(amp, w0[r]));
        }
      }
    }
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const int j = j0 + r;
      if (score && colok && j < j_hi) {
        if (touched) bcol[(size_t)j * kCol] = bv[r];
        fold_score(bv[r], __ldg(a.nmi + j), j, best, arg);
      }
    }
  }
  if (colok) {
    if (score) {
      if (best >= 0.f) atomicMax(&pack_out[c], pack_score(best, arg));
    } else if (j_lo == 0) {
      atomicMax(&pack_out[c], pack_score(a.cfmax[c], a.imax[c]));
    }
  }
}

// Block of the rank-th set bit of the dirty bitmap (s.wprefix holds the
// exclusive prefix of the word popcounts).
__device__ __forceinline__ int dirty_block(const Smem& s, const unsigned* bits,
                                           int nwords, int rank) {
  int lo = 0, hi = nwords - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (s.wprefix[mid] <= rank) lo = mid; else hi = mid - 1;
  }
  const unsigned word = bits[lo];
  const int bit = (int)__fns(word, 0, rank - s.wprefix[lo] + 1);
  return lo * 32 + bit;
}

// Outcome of one batch's peel, the same in every block of the team.
struct PeelOutcome {
  long long n_out;
  int iters;
  int status;
};

// The peel of one batch by a team of G co-resident blocks (this block has
// rank `rank` in it); epoch is the team barrier's count of passed barriers,
// carried across the batches a team processes.  The team first clears the
// batch's per-run state, then runs the iterations; the outcome goes to info
// (written by one thread) and is returned to every thread.  When the status
// is KS_OK every record and residual list of the batch is complete and
// visible to the team (the last pass ended at a team barrier).
template <int kRows>
__device__ PeelOutcome run_peel(const PeelArgs& a, const Smem& s, int rank, unsigned G,
                                unsigned& epoch) {
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const long long gwarp = (long long)rank * kWarps + warp;
  const long long nwarps = (long long)G * kWarps;
  stage_basis_t8(a.W, a.P, a.nt, s.W, kThreads);
  // a failed producer of the score matrix fails the peel
  if (rank == 0 && tid == 0 && a.upstream_err) {
    const int ue = ks_ld_volatile(a.upstream_err);
    if (ue) atomicCAS(a.err, 0, ue);
  }
  // per-batch state starts empty: registration counts, dirty bitmaps, both
  // rescoring buffers (pack[1] receives the initial scores), work counters and
  // the residual lists
  {
    const long long t0 = (long long)rank * kThreads + tid, ts = (long long)G * kThreads;
    for (long long i = t0; i < 2LL * a.nblk; i += ts) a.tcount[i] = 0;
    for (long long i = t0; i < 2LL * a.nwords; i += ts) a.dbits[i] = 0u;
    for (long long i = t0; i < 2LL * a.L; i += ts) a.pack[i] = 0ull;
    for (long long i = t0; i < a.nblk; i += ts) a.xcount[i] = 0;
    if (t0 < 2) a.wctr[t0] = 0u;
  }
  if (!ks_grid_sync(a.bar, G, epoch, a.err, a.limit_ns)) {
    const int e = ks_ld_volatile(a.err);
    if (rank == 0 && tid == 0) {
      a.info[0] = 0;
      a.info[1] = e;
      a.info[2] = 0;
      a.info[3] = 0;
    }
    return PeelOutcome{0, 0, e ? e : KS_ERR_TIMEOUT};
  }

  // initial scores of every column, folded into pack[1]
  {
    unsigned long long* pinit = a.pack + (size_t)a.L;
    const int rg = (a.K + kItemRows - 1) / kItemRows;
    const TouchList none{0, nullptr, nullptr, nullptr};
    const long long n_items = (long long)a.nblk * rg;
    for (long long w = gwarp; w < n_items; w += nwarps) {
      const int blk = (int)(w / rg), r = (int)(w % rg);
      update_warp_item<kRows>(a, none, blk, r * kItemRows, min(a.K, (r + 1) * kItemRows), pinit,
                              lane, true);
    }
  }

  long long n_out = 0;
  int it = 0;
  int status = KS_OK;
  KS_TRACE(0, 7, ks_globaltimer());
  bool ok = ks_grid_sync(a.bar, G, epoch, a.err, a.limit_ns);
  for (; ok && it < a.max_peels; ++it) {
    const int p = it & 1, q = p ^ 1;
    KS_TRACE(it, 0, ks_globaltimer());
    for (int ch = rank; ch < a.nchunks; ch += (int)G) detect_chunk(a, s, ch, it);
    KS_TRACE(it, 1, ks_globaltimer());
    if (!ks_grid_sync(a.bar, G, epoch, a.err, a.limit_ns)) break;
    KS_TRACE(it, 2, ks_globaltimer());

    const unsigned* bits = a.dbits + (size_t)p * a.nwords;
    int total, ndirty;
    two_prefix(a.chunk_cnt, a.nchunks, bits, a.nwords, s, total, ndirty);
    if (total == 0) break;
    if (n_out + total > a.capacity) {
      status = KS_ERR_OVERFLOW;
      if (rank == 0 && tid == 0) a.info[3] = n_out + total;
      break;
    }
    // one warp per chunk (the chunks' peak counts are independent loads)
    for (int ch = rank * kWarps + warp; ch < a.nchunks; ch += (int)G * kWarps) {
      const int c_n = a.chunk_cnt[ch];
      for (int i = lane; i < c_n; i += 32) {
        const long long slot = (long long)ch * kChunk + i;
        const long long o = n_out + s.prefix[ch] + i;
        const int tau = a.chunk_tau[slot];
        a.st[2 * o] = tau;
        a.st[2 * o + 1] = a.chunk_k[slot];
        a.amps[o] = a.chunk_amp[slot];
        a.th_amps[o] = a.chunk_th[slot];
        // blocks whose columns this spike's residual window covers
        const int xb0 = (tau - a.nt / 2) / kCol, xb1 = (tau + a.nt / 2) / kCol;
        for (int b = xb0; b <= xb1; ++b) {
          const int pos = atomicAdd(&a.xcount[b], 1);
          if (pos < kXCap) a.xlist[(size_t)b * kXCap + pos] = (int)o;
        }
      }
    }
    // registration lists, bitmap and work counter of the next iteration start empty
    for (int w = rank * kThreads + tid; w < a.nblk; w += (int)G * kThreads)
      a.tcount[(size_t)q * a.nblk + w] = 0;
    for (int w = rank * kThreads + tid; w < a.nwords; w += (int)G * kThreads)
      a.dbits[(size_t)q * a.nwords + w] = 0u;
    if (rank == 0 && tid == 0) a.wctr[q] = 0u;
    // update items: (dirty block in column order, row range), sized so that
    // there are about four per warp
    // rows per item: the split whose most loaded warp has the least work
    // (row groups of 16 plus one group's worth of per-item set-up)
    const int item_cap = nwarps >= kStaticWarps ? kItemRows : kItemRowsSmall;
    int rows = kItemRows;
    if (ndirty > 0) {
      long long best_cost = -1;
      for (int r = kRows; r <= item_cap; r += kRows) {
        const long long items = (long long)ndirty * ((a.K + r - 1) / r);
        const long long per_warp = (items + nwarps - 1) / nwarps;
        const long long cost = per_warp * (r / kRows + 1);
        if (best_cost < 0 || cost < best_cost) {
          best_cost = cost;
          rows = r;
        }
      }
    }
    const int rgroups = (a.K + rows - 1) / rows;
    const long long n_upd = (long long)ndirty * rgroups;
    const long long n_items = n_upd;
    if (rank == 0 && tid == 0) a.itoff[it] = (int)n_out;
    unsigned long long* pcur = a.pack + (size_t)p * a.L;
    KS_TRACE(it, 3, ks_globaltimer());
    // Items go to warps in item order, so consecutive items (neighbouring
    // blocks, which share the slabs of their peaks) run at about the same
    // time.  A small team takes every item from the counter: warps that ran
    // into slower memory take fewer of them (a static deal left the blocks
    // of a 14-block team up to 20 % of an iteration apart at the closing
    // barrier).  A large team deals all but its last round round-robin, so
    // thousands of warps do not queue on one counter.
    const long long rounds = n_items / nwarps;
    const long long n_static =
        (nwarps >= kStaticWarps && rounds > 1) ? (rounds - 1) * nwarps : 0;
    for (long long w = gwarp; w < n_static; w += nwarps) {
      const int blk = dirty_block(s, bits, a.nwords, (int)(w / rgroups));
      const int r = (int)(w % rgroups);
      const TouchList tl = load_touch_warp(a, s, p, blk, lane, warp);
      update_warp_item<kRows>(a, tl, blk, r * rows, min(a.K, (r + 1) * rows), pcur, lane);
    }
    while (true) {
      unsigned next = 0;
      if (lane == 0) next = atomicAdd(&a.wctr[p], 1u);
      const long long w = n_static + (long long)__shfl_sync(0xffffffffu, next, 0);
      if (w >= n_items) break;
      const int blk = dirty_block(s, bits, a.nwords, (int)(w / rgroups));
      const int r = (int)(w % rgroups);
      const TouchList tl = load_touch_warp(a, s, p, blk, lane, warp);
      update_warp_item<kRows>(a, tl, blk, r * rows, min(a.K, (r + 1) * rows), pcur, lane);
    }
    KS_TRACE(it, 4, ks_globaltimer());
    __syncthreads();
    KS_TRACE_CTA(it, ks_globaltimer());
    KS_TRACE(it, 5, total);
    KS_TRACE(it, 6, ndirty);
    n_out += total;
    ok = ks_grid_sync(a.bar, G, epoch, a.err, a.limit_ns);
  }
  // one read of the error word for the whole block
  const int e = __syncthreads_or(tid == 0 && ks_ld_volatile(a.err) != 0) ? ks_ld_volatile(a.err) : 0;
  if (rank == 0 && tid == 0) {
    a.info[0] = n_out;
    a.info[1] = e ? e : status;
    a.info[2] = it;
    if (status != KS_ERR_OVERFLOW) a.info[3] = n_out;
  }
  return PeelOutcome{n_out, it, e ? e : status};
}

__global__ void __launch_bounds__(kThreads, 2) peel_kernel(PeelArgs a) {
  extern __shared__ __align__(16) char smem_raw[];
  const Smem s = carve_smem(a, smem_raw);
  unsigned epoch = 0;
  run_peel<kRowsPerWarp>(a, s, blockIdx.x, gridDim.x, epoch);
}

constexpr int kXTile = kCol * (kCol + 1);   // floats of one warp's transpose tile

struct ResSmem {
  const float* W;  // Wt[t][8]: the basis transposed, components padded to 8
  int* xl_tau;     // warps*kXList
  int* xl_k;
  float* xl_amp;
  float* xt;       // warps*kXTile (tiled form only): 32 channels x 33 floats per warp
};

// ---------------------------------------------------------------- RESIDUAL
// After the loop: Xres[c, col] -= amp_s * sum_p U[k_s,p,c] W[p, col-tau_s+nt/2]
// for every spike s whose window covers col, applied in record order
// (iteration, then time) -- per element the order in which the reference's
// iterations subtract (:237).  Each element is read and written once.
//
// Gather, into the warp's list, the spikes of record positions
// [skip, skip + kXList) among those whose window meets columns [c0, c0+32):
// lanes binary-search the time-sorted run of one iteration each.  Returns the
// total number of such spikes.
__device__ int gather_residual(const PeelArgs& a, const ResSmem& s, int n_iter,
                               long long n_out, int c0, int skip, int lane, int warp) {
  __syncwarp();   // earlier readers of the warp's list are done
  const int half = a.nt / 2;
  const long long wlo = (long long)c0 - half, whi = (long long)c0 + kCol - 1 + half;
  int* ltau = s.xl_tau + warp * kXList;
  int* lk = s.xl_k + warp * kXList;
  float* lamp = s.xl_amp + warp * kXList;
  int total = 0;
  for (int i0 = 0; i0 < n_iter; i0 += 32) {
    const int i = i0 + lane;
    long long first = 0, last = 0;
    if (i < n_iter) {
      long long lo = a.itoff[i];
      const long long end = (i + 1 < n_iter) ? a.itoff[i + 1] : n_out;
      long long hi = end;
      while (lo < hi) {                       // first record with tau >= wlo
        const long long mid = (lo + hi) >> 1;
        if (a.st[2 * mid] < wlo) lo = mid + 1; else hi = mid;
      }
      first = lo;
      last = lo;
      while (last < end && a.st[2 * last] <= whi) ++last;
    }
    const int cnt = (int)(last - first);
    int incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const int base = total + incl - cnt;
    for (int e = 0; e < cnt; ++e) {
      const int pos = base + e - skip;
      if (pos >= 0 && pos < kXList) {
        const long long o = first + e;
        ltau[pos] = (int)a.st[2 * o];
        lk[pos] = (int)a.st[2 * o + 1];
        lamp[pos] = a.amps[o];
      }
    }
    total += __shfl_sync(0xffffffffu, incl, 31);
  }
  __syncwarp();
  return total;
}

// Load into the warp's list the spikes whose residual window meets block blk,
// in record order.  Returns their number; when it exceeds kXCap the per-block
// record list overflowed and the caller gathers with gather_residual instead.
__device__ int load_residual_list(const PeelArgs& a, const ResSmem& s, int blk, int lane,
                                  int warp) {
  __syncwarp();
  const int n = a.xcount[blk];
  if (n > kXCap) return n;
  const int o = lane < n ? a.xlist[(size_t)blk * kXCap + lane] : 0x7fffffff;
  int rank = 0;
  for (int j = 0; j < n; ++j) {
    const int oj = __shfl_sync(0xffffffffu, o, j);
    rank += (oj < o) ? 1 : 0;
  }
  if (lane < n) {
    s.xl_tau[warp * kXList + rank] = (int)a.st[2 * (long long)o];
    s.xl_k[warp * kXList + rank] = (int)a.st[2 * (long long)o + 1];
    s.xl_amp[warp * kXList + rank] = a.amps[o];
  }
  __syncwarp();
  return n;
}

// Residual of block blk for channels [32*cg, 32*cg + 32): lanes run over
// channels, each lane keeps its 32 residual values in registers while the
// listed spikes are subtracted in record order.  kTiled: the 32 x 32 tile
// moves a channel row at a time (lanes over columns, one coalesced access
// each) through a transpose in shared memory, instead of each lane touching
// its own row 32 times; the batched peel, whose update phase gains more from
// the L1 that this shared memory would take, uses the direct form.
template <bool kTiled>
__device__ void residual_item(const PeelArgs& a, const ResSmem& s, int n_iter, long long n_out,
                              int blk, int cg, int lane, int warp) {
  const int c0 = blk * kCol;
  const int half = a.nt / 2, nt = a.nt, P = a.P;
  const int c = cg * 32 + lane;
  const bool chok = c < a.C;
  int total = load_residual_list(a, s, blk, lane, warp);
  const bool overflow = total > kXCap;
  if (overflow) total = gather_residual(a, s, n_iter, n_out, c0, 0, lane, warp);
  if (total == 0) return;
  const int ncol = min(kCol, a.L - c0);
  float* xrow = a.Xres + (long long)c * a.L + c0;
  float* xt = kTiled ? s.xt + warp * kXTile : nullptr;
  const int cbase = cg * 32;
  const bool colok = lane < ncol;
  float x[kCol];
  if (kTiled) {
    {
      float v[kCol];
#pragma unroll
      for (int r = 0; r < kCol; ++r)
        v[r] = (colok && cbase + r < a.C) ? a.Xres[(long long)(cbase + r) * a.L + c0 + lane] : 0.f;
#pragma unroll
      for (int r = 0; r < kCol; ++r) xt[r * (kCol + 1) + lane] = v[r];
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < kCol; ++j) x[j] = xt[lane * (kCol + 1) + j];
  } else {
#pragma unroll
    for (int j = 0; j < kCol; ++j) x[j] = (chok && j < ncol) ? xrow[j] : 0.f;
  }
  const int epochs = (total + kXList - 1) / kXList;
  for (int ep = 0; ep < epochs; ++ep) {
    if (ep > 0) gather_residual(a, s, n_iter, n_out, c0, ep * kXList, lane, warp);
    const int n = min(kXList, total - ep * kXList);
    for (int e = 0; e < n; ++e) {
      const int tau = s.xl_tau[warp * kXList + e];
      const int k = s.xl_k[warp * kXList + e];
      const float amp = s.xl_amp[warp * kXList + e];
      const int t0 = c0 - tau + half;   // tap of column c0
      float u[8];
#pragma unroll
      for (int pp = 0; pp < 8; ++pp)
        u[pp] = (chok && pp < P) ? __ldg(a.U + ((long long)k * P + pp) * a.C + c) : 0.f;
      const float4* W4 = reinterpret_cast<const float4*>(s.W);
#pragma unroll
      for (int j = 0; j < kCol; ++j) {
        const int t = t0 + j;
        if (t >= 0 && t < nt) {
          // the tap's P components: two broadcast 16-byte loads
          const float4 wa = W4[2 * t], wb = W4[2 * t + 1];
          const float wt[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
          float wv = 0.f;
#pragma unroll
          for (int pp = 0; pp < 8; ++pp)
            if (pp < P) wv = fmaf(u[pp], wt[pp], wv);
          x[j] = __fsub_rn(x[j], __fmul_rn(amp, wv));
        }
      }
    }
  }
  if (kTiled) {
    __syncwarp();
#pragma unroll
    for (int j = 0; j < kCol; ++j) xt[lane * (kCol + 1) + j] = x[j];
    __syncwarp();
#pragma unroll
    for (int r = 0; r < kCol; ++r)
      if (colok && cbase + r < a.C)
        a.Xres[(long long)(cbase + r) * a.L + c0 + lane] = xt[r * (kCol + 1) + lane];
  } else {
#pragma unroll
    for (int j = 0; j < kCol; ++j)
      if (chok && j < ncol) xrow[j] = x[j];
  }
}

constexpr int kResThreads = 256;
constexpr int kResWarps = kResThreads / 32;

// One warp per (32-column block, 32 channels) of the residual; runs after the
// peel kernel on the same stream and reads its outcome from info.
__global__ void __launch_bounds__(kResThreads)
ks_residual_kernel(PeelArgs a) {
  extern __shared__ __align__(16) char smem_raw[];
  float* sW = reinterpret_cast<float*>(smem_raw);
  ResSmem s;
  s.W = sW;
  s.xl_tau = reinterpret_cast<int*>(sW + 8 * a.nt);
  s.xl_k = s.xl_tau + kResWarps * kXList;
  s.xl_amp = reinterpret_cast<float*>(s.xl_k + kResWarps * kXList);
  s.xt = s.xl_amp + kResWarps * kXList;
  stage_basis_t8(a.W, a.P, a.nt, sW, kResThreads);
  __syncthreads();
  const long long n_out = a.info[0];
  const int status = (int)a.info[1];
  const int n_iter = (int)a.info[2];
  if (status != KS_OK || n_out <= 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int xg = (a.C + 31) / 32;
  const long long n_items = (long long)a.nblk * xg;
  const long long w = (long long)blockIdx.x * kResWarps + warp;
  if (w >= n_items) return;
  residual_item<true>(a, s, n_iter, n_out, (int)(w / xg), (int)(w % xg), lane, warp);
}

size_t residual_smem_bytes(int P, int nt) {
  (void)P;
  return sizeof(float) * 8 * (size_t)nt +
         (size_t)kResWarps * kXList * (2 * sizeof(int) + sizeof(float)) +
         sizeof(float) * (size_t)kResWarps * kXTile;
}

__global__ void ks_nm_pair_kernel(const float* __restrict__ nm, int K, float2* __restrict__ nmi) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < K; j += gridDim.x * blockDim.x) {
    const float v = nm[j];
    const bool normal = v >= 1.17549435e-38f && v <= 3.40282347e38f;
    nmi[j] = make_float2(v, normal ? __frcp_rn(v) : __int_as_float(0x7fc00000));
  }
}

// ------------------------------------------------------------------ relayout
__global__ void ks_tile_rows_kernel(const float* __restrict__ B, long long ldb, int K,
                                    int L, int nblk, float* __restrict__ Bt) {
  const long long n = (long long)nblk * K * kCol;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % kCol);
    const long long bj = e / kCol;
    const int j = (int)(bj % K);
    const int blk = (int)(bj / K);
    const int col = blk * kCol + c;
    Bt[e] = col < L ? B[(long long)j * ldb + col] : 0.f;
  }
}

__global__ void ks_untile_rows_kernel(const float* __restrict__ Bt, int K, int L,
                                      float* __restrict__ B, long long ldb) {
  const long long n = (long long)K * L;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int col = (int)(e % L);
    const int j = (int)(e / L);
    B[(long long)j * ldb + col] = Bt[((long long)(col / kCol) * K + j) * kCol + (col % kCol)];
  }
}

__global__ void ks_ctc_transpose_kernel(const float* __restrict__ ctc, int K, int nlag,
                                        float* __restrict__ ctcT) {
  // ctcT[k][j][l] = ctc[j][k][l]; one row of nlag contiguous floats per (k, j)
  const long long rows = (long long)K * K;
  for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
    const int k = (int)(r / K), j = (int)(r % K);
    const float* src = ctc + ((long long)j * K + k) * nlag;
    float* dst = ctcT + r * nlag;
    for (int l = threadIdx.x; l < nlag; l += blockDim.x) dst[l] = src[l];
  }
}

// Scratch of one team (reused for every batch it processes), for batches of
// up to L padded samples: [ctl 256 B: barrier count, error word] [cfmax L]
// [imax L] [pack 2L] [chunk counts] [chunk buffers 4 x nchunks*kChunk]
// [tcount 2 nblk] [touch 2 nblk*kTouch] [dbits 2 nwords] [work counters 2].
// Only the control words need zeroing before a launch; the team clears the
// rest per batch.
struct TeamLayout {
  size_t cfmax, imax, pack, chunk_cnt, chunk_tau, chunk_k, chunk_amp, chunk_th, tcount,
      touch, dbits, wctr, bytes;
};

__host__ __device__ inline size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

__host__ __device__ inline TeamLayout team_layout(long long L) {
  const long long nchunks = (L + kChunk - 1) / kChunk, nblk = (L + kCol - 1) / kCol;
  const long long nwords = (nblk + 31) / 32;
  TeamLayout t;
  size_t o = 256;
  t.cfmax = o; o = al256(o + 4 * (size_t)L);
  t.imax = o; o = al256(o + 4 * (size_t)L);
  t.pack = o; o = al256(o + 16 * (size_t)L);
  t.chunk_cnt = o; o = al256(o + 4 * (size_t)nchunks);
  t.chunk_tau = o; o = al256(o + 4 * (size_t)nchunks * kChunk);
  t.chunk_k = o; o = al256(o + 4 * (size_t)nchunks * kChunk);
  t.chunk_amp = o; o = al256(o + 4 * (size_t)nchunks * kChunk);
  t.chunk_th = o; o = al256(o + 4 * (size_t)nchunks * kChunk);
  t.tcount = o; o = al256(o + 8 * (size_t)nblk);
  t.touch = o; o = al256(o + 2 * sizeof(Touch) * (size_t)nblk * kTouch);
  t.dbits = o; o = al256(o + 8 * (size_t)nwords);
  t.wctr = o; o = al256(o + 8);
  t.bytes = o;
  return t;
}

// Lists a batch keeps until its residual pass: [iteration offsets kMaxIters]
// [residual counts nblk] [residual lists nblk*kXCap].
struct ListLayout {
  size_t itoff, xcount, xlist, bytes;
};

__host__ __device__ inline ListLayout list_layout(long long L) {
  const long long nblk = (L + kCol - 1) / kCol;
  ListLayout t;
  size_t o = 0;
  t.itoff = o; o = al256(o + 4 * (size_t)kMaxIters);
  t.xcount = o; o = al256(o + 4 * (size_t)nblk);
  t.xlist = o; o = al256(o + 4 * (size_t)nblk * kXCap);
  t.bytes = o;
  return t;
}

// Point the scratch fields of a at a team region and a list region.
__host__ __device__ inline void bind_scratch(PeelArgs& a, char* team, char* lists) {
  const TeamLayout t = team_layout(a.L);
  const ListLayout l = list_layout(a.L);
  a.bar = reinterpret_cast<unsigned*>(team);
  a.err = reinterpret_cast<int*>(team + 64);
  a.cfmax = reinterpret_cast<float*>(team + t.cfmax);
  a.imax = reinterpret_cast<int*>(team + t.imax);
  a.pack = reinterpret_cast<unsigned long long*>(team + t.pack);
  a.chunk_cnt = reinterpret_cast<int*>(team + t.chunk_cnt);
  a.chunk_tau = reinterpret_cast<int*>(team + t.chunk_tau);
  a.chunk_k = reinterpret_cast<int*>(team + t.chunk_k);
  a.chunk_amp = reinterpret_cast<float*>(team + t.chunk_amp);
  a.chunk_th = reinterpret_cast<float*>(team + t.chunk_th);
  a.tcount = reinterpret_cast<int*>(team + t.tcount);
  a.touch = reinterpret_cast<Touch*>(team + t.touch);
  a.dbits = reinterpret_cast<unsigned*>(team + t.dbits);
  a.wctr = reinterpret_cast<unsigned*>(team + t.wctr);
  a.itoff = reinterpret_cast<int*>(lists + l.itoff);
  a.xcount = reinterpret_cast<int*>(lists + l.xcount);
  a.xlist = reinterpret_cast<int*>(lists + l.xlist);
  a.nchunks = (int)((a.L + kChunk - 1) / kChunk);
  a.nblk = (int)((a.L + kCol - 1) / kCol);
  a.nwords = (a.nblk + 31) / 32;
}

}  // namespace
