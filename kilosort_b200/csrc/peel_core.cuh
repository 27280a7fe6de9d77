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

constexpr int kThreads = 384;
constexpr int kWarps = kThreads / 32;
constexpr int kChunk = 256;          // detection chunk, one column per thread
constexpr int kCol = 32;             // update block, one column per lane
constexpr int kRowsPerWarp = 16;     // template rows in flight per lane (ungrouped update)
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
constexpr int kGroup = 32;           // template rows of one group (grouped update)
constexpr int kInitGroups = 2;       // groups per item of the initial scoring

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
  unsigned* wctr;             // [6] work counters by iteration parity: [0,1] update
                              //     items, [2,3] grouped units written, [4,5] taken
  int* itoff;                 // [kMaxIters] first record of each iteration
  int* xcount;                // [nblk] spikes whose residual window meets the block
  int* xlist;                 // [nblk * kXCap] their record indices (unordered)
  unsigned* bar;              // barrier arrival count (monotonic)
  int* err;
  const int* upstream_err;    // error word of the producer of Bt (may be null)
  // grouped update (null rperm: every row of a touched column is rewritten)
  const int* rperm;           // [K] template rows in group order (group g: rows
                              //     rperm[32g .. 32g+31])
  const float2* nmip;         // [K] {nm, 1/nm} in group order, nmip[r] = nmi[rperm[r]]
  const float* mg;            // [K][ng] largest |ctcT[k][j][l]| over the rows j
                              //     of group g and all lags
  unsigned long long* gbest;  // [nblk][ng][32] packed best score of each group
                              //     per column (pack_score)
  unsigned char* gexp;        // [nblk][ng][32] smallest exponent field of |B|
                              //     over each group's rows per column (noop_expo)
  int* blist;                 // [nblk][32] a dirty block's ordered touch list for
                              //     its units: n, tau[kTouch], k[kTouch], amp bits
  uint2* units;               // [nblk*ng] (block << 11 | group, columns to process)
  int ng;                     // groups, ceil(K / kGroup)
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
  unsigned char* eb;  // kWarps*kTouch*32  bound exponents of a warp's touching peaks
  float* stage;       // kWarps*2*kGroup*32 (grouped update only): a warp's tile of
                      //   B rows [kGroup][32] and of ctc rows [kGroup][32]
  float2* rtab;       // kWarps*kGroup (grouped update only): row index bits and nm
                      //   of the rows of the group a warp processes
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

__device__ __forceinline__ Smem carve_smem(const PeelArgs& a, char* base, bool grouped) {
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
  s.eb = reinterpret_cast<unsigned char*>(take(kWarps * kTouch * 32));
  s.stage = grouped ? reinterpret_cast<float*>(take(sizeof(float) * kWarps * 2 * kGroup * 32))
                    : nullptr;
  s.rtab = grouped ? reinterpret_cast<float2*>(take(sizeof(float2) * kWarps * kGroup)) : nullptr;
  return s;
}

size_t smem_bytes(int P, int nt, int nchunks, int nwords, bool grouped) {
  auto r = [](size_t b) { return (b + 15) & ~size_t(15); };
  const size_t wn = kChunk + 2 * (size_t)nt;
  (void)P;
  return r(sizeof(float) * 8 * nt) + r(sizeof(int) * (nchunks + 1)) +
         r(sizeof(int) * (nwords + 1)) + 3 * r(sizeof(float) * wn) +
         r(sizeof(int) * kChunk) + r(sizeof(int) * (kWarps + 1)) +
         3 * r(sizeof(int) * kWarps * kTouch) + r(kWarps * kTouch * 32) +
         (grouped ? r(sizeof(float) * kWarps * 2 * kGroup * 32) + r(sizeof(float2) * kWarps * kGroup)
                  : 0);
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

// Exponent field of |x| as the no-op test reads a score: the biased exponent
// of a normal number; 0 for zero, subnormal, infinite and NaN values, whose
// groups then always take the exact path.
__device__ __forceinline__ int noop_expo(float x) {
  const int e = (int)((__float_as_uint(x) >> 23) & 0xffu);
  return e == 255 ? 0 : e;
}

// Exponent field of a non-negative product bound (255 for infinity or NaN,
// which never passes the test).
__device__ __forceinline__ int bound_expo(float b) {
  return (int)((__float_as_uint(b) >> 23) & 0xffu);
}

// cp.async global -> shared: 4 bytes (L1-allocating) and 16 bytes (L2 only),
// and the wait for this thread's copies.
__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(float* dst, const float* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// ----------------------------------------------------------- grouped update
// Grouped form of update_warp_item.  The K template rows are cut into groups
// of kGroup rows in the order rperm (templates sorted by the channel centroid
// of their energy, so one group holds templates of neighbouring sites).
// Before touching a group, a column decides from per-group metadata alone
// whether the subtractions can change any of its rows:
//   the product that a subtraction rounds, p = fl(amp * ctc[j,k,l]), has
//   |p| <= fl(|amp| * mg[k][g]) = bnd, because |ctc[j,k,l]| <= mg[k][g] (the
//   group's largest magnitude over rows and lags) and rounding is monotone;
//   if bnd's exponent field Eb satisfies Eb <= gexp - 26, where gexp is the
//   smallest exponent field of |B[j,c]| over the group's rows, then
//   |p| < 2^(Eb-126) <= 2^(gexp-152) <= ulp(B[j,c]) / 4 for every row j of
//   the group, so fl(B[j,c] - p) = B[j,c] exactly (also when B[j,c] is a power
//   of two, where the spacing below it is ulp / 2), for each of the peaks
//   touching the column in turn.
// Zero, subnormal, infinite and NaN scores give gexp = 0, and an infinite or
// NaN bound gives Eb = 255, so those always take the exact path.  A (column,
// group) pair that passes is left as it is: its rows are not read, its
// cross-correlations are not loaded and its cached best (gbest) stands.  The
// other pairs are updated exactly as update_warp_item does (same peaks, same
// order, same roundings), and their gbest and gexp are rewritten.  The
// column's best is the packed maximum over all groups (larger score, then the
// smaller template index), which equals update_warp_item's in-order fold.
//
// An iteration's update runs in two phases separated by a team barrier, so
// that the uneven work (a dirty block needs anywhere from none to all of its
// groups) is spread evenly: group_scan_block (one warp per dirty block) reads
// only metadata, folds the cached bests of the groups its columns leave
// alone into the column maxima and appends each group that some column must
// process to the iteration's unit list; unit_run (units taken from a
// counter) processes one such group tile.

// Per-lane view of an ordered touch list: the first entry touching this
// column (-1: none) and the mask of the others.
struct LaneEntries {
  int e0;
  unsigned rest;
};

__device__ __forceinline__ LaneEntries lane_entries(const TouchList& tl, int c, bool colok, int nt) {
  LaneEntries le{-1, 0u};
  for (int e = 0; e < tl.n; ++e) {
    const int d = c - tl.tau[e];
    if (colok && d >= -nt && d <= nt) {
      if (le.e0 < 0) le.e0 = e;
      else le.rest |= 1u << e;
    }
  }
  return le;
}

// One group tile (group g of block blk): when some column of the warp has nd
// set, the warp stages the group's 32 rows of B (whole rows, 16-byte copies)
// and every nd column stages its first touching peak's cross-correlations,
// into the warp's shared tiles with cp.async (one round trip, no registers
// held in flight); the columns subtract their touching peaks in application
// order (further peaks stage their cross-correlations into the same tile),
// write the rows back when `store`, and rewrite the group's gbest and gexp.
// jl / nl: row index and {nm, 1/nm} of group position `lane` (rperm, nmip).
// Returns the group's packed best for nd columns (0 otherwise).  Called by
// the whole warp.
//
// The best over the group's rows is found without a division per row: with
// approx = fl(sq * fl(1/nm)) within a relative 2^-22 of the exact quotient
// cf = fl(sq / nm) (sq and the quotient normal), a row whose approx is below
// (1 - 2^-20) times the largest approx m of the group cannot reach the exact
// quotient of the row holding m, so only the rows at or above that level
// have their exact quotient computed and folded (larger score, then the
// smaller template index); rows with sq = 0 and a normal nm have the
// quotient +0 exactly, and rows whose approx is NaN or tiny are folded
// exactly too.
// kLazy selects the lean form of that fold (the batched launch): the same
// result with fewer instructions per row, the rare cases (zero scores, NaN or
// tiny approximations) found by second passes that run only when needed.
template <bool kLazy>
__device__ unsigned long long group_tile(const PeelArgs& a, const Smem& s, const TouchList& tl,
                                         int blk, int g, bool nd, const LaneEntries& le,
                                         bool store, int jl, float2 nl, int lane, int warp) {
  const int c = blk * kCol + lane;
  const int nt = a.nt, K = a.K, nlag = 2 * nt + 1;
  const int nrow = min(kGroup, K - g * kGroup);
  float* Bs = s.stage + (size_t)warp * (2 * kGroup * 32);
  float* Cs = Bs + kGroup * 32;
  float2* rtab = s.rtab + warp * kGroup;
  const float* brow = a.Bt + (size_t)blk * K * kCol;
  const float* cp0 = a.ctcT;
  float amp0 = 0.f;
  if (le.e0 >= 0) {
    cp0 = a.ctcT + (size_t)tl.k[le.e0] * K * nlag + (c - tl.tau[le.e0] + nt);
    amp0 = tl.amp[le.e0];
  }
  const bool any_nd = __any_sync(0xffffffffu, nd);
  const unsigned rest_any = __reduce_or_sync(0xffffffffu, nd ? le.rest : 0u);
  __syncwarp();                       // earlier readers of the tiles are done
  if (lane < nrow) rtab[lane] = make_float2(__int_as_float(jl), nl.x);
  // whole rows of B: lane copies 16 bytes (4 columns) of rows 4i + lane/8
#pragma unroll
  for (int i = 0; i < kGroup / 4; ++i) {
    const int r = 4 * i + (lane >> 3);
    const int j = __shfl_sync(0xffffffffu, jl, r);
    if (any_nd && r < nrow)
      cp_async16(Bs + r * 32 + (lane & 7) * 4, brow + (size_t)j * kCol + (lane & 7) * 4);
  }
  for (int r = 0; r < nrow; ++r) {
    const int j = __shfl_sync(0xffffffffu, jl, r);
    if (nd && le.e0 >= 0) cp_async4(Cs + r * 32 + lane, cp0 + (size_t)j * nlag);
  }
  cp_async_commit();
  cp_async_wait_all();
  __syncwarp();                       // every lane's rows of B have landed
  // a column touched by further peaks applies them here in application
  // order; otherwise its single peak is applied in the first pass below
  const bool fused = rest_any == 0u;
  if (!fused) {
    if (nd && le.e0 >= 0) {
      for (int r = 0; r < nrow; ++r)
        Bs[r * 32 + lane] = __fsub_rn(Bs[r * 32 + lane], __fmul_rn(amp0, Cs[r * 32 + lane]));
    }
    for (unsigned m = rest_any; m; m &= m - 1u) {
      const int e = __ffs(m) - 1;
      const bool mine = nd && ((le.rest >> e) & 1u);
      const float* cp = a.ctcT + (size_t)tl.k[e] * K * nlag + (c - tl.tau[e] + nt);
      for (int r = 0; r < nrow; ++r) {
        const int j = __shfl_sync(0xffffffffu, jl, r);
        if (mine) cp_async4(Cs + r * 32 + lane, cp + (size_t)j * nlag);
      }
      cp_async_commit();
      cp_async_wait_all();
      if (mine) {
        const float amp = tl.amp[e];
        for (int r = 0; r < nrow; ++r)
          Bs[r * 32 + lane] = __fsub_rn(Bs[r * 32 + lane], __fmul_rn(amp, Cs[r * 32 + lane]));
      }
    }
  }
  float best = -1.f;
  int arg = 0x7fffffff;
  int emin = 255;                             // smallest exponent field over the rows
  if constexpr (!kLazy) {
  // pass 1, branch-free over all kGroup rows (rows past nrow and columns
  // without nd only compute, their results unused): the (single peak)
  // subtraction, the write-back, the smallest exponent, and for the best
  // score the largest approx m with its first row rm, the largest approx m2
  // of the other rows, the smallest row index whose score is exactly 0
  // (sq = 0 and a normal nm), and the rows that need an exact quotient
  // whatever m is (approx NaN, or below 2^-100 with sq > 0).
  float* bdst = a.Bt + (size_t)blk * K * kCol + lane;
  const bool sub = fused && le.e0 >= 0;
  constexpr float kTiny = 7.8886091e-31f;     // 2^-100
  float m = -1.f, m2 = -1.f;
  int rm = -1, jz = 0x7fffffff;
  unsigned spec = 0u;
#pragma unroll 8
  for (int r = 0; r < kGroup; ++r) {
    const int j = __shfl_sync(0xffffffffu, jl, r);
    const float nmy = __shfl_sync(0xffffffffu, nl.y, r);
    const bool ok = nd && r < nrow;
    const float b0 = Bs[r * 32 + lane];
    const float b1 = __fsub_rn(b0, __fmul_rn(amp0, Cs[r * 32 + lane]));
    const float b = sub ? b1 : b0;
    if (ok && store) bdst[(size_t)j * kCol] = b;
    emin = ok ? min(emin, noop_expo(b)) : emin;
    const float rl = b > 0.f ? b : 0.f;
    const float sq = __fmul_rn(rl, rl);
    const float ap = __fmul_rn(sq, nmy);
    const bool big = ok && ap >= kTiny;
    const bool top = big && ap > m;
    m2 = top ? m : (big ? fmaxf(m2, ap) : m2);
    rm = top ? r : rm;
    m = top ? ap : m;
    jz = (ok && sq == 0.f && nmy == nmy && j < jz) ? j : jz;
    spec |= (ok && (ap != ap || (ap < kTiny && sq != 0.f))) ? (1u << r) : 0u;
  }
  // Candidates for the best: with m >= 2^-90 the rows whose approx is at
  // least (1 - 2^-20) m -- only rm, unless m2 reaches that level; below
  // 2^-90 every row with approx >= 2^-100.  Rows with a smaller approx
  // cannot reach the exact quotient of rm (or 2^-100 and the zeros), so the
  // result is that of folding every row.
  const bool regime_a = m >= 8.0779356e-28f;  // 2^-90
  const float thr = regime_a ? m * 0.99999905f : kTiny;
  const bool scan = !regime_a || m2 >= thr;
  if (jz != 0x7fffffff) {
    best = 0.f;
    arg = jz;
  }
  unsigned cand = spec;
  if (regime_a && !scan) cand |= 1u << rm;
  if (__any_sync(0xffffffffu, nd && scan)) {
#pragma unroll 8
    for (int r = 0; r < kGroup; ++r) {
      const float nmy = __shfl_sync(0xffffffffu, nl.y, r);
      const bool ok = nd && scan && r < nrow;
      const float b0 = Bs[r * 32 + lane];
      const float b1 = __fsub_rn(b0, __fmul_rn(amp0, Cs[r * 32 + lane]));
      const float b = sub ? b1 : b0;
      const float rl = b > 0.f ? b : 0.f;
      const float ap = __fmul_rn(__fmul_rn(rl, rl), nmy);
      cand |= (ok && ap >= thr) ? (1u << r) : 0u;
    }
  }
  // exact quotients of the candidates (usually only rm, converged)
  if (!nd) cand = 0u;
  for (unsigned mm = cand; mm; mm &= mm - 1u) {
    const int r = __ffs(mm) - 1;
    float b = Bs[r * 32 + lane];
    if (sub) b = __fsub_rn(b, __fmul_rn(amp0, Cs[r * 32 + lane]));
    const float2 jn = rtab[r];
    const int j = __float_as_int(jn.x);
    const float rl = b > 0.f ? b : 0.f;
    const float sq = __fmul_rn(rl, rl);
    const bool normal = jn.y >= 1.17549435e-38f && jn.y <= 3.40282347e38f;
    const float cf = (sq == 0.f && normal) ? 0.f : __fdiv_rn(sq, jn.y);
    if (cf > best || (cf == best && j < arg)) {
      best = cf;
      arg = j;
    }
  }
  } else {
  // pass 1 over the group's rows, branch-free in the columns (a column
  // without nd computes too, its results unused): the (single peak)
  // subtraction, the write-back, the smallest exponent, and for the best
  // score the largest approx m with its first row rm and the largest approx
  // m2 of the other rows.  Rows with an approx below 2^-100 take part in m
  // and m2 without changing what follows (the candidate level is at least
  // 2^-90 when m is, and below it every row >= 2^-100 is a candidate), NaN
  // approx never does.  Rows that need an exact quotient whatever m is
  // (approx NaN, or below 2^-100 with sq > 0) only raise a flag here and are
  // found by a second pass when some column has one.
  float* bdst = a.Bt + (size_t)blk * K * kCol + lane;
  const bool sub = fused && le.e0 >= 0;
  constexpr float kTiny = 7.8886091e-31f;     // 2^-100
  float m = -1.f, m2 = -1.f;
  int rm = -1;
  bool anyspec = false;
#pragma unroll 8
  for (int r = 0; r < nrow; ++r) {
    const int j = __shfl_sync(0xffffffffu, jl, r);
    const float nmy = __shfl_sync(0xffffffffu, nl.y, r);
    const float b0 = Bs[r * 32 + lane];
    const float b1 = __fsub_rn(b0, __fmul_rn(amp0, Cs[r * 32 + lane]));
    const float b = sub ? b1 : b0;
    if (nd && store) bdst[(size_t)j * kCol] = b;
    emin = min(emin, noop_expo(b));
    const float rl = b > 0.f ? b : 0.f;
    const float sq = __fmul_rn(rl, rl);
    const float ap = __fmul_rn(sq, nmy);
    const bool top = ap > m;
    m2 = top ? m : fmaxf(m2, ap);
    rm = top ? r : rm;
    m = top ? ap : m;
    anyspec |= (ap != ap) || (ap < kTiny && sq != 0.f);
  }
  // Candidates for the best: with m >= 2^-90 the rows whose approx is at
  // least (1 - 2^-20) m -- only rm, unless m2 reaches that level; below
  // 2^-90 every row with approx >= 2^-100.  Rows with a smaller approx
  // cannot reach the exact quotient of rm (or 2^-100 and the zeros), so the
  // result is that of folding every row.
  const bool regime_a = m >= 8.0779356e-28f;  // 2^-90
  const float thr = regime_a ? m * 0.99999905f : kTiny;
  const bool scan = !regime_a || m2 >= thr;
  unsigned cand = 0u;
  if (regime_a && !scan) cand |= 1u << rm;
  if (__any_sync(0xffffffffu, nd && (scan || anyspec))) {
#pragma unroll 8
    for (int r = 0; r < nrow; ++r) {
      const float nmy = __shfl_sync(0xffffffffu, nl.y, r);
      const float b0 = Bs[r * 32 + lane];
      const float b1 = __fsub_rn(b0, __fmul_rn(amp0, Cs[r * 32 + lane]));
      const float b = sub ? b1 : b0;
      const float rl = b > 0.f ? b : 0.f;
      const float sq = __fmul_rn(rl, rl);
      const float ap = __fmul_rn(sq, nmy);
      const bool sp = ap != ap || (ap < kTiny && sq != 0.f);
      cand |= ((scan && ap >= thr) || sp) ? (1u << r) : 0u;
    }
  }
  // exact quotients of the candidates (usually only rm, converged)
  if (!nd) cand = 0u;
  for (unsigned mm = cand; mm; mm &= mm - 1u) {
    const int r = __ffs(mm) - 1;
    float b = Bs[r * 32 + lane];
    if (sub) b = __fsub_rn(b, __fmul_rn(amp0, Cs[r * 32 + lane]));
    const float2 jn = rtab[r];
    const int j = __float_as_int(jn.x);
    const float rl = b > 0.f ? b : 0.f;
    const float sq = __fmul_rn(rl, rl);
    const bool normal = jn.y >= 1.17549435e-38f && jn.y <= 3.40282347e38f;
    const float cf = (sq == 0.f && normal) ? 0.f : __fdiv_rn(sq, jn.y);
    if (cf > best || (cf == best && j < arg)) {
      best = cf;
      arg = j;
    }
  }
  // rows whose score is exactly 0 (sq = 0 and 1/nm not NaN) can only matter
  // when no candidate scored above 0: fold them then (score 0, smaller
  // template index first)
  if (__any_sync(0xffffffffu, nd && !(best > 0.f))) {
    for (int r = 0; r < nrow; ++r) {
      const int j = __shfl_sync(0xffffffffu, jl, r);
      const float nmy = __shfl_sync(0xffffffffu, nl.y, r);
      float b = Bs[r * 32 + lane];
      if (sub) b = __fsub_rn(b, __fmul_rn(amp0, Cs[r * 32 + lane]));
      const float rl = b > 0.f ? b : 0.f;
      const float sq = __fmul_rn(rl, rl);
      if (nd && sq == 0.f && nmy == nmy && (0.f > best || (0.f == best && j < arg))) {
        best = 0.f;
        arg = j;
      }
    }
  }
  }
  unsigned long long gb = 0ull;
  if (nd) {
    gb = best >= 0.f ? pack_score(best, arg) : 0ull;
    const size_t mi = ((size_t)blk * a.ng + g) * 32 + lane;
    a.gbest[mi] = gb;
    a.gexp[mi] = (unsigned char)emin;
  }
  return gb;
}

// Row indices and {nm, 1/nm} of group g, lane r holding position r.
__device__ __forceinline__ void group_rows(const PeelArgs& a, int g, int lane, int& jl, float2& nl) {
  const int rr = g * kGroup + lane;
  jl = 0;
  nl = make_float2(1.f, 1.f);
  if (rr < a.K) {
    jl = __ldg(a.rperm + rr);
    nl = __ldg(a.nmip + rr);
  }
}

// Initial scores of groups [g_lo, g_hi) of block blk (nothing subtracted):
// every group's gbest and gexp, and the column maxima folded into pack_out.
template <bool kLazy>
__device__ void group_init_item(const PeelArgs& a, const Smem& s, int blk, int g_lo, int g_hi,
                                unsigned long long* pack_out, int lane, int warp) {
  const int c = blk * kCol + lane;
  const bool colok = c < a.L;
  const TouchList none{0, nullptr, nullptr, nullptr};
  const LaneEntries le{-1, 0u};
  unsigned long long colbest = 0ull;
  for (int g = g_lo; g < g_hi; ++g) {
    int jl;
    float2 nl;
    group_rows(a, g, lane, jl, nl);
    const unsigned long long gb =
        group_tile<kLazy>(a, s, none, blk, g, colok, le, false, jl, nl, lane, warp);
    colbest = gb > colbest ? gb : colbest;
  }
  if (colok && colbest) atomicMax(&pack_out[c], colbest);
}

// Phase A for dirty block blk (iteration parity p): publish the block's
// ordered touch list for its units, decide per column and group from the
// metadata, fold the cached bests of the groups a column leaves alone (and
// the settled score of a column no peak touches) into pack_out, and append
// the groups some column must process to the unit list.
__device__ void group_scan_block(const PeelArgs& a, const Smem& s, int p, int blk,
                                 unsigned long long* pack_out, int lane, int warp) {
  const TouchList tl = load_touch_warp(a, s, p, blk, lane, warp);
  int* bl = a.blist + (size_t)blk * 32;
  if (lane == 0) bl[0] = tl.n;
  if (lane < tl.n) {
    bl[1 + lane] = tl.tau[lane];
    bl[1 + kTouch + lane] = tl.k[lane];
    bl[1 + 2 * kTouch + lane] = __float_as_int(tl.amp[lane]);
  }
  const int c = blk * kCol + lane;
  const bool colok = c < a.L;
  const int nt = a.nt, ng = a.ng;
  unsigned tmask = 0u;
  for (int e = 0; e < tl.n; ++e) {
    const int d = c - tl.tau[e];
    if (colok && d >= -nt && d <= nt) tmask |= 1u << e;
  }
  const bool touched = tmask != 0u;
  const size_t meta = (size_t)blk * ng * 32 + lane;
  unsigned char* eb = s.eb + warp * (kTouch * 32);
  unsigned* ucount = a.wctr + 2 + p;
  unsigned long long colbest = 0ull;
  for (int gc = 0; gc < ng; gc += 32) {
    const int gn = min(32, ng - gc);
    const unsigned gmask = gn == 32 ? 0xffffffffu : ((1u << gn) - 1u);
    // exponent fields of the product bounds of every touching peak, for the
    // groups gc + lane
    __syncwarp();
    for (int e = 0; e < tl.n; ++e) {
      int x = 255;
      if (lane < gn)
        x = bound_expo(__fmul_rn(fabsf(tl.amp[e]), __ldg(a.mg + (size_t)tl.k[e] * ng + gc + lane)));
      eb[e * 32 + lane] = (unsigned char)x;
    }
    __syncwarp();
    unsigned need = 0u;
    if (touched) {
#pragma unroll 8
      for (int i = 0; i < gn; ++i) {
        const int ex = a.gexp[meta + (size_t)(gc + i) * 32];
        bool nd = false;
        for (unsigned m = tmask; m; m &= m - 1u) {
          const int e = __ffs(m) - 1;
          nd |= (int)eb[e * 32 + i] + 26 > ex;
        }
        if (nd) need |= 1u << i;
      }
      const unsigned keep = ~need & gmask;
#pragma unroll 8
      for (int i = 0; i < gn; ++i) {
        if ((keep >> i) & 1u) {
          const unsigned long long gb = a.gbest[meta + (size_t)(gc + i) * 32];
          colbest = gb > colbest ? gb : colbest;
        }
      }
    }
    const unsigned proc = __reduce_or_sync(0xffffffffu, need);
    if (proc) {
      unsigned base = 0u;
      if (lane == 0) base = atomicAdd(ucount, (unsigned)__popc(proc));
      base = __shfl_sync(0xffffffffu, base, 0);
      unsigned cols = 0u;             // lane i: the columns that process group gc + i
      for (unsigned m = proc; m; m &= m - 1u) {
        const int i = __ffs(m) - 1;
        const unsigned b = __ballot_sync(0xffffffffu, (need >> i) & 1u);
        if (lane == i) cols = b;
      }
      if ((proc >> lane) & 1u)
        a.units[base + __popc(proc & ((1u << lane) - 1u))] =
            make_uint2(((unsigned)blk << 11) | (unsigned)(gc + lane), cols);
    }
  }
  if (colok) {
    if (touched) {
      if (colbest) atomicMax(&pack_out[c], colbest);
    } else {
      atomicMax(&pack_out[c], pack_score(a.cfmax[c], a.imax[c]));
    }
  }
}

// Phase B: one unit (a group tile that some columns of a block must
// process), its block's ordered touch list read back from the scan.
// unit_fetch issues the unit's loads (the block's list, the group's rows);
// unit_run uses them, so a warp fetches its next unit before running the
// current one.
struct UnitFetch {
  uint2 u;
  int v;        // word `lane` of the block's list (n, tau[], k[], amp bits[])
  int jl;       // row index of group position `lane`
  float2 nl;    // its {nm, 1/nm}
};

__device__ __forceinline__ UnitFetch unit_fetch(const PeelArgs& a, uint2 u, int lane) {
  UnitFetch f;
  f.u = u;
  const int blk = (int)(u.x >> 11), g = (int)(u.x & 2047u);
  f.v = lane < 1 + 3 * kTouch ? a.blist[(size_t)blk * 32 + lane] : 0;
  group_rows(a, g, lane, f.jl, f.nl);
  return f;
}

template <bool kLazy>
__device__ void unit_run(const PeelArgs& a, const Smem& s, const UnitFetch& f,
                         unsigned long long* pack_out, int lane, int warp) {
  const int blk = (int)(f.u.x >> 11), g = (int)(f.u.x & 2047u);
  const bool nd = (f.u.y >> lane) & 1u;
  const int n = __shfl_sync(0xffffffffu, f.v, 0);
  int* tau = s.tl_tau + warp * kTouch;
  int* kk = s.tl_k + warp * kTouch;
  float* amp = s.tl_amp + warp * kTouch;
  const int tv = __shfl_sync(0xffffffffu, f.v, 1 + (lane & (kTouch - 1)));
  const int kv = __shfl_sync(0xffffffffu, f.v, 1 + kTouch + (lane & (kTouch - 1)));
  const int av = __shfl_sync(0xffffffffu, f.v, 1 + 2 * kTouch + (lane & (kTouch - 1)));
  __syncwarp();
  if (lane < n) {
    tau[lane] = tv;
    kk[lane] = kv;
    amp[lane] = __int_as_float(av);
  }
  __syncwarp();
  const TouchList tl{n, tau, kk, amp};
  const int c = blk * kCol + lane;
  const LaneEntries le = lane_entries(tl, c, c < a.L, a.nt);
  const unsigned long long gb =
      group_tile<kLazy>(a, s, tl, blk, g, nd, le, true, f.jl, f.nl, lane, warp);
  if (nd && gb) atomicMax(&pack_out[c], gb);
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
template <int kRows, bool kGrouped, bool kLazy = false>
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
    if (t0 < 6) a.wctr[t0] = 0u;
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
    if (kGrouped) {
      // items of kInitGroups groups: the group metadata of every column too
      const int rg = (a.ng + kInitGroups - 1) / kInitGroups;
      const long long n_items = (long long)a.nblk * rg;
      for (long long w = gwarp; w < n_items; w += nwarps) {
        const int blk = (int)(w / rg), r = (int)(w % rg);
        group_init_item<kLazy>(a, s, blk, r * kInitGroups, min(a.ng, (r + 1) * kInitGroups), pinit,
                        lane, warp);
      }
    } else {
      const int rg = (a.K + kItemRows - 1) / kItemRows;
      const TouchList none{0, nullptr, nullptr, nullptr};
      const long long n_items = (long long)a.nblk * rg;
      for (long long w = gwarp; w < n_items; w += nwarps) {
        const int blk = (int)(w / rg), r = (int)(w % rg);
        update_warp_item<kRows>(a, none, blk, r * kItemRows, min(a.K, (r + 1) * kItemRows),
                                pinit, lane, true);
      }
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
    if (rank == 0 && tid == 0) {
      a.wctr[q] = 0u;
      a.wctr[2 + q] = 0u;
      a.wctr[4 + q] = 0u;
    }
    if (rank == 0 && tid == 0) a.itoff[it] = (int)n_out;
    unsigned long long* pcur = a.pack + (size_t)p * a.L;
    KS_TRACE(it, 3, ks_globaltimer());
    if (kGrouped) {
      // phase A: one warp per dirty block, dealt round-robin (metadata only,
      // about the same work per block)
      for (long long w = gwarp; w < ndirty; w += nwarps)
        group_scan_block(a, s, p, dirty_block(s, bits, a.nwords, (int)w), pcur, lane, warp);
      if (!ks_grid_sync(a.bar, G, epoch, a.err, a.limit_ns)) break;
      // phase B: the units, taken from a counter in claims of about a quarter
      // of a warp's share (at most 32), so thousands of warps do not queue on
      // it; a warp reads its claim's records at once and fetches each unit's
      // inputs while it runs the one before
      const unsigned n_units = ks_ld_acquire(a.wctr + 2 + p);
      const unsigned claim =
          (unsigned)min(32LL, max(1LL, (long long)n_units / (nwarps * 4)));
      while (true) {
        unsigned first = 0;
        if (lane == 0) first = atomicAdd(&a.wctr[4 + p], claim);
        first = __shfl_sync(0xffffffffu, first, 0);
        if (first >= n_units) break;
        const int nu = (int)(min(n_units, first + claim) - first);
        const uint2 rec = lane < nu ? a.units[first + lane] : make_uint2(0u, 0u);
        UnitFetch cur = unit_fetch(
            a, make_uint2(__shfl_sync(0xffffffffu, rec.x, 0), __shfl_sync(0xffffffffu, rec.y, 0)),
            lane);
        for (int i = 0; i < nu; ++i) {
          UnitFetch nxt = cur;
          if (i + 1 < nu)
            nxt = unit_fetch(a, make_uint2(__shfl_sync(0xffffffffu, rec.x, i + 1),
                                           __shfl_sync(0xffffffffu, rec.y, i + 1)),
                             lane);
          unit_run<kLazy>(a, s, cur, pcur, lane, warp);
          cur = nxt;
        }
      }
    } else {
      // update items: (dirty block in column order, row range): the split
      // whose most loaded warp has the least work (row steps of kRows plus one
      // step's worth of per-item set-up)
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
      const long long n_items = (long long)ndirty * rgroups;
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

// kGrouped: the grouped update (a.rperm, a.nmip, a.mg and the group metadata
// set); the ungrouped form needs no group metadata.
template <bool kGrouped>
__global__ void __launch_bounds__(kThreads, 2) peel_kernel(PeelArgs a) {
  extern __shared__ __align__(16) char smem_raw[];
  const Smem s = carve_smem(a, smem_raw, kGrouped);
  unsigned epoch = 0;
  run_peel<kRowsPerWarp, kGrouped>(a, s, blockIdx.x, gridDim.x, epoch);
}

constexpr int kXTile = kCol * (kCol + 1);   // floats of one warp's transpose tile
// the batched peel's residual lists and transpose tiles fit in the stage tiles
static_assert(3 * kXList * 4 + kXTile * 4 <= 2 * kGroup * 32 * 4, "residual scratch exceeds a stage tile");

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

// ------------------------------------------------------------ group order
// Setup of the grouped update.  The order only decides how many (column,
// group) pairs the no-op test can leave alone; any order gives the same
// results.
//
// Spatial key of each template: the channel centroid sum_c c*e_c / sum_c e_c
// of its energy e_c = sum_p U[k,p,c]^2 (0 for a template without energy).
// One warp per template, fixed summation order.
__global__ void ks_template_key_kernel(const float* __restrict__ U, int K, int P, int C,
                                       float* __restrict__ key) {
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= K) return;
  double se = 0.0, sc = 0.0;
  for (int c = lane; c < C; c += 32) {
    float e = 0.f;
    for (int p = 0; p < P; ++p) {
      const float u = U[((size_t)w * P + p) * C + c];
      e = fmaf(u, u, e);
    }
    se += e;
    sc += (double)c * e;
  }
  for (int o = 16; o; o >>= 1) {
    se += __shfl_xor_sync(0xffffffffu, se, o);
    sc += __shfl_xor_sync(0xffffffffu, sc, o);
  }
  if (lane == 0) key[w] = se > 0.0 ? (float)(sc / se) : 0.f;
}

__device__ __forceinline__ unsigned sortable_key(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// rperm[r] = the template of rank r in ascending key order (the smaller
// template index first on equal keys): each thread counts the keys below its
// own, staged through shared memory 1024 at a time.
__global__ void __launch_bounds__(256) ks_group_order_kernel(const float* __restrict__ key, int K,
                                                             int* __restrict__ rperm) {
  __shared__ unsigned sk[1024];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned mine = k < K ? sortable_key(key[k]) : 0u;
  int rank = 0;
  for (int j0 = 0; j0 < K; j0 += 1024) {
    const int n = min(1024, K - j0);
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) sk[i] = sortable_key(key[j0 + i]);
    __syncthreads();
    if (k < K)
      for (int i = 0; i < n; ++i) {
        const unsigned v = sk[i];
        rank += (v < mine || (v == mine && j0 + i < k)) ? 1 : 0;
      }
  }
  if (k < K) rperm[rank] = k;
}

// mg[k][g] = the largest |ctcT[k][j][l]| over the rows j of group g (rows
// rperm[32g ..]) and all lags l, by the integer maximum of the magnitude bits
// (so a NaN anywhere gives a NaN bound, which never passes the no-op test).
// One block of 256 threads per (template, group).
__global__ void __launch_bounds__(256) ks_group_bound_kernel(const float* __restrict__ ctcT,
                                                             const int* __restrict__ rperm, int K,
                                                             int nlag, int ng,
                                                             float* __restrict__ mg) {
  __shared__ unsigned wm[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long items = (long long)K * ng;
  for (long long item = blockIdx.x; item < items; item += gridDim.x) {
    const int k = (int)(item / ng), g = (int)(item % ng);
    unsigned m = 0u;
    for (int r = warp; r < kGroup; r += 8) {
      const int rr = g * kGroup + r;
      if (rr >= K) break;
      const float* row = ctcT + ((size_t)k * K + rperm[rr]) * nlag;
      for (int l = lane; l < nlag; l += 32) m = max(m, __float_as_uint(row[l]) & 0x7fffffffu);
    }
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    __syncthreads();
    if (lane == 0) wm[warp] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned x = 0u;
      for (int w = 0; w < 8; ++w) x = max(x, wm[w]);
      mg[item] = __uint_as_float(x);
    }
  }
}

// nmip[r] = nmi[rperm[r]]: {nm, 1/nm} of the template rows in group order.
__global__ void ks_group_nmi_kernel(const float2* __restrict__ nmi, const int* __restrict__ rperm,
                                    int K, float2* __restrict__ nmip) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < K; r += gridDim.x * blockDim.x)
    nmip[r] = nmi[rperm[r]];
}

// Scratch of one team (reused for every batch it processes), for batches of
// up to L padded samples and K templates: [ctl 256 B: barrier count, error
// word] [cfmax L] [imax L] [pack 2L] [chunk counts] [chunk buffers 4 x
// nchunks*kChunk] [tcount 2 nblk] [touch 2 nblk*kTouch] [dbits 2 nwords]
// [work counters 6], and for the grouped update [gbest nblk*ng*32 u64]
// [gexp nblk*ng*32 u8] [blist nblk*32 int] [units nblk*ng uint2] (K = 0:
// none).  Only the control words need zeroing before a launch; the team
// clears the rest per batch (the initial scoring writes every gbest and gexp
// entry).
struct TeamLayout {
  size_t cfmax, imax, pack, chunk_cnt, chunk_tau, chunk_k, chunk_amp, chunk_th, tcount,
      touch, dbits, wctr, gbest, gexp, blist, units, bytes;
};

__host__ __device__ inline size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

__host__ __device__ inline int n_groups(long long K) { return (int)((K + kGroup - 1) / kGroup); }

__host__ __device__ inline TeamLayout team_layout(long long L, long long K) {
  const long long nchunks = (L + kChunk - 1) / kChunk, nblk = (L + kCol - 1) / kCol;
  const long long nwords = (nblk + 31) / 32;
  const size_t meta = (size_t)nblk * n_groups(K) * 32;
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
  t.wctr = o; o = al256(o + 24);
  t.gbest = o; o = al256(o + 8 * meta);
  t.gexp = o; o = al256(o + meta);
  t.blist = o; o = al256(o + (K > 0 ? 128 * (size_t)nblk : 0));
  t.units = o; o = al256(o + 8 * (size_t)nblk * n_groups(K));
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

// Point the scratch fields of a at a team region and a list region; with
// grouped, also the group metadata (a.K must be set).
__host__ __device__ inline void bind_scratch(PeelArgs& a, char* team, char* lists,
                                             bool grouped) {
  const TeamLayout t = team_layout(a.L, grouped ? a.K : 0);
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
  a.gbest = grouped ? reinterpret_cast<unsigned long long*>(team + t.gbest) : nullptr;
  a.gexp = grouped ? reinterpret_cast<unsigned char*>(team + t.gexp) : nullptr;
  a.blist = grouped ? reinterpret_cast<int*>(team + t.blist) : nullptr;
  a.units = grouped ? reinterpret_cast<uint2*>(team + t.units) : nullptr;
  a.ng = grouped ? n_groups(a.K) : 0;
  a.nchunks = (int)((a.L + kChunk - 1) / kChunk);
  a.nblk = (int)((a.L + kCol - 1) / kCol);
  a.nwords = (a.nblk + 31) / 32;
}

}  // namespace
