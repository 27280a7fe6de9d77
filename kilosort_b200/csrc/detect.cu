// Universal-template spike detection on the device, kilosort/spikedetect.py:133-197
// (template_match and yweighted) plus the PC features of run() (:265-266).
//
//   B[c, k, t]  = conv1d(X[c], wTEMP[k]) (padding nt/2)          FP32 temporal kernel, rows (c, k)
//   A[s, k]     = sum_j weigh[s, j, f] * B[iC[j, f], k, t]       per position f and sample t
//   As[f, t]    = max |A|,  imax[f, t] = (1 + argmax) * sign(A[argmax])   (index s*nk + k)
//   Amax[f, t]  = max over the nC2 nearest positions iC2[:, f] of As     (0 for t < nt, t >= L-nt)
//   peak        = maxpool_{+-nt0}(Amax)[f, t] == As[f, t] and As[f, t] > Th_universal
//   spikes in (f, t) order; adist[j] = B[iC[j, f], |imax|-1 mod nk, t] * sign(imax);
//   y = sum_j relu(adist_j)/sum relu(adist) * yc[iC[j, f]];
//   tF[s, j, p] = sum_u X[iC[j, f], t - nt/2 + u] * wPCA[p, u]
//
// Kernels: ks_detect_scores_tiled_kernel (a block per tile of 32 positions,
// persistent over 32-sample time tiles: the union of the positions' nearest
// channels is staged, double-buffered by cp.async, the (s, k) sums of one
// position over 32 samples per warp in registers; A is never stored;
// ks_detect_scores_kernel is the form for more than 8192 channels),
// ks_detect_peaks_kernel (a block per (f, 256-sample tile): only where the
// score exceeds the threshold, the maximum over the neighbour rows and the
// +-nt0 window, left at the first larger value; peak bits by warp ballot),
// count / scan / emit in (f, t) order, and one gather
// kernel per spike (adist, y) and per (spike, channel) warp (features).
#include "ks_common.cuh"
#include "project.cuh"

#include <algorithm>
#include <cmath>

namespace {

constexpr int kMaxNK = 8;        // universal waveforms
constexpr int kMaxNS = 8;        // template sizes
constexpr int kMaxNC = 32;       // nearest channels
constexpr int kTile = 256;       // samples per block
constexpr int kChunkWords = 32;  // peak-bit words per counting chunk (1024 samples)

__global__ void __launch_bounds__(kTile)
ks_detect_scores_kernel(const float* __restrict__ BT, long long ldb, int nk, int C,
                        const long long* __restrict__ iC, int nC,
                        const float* __restrict__ weigh, int ns, int Nfilt, int L,
                        float* __restrict__ As, signed char* __restrict__ imaxs, int* err) {
  __shared__ int sc[kMaxNC];
  __shared__ float sw[kMaxNS * kMaxNC];
  const int f = blockIdx.x;
  const int t = blockIdx.y * kTile + threadIdx.x;
  for (int j = threadIdx.x; j < nC; j += kTile) {
    long long c = iC[(long long)j * Nfilt + f];
    if (c < 0 || c >= C) {
      atomicCAS(err, 0, KS_ERR_ARG);   // reported; channel 0 stands in
      c = 0;
    }
    sc[j] = (int)c;
  }
  for (int e = threadIdx.x; e < ns * nC; e += kTile) {
    const int s = e / nC, j = e - s * nC;
    sw[e] = weigh[((long long)s * nC + j) * Nfilt + f];
  }
  __syncthreads();
  if (t >= L) return;
  float a[kMaxNS][kMaxNK];
#pragma unroll
  for (int s = 0; s < kMaxNS; ++s)
#pragma unroll
    for (int k = 0; k < kMaxNK; ++k) a[s][k] = 0.f;
  for (int j = 0; j < nC; ++j) {
    const float* b = BT + (long long)sc[j] * nk * ldb + t;
    float bk[kMaxNK];
#pragma unroll
    for (int k = 0; k < kMaxNK; ++k) bk[k] = k < nk ? __ldg(b + (long long)k * ldb) : 0.f;
#pragma unroll
    for (int s = 0; s < kMaxNS; ++s) {
      if (s < ns) {
        const float w = sw[s * nC + j];
#pragma unroll
        for (int k = 0; k < kMaxNK; ++k)
          if (k < nk) a[s][k] = fmaf(w, bk[k], a[s][k]);
      }
    }
  }
  // largest magnitude, first index in (s, k) order
  float best = -1.f, bval = 0.f;
  int bidx = 0;
#pragma unroll
  for (int s = 0; s < kMaxNS; ++s)
#pragma unroll
    for (int k = 0; k < kMaxNK; ++k)
      if (s < ns && k < nk) {
        const float m = fabsf(a[s][k]);
        if (m > best) {
          best = m;
          bval = a[s][k];
          bidx = s * nk + k;
        }
      }
  const int sg = bval > 0.f ? 1 : (bval < 0.f ? -1 : 0);
  As[(long long)f * L + t] = best;
  imaxs[(long long)f * L + t] = (signed char)((1 + bidx) * sg);
}

// The same sums for a tile of kFT consecutive positions x kTT samples: the
// block first collects the union of its positions' nearest channels (a
// bitmap over channels, compacted in channel order), stages those channels'
// convolution rows for its samples in shared memory, then each warp computes
// one position over 32 consecutive samples per round.  A tile whose union
// exceeds kMaxU channels reads its rows from global memory instead.
constexpr int kFT = 32;          // positions per block
constexpr int kTT = 32;          // samples per time tile
constexpr int kMaxU = 48;        // staged channels
constexpr int kMaxCBits = 8192;  // channels covered by the bitmap

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait1() {
  asm volatile("cp.async.wait_group 1;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait0() {
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// Persistent over time: block (position tile, y) takes the time tiles y,
// y + gridDim.y, ...; the union of its positions' channels and their weights
// are set up once, and the channels' convolution rows of the next time tile
// are copied (cp.async, 16-byte pieces) while the current one is summed.
template <int NS, int NK>
__global__ void __launch_bounds__(256)
ks_detect_scores_tiled_kernel(const float* __restrict__ BT, long long ldb, int nk_rt, int C,
                              const long long* __restrict__ iC, int nC,
                              const float* __restrict__ weigh, int ns_rt, int Nfilt, int L,
                              int n_ttiles, float* __restrict__ As,
                              signed char* __restrict__ imaxs, int* err) {
  // NS, NK: compile-time bounds of the sizes and waveforms; ns_rt, nk_rt the
  // actual counts (equal to the bounds in the specialised instantiation)
  extern __shared__ __align__(16) float sm[];
  float* sB = sm;                                                // [2][kMaxU][NK][kTT]
  float* sw = sB + 2 * kMaxU * NK * kTT;                         // [kFT][nC][NS]
  unsigned* bitmap = reinterpret_cast<unsigned*>(sw + kFT * NS * nC);   // [kMaxCBits / 32]
  int* wpre = reinterpret_cast<int*>(bitmap + kMaxCBits / 32);   // [kMaxCBits / 32]
  int* ulist = wpre + kMaxCBits / 32;                            // [kMaxU]
  int* cidx = ulist + kMaxU;                                     // [kMaxNC][kFT] channel
  int* loc = cidx + kMaxNC * kFT;                                // [kMaxNC][kFT] union slot
  __shared__ int nU;
  const int ns = NS == kMaxNS ? ns_rt : NS;
  const int nk = NK == kMaxNK ? nk_rt : NK;
  const int f0 = blockIdx.x * kFT;
  const int nwc = (C + 31) >> 5;
  for (int w = threadIdx.x; w < nwc; w += blockDim.x) bitmap[w] = 0u;
  __syncthreads();
  for (int e = threadIdx.x; e < nC * kFT; e += blockDim.x) {
    const int j = e / kFT, fl = e % kFT;
    const int f = f0 + fl;
    int c = 0;
    if (f < Nfilt) {
      const long long cc = iC[(long long)j * Nfilt + f];
      if (cc < 0 || cc >= C) atomicCAS(err, 0, KS_ERR_ARG);   // channel 0 stands in
      else c = (int)cc;
    }
    cidx[e] = c;
    atomicOr(bitmap + (c >> 5), 1u << (c & 31));
  }
  // weights [fl][j][q] (zero for missing sizes and positions)
  for (int e = threadIdx.x; e < kFT * nC * NS; e += blockDim.x) {
    const int fl = e / (nC * NS), r = e - fl * nC * NS, j = r / NS, q = r % NS;
    const int f = f0 + fl;
    sw[e] = (f < Nfilt && q < ns) ? weigh[((long long)q * nC + j) * Nfilt + f] : 0.f;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    // exclusive prefix of the bitmap words' population counts
    int run = 0;
    for (int w0 = 0; w0 < nwc; w0 += 32) {
      const int w = w0 + threadIdx.x;
      const int cnt = w < nwc ? __popc(bitmap[w]) : 0;
      int incl = cnt;
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if ((int)threadIdx.x >= o) incl += v;
      }
      if (w < nwc) wpre[w] = run + incl - cnt;
      run += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (threadIdx.x == 0) nU = run;
  }
  __syncthreads();
  const bool staged = nU <= kMaxU;
  for (int e = threadIdx.x; e < nC * kFT; e += blockDim.x) {
    const int c = cidx[e];
    loc[e] = wpre[c >> 5] + __popc(bitmap[c >> 5] & ((1u << (c & 31)) - 1u));
    if (staged) ulist[loc[e]] = c;
  }
  __syncthreads();
  // rows (u, k) of a time tile: kTT floats = kTT/4 16-byte pieces each
  auto fetch = [&](int tt, int buf) {
    if (staged) {
      const int n = nU * nk * (kTT / 4);
      float* dst = sB + buf * kMaxU * NK * kTT;
      for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const int row = e / (kTT / 4), piece = e % (kTT / 4);
        const int u = row / nk, k = row % nk;
        cp_async16(dst + (u * NK + k) * kTT + piece * 4,
                   BT + ((long long)ulist[u] * nk + k) * ldb + (long long)tt * kTT + piece * 4);
      }
    }
    cp_async_commit();
  };
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int buf = 0;
  if ((int)blockIdx.y < n_ttiles) fetch(blockIdx.y, 0);
  for (int tt = blockIdx.y; tt < n_ttiles; tt += gridDim.y) {
    const int next = tt + gridDim.y;
    if (next < n_ttiles) fetch(next, buf ^ 1);
    else cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    const float* cur = sB + buf * kMaxU * NK * kTT;
    const int t = tt * kTT + lane;
    for (int fl = warp; fl < kFT; fl += 8) {
      const int f = f0 + fl;
      float a[NS][NK];
#pragma unroll
      for (int q = 0; q < NS; ++q)
#pragma unroll
        for (int k = 0; k < NK; ++k) a[q][k] = 0.f;
      for (int j = 0; j < nC; ++j) {
        float bk[NK];
        if (staged) {
          const float* b = cur + (loc[j * kFT + fl] * NK) * kTT + lane;
#pragma unroll
          for (int k = 0; k < NK; ++k) bk[k] = b[k * kTT];
        } else {
          const float* b = BT + (long long)cidx[j * kFT + fl] * nk * ldb + t;
#pragma unroll
          for (int k = 0; k < NK; ++k) bk[k] = k < nk ? __ldg(b + (long long)k * ldb) : 0.f;
        }
        const float* w = sw + (fl * nC + j) * NS;
#pragma unroll
        for (int q = 0; q < NS; ++q) {
          const float wq = w[q];
#pragma unroll
          for (int k = 0; k < NK; ++k) a[q][k] = fmaf(wq, bk[k], a[q][k]);
        }
      }
      // largest magnitude, first index in (size, waveform) order: the
      // maximum first (NaN never wins, as in a strict > scan), then the first
      // entry that reaches it
      float best = -1.f, bval = 0.f;
      int bidx = 0;
#pragma unroll
      for (int q = 0; q < NS; ++q)
#pragma unroll
        for (int k = 0; k < NK; ++k)
          if (q < ns && k < nk) best = fmaxf(best, fabsf(a[q][k]));
      bool found = false;
#pragma unroll
      for (int q = NS - 1; q >= 0; --q)
#pragma unroll
        for (int k = NK - 1; k >= 0; --k)
          if (q < ns && k < nk && fabsf(a[q][k]) == best) {
            found = true;
            bval = a[q][k];
            bidx = q * nk + k;
          }
      if (!found) best = -1.f;
      if (f < Nfilt && t < L) {
        const int sg = bval > 0.f ? 1 : (bval < 0.f ? -1 : 0);
        As[(long long)f * L + t] = best;
        imaxs[(long long)f * L + t] = (signed char)((1 + bidx) * sg);
      }
    }
    __syncthreads();          // the buffer is read: the next fetch may reuse it
    buf ^= 1;
  }
  cp_async_wait0();
}

size_t scores_tiled_smem(int NK, int NS, int nC) {
  return sizeof(unsigned) * (kMaxCBits / 32) * 2 + sizeof(int) * (kMaxU + 2 * kMaxNC * kFT) +
         sizeof(float) * ((size_t)kFT * NS * nC + 2 * (size_t)kMaxU * NK * kTT);
}

template <int NS, int NK>
int launch_scores_tiled(const float* BT, long long ldb, int nk, int C, const long long* iC,
                        int nC, const float* weigh, int ns, int Nfilt, int L, float* As,
                        signed char* ims, int* err, cudaStream_t s) {
  const size_t smem = scores_tiled_smem(NK, NS, nC);
  KS_CUDA(cudaFuncSetAttribute(ks_detect_scores_tiled_kernel<NS, NK>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  ks::DeviceInfo dev;
  int rc = ks::device_info(&dev);
  if (rc) return rc;
  int occ = 0;
  KS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ks_detect_scores_tiled_kernel<NS, NK>,
                                                        256, smem));
  const int ftiles = (Nfilt + kFT - 1) / kFT;
  const int n_ttiles = (L + kTT - 1) / kTT;
  // about one wave of resident blocks, each walking its share of the time tiles
  const int gy = std::max(1, std::min(n_ttiles, std::max(occ, 1) * dev.sm_count / ftiles));
  const dim3 grid((unsigned)ftiles, (unsigned)gy);
  ks_detect_scores_tiled_kernel<NS, NK><<<grid, 256, smem, s>>>(BT, ldb, nk, C, iC, nC, weigh,
                                                                ns, Nfilt, L, n_ttiles, As, ims,
                                                                err);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

// Peak test, one block per (f, tile), one thread per sample.  The reference's
// test, pooled == As[f, t] && As[f, t] > th with pooled the max-pool over
// +-nt0 of the neighbour maximum (0 at the batch edges), needs the neighbour
// maximum only where As[f, t] > th: there the thread walks the nC2 neighbour
// rows over the window, keeping the running maximum from 0 as the max-pool
// does, and stops after the first row that lifts it above As[f, t] (the
// sample is then no peak; most candidates stop at the first rows, the nearest
// positions).  Maxima are exact, so the order of the walk does not matter.
// (A warp walking one candidate at a time, a lane per row, measured 6x
// slower: candidates are many and most stop within one row.)
__global__ void __launch_bounds__(kTile)
ks_detect_peaks_kernel(const float* __restrict__ As, const long long* __restrict__ iC2,
                       int nC2, int Nfilt, int L, int nt, int nt0, float th,
                       unsigned* __restrict__ bits, int nwords) {
  extern __shared__ float sm[];
  int* snb = reinterpret_cast<int*>(sm);           // [nC2]
  const int f = blockIdx.x;
  const int t0 = blockIdx.y * kTile;
  for (int j = threadIdx.x; j < nC2; j += kTile) {
    long long g = iC2[(long long)j * Nfilt + f];
    snb[j] = (int)(g < 0 ? f : (g >= Nfilt ? f : g));
  }
  __syncthreads();
  const int t = t0 + threadIdx.x;
  bool peak = false;
  if (t < L) {
    const float a = As[(long long)f * L + t];
    if (a > th) {
      // neighbour values exist for samples nt .. L-nt-1 only (0 elsewhere)
      const int lo = max(t - nt0, nt), hi = min(t + nt0, L - nt - 1);
      float m = 0.f;
      for (int j = 0; j < nC2 && !(m > a); ++j) {
        const float* row = As + (long long)snb[j] * L;
        for (int u = lo; u <= hi; ++u) m = fmaxf(m, row[u]);
      }
      peak = m == a;
    }
  }
  const unsigned w = __ballot_sync(0xffffffffu, peak);
  const int word = (t0 >> 5) + (threadIdx.x >> 5);
  if ((threadIdx.x & 31) == 0 && word < nwords) bits[(long long)f * nwords + word] = w;
}

__global__ void ks_detect_count_kernel(const unsigned* __restrict__ bits, int Nfilt, int nwords,
                                       int nchunks, long long* __restrict__ counts) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)Nfilt * nchunks) return;
  const int f = (int)(e / nchunks), ch = (int)(e % nchunks);
  const unsigned* b = bits + (long long)f * nwords;
  int n = 0;
  for (int w = ch * kChunkWords; w < min(nwords, (ch + 1) * kChunkWords); ++w) n += __popc(b[w]);
  counts[e] = n;
}

// Exclusive scan of n counts in place (one block), total in *total.
__global__ void __launch_bounds__(1024)
ks_detect_scan_kernel(long long* __restrict__ counts, long long n, long long* __restrict__ total) {
  __shared__ long long part[1024];
  const long long per = (n + 1023) / 1024;
  const long long a = threadIdx.x * per, b = min(n, a + per);
  long long s = 0;
  for (long long i = a; i < b; ++i) s += counts[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const long long v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  long long run = part[threadIdx.x] - s;
  for (long long i = a; i < b; ++i) {
    const long long c = counts[i];
    counts[i] = run;
    run += c;
  }
  if (threadIdx.x == 1023) *total = part[1023];
}

__global__ void ks_detect_emit_kernel(const unsigned* __restrict__ bits, int Nfilt, int nwords,
                                      int nchunks, const long long* __restrict__ offsets,
                                      long long capacity, long long* __restrict__ xy) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)Nfilt * nchunks) return;
  const int f = (int)(e / nchunks), ch = (int)(e % nchunks);
  const unsigned* b = bits + (long long)f * nwords;
  long long o = offsets[e];
  for (int w = ch * kChunkWords; w < min(nwords, (ch + 1) * kChunkWords); ++w) {
    unsigned m = b[w];
    while (m) {
      const int bit = __ffs(m) - 1;
      m &= m - 1;
      if (o < capacity) {
        xy[2 * o] = f;
        xy[2 * o + 1] = (long long)w * 32 + bit;
      }
      ++o;
    }
  }
}

// Per spike: signed index, amplitude, adist over the nearest channels and
// the relu-weighted y position (float32, j in order).
__global__ void ks_detect_gather_kernel(const long long* __restrict__ xy, const long long* __restrict__ n_ptr,
                                        long long capacity, const float* __restrict__ As,
                                        const signed char* __restrict__ imaxs,
                                        const float* __restrict__ BT, long long ldb, int nk, int C,
                                        const long long* __restrict__ iC, int nC, int Nfilt,
                                        int L, const float* __restrict__ yc,
                                        long long* __restrict__ imax, float* __restrict__ amp,
                                        float* __restrict__ adist, float* __restrict__ yct) {
  const long long n = min(*n_ptr, capacity);
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int f = (int)xy[2 * s];
  const int t = (int)xy[2 * s + 1];
  const int im = imaxs[(long long)f * L + t];
  const int sg = im > 0 ? 1 : (im < 0 ? -1 : 0);
  const int idx = abs(im) - 1;
  imax[s] = idx;
  amp[s] = As[(long long)f * L + t];
  const int k = ((idx % nk) + nk) % nk;
  float rs = 0.f;
  float r[kMaxNC];
#pragma unroll
  for (int j = 0; j < kMaxNC; ++j) {
    r[j] = 0.f;
    if (j < nC) {
      long long c = iC[(long long)j * Nfilt + f];
      if (c < 0 || c >= C) c = 0;
      const float v = BT[((long long)c * nk + k) * ldb + t] * (float)sg;
      adist[(long long)j * capacity + s] = v;
      r[j] = fmaxf(v, 0.f);
      rs = __fadd_rn(rs, r[j]);
    }
  }
  float y = 0.f;
#pragma unroll
  for (int j = 0; j < kMaxNC; ++j)
    if (j < nC) {
      long long c = iC[(long long)j * Nfilt + f];
      if (c < 0 || c >= C) c = 0;
      y = __fadd_rn(y, __fmul_rn(__fdiv_rn(r[j], rs), yc[c]));
    }
  yct[s] = y;
}

// tF[s, j, p] = sum_u X[iC[j, f], t - nt/2 + u] * wPCA[p, u]: one warp per
// (spike, channel), grid-stride over the spikes found.
__global__ void __launch_bounds__(256)
ks_detect_features_kernel(const float* __restrict__ X, int C, int L,
                          const long long* __restrict__ xy, const long long* __restrict__ n_ptr,
                          long long capacity, const long long* __restrict__ iC, int nC,
                          int Nfilt, const float* __restrict__ W, int P, int nt,
                          float* __restrict__ tF) {
  extern __shared__ float sW[];   // [P][nt]
  const long long n = min(*n_ptr, capacity);
  if ((long long)blockIdx.x * 8 >= n * nC) return;     // the whole block has no work
  for (int i = threadIdx.x; i < P * nt; i += blockDim.x) sW[i] = W[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (long long e = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; e < n * nC;
       e += ((long long)gridDim.x * blockDim.x) >> 5) {
    const long long s = e / nC;
    const int j = (int)(e - s * nC);
    const int f = (int)xy[2 * s];
    const int t = (int)xy[2 * s + 1];
    long long c = iC[(long long)j * Nfilt + f];
    if (c < 0 || c >= C) c = 0;
    const float* x = X + c * L + (t - nt / 2);
    float part[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) part[p] = 0.f;
    for (int u = lane; u < nt; u += 32) {
      const float xv = x[u];
#pragma unroll
      for (int p = 0; p < 8; ++p)
        if (p < P) part[p] = fmaf(xv, sW[p * nt + u], part[p]);
    }
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      if (p < P) {
        float v = part[p];
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) tF[(s * nC + j) * P + p] = v;
      }
    }
  }
}

__global__ void ks_detect_finish_kernel(const long long* __restrict__ total, long long capacity,
                                        const int* __restrict__ err, long long* __restrict__ info) {
  const long long n = *total;
  const int e = *err;
  info[0] = n < capacity ? n : capacity;
  info[1] = e ? e : (n > capacity ? KS_ERR_OVERFLOW : KS_OK);
  info[2] = 0;
  info[3] = n;
}

struct DetectLayout {
  int64_t Lpad, nwords, nchunks;
  size_t ctl, bt, as, im, bits, counts, bytes;
};

DetectLayout detect_layout(int64_t C, int64_t L, int64_t nk, int64_t Nfilt) {
  DetectLayout d{};
  d.Lpad = ks::round_up(L, 128);
  d.nwords = (L + 31) / 32;
  d.nchunks = (d.nwords + kChunkWords - 1) / kChunkWords;
  size_t o = 0;
  auto take = [&](size_t b) {
    const size_t at = o;
    o = ks::align256(o + b);
    return at;
  };
  d.ctl = take(256);                               // err, total
  d.bt = take(sizeof(float) * (size_t)C * nk * d.Lpad);
  d.as = take(sizeof(float) * (size_t)Nfilt * L);
  d.im = take((size_t)Nfilt * L);
  d.bits = take(sizeof(unsigned) * (size_t)Nfilt * d.nwords);
  d.counts = take(sizeof(long long) * (size_t)Nfilt * d.nchunks);
  d.bytes = o;
  return d;
}

}  // namespace

extern "C" KS_API size_t ks_detect_workspace_size(int64_t C, int64_t L, int64_t nk,
                                                  int64_t Nfilt) {
  if (C < 1 || L < 1 || nk < 1 || Nfilt < 1) return 0;
  return detect_layout(C, L, nk, Nfilt).bytes;
}

extern "C" KS_API int ks_detect(const float* X, int64_t C, int64_t L, const float* wTEMP,
                                int64_t nk, int64_t nt, const int64_t* iC, int64_t nC,
                                const int64_t* iC2, int64_t nC2, const float* weigh,
                                int64_t nsizes, int64_t Nfilt, int64_t nt0, float th,
                                const float* wPCA, int64_t P, const float* yc, int64_t capacity,
                                int64_t* xy, int64_t* imax, float* amp, float* adist, float* yct,
                                float* tF, int64_t* info, void* workspace,
                                size_t workspace_bytes, void* stream) {
  using namespace ks;
  if (!X || !wTEMP || !iC || !iC2 || !weigh || !wPCA || !yc || !info)
    return fail(KS_ERR_ARG, "ks_detect: null pointer");
  if (C < 1 || L < 1 || nk < 1 || nt < 1 || nt % 2 == 0 || nC < 1 || nC2 < 1 || nsizes < 1 ||
      Nfilt < 1 || nt0 < 0 || P < 1 || capacity < 0)
    return fail(KS_ERR_ARG, "ks_detect: bad sizes (odd nt, counts >= 1)");
  if (nk > kMaxNK || nsizes > kMaxNS || nC > kMaxNC || P > 8 || nt > 1023)
    return fail(KS_ERR_UNSUPPORTED, "ks_detect: nk, sizes <= 8, nC <= 32, P <= 8, nt <= 1023");
  if (L > 0x7fffffffLL / 2 || Nfilt > 65535 || (long long)Nfilt * L > (1LL << 40))
    return fail(KS_ERR_UNSUPPORTED, "ks_detect: batch too long or too many positions");
  if (capacity > 0 && (!xy || !imax || !amp || !adist || !yct || !tF))
    return fail(KS_ERR_ARG, "ks_detect: null output");
  const DetectLayout d = detect_layout(C, L, nk, Nfilt);
  if (!workspace || workspace_bytes < d.bytes)
    return fail(KS_ERR_WORKSPACE, "ks_detect: workspace too small");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long* iCl = reinterpret_cast<const long long*>(iC);
  const long long* iC2l = reinterpret_cast<const long long*>(iC2);
  long long* xyl = reinterpret_cast<long long*>(xy);
  long long* imaxl = reinterpret_cast<long long*>(imax);
  long long* infol = reinterpret_cast<long long*>(info);
  char* base = static_cast<char*>(workspace);
  int* err = reinterpret_cast<int*>(base + d.ctl);
  long long* total = reinterpret_cast<long long*>(base + d.ctl + 8);
  float* BT = reinterpret_cast<float*>(base + d.bt);
  float* As = reinterpret_cast<float*>(base + d.as);
  signed char* ims = reinterpret_cast<signed char*>(base + d.im);
  unsigned* bits = reinterpret_cast<unsigned*>(base + d.bits);
  long long* counts = reinterpret_cast<long long*>(base + d.counts);
  KS_CUDA(cudaMemsetAsync(base + d.ctl, 0, 16, s));

  // 1. the universal waveforms convolved with the batch: rows (c, k)
  int rc = launch_temporal_rows(X, wTEMP, C, L, nk, nt, d.Lpad, BT, d.Lpad, s);
  if (rc) return rc;
  // 2. scores over sizes and waveforms
  if (C <= kMaxCBits) {
    // the reference's defaults (5 sizes, 6 waveforms) have their own instantiation
    rc = (nsizes == 5 && nk == 6)
             ? launch_scores_tiled<5, 6>(BT, d.Lpad, (int)nk, (int)C, iCl, (int)nC, weigh,
                                         (int)nsizes, (int)Nfilt, (int)L, As, ims, err, s)
             : launch_scores_tiled<kMaxNS, kMaxNK>(BT, d.Lpad, (int)nk, (int)C, iCl, (int)nC,
                                                   weigh, (int)nsizes, (int)Nfilt, (int)L, As,
                                                   ims, err, s);
    if (rc) return rc;
  } else {
    const dim3 grid((unsigned)Nfilt, (unsigned)((L + kTile - 1) / kTile));
    ks_detect_scores_kernel<<<grid, kTile, 0, s>>>(BT, d.Lpad, (int)nk, (int)C, iCl, (int)nC, weigh,
                                                   (int)nsizes, (int)Nfilt, (int)L, As, ims, err);
    KS_CUDA(cudaGetLastError());
  }
  // 3. neighbour maximum, max-pool, peaks
  {
    const size_t smem = sizeof(int) * (size_t)nC2;
    if (smem > 200 * 1024) return fail(KS_ERR_UNSUPPORTED, "ks_detect: nC2 too large");
    KS_CUDA(cudaFuncSetAttribute(ks_detect_peaks_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    const dim3 grid((unsigned)Nfilt, (unsigned)((L + kTile - 1) / kTile));
    ks_detect_peaks_kernel<<<grid, kTile, smem, s>>>(As, iC2l, (int)nC2, (int)Nfilt, (int)L,
                                                     (int)nt, (int)nt0, th, bits, (int)d.nwords);
    KS_CUDA(cudaGetLastError());
  }
  // 4. (f, t)-ordered compaction
  const long long ncnt = (long long)Nfilt * d.nchunks;
  const unsigned cb = (unsigned)((ncnt + 255) / 256);
  ks_detect_count_kernel<<<cb, 256, 0, s>>>(bits, (int)Nfilt, (int)d.nwords, (int)d.nchunks, counts);
  KS_CUDA(cudaGetLastError());
  ks_detect_scan_kernel<<<1, 1024, 0, s>>>(counts, ncnt, total);
  KS_CUDA(cudaGetLastError());
  if (capacity > 0) {
    ks_detect_emit_kernel<<<cb, 256, 0, s>>>(bits, (int)Nfilt, (int)d.nwords, (int)d.nchunks, counts,
                                             capacity, xyl);
    KS_CUDA(cudaGetLastError());
    // 5. per-spike outputs (grids sized for the capacity; threads past the count return)
    ks_detect_gather_kernel<<<(unsigned)((capacity + 127) / 128), 128, 0, s>>>(
        xyl, total, capacity, As, ims, BT, d.Lpad, (int)nk, (int)C, iCl, (int)nC, (int)Nfilt, (int)L,
        yc, imaxl, amp, adist, yct);
    KS_CUDA(cudaGetLastError());
    DeviceInfo dev;
    if ((rc = device_info(&dev))) return rc;
    const long long warps = capacity * nC;
    const unsigned fb = (unsigned)std::min<long long>((warps + 7) / 8, (long long)dev.sm_count * 16);
    ks_detect_features_kernel<<<fb, 256, sizeof(float) * P * nt, s>>>(
        X, (int)C, (int)L, xyl, total, capacity, iCl, (int)nC, (int)Nfilt, wPCA, (int)P, (int)nt, tF);
    KS_CUDA(cudaGetLastError());
  }
  ks_detect_finish_kernel<<<1, 1, 0, s>>>(total, capacity, err, infol);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}
