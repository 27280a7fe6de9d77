// Universal templates learned from data (kilosort/spikedetect.py:33-92,
// templates_from_data): isolated single-channel peaks, their snippets, the
// Gram matrix of the unit-norm snippets (whose leading eigenvectors are the
// truncated-SVD basis wPCA) and the k-means steps that give wTEMP.
//
// ks_snippets -- kilosort/spikedetect.py:33-48 (extract_snippets) on one
// padded batch X [C, L] f32:
//   peak[c, t] = |X[c, t]| is the maximum of |X| over channels c-4..c+4 and
//                samples t-5..t+5 (inside the batch) and exceeds th;
//   iso[c, t]  = peak[c, t] and the peaks in channels c-6..c+6 and samples
//                t-30..t+30 number one, tested as the reference tests it:
//                fl(fl(n / area) * area) == 1 with area = 13*61 (the mean
//                pool times its area, in float32); zero for t < nt and
//                t >= L - nt;
//   snippets of every iso point in (channel, sample) order -- the order of
//   torch.nonzero -- clips[i, j] = X[c, t - twav_min + j], j < nt.
// Both window maxima and sums are separable: a pass along the samples, then
// one along the channels.  The compaction counts each channel row, scans the
// counts and writes each row's points in sample order (a block per row).
#include "ks_common.cuh"

#include <algorithm>

namespace {

constexpr int kLocC = 4, kLocT = 5;     // peak window (channels, samples)
constexpr int kIsoC = 6, kIsoT = 30;    // isolation window

// |X| maximum over samples t-kLocT..t+kLocT of each row.
__global__ void ks_snip_tmax_kernel(const float* __restrict__ X, int C, int L,
                                    float* __restrict__ tmax) {
  const long long n = (long long)C * L;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(e % L);
    const float* row = X + (e - t);
    float m = fabsf(row[t]);
    for (int d = 1; d <= kLocT; ++d) {
      if (t - d >= 0) m = fmaxf(m, fabsf(row[t - d]));
      if (t + d < L) m = fmaxf(m, fabsf(row[t + d]));
    }
    tmax[e] = m;
  }
}

// peak[c, t] from the channel maximum of tmax over c-kLocC..c+kLocC.
__global__ void ks_snip_peak_kernel(const float* __restrict__ X,
                                    const float* __restrict__ tmax, int C, int L, float th,
                                    unsigned char* __restrict__ peak) {
  const long long n = (long long)C * L;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e / L);
    const int t = (int)(e % L);
    float m = tmax[e];
    for (int d = 1; d <= kLocC; ++d) {
      if (c - d >= 0) m = fmaxf(m, tmax[(long long)(c - d) * L + t]);
      if (c + d < C) m = fmaxf(m, tmax[(long long)(c + d) * L + t]);
    }
    const float a = fabsf(X[e]);
    peak[e] = (m == a && a > th) ? 1 : 0;
  }
}

// Count of peaks over samples t-kIsoT..t+kIsoT of each row.
__global__ void ks_snip_tsum_kernel(const unsigned char* __restrict__ peak, int C, int L,
                                    unsigned short* __restrict__ tsum) {
  const long long n = (long long)C * L;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(e % L);
    const unsigned char* row = peak + (e - t);
    int s = 0;
    const int lo = max(0, t - kIsoT), hi = min(L - 1, t + kIsoT);
    for (int u = lo; u <= hi; ++u) s += row[u];
    tsum[e] = (unsigned short)s;
  }
}

// iso[c, t]: the peak is alone in its isolation window (the reference's
// float32 test) and lies nt or more samples from both batch edges.
__global__ void ks_snip_iso_kernel(const unsigned char* __restrict__ peak,
                                   const unsigned short* __restrict__ tsum, int C, int L, int nt,
                                   unsigned char* __restrict__ iso) {
  const long long n = (long long)C * L;
  const float area = (float)((2 * kIsoC + 1) * (2 * kIsoT + 1));
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e / L);
    const int t = (int)(e % L);
    int s = 0;
    if (peak[e]) {
      const int lo = max(0, c - kIsoC), hi = min(C - 1, c + kIsoC);
      for (int u = lo; u <= hi; ++u) s += tsum[(long long)u * L + t];
    }
    const float sum = __fmul_rn(__fdiv_rn((float)s, area), area);
    iso[e] = (peak[e] && sum == 1.f && t >= nt && t < L - nt) ? 1 : 0;
  }
}

// Points of each channel row (a block per row).
__global__ void ks_snip_count_kernel(const unsigned char* __restrict__ iso, int L,
                                     int* __restrict__ rows) {
  __shared__ int part[32];
  const unsigned char* row = iso + (long long)blockIdx.x * L;
  int s = 0;
  for (int t = threadIdx.x; t < L; t += blockDim.x) s += row[t];
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int tot = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += part[w];
    rows[blockIdx.x] = tot;
  }
}

// Exclusive scan of the row counts (one block, rows in order); offs[C] is the
// batch's total.
__global__ void ks_snip_scan_kernel(const int* __restrict__ rows, int C, int* __restrict__ offs) {
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int c = 0; c < C; ++c) {
      offs[c] = acc;
      acc += rows[c];
    }
    offs[C] = acc;
  }
}

// Snippets of row blockIdx.x in sample order: a block-wide scan per tile of
// blockDim.x samples gives each point its rank.  Points at or beyond cap are
// counted but not written.
__global__ void ks_snip_gather_kernel(const float* __restrict__ X, const unsigned char* __restrict__ iso,
                                      const int* __restrict__ offs, int L, int nt, int twav_min,
                                      long long base, long long cap, float* __restrict__ clips) {
  __shared__ int wsum[33];
  const int c = blockIdx.x;
  const unsigned char* row = iso + (long long)c * L;
  const float* xr = X + (long long)c * L;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  long long next = base + offs[c];
  for (int t0 = 0; t0 < L; t0 += blockDim.x) {
    const int t = t0 + threadIdx.x;
    const int f = (t < L && row[t]) ? 1 : 0;
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wsum[warp] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int w = 0; w < nw; ++w) {
        const int v = wsum[w];
        wsum[w] = acc;
        acc += v;
      }
      wsum[32] = acc;
    }
    __syncthreads();
    if (f) {
      const long long i = next + wsum[warp] + __popc(bal & ((1u << lane) - 1u));
      if (i < cap) {
        const float* src = xr + (t - twav_min);
        float* dst = clips + i * nt;
        for (int j = 0; j < nt; ++j) dst[j] = src[j];
      }
    }
    next += wsum[32];
    __syncthreads();
  }
}

// --------------------------------------------------------------- Gram matrix
// Each snippet scaled to unit norm (in place; the norm in double), and the
// per-block partials of G = sum_i x_i x_i^T (double), blocks taking fixed
// chunks of snippets so the final sum (ks_gram_reduce_kernel, blocks in
// order) is reproducible.  Thread e of a block owns entries e, e+blockDim, ...
// of the nt x nt matrix.
constexpr int kGramChunk = 64;   // snippets staged per step

__global__ void ks_snip_normalize_kernel(float* __restrict__ clips, long long n, int nt) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    float* x = clips + i * nt;
    double s = 0.0;
    for (int j = 0; j < nt; ++j) s += (double)x[j] * x[j];
    const double r = s > 0.0 ? 1.0 / sqrt(s) : 0.0;
    for (int j = 0; j < nt; ++j) x[j] = (float)(x[j] * r);
  }
}

__global__ void ks_gram_partial_kernel(const float* __restrict__ clips, long long n, int nt,
                                       long long per_block, double* __restrict__ partial) {
  extern __shared__ float sx[];                    // kGramChunk x nt
  const long long i0 = blockIdx.x * per_block;
  const long long i1 = min(n, i0 + per_block);
  const int ne = nt * nt;
  double acc[16];
  for (int q = 0; q < 16; ++q) acc[q] = 0.0;
  for (long long c0 = i0; c0 < i1; c0 += kGramChunk) {
    const int m = (int)min((long long)kGramChunk, i1 - c0);
    __syncthreads();
    for (int e = threadIdx.x; e < m * nt; e += blockDim.x) sx[e] = clips[c0 * nt + e];
    __syncthreads();
    for (int q = 0; q < 16; ++q) {
      const int e = threadIdx.x + q * blockDim.x;
      if (e >= ne) break;
      const int a = e / nt, b = e % nt;
      double s = 0.0;
      for (int r = 0; r < m; ++r) s += (double)sx[r * nt + a] * sx[r * nt + b];
      acc[q] += s;
    }
  }
  for (int q = 0; q < 16; ++q) {
    const int e = threadIdx.x + q * blockDim.x;
    if (e < ne) partial[(long long)blockIdx.x * ne + e] = acc[q];
  }
}

__global__ void ks_gram_reduce_kernel(const double* __restrict__ partial, int nblocks, int ne,
                                      double* __restrict__ G) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partial[(long long)b * ne + e];
    G[e] = s;
  }
}

// ----------------------------------------------------------------- k-means
// Lloyd steps and k-means++ seeding over the unit-norm snippets X [n, d]
// (kilosort/spikedetect.py:78-85 runs sklearn's KMeans there).  Distances in
// double; each block takes fixed chunks of kKmChunk points, staged in shared
// memory, and reduces its per-cluster sums in point order, so every result
// is reproducible.
constexpr int kKmChunk = 128;
constexpr int kKmThreads = 256;

__device__ __forceinline__ double sqdist(const float* x, const float* c, int d) {
  double s = 0.0;
  for (int a = 0; a < d; ++a) {
    const double v = (double)x[a] - (double)c[a];
    s += v * v;
  }
  return s;
}

// Assignment to the nearest center (first index on ties), with per-block
// partial sums [k][d], counts [k], inertia and number of changed labels.
__global__ void __launch_bounds__(kKmThreads)
ks_km_assign_kernel(const float* __restrict__ X, long long n, int d,
                    const float* __restrict__ centers, int k, long long per_block,
                    int* __restrict__ labels, double* __restrict__ psum,
                    long long* __restrict__ pcnt, double* __restrict__ pstat) {
  extern __shared__ double smem_d[];
  double* sdist = smem_d;                                            // kKmChunk distances
  int* slab = reinterpret_cast<int*>(sdist + kKmChunk);              // kKmChunk labels
  float* sc = reinterpret_cast<float*>(slab + kKmChunk);             // k x d centers
  float* sx = sc + k * d;                                            // kKmChunk x d points
  for (int e = threadIdx.x; e < k * d; e += blockDim.x) sc[e] = centers[e];
  const long long i0 = blockIdx.x * per_block;
  const long long i1 = min(n, i0 + per_block);
  const int ke = k * d;
  double acc[16];
  long long cnt = 0;
  for (int q = 0; q < 16; ++q) acc[q] = 0.0;
  double inertia = 0.0;
  long long changed = 0;
  for (long long c0 = i0; c0 < i1; c0 += kKmChunk) {
    const int m = (int)min((long long)kKmChunk, i1 - c0);
    __syncthreads();
    for (int e = threadIdx.x; e < m * d; e += blockDim.x) sx[e] = X[c0 * d + e];
    __syncthreads();
    if (threadIdx.x < m) {
      const float* x = sx + threadIdx.x * d;
      int best = 0;
      double bd = sqdist(x, sc, d);
      for (int j = 1; j < k; ++j) {
        const double v = sqdist(x, sc + j * d, d);
        if (v < bd) {
          bd = v;
          best = j;
        }
      }
      const long long i = c0 + threadIdx.x;
      if (labels[i] != best) {
        labels[i] = best;
        slab[threadIdx.x] = best | (1 << 30);
      } else {
        slab[threadIdx.x] = best;
      }
      sdist[threadIdx.x] = bd;
    }
    __syncthreads();
    for (int q = 0; q < 16; ++q) {
      const int e = threadIdx.x + q * blockDim.x;
      if (e >= ke) break;
      const int j = e / d, a = e % d;
      double s = 0.0;
      for (int r = 0; r < m; ++r)
        if ((slab[r] & 0xffff) == j) s += sx[r * d + a];
      acc[q] += s;
    }
    if (threadIdx.x < k) {
      for (int r = 0; r < m; ++r) cnt += ((slab[r] & 0xffff) == (int)threadIdx.x) ? 1 : 0;
    }
    if (threadIdx.x == 0) {
      for (int r = 0; r < m; ++r) {
        inertia += sdist[r];
        changed += (slab[r] >> 30) & 1;
      }
    }
  }
  for (int q = 0; q < 16; ++q) {
    const int e = threadIdx.x + q * blockDim.x;
    if (e < ke) psum[(long long)blockIdx.x * ke + e] = acc[q];
  }
  if (threadIdx.x < k) pcnt[(long long)blockIdx.x * k + threadIdx.x] = cnt;
  if (threadIdx.x == 0) {
    pstat[2 * blockIdx.x] = inertia;
    pstat[2 * blockIdx.x + 1] = (double)changed;
  }
}

// Sum of the block partials in block order: sums [k][d], counts [k],
// stats {inertia, changed}.
__global__ void ks_km_reduce_kernel(const double* __restrict__ psum,
                                    const long long* __restrict__ pcnt,
                                    const double* __restrict__ pstat, int nblocks, int k, int d,
                                    double* __restrict__ sums, long long* __restrict__ counts,
                                    double* __restrict__ stats) {
  const int ke = k * d;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ke + k + 2;
       e += gridDim.x * blockDim.x) {
    if (e < ke) {
      double s = 0.0;
      for (int b = 0; b < nblocks; ++b) s += psum[(long long)b * ke + e];
      sums[e] = s;
    } else if (e < ke + k) {
      long long s = 0;
      for (int b = 0; b < nblocks; ++b) s += pcnt[(long long)b * k + (e - ke)];
      counts[e - ke] = s;
    } else {
      const int w = e - ke - k;
      double s = 0.0;
      for (int b = 0; b < nblocks; ++b) s += pstat[2 * b + w];
      stats[w] = s;
    }
  }
}

// d2[i] = squared distance of point i to c (init) or the smaller of d2[i]
// and that distance.
__global__ void ks_km_mindist_kernel(const float* __restrict__ X, long long n, int d,
                                     const float* __restrict__ c, int init,
                                     double* __restrict__ d2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = sqdist(X + i * d, c, d);
    d2[i] = init ? v : fmin(d2[i], v);
  }
}

// Per-block partial potentials of T candidate centers: sum over the block's
// chunk of min(d2[i], |x_i - cand_t|^2), points in order.
__global__ void __launch_bounds__(kKmThreads)
ks_km_candidates_kernel(const float* __restrict__ X, long long n, int d,
                        const float* __restrict__ cand, int T, const double* __restrict__ d2,
                        long long per_block, double* __restrict__ ppot) {
  __shared__ double part[kKmThreads];
  const long long i0 = blockIdx.x * per_block;
  const long long i1 = min(n, i0 + per_block);
  for (int t = 0; t < T; ++t) {
    double s = 0.0;
    for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x)
      s += fmin(d2[i], sqdist(X + i * d, cand + t * d, d));
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double tot = 0.0;
      for (int r = 0; r < (int)blockDim.x; ++r) tot += part[r];
      ppot[(long long)blockIdx.x * T + t] = tot;
    }
    __syncthreads();
  }
}

__global__ void ks_km_pot_reduce_kernel(const double* __restrict__ ppot, int nblocks, int T,
                                        double* __restrict__ pots) {
  const int t = threadIdx.x;
  if (t < T) {
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += ppot[(long long)b * T + t];
    pots[t] = s;
  }
}

}  // namespace

namespace {

struct SnipLayout {
  size_t tmax, peak, tsum, iso, rows, offs, bytes;
};

SnipLayout snip_layout(int64_t C, int64_t L) {
  SnipLayout s;
  size_t o = 0;
  auto take = [&](size_t b) {
    const size_t at = o;
    o = ks::align256(o + b);
    return at;
  };
  s.tmax = take(4 * (size_t)C * L);
  s.peak = take((size_t)C * L);
  s.tsum = take(2 * (size_t)C * L);
  s.iso = take((size_t)C * L);
  s.rows = take(4 * (size_t)C);
  s.offs = take(4 * (size_t)(C + 1));
  s.bytes = o;
  return s;
}

unsigned grid_for(long long n, int threads) {
  return (unsigned)std::min<long long>((n + threads - 1) / threads, 8192);
}

int blocks_for(long long n, int per_chunk, long long* per_block) {
  // about four chunks per block, at most 1184 blocks (8 per SM)
  long long nb = std::max<long long>(1, std::min<long long>(1184, (n + 4 * per_chunk - 1) /
                                                                       (4 * per_chunk)));
  *per_block = (n + nb - 1) / nb;
  return (int)nb;
}

}  // namespace

extern "C" KS_API size_t ks_snippets_workspace_size(int64_t C, int64_t L) {
  if (C < 1 || L < 1) return 0;
  return snip_layout(C, L).bytes;
}

extern "C" KS_API int ks_snippets(const float* X, int64_t C, int64_t L, int64_t nt,
                                  int64_t twav_min, float th, int64_t base, int64_t capacity,
                                  float* clips, int32_t* count, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  using namespace ks;
  if (!X || !count || (capacity > 0 && !clips)) return fail(KS_ERR_ARG, "ks_snippets: null pointer");
  if (C < 1 || L < 1 || nt < 1 || twav_min < 0 || twav_min >= nt || 2 * nt >= L || base < 0 ||
      capacity < 0)
    return fail(KS_ERR_ARG, "ks_snippets: need C, L, nt >= 1, 0 <= twav_min < nt, 2*nt < L");
  if (C * L >= (1LL << 31)) return fail(KS_ERR_UNSUPPORTED, "ks_snippets: batch too large");
  const SnipLayout sl = snip_layout(C, L);
  if (!workspace || workspace_bytes < sl.bytes)
    return fail(KS_ERR_WORKSPACE, "ks_snippets: workspace too small");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  char* w = static_cast<char*>(workspace);
  float* tmax = reinterpret_cast<float*>(w + sl.tmax);
  unsigned char* peak = reinterpret_cast<unsigned char*>(w + sl.peak);
  unsigned short* tsum = reinterpret_cast<unsigned short*>(w + sl.tsum);
  unsigned char* iso = reinterpret_cast<unsigned char*>(w + sl.iso);
  int* rows = reinterpret_cast<int*>(w + sl.rows);
  int* offs = reinterpret_cast<int*>(w + sl.offs);
  const long long n = C * L;
  ks_snip_tmax_kernel<<<grid_for(n, 256), 256, 0, s>>>(X, (int)C, (int)L, tmax);
  ks_snip_peak_kernel<<<grid_for(n, 256), 256, 0, s>>>(X, tmax, (int)C, (int)L, th, peak);
  ks_snip_tsum_kernel<<<grid_for(n, 256), 256, 0, s>>>(peak, (int)C, (int)L, tsum);
  ks_snip_iso_kernel<<<grid_for(n, 256), 256, 0, s>>>(peak, tsum, (int)C, (int)L, (int)nt, iso);
  ks_snip_count_kernel<<<(unsigned)C, 256, 0, s>>>(iso, (int)L, rows);
  ks_snip_scan_kernel<<<1, 32, 0, s>>>(rows, (int)C, offs);
  ks_snip_gather_kernel<<<(unsigned)C, 256, 0, s>>>(X, iso, offs, (int)L, (int)nt,
                                                     (int)twav_min, base, capacity, clips);
  KS_CUDA(cudaGetLastError());
  KS_CUDA(cudaMemcpyAsync(count, offs + C, sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
  return KS_OK;
}

extern "C" KS_API size_t ks_snippet_gram_workspace_size(int64_t n, int64_t nt) {
  if (n < 0 || nt < 1 || nt > 64) return 0;
  long long per_block;
  const int nb = blocks_for(std::max<int64_t>(n, 1), kGramChunk, &per_block);
  return ks::align256(8 * (size_t)nb * nt * nt);
}

extern "C" KS_API int ks_snippet_gram(float* clips, int64_t n, int64_t nt, double* G,
                                      void* workspace, size_t workspace_bytes, void* stream) {
  using namespace ks;
  if (!G || (n > 0 && !clips)) return fail(KS_ERR_ARG, "ks_snippet_gram: null pointer");
  if (n < 0 || nt < 1 || nt > 64) return fail(KS_ERR_ARG, "ks_snippet_gram: need n >= 0, 1 <= nt <= 64");
  long long per_block;
  const int nb = blocks_for(std::max<int64_t>(n, 1), kGramChunk, &per_block);
  if (!workspace || workspace_bytes < ks_snippet_gram_workspace_size(n, nt))
    return fail(KS_ERR_WORKSPACE, "ks_snippet_gram: workspace too small");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* partial = static_cast<double*>(workspace);
  if (n > 0) ks_snip_normalize_kernel<<<grid_for(n, 256), 256, 0, s>>>(clips, n, (int)nt);
  ks_gram_partial_kernel<<<nb, 256, sizeof(float) * kGramChunk * nt, s>>>(clips, n, (int)nt,
                                                                          per_block, partial);
  ks_gram_reduce_kernel<<<(unsigned)((nt * nt + 255) / 256), 256, 0, s>>>(partial, nb,
                                                                          (int)(nt * nt), G);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

extern "C" KS_API size_t ks_kmeans_workspace_size(int64_t n, int64_t d, int64_t k) {
  if (n < 1 || d < 1 || d > 64 || k < 1 || k > 64 || k * d > 16 * kKmThreads) return 0;
  long long per_block;
  const int nb = blocks_for(n, kKmChunk, &per_block);
  return ks::align256(8 * (size_t)nb * k * d) + ks::align256(8 * (size_t)nb * k) +
         ks::align256(16 * (size_t)nb) + ks::align256(8 * (size_t)nb * 64);
}

// One Lloyd step: labels (int32 [n], in/out; set them to -1 before the first
// step) of the nearest of the k centers [k, d], and the sums [k, d] (double),
// counts [k] (int64) and stats {inertia, changed labels} (double) of that
// assignment, all on the device.
extern "C" KS_API int ks_kmeans_step(const float* X, int64_t n, int64_t d, const float* centers,
                                     int64_t k, int32_t* labels, double* sums, int64_t* counts,
                                     double* stats, void* workspace, size_t workspace_bytes,
                                     void* stream) {
  using namespace ks;
  if (!X || !centers || !labels || !sums || !counts || !stats)
    return fail(KS_ERR_ARG, "ks_kmeans_step: null pointer");
  const size_t need = ks_kmeans_workspace_size(n, d, k);
  if (need == 0) return fail(KS_ERR_ARG, "ks_kmeans_step: need n >= 1, 1 <= d, k <= 64, k*d <= 4096");
  if (!workspace || workspace_bytes < need)
    return fail(KS_ERR_WORKSPACE, "ks_kmeans_step: workspace too small");
  long long per_block;
  const int nb = blocks_for(n, kKmChunk, &per_block);
  char* w = static_cast<char*>(workspace);
  double* psum = reinterpret_cast<double*>(w);
  long long* pcnt = reinterpret_cast<long long*>(w + align256(8 * (size_t)nb * k * d));
  double* pstat = reinterpret_cast<double*>(w + align256(8 * (size_t)nb * k * d) +
                                            align256(8 * (size_t)nb * k));
  const size_t smem = sizeof(double) * kKmChunk + sizeof(int) * kKmChunk +
                      sizeof(float) * (size_t)(k + kKmChunk) * d;
  KS_CUDA(cudaFuncSetAttribute(ks_km_assign_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  ks_km_assign_kernel<<<nb, kKmThreads, smem, s>>>(X, n, (int)d, centers, (int)k, per_block,
                                                   labels, psum, pcnt, pstat);
  ks_km_reduce_kernel<<<(unsigned)((k * d + k + 2 + 255) / 256), 256, 0, s>>>(
      psum, reinterpret_cast<const long long*>(pcnt), pstat, nb, (int)k, (int)d, sums,
      reinterpret_cast<long long*>(counts), stats);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

// k-means++ seeding helpers: d2 [n] (double) = squared distance of each point
// to center c [d] (init != 0) or the smaller of d2 and that distance; and the
// potentials pots [T] (double) = sum_i min(d2[i], |x_i - cand_t|^2) of T
// candidate centers cand [T, d] (T <= 64).
extern "C" KS_API int ks_kmeans_mindist(const float* X, int64_t n, int64_t d, const float* c,
                                        int init, double* d2, void* stream) {
  using namespace ks;
  if (!X || !c || !d2 || n < 1 || d < 1) return fail(KS_ERR_ARG, "ks_kmeans_mindist: bad arguments");
  ks_km_mindist_kernel<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      X, n, (int)d, c, init, d2);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

extern "C" KS_API int ks_kmeans_candidates(const float* X, int64_t n, int64_t d, const float* cand,
                                           int64_t T, const double* d2, double* pots,
                                           void* workspace, size_t workspace_bytes, void* stream) {
  using namespace ks;
  if (!X || !cand || !d2 || !pots || n < 1 || d < 1 || T < 1 || T > 64)
    return fail(KS_ERR_ARG, "ks_kmeans_candidates: bad arguments");
  long long per_block;
  const int nb = blocks_for(n, kKmChunk, &per_block);
  if (!workspace || workspace_bytes < 8 * (size_t)nb * T)
    return fail(KS_ERR_WORKSPACE, "ks_kmeans_candidates: workspace too small");
  double* ppot = static_cast<double*>(workspace);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  ks_km_candidates_kernel<<<nb, kKmThreads, 0, s>>>(X, n, (int)d, cand, (int)T, d2, per_block,
                                                    ppot);
  ks_km_pot_reduce_kernel<<<1, 64, 0, s>>>(ppot, nb, (int)T, pots);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}
