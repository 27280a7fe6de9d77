// The parts of the Phy export (kilosort/io.py:248-470, save_to_phy) that the
// matching path produces: duplicate-spike removal and the template
// waveforms.  (Spike positions and amplitudes are in postprocess.cu.)
//
// ks_remove_duplicates -- kilosort/postprocessing.py:10-30.  Spikes are taken
// in index order; a spike is kept when its time is at least dt after the
// last kept spike of the same cluster (the first spike of a cluster is
// always kept).  On the device: the spike indices are grouped by cluster with
// a stable radix sort of (cluster, index) pairs (CUB), so each cluster's
// spikes form one run in index order, and one thread walks each run applying
// that rule.  The result is the reference's keep mask exactly, for any order
// of the input times.
//
// ks_phy_templates -- kilosort/io.py:383-385: the waveform of each cluster
// from its PC loadings, templates[k, t, c] = sum_p Wall[k, c, p] * W[p, t]
// (products rounded, then summed over p in order), written in Phy's
// [K, nt, C] layout.
#include "ks_common.cuh"

#include <cub/device/device_radix_sort.cuh>

namespace {

__global__ void ks_dup_prepare_kernel(const int32_t* __restrict__ clusters, int N,
                                      int32_t* __restrict__ keys, int32_t* __restrict__ idx) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    keys[i] = clusters[i];
    idx[i] = i;
  }
}

// One thread per run of equal clusters in the sorted order: the run's spikes
// in index order, the greedy rule of the reference.
__global__ void ks_dup_scan_kernel(const int32_t* __restrict__ keys,
                                   const int32_t* __restrict__ idx,
                                   const int64_t* __restrict__ times, int N, int64_t dt,
                                   uint8_t* __restrict__ keep) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    if (i > 0 && keys[i - 1] == keys[i]) continue;     // not the start of a run
    const int32_t c = keys[i];
    int64_t t0 = 0;
    bool first = true;
    for (int j = i; j < N && keys[j] == c; ++j) {
      const int s = idx[j];
      const int64_t t = times[s];
      if (first) {
        t0 = t - dt;
        first = false;
      }
      if (t >= t0 + dt) {
        t0 = t;
        keep[s] = 1;
      } else {
        keep[s] = 0;
      }
    }
  }
}

__global__ void ks_phy_templates_kernel(const float* __restrict__ Wall,
                                        const float* __restrict__ W, int K, int C, int P,
                                        int nt, float* __restrict__ templates) {
  const long long n = (long long)K * nt * C;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % C);
    const long long kt = e / C;
    const int t = (int)(kt % nt);
    const int k = (int)(kt / nt);
    const float* wk = Wall + ((size_t)k * C + c) * P;
    float acc = __fmul_rn(wk[0], W[t]);
    for (int p = 1; p < P; ++p) acc = __fadd_rn(acc, __fmul_rn(wk[p], W[(size_t)p * nt + t]));
    templates[e] = acc;
  }
}

// Workspace: [keys in] [idx in] [keys out] [idx out] [CUB temp].
struct DupLayout {
  size_t keys_in, idx_in, keys_out, idx_out, temp, temp_bytes, bytes;
};

int dup_layout(int64_t N, DupLayout* d) {
  size_t temp_bytes = 0;
  const cudaError_t e = cub::DeviceRadixSort::SortPairs(
      nullptr, temp_bytes, static_cast<const int32_t*>(nullptr), static_cast<int32_t*>(nullptr),
      static_cast<const int32_t*>(nullptr), static_cast<int32_t*>(nullptr), (int)N);
  if (e != cudaSuccess) return ks::cuda_fail(e, "cub::DeviceRadixSort::SortPairs (size query)");
  size_t o = 0;
  auto take = [&](size_t b) {
    const size_t at = o;
    o = ks::align256(o + b);
    return at;
  };
  d->keys_in = take(4 * (size_t)N);
  d->idx_in = take(4 * (size_t)N);
  d->keys_out = take(4 * (size_t)N);
  d->idx_out = take(4 * (size_t)N);
  d->temp = take(temp_bytes);
  d->temp_bytes = temp_bytes;
  d->bytes = o;
  return KS_OK;
}

}  // namespace

extern "C" KS_API size_t ks_remove_duplicates_workspace_size(int64_t N) {
  if (N < 0 || N >= (1LL << 31)) return 0;
  DupLayout d;
  if (dup_layout(N, &d)) return 0;
  return d.bytes;
}

extern "C" KS_API int ks_remove_duplicates(const int64_t* spike_times,
                                           const int32_t* spike_clusters, int64_t N,
                                           int64_t dt, uint8_t* keep, void* workspace,
                                           size_t workspace_bytes, void* stream) {
  using namespace ks;
  if (N < 0) return fail(KS_ERR_ARG, "ks_remove_duplicates: negative N");
  if (N >= (1LL << 31)) return fail(KS_ERR_UNSUPPORTED, "ks_remove_duplicates: too many spikes");
  if (N == 0) return KS_OK;
  if (!spike_times || !spike_clusters || !keep)
    return fail(KS_ERR_ARG, "ks_remove_duplicates: null pointer");
  DupLayout d;
  int rc = dup_layout(N, &d);
  if (rc) return rc;
  if (!workspace || workspace_bytes < d.bytes)
    return fail(KS_ERR_WORKSPACE, "ks_remove_duplicates: workspace too small");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  char* base = static_cast<char*>(workspace);
  int32_t* keys_in = reinterpret_cast<int32_t*>(base + d.keys_in);
  int32_t* idx_in = reinterpret_cast<int32_t*>(base + d.idx_in);
  int32_t* keys_out = reinterpret_cast<int32_t*>(base + d.keys_out);
  int32_t* idx_out = reinterpret_cast<int32_t*>(base + d.idx_out);
  const unsigned grid = (unsigned)std::min<int64_t>((N + 255) / 256, 4096);
  ks_dup_prepare_kernel<<<grid, 256, 0, s>>>(spike_clusters, (int)N, keys_in, idx_in);
  KS_CUDA(cudaGetLastError());
  size_t temp_bytes = d.temp_bytes;
  KS_CUDA(cub::DeviceRadixSort::SortPairs(base + d.temp, temp_bytes, keys_in, keys_out, idx_in,
                                          idx_out, (int)N, 0, 32, s));
  ks_dup_scan_kernel<<<grid, 256, 0, s>>>(keys_out, idx_out, spike_times, (int)N, dt, keep);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

extern "C" KS_API int ks_phy_templates(const float* Wall, const float* W, int64_t K, int64_t C,
                                       int64_t P, int64_t nt, float* templates, void* stream) {
  using namespace ks;
  if (K < 0 || C < 1 || P < 1 || nt < 1)
    return fail(KS_ERR_ARG, "ks_phy_templates: need K >= 0 and C, P, nt >= 1");
  if (K == 0) return KS_OK;
  if (!Wall || !W || !templates) return fail(KS_ERR_ARG, "ks_phy_templates: null pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long n = K * nt * C;
  const unsigned grid = (unsigned)std::min<long long>((n + 255) / 256, 65535);
  ks_phy_templates_kernel<<<grid, 256, 0, s>>>(Wall, W, (int)K, (int)C, (int)P, (int)nt,
                                               templates);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}
