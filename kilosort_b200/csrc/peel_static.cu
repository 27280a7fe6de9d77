// ks_peel_static: the greedy peel without a caller-supplied workspace.
//
// Some callers cannot allocate device memory when they match a batch: an
// acquisition loop that must not call cudaMalloc on its hot path (the call
// can synchronise the whole device and has no latency bound), or a host
// plugin that receives device buffers from its host application but owns no
// device allocator of its own.  They hand over inputs and outputs only; the
// peel's scratch lives in a fixed array of this library's device image.
//
// The array below is a file-scope __device__ object of kPeelStaticBytes
// bytes (7 MiB); every GPU that loads the library holds one copy until the
// process exits.  It holds the scratch of batches of up to
// KS_PEEL_STATIC_MAX_L padded samples with up to KS_PEEL_STATIC_MAX_K
// templates (shorter batches leave room for more templates); any shape whose
// scratch does not fit is rejected with KS_ERR_UNSUPPORTED and a message.
// This entry point runs the peel's ungrouped update, whose scratch does not
// grow with the number of templates times the batch length.
//
// In host code the name of the array only stands for the device object; the
// kernel needs its device address, which cudaGetSymbolAddress returns.  A
// call on a stream that is not being captured looks the address up again
// with the device current (so a device whose context was reset gets the
// address of its new image) and caches it; a call inside a stream capture
// uses the cached address, so the first call on each device must come
// before any capture.
//
// All calls share the array and it keeps the previous call's contents.  The
// parts that must start at zero (barrier, counters, registration lists and
// rescoring slots) are cleared by every call; calls whose kernels overlap on
// the GPU (different streams, or several host threads) race on the array and
// must be serialised by the caller.
#include "ks_common.cuh"
#include "project.cuh"

#include <mutex>

namespace {

constexpr size_t kPeelStaticBytes = 7u << 20;

static __device__ __align__(256) unsigned char g_peel_scratch[kPeelStaticBytes];

struct StaticScratch {
  std::mutex mu;
  void* addr[64] = {};
};

StaticScratch& static_scratch() {
  static StaticScratch s;
  return s;
}

// Device address of the array on the current device: looked up again when
// the stream is not capturing, the cached value inside a capture.
int scratch_address(int device, cudaStream_t stream, void** out) {
  if (device < 0 || device >= 64) return ks::fail(KS_ERR_UNSUPPORTED, "ks_peel_static: device index out of range");
  StaticScratch& s = static_scratch();
  std::lock_guard<std::mutex> lock(s.mu);
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess) {
    (void)cudaGetLastError();
    cs = cudaStreamCaptureStatusActive;   // unknown: do not call into the runtime
  }
  if (cs == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_peel_scratch);
    if (e != cudaSuccess) return ks::cuda_fail(e, "cudaGetSymbolAddress(g_peel_scratch)");
    s.addr[device] = p;
  } else if (!s.addr[device]) {
    return ks::fail(KS_ERR_UNSUPPORTED,
                    "ks_peel_static: the first call on a device must come before any stream capture");
  }
  *out = s.addr[device];
  return KS_OK;
}

}  // namespace

extern "C" KS_API int ks_peel_static(float* Bt, float* Xres, const float* U, const float* W,
                                     const float* ctcT, const float* nm, int64_t C, int64_t L,
                                     int64_t K, int64_t P, int64_t nt, float th2,
                                     int64_t max_peels, int64_t capacity, int64_t* st,
                                     float* amps, float* th_amps, int64_t* info, void* stream) {
  using namespace ks;
  if (L < 1 || L > KS_PEEL_STATIC_MAX_L)
    return fail(KS_ERR_UNSUPPORTED,
                "ks_peel_static: batch length must be 1.." + std::to_string(KS_PEEL_STATIC_MAX_L) +
                    " padded samples (the fixed scratch array is sized for that)");
  const size_t need = peel_scratch_size(L, K, false);
  if (need > kPeelStaticBytes)
    return fail(KS_ERR_UNSUPPORTED,
                "ks_peel_static: the scratch of L=" + std::to_string(L) + ", K=" + std::to_string(K) +
                    " exceeds the fixed array (" + std::to_string(KS_PEEL_STATIC_MAX_L) +
                    " samples hold up to " + std::to_string(KS_PEEL_STATIC_MAX_K) + " templates)");
  DeviceInfo dev;
  int rc = device_info(&dev);
  if (rc) return rc;
  void* ws = nullptr;
  rc = scratch_address(dev.device, static_cast<cudaStream_t>(stream), &ws);
  if (rc) return rc;
  return launch_peel_tiled(Bt, Xres, U, W, ctcT, nm, C, L, K, P, nt, th2, max_peels, capacity, st,
                           amps, th_amps, info, ws, kPeelStaticBytes,
                           static_cast<cudaStream_t>(stream), wait_limit_ns(), nullptr, false);
}
