// extern "C" entry points declared in include/ks_b200.h.
#include "ks_common.cuh"
#include "project.cuh"

#include <algorithm>
#include <cstdlib>
#include <string>

namespace ks {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return KS_ERR_CUDA;
}

int device_info(DeviceInfo* out) {
  static thread_local DeviceInfo cache[64];
  int dev = 0;
  KS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(KS_ERR_UNSUPPORTED, "device index out of range");
  DeviceInfo& d = cache[dev];
  if (d.device != dev) {
    cudaDeviceProp prop;
    KS_CUDA(cudaGetDeviceProperties(&prop, dev));
    d.sm_count = prop.multiProcessorCount;
    d.cc_major = prop.major;
    d.cc_minor = prop.minor;
    d.smem_optin = prop.sharedMemPerBlockOptin;
    d.device = dev;
  }
  if (d.cc_major != 10)
    return fail(KS_ERR_UNSUPPORTED, "this library is built for sm_100a (B200) only");
  *out = d;
  return KS_OK;
}

// Per host thread: events recorded at the stage boundaries of the calls it
// makes while tracing is on.
struct TraceState {
  bool on = false;
  int device = -1;
  cudaEvent_t ev[kTraceMarks] = {};
};
static thread_local TraceState g_trace;

void trace_mark(int slot, cudaStream_t stream) {
  if (g_trace.on && slot >= 0 && slot < kTraceMarks) cudaEventRecord(g_trace.ev[slot], stream);
}

unsigned long long wait_limit_ns() {
  static unsigned long long v = [] {
    const char* s = std::getenv("KS_B200_WAIT_LIMIT_NS");
    unsigned long long x = s ? std::strtoull(s, nullptr, 10) : 0ull;
    return x ? x : kWaitLimitNs;
  }();
  return v;
}

size_t ctc_workspace_size(int64_t K, int64_t P, int64_t C, int64_t nt);
int launch_ctc(const float* U, const float* W, int64_t K, int64_t P, int64_t C,
               int64_t nt, float* ctc, void* ws, size_t ws_bytes, cudaStream_t stream);
int launch_features(const float* Xres, const int64_t* st, const float* amps,
                    const float* W, const int64_t* iCC, const int64_t* iU,
                    const float* Ucc, int64_t C, int64_t L, int64_t K, int64_t P,
                    int64_t nt, int64_t nC, int64_t N, float* tF, cudaStream_t stream, const int64_t* n_dev = nullptr);
int launch_template_channels(const float* U, const int64_t* iCC, int64_t K,
                             int64_t P, int64_t C, int64_t nC, int64_t* iU,
                             float* Ucc, cudaStream_t stream);

// Workspace of run_matching: nm, tiled B, projection scratch, transposed ctc
// (only when ctc arrives in the reference layout), peel scratch.
struct MatchLayout {
  size_t nm_off, b_off, proj_off, ctc_off, peel_off, bytes;
};

static size_t ctcT_bytes(int64_t K, int64_t nt, int ctc_layout) {
  return ctc_layout == KS_CTC_KJL ? 0 : align256(sizeof(float) * (size_t)K * K * (2 * nt + 1));
}

static MatchLayout match_layout(int64_t C, int64_t L, int64_t K, int64_t P, int64_t nt,
                                int precision, int ctc_layout) {
  MatchLayout m;
  size_t off = 0;
  m.nm_off = off;
  off = align256(off + sizeof(float) * K);
  m.b_off = off;
  off = align256(off + sizeof(float) * (size_t)tiled_rows_floats(L, K));
  m.proj_off = off;
  off = align256(off + proj_layout(C, L, K, P, precision).bytes);
  m.ctc_off = off;
  off += ctcT_bytes(K, nt, ctc_layout);
  m.peel_off = off;
  off = align256(off + peel_scratch_size(L, K, true));
  m.bytes = off;
  return m;
}

// Workspace of the standalone peel: tiled copy of B, transposed ctc, scratch.
struct PeelWsLayout {
  size_t b_off, ctc_off, peel_off, bytes;
};

static PeelWsLayout peel_ws_layout(int64_t L, int64_t K, int64_t nt, int b_layout,
                                   int ctc_layout) {
  PeelWsLayout m;
  size_t off = 0;
  m.b_off = off;
  if (b_layout != KS_B_TILED) off = align256(off + sizeof(float) * (size_t)tiled_rows_floats(L, K));
  m.ctc_off = off;
  off += ctcT_bytes(K, nt, ctc_layout);
  m.peel_off = off;
  off = align256(off + peel_scratch_size(L, K, true));
  m.bytes = off;
  return m;
}

__global__ void ks_wait_never_kernel(unsigned long long limit_ns, int* status,
                                     const int* flag) {
  const unsigned long long t0 = ks_globaltimer();
  int st = KS_OK;
  while (ks_ld_volatile(flag) == 0) {
    __nanosleep(1000);
    if (ks_globaltimer() - t0 > limit_ns) {
      st = KS_ERR_TIMEOUT;
      break;
    }
  }
  *status = st;
}

}  // namespace ks

using namespace ks;

extern "C" {

int ks_version(void) { return 1; }

const char* ks_status_string(int status) {
  switch (status) {
    case KS_OK: return "ok";
    case KS_ERR_ARG: return "invalid argument";
    case KS_ERR_CUDA: return "CUDA error";
    case KS_ERR_OVERFLOW: return "spike buffer overflow";
    case KS_ERR_TIMEOUT: return "device-side wait timed out";
    case KS_ERR_WORKSPACE: return "workspace too small";
    case KS_ERR_UNSUPPORTED: return "unsupported device or shape";
    case KS_ERR_DEGENERATE: return "score plateau beyond the tie buffer";
    default: return "unknown status";
  }
}

const char* ks_last_error(void) { return g_last_error.c_str(); }

int ks_template_energy(const float* U, int64_t K, int64_t P, int64_t C, float* nm,
                       void* stream) {
  return launch_template_energy(U, K, P, C, nm, static_cast<cudaStream_t>(stream));
}

size_t ks_project_workspace_size(int64_t C, int64_t L, int64_t K, int64_t P,
                                 int precision) {
  return proj_layout(C, L, K, P, precision).bytes;
}

int ks_project(const float* X, const float* U, const float* W, int64_t C,
               int64_t L, int64_t K, int64_t P, int64_t nt, int precision,
               float* B, int64_t ldb, int b_layout, int* status, void* workspace,
               size_t workspace_bytes, void* stream) {
  if (!X || !U || !W || !B) return fail(KS_ERR_ARG, "ks_project: null pointer");
  if (b_layout != KS_B_ROWS && b_layout != KS_B_TILED)
    return fail(KS_ERR_ARG, "ks_project: unknown B layout");
  DeviceInfo d;
  int rc = device_info(&d);
  if (rc) return rc;
  return launch_project(X, U, W, C, L, K, P, nt, precision, B, ldb, b_layout == KS_B_TILED,
                        workspace, workspace_bytes, status, static_cast<cudaStream_t>(stream));
}

size_t ks_peel_workspace_size(int64_t L, int64_t K, int64_t nt, int b_layout,
                              int ctc_layout) {
  return peel_ws_layout(L, K, nt, b_layout, ctc_layout).bytes;
}

int ks_peel(float* B, int64_t ldb, int b_layout, float* Xres, const float* U, const float* W,
            const float* ctc, int ctc_layout, const float* nm, int64_t C, int64_t L,
            int64_t K, int64_t P, int64_t nt, float th2, int64_t max_peels,
            int64_t capacity, int64_t* st, float* amps, float* th_amps, int64_t* info,
            void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!B || !ctc) return fail(KS_ERR_ARG, "ks_peel: null pointer");
  if (ctc_layout != KS_CTC_JKL && ctc_layout != KS_CTC_KJL)
    return fail(KS_ERR_ARG, "ks_peel: unknown ctc layout");
  if (b_layout != KS_B_ROWS && b_layout != KS_B_TILED)
    return fail(KS_ERR_ARG, "ks_peel: unknown B layout");
  if (K < 1 || L < 1 || nt < 1) return fail(KS_ERR_ARG, "ks_peel: bad sizes");
  if (b_layout == KS_B_ROWS && ldb < L) return fail(KS_ERR_ARG, "ks_peel: ldb < L");
  const PeelWsLayout m = peel_ws_layout(L, K, nt, b_layout, ctc_layout);
  if (!workspace || workspace_bytes < m.bytes)
    return fail(KS_ERR_WORKSPACE, "ks_peel: workspace too small");
  char* base = static_cast<char*>(workspace);
  float* Bt = b_layout == KS_B_TILED ? B : reinterpret_cast<float*>(base + m.b_off);
  const float* ctcT = ctc;
  int rc;
  if (ctc_layout == KS_CTC_JKL) {
    float* t = reinterpret_cast<float*>(base + m.ctc_off);
    rc = launch_ctc_transpose(ctc, K, nt, t, s);
    if (rc) return rc;
    ctcT = t;
  }
  if (b_layout == KS_B_ROWS) {
    rc = launch_tile_rows(B, ldb, K, L, Bt, s);
    if (rc) return rc;
  }
  rc = launch_peel_tiled(Bt, Xres, U, W, ctcT, nm, C, L, K, P, nt, th2, max_peels, capacity,
                         st, amps, th_amps, info, base + m.peel_off, m.bytes - m.peel_off, s,
                         wait_limit_ns(), nullptr, true);
  if (rc) return rc;
  return b_layout == KS_B_ROWS ? launch_untile_rows(Bt, K, L, B, ldb, s) : KS_OK;
}

size_t ks_run_matching_workspace_size(int64_t C, int64_t L, int64_t K, int64_t P,
                                      int64_t nt, int precision, int ctc_layout) {
  return match_layout(C, L, K, P, nt, precision, ctc_layout).bytes;
}

int ks_run_matching(const float* X, const float* U, const float* W, const float* ctc,
                    int ctc_layout, int64_t C, int64_t L, int64_t K, int64_t P, int64_t nt,
                    float th2, int64_t max_peels, int precision, int64_t capacity,
                    int64_t* st, float* amps, float* th_amps, float* Xres, int64_t* info,
                    void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!X || !Xres || !ctc) return fail(KS_ERR_ARG, "ks_run_matching: null pointer");
  if (C < 1 || L < 1 || K < 1 || P < 1 || nt < 1) return fail(KS_ERR_ARG, "ks_run_matching: bad sizes");
  if (precision != KS_PROJ_FP32 && precision != KS_PROJ_BF16X3)
    return fail(KS_ERR_ARG, "ks_run_matching: unknown precision");
  if (ctc_layout != KS_CTC_JKL && ctc_layout != KS_CTC_KJL)
    return fail(KS_ERR_ARG, "ks_run_matching: unknown ctc layout");
  const MatchLayout m = match_layout(C, L, K, P, nt, precision, ctc_layout);
  if (!workspace || workspace_bytes < m.bytes)
    return fail(KS_ERR_WORKSPACE, "ks_run_matching: workspace too small");
  DeviceInfo d;
  int rc = device_info(&d);
  if (rc) return rc;
  char* base = static_cast<char*>(workspace);
  float* nm = reinterpret_cast<float*>(base + m.nm_off);
  float* Bt = reinterpret_cast<float*>(base + m.b_off);
  const float* ctcT = ctc;
  if (ctc_layout == KS_CTC_JKL) {
    float* t = reinterpret_cast<float*>(base + m.ctc_off);
    rc = launch_ctc_transpose(ctc, K, nt, t, s);
    if (rc) return rc;
    ctcT = t;
  }
  trace_mark(0, s);
  if (Xres != X)
    KS_CUDA(cudaMemcpyAsync(Xres, X, sizeof(float) * C * L, cudaMemcpyDeviceToDevice, s));
  rc = launch_template_energy(U, K, P, C, nm, s);
  if (rc) return rc;
  trace_mark(1, s);
  rc = launch_project(X, U, W, C, L, K, P, nt, precision, Bt, 0, true, base + m.proj_off,
                      m.ctc_off - m.proj_off, nullptr, s);
  if (rc) return rc;
  // the projection's error word is the first int of its workspace
  return launch_peel_tiled(Bt, Xres, U, W, ctcT, nm, C, L, K, P, nt, th2, max_peels,
                           capacity, st, amps, th_amps, info, base + m.peel_off,
                           m.bytes - m.peel_off, s, wait_limit_ns(),
                           reinterpret_cast<const int*>(base + m.proj_off), true);
}

int ks_ctc_transpose(const float* ctc, int64_t K, int64_t nt, float* ctcT, void* stream) {
  return launch_ctc_transpose(ctc, K, nt, ctcT, static_cast<cudaStream_t>(stream));
}

int ks_features(const float* Xres, const int64_t* st, const float* amps,
                const float* W, const int64_t* iCC, const int64_t* iU,
                const float* Ucc, int64_t C, int64_t L, int64_t K, int64_t P,
                int64_t nt, int64_t nC, int64_t n_spikes, float* tF, void* stream) {
  return launch_features(Xres, st, amps, W, iCC, iU, Ucc, C, L, K, P, nt, nC, n_spikes,
                         tF, static_cast<cudaStream_t>(stream));
}

int ks_features_counted(const float* Xres, const int64_t* st, const float* amps,
                        const float* W, const int64_t* iCC, const int64_t* iU,
                        const float* Ucc, int64_t C, int64_t L, int64_t K, int64_t P,
                        int64_t nt, int64_t nC, const int64_t* n_spikes_dev,
                        int64_t max_spikes, float* tF, void* stream) {
  if (!n_spikes_dev) return fail(KS_ERR_ARG, "ks_features_counted: null count");
  return launch_features(Xres, st, amps, W, iCC, iU, Ucc, C, L, K, P, nt, nC, max_spikes,
                         tF, static_cast<cudaStream_t>(stream), n_spikes_dev);
}

int ks_template_channels(const float* U, const int64_t* iCC, int64_t K, int64_t P,
                         int64_t C, int64_t nC, int64_t* iU, float* Ucc,
                         void* stream) {
  return launch_template_channels(U, iCC, K, P, C, nC, iU, Ucc,
                                  static_cast<cudaStream_t>(stream));
}

size_t ks_ctc_workspace_size(int64_t K, int64_t P, int64_t C, int64_t nt) {
  return ctc_workspace_size(K, P, C, nt);
}

int ks_ctc(const float* U, const float* W, int64_t K, int64_t P, int64_t C,
           int64_t nt, float* ctc, void* workspace, size_t workspace_bytes,
           void* stream) {
  return launch_ctc(U, W, K, P, C, nt, ctc, workspace, workspace_bytes,
                    static_cast<cudaStream_t>(stream));
}

int ks_trace_stages(int enable) {
  if (!enable) {
    g_trace.on = false;
    return KS_OK;
  }
  DeviceInfo d;
  int rc = device_info(&d);
  if (rc) return rc;
  if (g_trace.device != d.device) {
    for (int i = 0; i < kTraceMarks; ++i)
      if (g_trace.ev[i]) cudaEventDestroy(g_trace.ev[i]);
    for (int i = 0; i < kTraceMarks; ++i) KS_CUDA(cudaEventCreate(&g_trace.ev[i]));
    g_trace.device = d.device;
  }
  g_trace.on = true;
  return KS_OK;
}

int ks_trace_read(float* ms, int n) {
  if (!ms || n < 1 || n > kTraceMarks - 1) return fail(KS_ERR_ARG, "ks_trace_read: 1..4 intervals");
  if (g_trace.device < 0) return fail(KS_ERR_ARG, "ks_trace_read: tracing was never enabled");
  KS_CUDA(cudaEventSynchronize(g_trace.ev[n]));
  for (int i = 0; i < n; ++i) KS_CUDA(cudaEventElapsedTime(&ms[i], g_trace.ev[i], g_trace.ev[i + 1]));
  return KS_OK;
}

int ks_selftest_wait(int64_t timeout_ns, int* status, void* stream) {
  if (!status || timeout_ns <= 0 || timeout_ns > 10000000000LL)
    return fail(KS_ERR_ARG, "ks_selftest_wait: need 0 < timeout_ns <= 1e10 and a status pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the flag lives in the status word's neighbour: status[1] is cleared and
  // never set, so the wait can only end through its limit
  KS_CUDA(cudaMemsetAsync(status, 0, 2 * sizeof(int), s));
  ks_wait_never_kernel<<<1, 1, 0, s>>>((unsigned long long)timeout_ns, status, status + 1);
  KS_CUDA(cudaGetLastError());
  return KS_OK;
}

}  // extern "C"
