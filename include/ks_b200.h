/*
 * ks_b200.h -- C ABI of the B200-native Kilosort4 template-matching path.
 *
 * Every entry point takes raw device pointers (row-major, contiguous unless a
 * leading dimension is given), int64 sizes, a CUDA stream (cudaStream_t passed
 * as void*) and, where scratch is needed, a caller-owned device workspace whose
 * size is returned by the matching *_workspace_size() query.  The library never
 * allocates device memory and never synchronises the stream, except where a
 * function says so.  Return value: 0 (KS_OK) or a KS_ERR_* code; a readable
 * message for the last failure on the calling thread is in ks_last_error().
 *
 * Device-side outcomes of the greedy peel (spike count, iterations, overflow,
 * watchdog) are written to a caller-provided int64 "info" array on the device:
 *   info[0] = spikes written, info[1] = status (KS_OK or KS_ERR_*),
 *   info[2] = iterations run, info[3] = spikes the batch needed (when it
 *   overflowed the capacity).
 *
 * Shapes use the reference's names: C = n channels, L = padded batch length
 * (NT + 2*nt), K = n templates, P = n_pcs, nt = template length (odd).
 */
#ifndef KS_B200_H
#define KS_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define KS_API __attribute__((visibility("default")))
#else
#define KS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define KS_OK 0
#define KS_ERR_ARG 1          /* invalid argument (size, alignment, null) */
#define KS_ERR_CUDA 2         /* a CUDA runtime call failed */
#define KS_ERR_OVERFLOW 3     /* more spikes than the output capacity */
#define KS_ERR_TIMEOUT 4      /* a bounded device-side wait ran out */
#define KS_ERR_WORKSPACE 5    /* workspace smaller than *_workspace_size() */
#define KS_ERR_UNSUPPORTED 6  /* device or shape not supported by this library */
#define KS_ERR_DEGENERATE 7   /* exact score plateaus beyond the tie buffer */

/* layout of the score matrix B */
#define KS_B_ROWS 0           /* B[k][tau] row-major with leading dimension ldb */
#define KS_B_TILED 1          /* Bt[tau/32][k][tau%32]: 32-column blocks, ceil(L/32)*K*32 floats */

/* layout of the template cross-correlations */
#define KS_CTC_JKL 0          /* ctc[j][k][lag], as prepare_matching returns it */
#define KS_CTC_KJL 1          /* ctcT[k][j][lag] = ctc[j][k][lag] (ks_ctc_transpose) */

/* projection precision */
#define KS_PROJ_FP32 0        /* plain FP32 (SIMT) contraction */
#define KS_PROJ_BF16X3 1      /* split-BF16 hi/lo, three tcgen05 MMAs, FP32 accumulate */

KS_API int ks_version(void);
KS_API const char* ks_status_string(int status);
KS_API const char* ks_last_error(void);

/*
 * Template energy, nm[k] = sum_{p,c} U[k,p,c]^2.
 * Replaces kilosort/template_matching.py:176.
 */
KS_API int ks_template_energy(const float* U, int64_t K, int64_t P, int64_t C,
                       float* nm, void* stream);

/*
 * Score matrix B[k, tau] = sum_{p,c} U[k,p,c] * sum_t W[p,t] X[c, tau - nt/2 + t]
 * (zero padding), written in b_layout (row-major with ldb >= L, or tiled).
 * status (device int, may be NULL) receives KS_OK or the device-side error of
 * the contraction (KS_ERR_TIMEOUT if a bounded wait ran out; B is then
 * undefined).
 * Replaces kilosort/template_matching.py:180-181 (conv1d + einsum).
 */
KS_API size_t ks_project_workspace_size(int64_t C, int64_t L, int64_t K, int64_t P,
                                 int precision);
KS_API int ks_project(const float* X, const float* U, const float* W,
               int64_t C, int64_t L, int64_t K, int64_t P, int64_t nt,
               int precision, float* B, int64_t ldb, int b_layout, int* status,
               void* workspace, size_t workspace_bytes, void* stream);

/*
 * Greedy peel on a score matrix (B in b_layout, modified in place) and a residual
 * (Xres [C, L], modified in place): up to max_peels iterations of detect /
 * record / subtract.  Outputs st [capacity, 2] int64 (tau, template),
 * amps [capacity], th_amps [capacity] float32, in the reference's order
 * (iteration, then tau).  th2 = Th_learned^2 rounded to float32.  ctc is in
 * the layout ctc_layout names; with KS_CTC_JKL a transposed copy is made in
 * the workspace on every call, and a row-major B is tiled into the workspace
 * and written back at the end.
 * Replaces kilosort/template_matching.py:183-244.
 */
KS_API size_t ks_peel_workspace_size(int64_t L, int64_t K, int64_t nt, int b_layout,
                                     int ctc_layout);
KS_API int ks_peel(float* B, int64_t ldb, int b_layout, float* Xres, const float* U, const float* W,
            const float* ctc, int ctc_layout, const float* nm,
            int64_t C, int64_t L, int64_t K, int64_t P, int64_t nt,
            float th2, int64_t max_peels, int64_t capacity,
            int64_t* st, float* amps, float* th_amps, int64_t* info,
            void* workspace, size_t workspace_bytes, void* stream);

/*
 * Whole per-batch matching: Xres <- X, nm, scores, peel.  Callers that match
 * many batches with one ctc pass it transposed once (KS_CTC_KJL).
 * Replaces kilosort/template_matching.py:170-244 (run_matching).
 */
KS_API size_t ks_run_matching_workspace_size(int64_t C, int64_t L, int64_t K,
                                      int64_t P, int64_t nt, int precision,
                                      int ctc_layout);
KS_API int ks_run_matching(const float* X, const float* U, const float* W,
                    const float* ctc, int ctc_layout, int64_t C, int64_t L,
                    int64_t K, int64_t P, int64_t nt, float th2,
                    int64_t max_peels, int precision, int64_t capacity,
                    int64_t* st, float* amps, float* th_amps, float* Xres,
                    int64_t* info, void* workspace, size_t workspace_bytes,
                    void* stream);

/*
 * ctcT[k][j][lag] = ctc[j][k][lag] (not in place).  The layout the peel
 * streams: a peak of template k subtracts one contiguous slab.
 * Helper of kilosort/template_matching.py:238 (reads ctc[:, k, :]).
 */
KS_API int ks_ctc_transpose(const float* ctc, int64_t K, int64_t nt, float* ctcT,
                            void* stream);

/*
 * Per-spike PC features: tF[s, i, p] = sum_t Xres[iCC[i, iU[k_s]], tau_s - nt/2 + t]
 * * W[p, t] + amps[s] * Ucc[i, k_s, p], for s < n_spikes (st/amps as written
 * by ks_peel).  tF is [n_spikes, nC, P].
 * Replaces kilosort/template_matching.py:85-86 (with the transpose at :108).
 */
KS_API int ks_features(const float* Xres, const int64_t* st, const float* amps,
                const float* W, const int64_t* iCC, const int64_t* iU,
                const float* Ucc, int64_t C, int64_t L, int64_t K, int64_t P,
                int64_t nt, int64_t nC, int64_t n_spikes, float* tF,
                void* stream);

/*
 * ks_features for the first min(max_spikes, *n_spikes_dev) spikes, the count
 * read on the device (an int64 a peel wrote, e.g. word 0 of its info), so the
 * features can be enqueued behind the peel without reading the count back.
 * tF holds max_spikes rows; rows past the count are left as they are.
 * Replaces kilosort/template_matching.py:85-86 like ks_features.
 */
KS_API int ks_features_counted(const float* Xres, const int64_t* st, const float* amps,
                               const float* W, const int64_t* iCC, const int64_t* iU,
                               const float* Ucc, int64_t C, int64_t L, int64_t K, int64_t P,
                               int64_t nt, int64_t nC, const int64_t* n_spikes_dev,
                               int64_t max_spikes, float* tF, void* stream);

/*
 * Per-template peak channel and feature loadings: iU[k] = argmax_c
 * sum_p U[k,p,c]^2 (first index on ties), Ucc[i,k,p] = U[k,p,iCC[i,iU[k]]].
 * Replaces the device part of kilosort/template_matching.py:50-51.
 */
KS_API int ks_template_channels(const float* U, const int64_t* iCC, int64_t K,
                         int64_t P, int64_t C, int64_t nC, int64_t* iU,
                         float* Ucc, void* stream);

/*
 * Template cross-correlations ctc [K, K, 2*nt+1].
 * Replaces kilosort/template_matching.py:155-167 (prepare_matching).
 */
KS_API size_t ks_ctc_workspace_size(int64_t K, int64_t P, int64_t C, int64_t nt);
KS_API int ks_ctc(const float* U, const float* W, int64_t K, int64_t P, int64_t C,
           int64_t nt, float* ctc, void* workspace, size_t workspace_bytes,
           void* stream);

/*
 * Greedy peel for callers that cannot allocate device memory while they match
 * a batch, for instance an acquisition loop that must not call cudaMalloc on
 * its hot path (it can synchronise the device and has no latency bound), or a
 * host plugin that is handed device buffers but owns no device allocator.
 * Same outputs as ks_peel with a tiled score matrix (KS_B_TILED) and
 * transposed cross-correlations (KS_CTC_KJL); instead of a workspace it uses
 * a fixed 7 MiB array in the library's device image (one per GPU that loads
 * the library, held until the process exits).  The array holds batches of up
 * to KS_PEEL_STATIC_MAX_L padded samples with up to KS_PEEL_STATIC_MAX_K
 * templates (shorter batches leave room for more); a shape whose scratch does
 * not fit returns KS_ERR_UNSUPPORTED with a message naming both limits.  A
 * call on a stream that is not capturing looks the array's device address up
 * (and caches it); inside a stream capture the cached address is used, so make
 * the first call on a device before any capture.  Every call shares the array
 * (it keeps the last call's contents; what must start at zero is cleared per
 * call), so calls whose kernels overlap on the GPU race and must be
 * serialised by the caller.  No counterpart in the reference.
 */
#define KS_PEEL_STATIC_MAX_L 131072
#define KS_PEEL_STATIC_MAX_K 56896
KS_API int ks_peel_static(float* Bt, float* Xres, const float* U, const float* W,
                          const float* ctcT, const float* nm, int64_t C, int64_t L,
                          int64_t K, int64_t P, int64_t nt, float th2,
                          int64_t max_peels, int64_t capacity, int64_t* st,
                          float* amps, float* th_amps, int64_t* info, void* stream);

/*
 * Many batches of several recordings in a few launches.
 * Replaces the per-batch loop of kilosort/template_matching.py:79-84
 * (extract: padded_batch_to_torch, then run_matching per batch), for up to
 * KS_MAX_BATCHES batches of up to KS_MAX_RECORDINGS recordings (template sets)
 * per call; batch lengths may differ.  Each batch gets exactly the outputs
 * ks_run_matching gives it (st, amps, th_amps, Xres, info), computed in this
 * order on the stream: per recording the template energies and the reordered
 * templates; per batch Xres = X and the temporal projection; the score
 * contraction of every batch (split-BF16: one grouped tensor-core launch;
 * FP32: one launch per batch); one cooperative peel launch whose grid is split
 * into `teams` groups of co-resident blocks, each peeling its share of the
 * batches (longest first) and then applying that batch's residual, with no
 * host round trip.  teams <= 0 picks a default.  With an aux_stream other
 * than stream and groups > 1 the batches (longest first) are split into
 * `groups` consecutive groups: the projections of group g+1 run on
 * aux_stream while group g is peeled on stream (the peel then runs one block
 * per SM, leaving room for the projection kernels); stream waits for
 * aux_stream before returning control of the work to the caller's later
 * launches.  info[1] of a batch that no team reached (after an error) stays
 * -1.  Nothing is copied from host memory and the host is not synchronised,
 * so the call can be captured in a CUDA graph (the descriptors are read at
 * call time).  ctcT is the transposed layout (KS_CTC_KJL).  Xres may equal X
 * (in place); otherwise they must not overlap.
 */
#define KS_MAX_BATCHES 256
#define KS_MAX_RECORDINGS 8
typedef struct ks_rec_desc {
  const float* U;          /* [K, P, C] */
  const float* W;          /* [P, nt]   wPCA */
  const float* ctcT;       /* [K, K, 2*nt+1] transposed cross-correlations */
  int64_t C, K, P, nt;
  float th2;               /* float(Th_learned**2) */
  int64_t max_peels;
  int64_t capacity;        /* spike rows of each batch's outputs */
} ks_rec_desc;
typedef struct ks_batch_desc {
  const float* X;          /* [C, L] */
  float* Xres;             /* [C, L] */
  int64_t L;
  int64_t rec;             /* index into the recording descriptors */
  int64_t* st;             /* [capacity, 2] */
  float* amps;             /* [capacity] */
  float* th_amps;          /* [capacity] */
  int64_t* info;           /* [4] */
} ks_batch_desc;
KS_API size_t ks_match_batches_workspace_size(const ks_rec_desc* recs, int64_t n_recs,
                                              const ks_batch_desc* batches,
                                              int64_t n_batches, int precision,
                                              int64_t teams);
KS_API int ks_match_batches(const ks_rec_desc* recs, int64_t n_recs,
                            const ks_batch_desc* batches, int64_t n_batches,
                            int precision, int64_t teams, int64_t groups,
                            void* workspace, size_t workspace_bytes, void* stream,
                            void* aux_stream);

/*
 * Fixed-assignment reconstruction loss and its adjoint, for template
 * refinement.  For spikes s = (tau_s = st[s][0], k_s = st[s][1]) with
 * amplitudes amps[s]:
 *   R[c, tau] = sum_s amps[s] * sum_p U[k_s,p,c] W[p, tau - tau_s + nt/2]
 * (the subtraction of kilosort/template_matching.py:237 applied to a fixed
 * spike set; window taps outside [0, L) are dropped), Xres = X - R and
 * loss = sum (X - R)^2, written to *loss (device double).  ks_recon_adjoint
 * takes that Xres and the upstream gradient dloss (device float) and writes
 * dU [K,P,C], dW [P,nt] and damps [n_spikes] of dloss * loss; it recomputes
 * the template waveforms U x W per block instead of storing them.  Both are
 * deterministic (fixed summation orders).  A spike with tau outside [0, L) or
 * a template outside [0, K) sets *status (device int) to KS_ERR_ARG and is
 * skipped.  No counterpart in the reference (it has no gradient of the
 * matching); the forward reproduces its residual subtraction.
 */
KS_API size_t ks_recon_workspace_size(int64_t C, int64_t L, int64_t K, int64_t P,
                                      int64_t nt, int64_t n_spikes);
KS_API int ks_recon_loss(const float* X, const int64_t* st, const float* amps,
                         int64_t n_spikes, const float* U, const float* W, int64_t C,
                         int64_t L, int64_t K, int64_t P, int64_t nt, float* Xres,
                         double* loss, int* status, void* workspace,
                         size_t workspace_bytes, void* stream);
KS_API int ks_recon_adjoint(const float* Xres, const int64_t* st, const float* amps,
                            int64_t n_spikes, const float* U, const float* W, int64_t C,
                            int64_t L, int64_t K, int64_t P, int64_t nt,
                            const float* dloss, float* dU, float* dW, float* damps,
                            int* status, void* workspace, size_t workspace_bytes,
                            void* stream);

/*
 * Universal-template spike detection on one batch X [C, L] (whitened, padded):
 *   B = conv1d(X, wTEMP [nk, nt]) (padding nt/2), for each template position
 *   f < Nfilt and sample t the weighted sums A[s, k] = sum_j weigh[s, j, f] *
 *   B[iC[j, f], k, t] (iC [nC, Nfilt] int64, weigh [nsizes, nC, Nfilt]), the
 *   largest |A| with its signed index (1 + s*nk + k) * sign, the maximum of
 *   that over the nC2 nearest positions iC2 [nC2, Nfilt] (zero for t < nt and
 *   t >= L - nt), a (2*nt0+1) max-pool in time, peaks above th.  Outputs in
 *   (position, time) order, at most `capacity`: xy [cap, 2] (f, t), imax [cap]
 *   (s*nk + k), amp [cap], adist [nC, cap], yct [cap] (yc [C] f32), tF
 *   [cap, nC, P] (wPCA [P, nt]).  info (device int64[4]): [0] spikes written,
 *   [1] KS_OK / KS_ERR_OVERFLOW / KS_ERR_ARG (a channel index outside [0, C)),
 *   [3] spikes found.  nk, nsizes <= 8, nC <= 32, P <= 8.
 *   Replaces kilosort/spikedetect.py:133-197 (template_match, yweighted) and
 *   the features of run() (:265-266).
 */
KS_API size_t ks_detect_workspace_size(int64_t C, int64_t L, int64_t nk, int64_t Nfilt);
KS_API int ks_detect(const float* X, int64_t C, int64_t L, const float* wTEMP, int64_t nk,
                     int64_t nt, const int64_t* iC, int64_t nC, const int64_t* iC2,
                     int64_t nC2, const float* weigh, int64_t nsizes, int64_t Nfilt,
                     int64_t nt0, float th, const float* wPCA, int64_t P, const float* yc,
                     int64_t capacity, int64_t* xy, int64_t* imax, float* amp, float* adist,
                     float* yct, float* tF, int64_t* info, void* workspace,
                     size_t workspace_bytes, void* stream);

/*
 * Universal templates learned from data (templates_from_data).
 * ks_snippets: on one padded batch X [C, L], the isolated single-channel
 * peaks -- |X[c,t]| the maximum of |X| over channels c-4..c+4 and samples
 * t-5..t+5 and above th, alone among the peaks of channels c-6..c+6 and
 * samples t-30..t+30 (the reference's float32 mean-pool test), nt or more
 * samples from both edges -- in (channel, sample) order, and their snippets
 * clips[base + i, j] = X[c, t - twav_min + j] (j < nt) for base + i <
 * capacity; count (device int32) receives the batch's number of peaks.
 * Replaces kilosort/spikedetect.py:33-48 (extract_snippets).
 * ks_snippet_gram: scales each of the n snippets [n, nt] to unit norm in
 * place and writes G = sum_i x_i x_i^T [nt, nt] (double; nt <= 64), whose
 * leading eigenvectors are the truncated-SVD basis of the snippets.
 * Replaces the data side of kilosort/spikedetect.py:70-73 (TruncatedSVD).
 * ks_kmeans_step / ks_kmeans_mindist / ks_kmeans_candidates: one Lloyd step
 * (labels int32 [n] in/out, -1 before the first step; sums [k, d] double,
 * counts [k] int64, stats {inertia, changed labels} double), and the distance
 * and candidate-potential steps of k-means++ seeding, over X [n, d] f32
 * (d, k <= 64).  Replace the data side of kilosort/spikedetect.py:78-85
 * (KMeans).
 */
KS_API size_t ks_snippets_workspace_size(int64_t C, int64_t L);
KS_API int ks_snippets(const float* X, int64_t C, int64_t L, int64_t nt, int64_t twav_min,
                       float th, int64_t base, int64_t capacity, float* clips, int32_t* count,
                       void* workspace, size_t workspace_bytes, void* stream);
KS_API size_t ks_snippet_gram_workspace_size(int64_t n, int64_t nt);
KS_API int ks_snippet_gram(float* clips, int64_t n, int64_t nt, double* G, void* workspace,
                           size_t workspace_bytes, void* stream);
KS_API size_t ks_kmeans_workspace_size(int64_t n, int64_t d, int64_t k);
KS_API int ks_kmeans_step(const float* X, int64_t n, int64_t d, const float* centers, int64_t k,
                          int32_t* labels, double* sums, int64_t* counts, double* stats,
                          void* workspace, size_t workspace_bytes, void* stream);
KS_API int ks_kmeans_mindist(const float* X, int64_t n, int64_t d, const float* c, int init,
                             double* d2, void* stream);
KS_API int ks_kmeans_candidates(const float* X, int64_t n, int64_t d, const float* cand,
                                int64_t T, const double* d2, double* pots, void* workspace,
                                size_t workspace_bytes, void* stream);

/*
 * Template similarity, sim[i, j] = max over lags l of
 *   sum_{k,m} (sum_c Wn[i,c,k] Wn[j,c,m]) * WtW[k,m,l],  Wn = Wall / (1e-6 + ||Wall||),
 * with WtW the flipped full cross-correlation of the wPCA rows (as ks_ctc).
 * Wall [K, C, P] (the clustering's layout), W [P, nt], sim [K, K], all f32.
 * Replaces kilosort/CCG.py:94-102 (similarity, used for Phy's
 * similar_templates at kilosort/io.py:377); the lags are never stored.
 */
KS_API size_t ks_similarity_workspace_size(int64_t K, int64_t C, int64_t P, int64_t nt);
KS_API int ks_similarity(const float* Wall, const float* W, int64_t K, int64_t C, int64_t P,
                         int64_t nt, float* sim, void* workspace, size_t workspace_bytes,
                         void* stream);

/*
 * Whitening of raw int16 samples (the streaming front end):
 *   X[c, t] = sum_c' Wrot[c, c'] * scale * raw[t * ld_raw + c']   (t < T, c < C)
 * with raw in the recording's layout (samples x channels), X row-major
 * [C, ldx].  Split-BF16 on the tensor cores: int16 values are exact as bf16
 * hi + lo, the matrix (scale folded in) is split as in the score
 * contraction.  status (device int) receives KS_OK or the contraction's
 * device error.  Replaces the whitening step of kilosort/io.py:1019-1025
 * (X = whiten_mat @ X) for raw batches.
 */
KS_API size_t ks_whiten_int16_workspace_size(int64_t T, int64_t C);
KS_API int ks_whiten_int16(const int16_t* raw, int64_t T, int64_t C, int64_t ld_raw,
                           const float* Wrot, float scale, float* X, int64_t ldx,
                           int* status, void* workspace, size_t workspace_bytes,
                           void* stream);

/*
 * Preprocessing of one raw int16 batch (the padded window, file layout
 * raw[t * ld_raw + ch], t < L), as kilosort/io.py:994-1026 (BinaryFiltered.filter):
 *   X = raw[:, chan_map] (C channels; chan_map NULL: the first C), negated when
 *   invert_sign; minus each channel's mean over the batch; minus each sample's
 *   lower median over channels when do_car; the circular high-pass
 *   X'[c, n] = sum_j hp_taps[j] X[c, (n + j - hp_centre) mod L] (the centre
 *   taps of the reference's filter, 1 <= ntaps <= min(1023, L), hp_centre the
 *   centre tap's index less the filter's offset from L/2; NULL: none); all
 *   zeros when artifact_threshold is finite and any |X'| >= it; then
 *   X = whiten @ X' (f32 [C][C] on the device, the drift matrix folded in by
 *   the caller; NULL: no whitening).  Output X [C][ldx] f32.  flags (device
 *   int[2]): [0] KS_OK, KS_ERR_ARG (a chan_map entry outside [0, ld_raw)) or
 *   the contraction's device error; [1] 1 when the artifact test zeroed the
 *   batch.  C <= 1024.
 */
KS_API size_t ks_preprocess_workspace_size(int64_t L, int64_t C, int whiten);
KS_API int ks_preprocess_int16(const int16_t* raw, int64_t L, int64_t ld_raw,
                               const int64_t* chan_map, int64_t C, int invert_sign,
                               int do_car, const float* hp_taps, int64_t ntaps,
                               int64_t hp_centre, float artifact_threshold,
                               const float* whiten, float* X,
                               int64_t ldx, int* flags, void* workspace,
                               size_t workspace_bytes, void* stream);

/*
 * Output consumers of extract: per spike s (template templ[s], features
 * tF [N, nC, P] as extract returns them), the position estimate
 *   w_i = m_i ||tF[s,i,:]|| / sum_j m_j ||tF[s,j,:]||, m_i = iCC_mask[i, iU[k]]
 *   xs[s] = sum_i xc[iCC[i, iU[k]]] w_i,  ys[s] likewise  (double)
 * and the amplitude amps[s] = ||tF[s,:,:]|| (float).  iCC [nC, C] int64,
 * iCC_mask [nC, C] uint8, iU [K] int64, xc/yc [C] double.  A template index
 * outside [0, K) sets *status (device int) to KS_ERR_ARG and gives zeros.
 * Replaces kilosort/postprocessing.py:33-62 (compute_spike_positions) and the
 * amplitudes of kilosort/io.py:353.
 */
KS_API int ks_spike_positions(const float* tF, const int64_t* templ, const int64_t* iCC,
                              const uint8_t* iCC_mask, const int64_t* iU, const double* xc,
                              const double* yc, int64_t N, int64_t nC, int64_t P, int64_t C,
                              int64_t K, double* xs, double* ys, float* amps, int* status,
                              void* stream);

/*
 * Duplicate-spike removal of the Phy export: spikes in index order, a spike
 * kept (keep[s] = 1) when its time is at least dt after the last kept spike
 * of the same cluster, the first spike of each cluster always kept (keep is
 * uint8 [N]).  spike_times int64 [N], spike_clusters int32 [N] (any order of
 * times).  Scratch: ks_remove_duplicates_workspace_size(N) bytes.
 * Replaces kilosort/postprocessing.py:10-30 (remove_duplicates, called by
 * kilosort/io.py:356-358).
 */
KS_API size_t ks_remove_duplicates_workspace_size(int64_t N);
KS_API int ks_remove_duplicates(const int64_t* spike_times, const int32_t* spike_clusters,
                                int64_t N, int64_t dt, uint8_t* keep, void* workspace,
                                size_t workspace_bytes, void* stream);

/*
 * Template waveforms of the Phy export, templates[k, t, c] = sum_p
 * Wall[k, c, p] * W[p, t] (products rounded, then summed over p in order),
 * Wall [K, C, P], W [P, nt] (wPCA), templates [K, nt, C], all f32.
 * Replaces kilosort/io.py:383-385 (templates.npy).
 */
KS_API int ks_phy_templates(const float* Wall, const float* W, int64_t K, int64_t C, int64_t P,
                            int64_t nt, float* templates, void* stream);

/*
 * Stage timing of ks_run_matching, for profiling the public call as it runs
 * (no work is skipped or added).  While enabled on the calling host thread,
 * ks_run_matching records CUDA events at five points on its stream: start,
 * after the template energies, after the projection, after the peel kernel,
 * after the residual kernel.  ks_trace_read waits for the last of the first
 * n+1 events of the thread's most recent traced call and writes n <= 4
 * intervals in ms: [energy + copy, projection, peel kernel, residual]
 * (ks_match_batches records the same five points around its stages:
 * [per-recording set-up, projections, peel launch, residual launch]).  The
 * events are the library's, created on the current device by the first
 * ks_trace_stages(1).  No reference counterpart (the reference has no
 * tracing of this path).
 */
KS_API int ks_trace_stages(int enable);
KS_API int ks_trace_read(float* ms, int n);

/*
 * Watchdog self-test: one thread waits on a device flag that nothing sets,
 * bounded by timeout_ns, and writes KS_ERR_TIMEOUT to status[0] when the wait
 * runs out.  status points to two device ints (status[1] is the flag, cleared
 * here).  No reference counterpart (tests the device-side bounded waits).
 */
KS_API int ks_selftest_wait(int64_t timeout_ns, int* status, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* KS_B200_H */
