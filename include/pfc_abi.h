/*
 * pfc_abi.h — C-ABI of libpf_kernels.so, the B200 (sm_100a) particle-filter and
 * CBGL global-localization library.
 *
 * The first block (18 functions) is the drop-in surface: same names, argument
 * meaning, return codes and ownership rules as the reference library that the
 * Rust crate `pf_core` links (`-l dylib=pf_kernels`, crates/pf_core/build.rs:15).
 * Every declaration cites the Rust binding it satisfies and the reference
 * definition it replaces.  The second block holds additive entry points with no
 * reference counterpart (fused cycle, parity hooks, fed-input scoring, batched
 * filters); existing signatures are never changed by them.
 *
 * Conventions shared by all entry points
 *   - 0 = success, -1 = error (a message goes to stderr and to
 *     pfc_last_error_message()); *_create returns NULL on failure.
 *   - Handles are opaque; the library owns all device memory behind them.
 *   - Host arrays are caller-owned and are fully consumed before the call
 *     returns; host outputs are written before the call returns.
 *   - One handle must not be used by two host threads at once (as in the
 *     reference: no internal locking).  Each handle runs its device work on its
 *     own CUDA stream on the device that was current at *_create time.
 */
#ifndef PFC_ABI_H
#define PFC_ABI_H

#ifdef __cplusplus
extern "C" {
#endif

/* Only the entry points below are exported from the shared library. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* One observation as the Rust side marshals it: `CObservation`,
 * crates/pf_core/src/cuda.rs:18-27 (#[repr(C)], 24 bytes), identical to the
 * reference's device record `ObsF`, src/cuda/pf_kernels.cu:79-84. */
typedef struct CObservation {
    int id;      /* landmark id (index into the dense landmark table)        */
    int mode;    /* 0 = Cartesian body-frame offset, 1 = range + unit bearing  */
    float dx, dy, dz; /* Cartesian offset, or unit bearing direction (body)   */
    float range; /* range in metres (mode 1 only)                              */
} CObservation;

/* ======================================================================
 * Drop-in block: particle filter (pfc_*).
 * Rust declarations: crates/pf_core/src/cuda.rs:33-88.
 * ==================================================================== */

/* Allocate a filter handle.  cap_obs outside [1,4096] becomes 64.
 * Replaces pf_kernels.cu:485-503; Rust: cuda.rs:34. */
void* pfc_create(int cap_obs);

/* Free a handle (NULL is accepted).  Returns 0.  Rust declares it without a
 * return value (cuda.rs:35), the reference C definition returns int
 * (pf_kernels.cu:505-517); both bind to this symbol. */
int pfc_destroy(void* h);

/* (Re)allocate for n particles; seed 0 becomes 42; resets the generation
 * counter.  Replaces pf_kernels.cu:519-551; Rust: cuda.rs:36. */
int pfc_init(void* h, int n, unsigned int seed);

/* Upload the dense landmark table: 3 floats per id, zeros for holes.
 * count == 0 clears the table.  Replaces pf_kernels.cu:553-565;
 * Rust: cuda.rs:37-41. */
int pfc_upload_landmarks(void* h, const float* xyz, int count);

/* Gaussian prior around (x,y,z | qw,qx,qy,qz); weights become 1/n.
 * Replaces pf_kernels.cu:567-582; Rust: cuda.rs:42-53. */
int pfc_reinit(void* h, float x, float y, float z, float qw, float qx, float qy,
               float qz, const float* pos_std3, const float* rot_std3);

/* Odometry delta (body frame) + process noise.  Replaces
 * pf_kernels.cu:584-598; Rust: cuda.rs:54-60. */
int pfc_predict(void* h, float tx, float ty, float tz, float qw, float qx,
                float qy, float qz, const float* tstd3, const float* rstd3);

/* Gated log-likelihoods + softmax.  nobs is clamped to cap_obs; nobs <= 0 or
 * an invalid normaliser resets the weights to uniform.  Observations whose id
 * is outside [0, landmark count) are skipped.  Replaces pf_kernels.cu:600-636;
 * Rust: cuda.rs:61-68. */
int pfc_weight(void* h, const CObservation* obs, int nobs, float sigma_r,
               float sigma_b, float gate);

/* Systematic resampling + optional uniform re-injection of
 * floor(ratio*n) particles; weights become 1/n.  An invalid weight total
 * resets the weights to uniform and leaves the particles in place.
 * Replaces pf_kernels.cu:638-676; Rust: cuda.rs:69. */
int pfc_resample(void* h, float random_inject_ratio);

/* 14 FP64 sums: [0..2] sum w*p, [3..12] upper triangle of sum w q q^T in the
 * order M00,M01,M02,M03,M11,M12,M13,M22,M23,M33, [13] sum w^2.
 * Replaces pf_kernels.cu:695-705; Rust: cuda.rs:70, unpacked at :277-285. */
int pfc_est_sums(void* h, double* out14);

/* 12 FP64 sums around the given means: [0..5] position covariance upper
 * triangle Pxx,Pxy,Pxz,Pyy,Pyz,Pzz; [6..11] attitude tangent covariance
 * Axx..Azz of the canonical axis-angle of qm^-1 * q.
 * Replaces pf_kernels.cu:709-722; Rust: cuda.rs:71-81. */
int pfc_covs(void* h, float mx, float my, float mz, float qw, float qx,
             float qy, float qz, double* out12);

/* Copy out positions (3n floats, xyz interleaved) and quaternions (4n floats,
 * w,x,y,z interleaved).  Replaces pf_kernels.cu:724-733; Rust: cuda.rs:82-86. */
int pfc_snapshot(void* h, float* pos3n, float* quat4n);

/* 1 when a CUDA device of compute capability >= 3 is present, else 0.
 * Replaces pf_kernels.cu:477-483; Rust: cuda.rs:87. */
int pfc_device_available(void);

/* ======================================================================
 * Drop-in block: global localization (pfgl_*).
 * Rust declarations: crates/pf_core/src/global_loc.rs:261-271.
 * ==================================================================== */

/* Occupancy grid: W*H bytes row-major, row 0 = lowest y, any nonzero byte is
 * occupied.  cap_hyp = largest hypothesis batch.  NULL on failure.
 * Replaces pf_kernels.cu:898-952; Rust: global_loc.rs:263-264. */
void* pfgl_create(int W, int H, float res, float ox, float oy,
                  const unsigned char* occ, int cap_hyp);

/* Free a handle (NULL accepted).  Replaces pf_kernels.cu:954-963;
 * Rust: global_loc.rs:265. */
int pfgl_destroy(void* h);

/* Number of free (zero) cells, or -1.  Replaces pf_kernels.cu:965-968;
 * Rust: global_loc.rs:266. */
int pfgl_free_cells(void* h);

/* Disperse n hypotheses uniformly over free cells, yaw uniform in [-pi,pi).
 * Replaces pf_kernels.cu:971-979; Rust: global_loc.rs:267. */
int pfgl_generate(void* h, int n, unsigned long long seed);

/* CAER = sum_r |scan[r] - raycast_r| for every current hypothesis.
 * Ray r points at theta + span*r/(nrays-1).  Replaces pf_kernels.cu:982-993;
 * Rust: global_loc.rs:268-269. */
int pfgl_score(void* h, const float* scan, int nrays, float rmax,
               float ang_span);

/* Bottom-k hypotheses by CAER ascending (ties: lower index first), written
 * as k*(x,y,theta).  Returns the count written (k clamped to the batch) or -1.
 * Replaces pf_kernels.cu:996-1023; Rust: global_loc.rs:270. */
int pfgl_topk(void* h, int k, float* out3k);

/* ======================================================================
 * Additive block (no reference counterpart).
 * ==================================================================== */

/* Last error message of the calling thread ("" when none). */
const char* pfc_last_error_message(void);

/* Library version, major*10000 + minor*100 + patch. */
int pfc_version(void);

/* Odometry record for the fused cycle (same meaning as pfc_predict's
 * arguments). */
typedef struct PfcOdom {
    float t[3];     /* body-frame translation                */
    float q[4];     /* rotation (w,x,y,z)                     */
    float tstd[3];  /* translation noise std dev per axis     */
    float rstd[3];  /* rotation noise std dev per axis        */
} PfcOdom;

/* Parameters of one fused cycle (the fields of PfConfig that
 * ParticleFilter::update reads, crates/pf_core/src/particle_filter.rs:111-124). */
typedef struct PfcCycleParams {
    float sigma_r, sigma_b, gate;
    double resample_ess_ratio;   /* resample when ess < ratio * n (0 = never) */
    float random_inject_ratio;
    int   reserved;
} PfcCycleParams;

/* Layout of the fused-cycle estimate (doubles). */
enum {
    PFC_EST_POS = 0,      /* 3: mean position                              */
    PFC_EST_QUAT = 3,     /* 4: mean attitude (w,x,y,z), w >= 0            */
    PFC_EST_POSCOV = 7,   /* 6: Pxx,Pxy,Pxz,Pyy,Pyz,Pzz                    */
    PFC_EST_ATTCOV = 13,  /* 6: Axx,Axy,Axz,Ayy,Ayz,Azz                    */
    PFC_EST_ESS = 19,     /* 1: effective sample size of the returned cloud */
    PFC_EST_RESAMPLED = 20, /* 1: 1.0 when the cycle resampled             */
    PFC_EST_ESS_PRE = 21, /* 1: ESS before resampling                       */
    PFC_EST_LEN = 24
};

/* One full ParticleFilter::update on the device with a single host sync:
 * predict -> weight -> estimate -> (ess < ratio*n ? resample + estimate).
 * The Markley mean and the resample decision run on the device. */
int pfc_cycle(void* h, const PfcOdom* odom, const CObservation* obs, int nobs,
              const PfcCycleParams* prm, double* est_out);

/* Same, with the observations already resident in device memory
 * (d_obs = device pointer to nobs CObservation records).  est_out may be a
 * host pointer (synchronous) or NULL (asynchronous; read it with
 * pfc_cycle_result). */
int pfc_cycle_device(void* h, const PfcOdom* odom, const void* d_obs, int nobs,
                     const PfcCycleParams* prm, double* est_out);

/* Wait for the last asynchronous cycle and copy its estimate. */
int pfc_cycle_result(void* h, double* est_out);

/* 1 (default): a fused cycle with observations is replayed from a CUDA graph
 * captured on first use (re-captured when n, the landmark table, the cycle
 * parameters or the weighting variant change); 0: direct kernel launches.
 * Both give identical results.  Cycles run with per-kernel profiling
 * (pfc_profile) always use direct launches. */
int pfc_set_graph(void* h, int on);

/* Sharded filter (no counterpart in the reference): one filter of n
 * particles over `world` ranks (one handle per rank, normally one GPU each).
 * Every rank's handle holds the whole cloud; a cycle predicts and weights
 * only the rank's slice [rank*chunk, min((rank+1)*chunk, n)), then the
 * caller exchanges the slices (an all-gather over the ranks of the seven
 * live planes, the log-likelihoods and the f32 softmax block partials, at
 * chunk particles or chunk/256 partials per rank), and every rank finishes
 * the cycle (softmax, ESS decision, resample, injection, estimate) on the
 * whole cloud.  With the same seed, landmarks and inputs on every rank the
 * cycle's result and particles equal pfc_cycle's on one handle, bit for
 * bit.
 *   pfc_shard_init:   instead of pfc_init (chunk = ceil(n/world) rounded
 *                     up to 2048; planes padded to world*chunk);
 *   pfc_shard_layout: chunk and plane length (n_pad);
 *   pfc_shard_weight: predict + weighting of the slice (asynchronous);
 *   pfc_shard_views:  device pointers of the live planes (7), ll and the
 *                     softmax partials (float2 per 256 particles), after
 *                     the slice's kernels completed (synchronises);
 *   pfc_shard_finish: the rest of the cycle once every slice is in place;
 *                     est_out as pfc_cycle's. */
int pfc_shard_init(void* h, int n, int world, int rank, unsigned int seed);
int pfc_shard_layout(void* h, int* chunk, int* n_pad);
int pfc_shard_weight(void* h, const PfcOdom* odom, const CObservation* obs, int nobs,
                     const PfcCycleParams* prm);
int pfc_shard_views(void* h, float** planes7, float** ll, float** part);
int pfc_shard_finish(void* h, const PfcCycleParams* prm, double* est_out);

/* The CUDA stream (cudaStream_t) the handle runs on. */
void* pfc_stream(void* h);

/* Particle count of the handle (0 before pfc_init). */
int pfc_size(void* h);

/* Normalised f32 weights (n floats) as the resampler and the estimator
 * see them. */
int pfc_get_weights(void* h, float* w);

/* f32 log-likelihoods from the last pfc_weight (n floats). */
int pfc_get_ll(void* h, float* ll);

/* Overwrite the particle set: AoS positions (3n) and quaternions (4n, w first)
 * as pfc_snapshot returns them; w = n weights or NULL for uniform 1/n. */
int pfc_set_state(void* h, const float* pos3n, const float* quat4n,
                  const float* w);

/* Global-localization hand-off: reinitialise around k planar poses
 * (x, y, yaw) held in DEVICE memory, e.g. pfgl_topk_device's result.
 * Particle i starts from pose i mod k at height z with attitude = yaw about
 * +z, perturbed like pfc_reinit (position N(0, pos_std3^2), attitude
 * exp(N(0, rot_std3^2))); weights become 1/n.  The poses must be complete
 * when the call is made (pfgl_topk_device's are). */
int pfc_reinit_poses(void* h, const float* d_pose3k, int k, float z,
                     const float* pos_std3, const float* rot_std3);

/* Resample with an explicit offset fraction u01 in [0,1) instead of the
 * handle's LCG draw (the LCG is left untouched); injection as pfc_resample. */
int pfc_resample_u01(void* h, double u01, float random_inject_ratio);

/* Accepted for compatibility and has no effect: every resample forms the
 * ancestor indices (its gather reads them), so they are always available. */
int pfc_record_ancestors(void* h, int on);

/* Ancestor index of every particle in the last resample (n ints). */
int pfc_get_ancestors(void* h, int* anc);

/* The reference's pick rule (pf_kernels.cu:304-321) applied to a caller
 * cumulative-weight array: anc[i] = first j with cum[j] >= u0 + i*(total/n),
 * clamped to n-1, evaluated on the device.  Host arrays of n entries. */
int pfc_pick_from_cum(void* h, const double* cum, int n, double u0,
                      double total, int* anc);

/* Tell the library the caller's resampling rule (ParticleFilter::update,
 * crates/pf_core/src/particle_filter.rs:111-124): after every pfc_weight the
 * caller reads the estimate's ESS and resamples when it is below
 * resample_ess_ratio * n, discarding that estimate.  The estimate and
 * covariance passes queued with it then report only sum w^2 on the device;
 * pfc_est_sums and pfc_covs still return the full values (computed on
 * demand), so results are unchanged.  0 (the default) turns it off.
 * Returns -1 for a NaN ratio. */
int pfc_set_ess_hint(void* h, double resample_ess_ratio);

/* ESS of the current cloud's estimate: 1 / out14[13] of pfc_est_sums (0 when
 * that sum is not positive), without the other sums when the ess hint lets
 * the library skip them. */
int pfc_est_ess(void* h, double* ess);

/* The weight normalisation's quotient e / S both ways on the device: fast[i]
 * from the FP64 product e * RN(1/S) (the form the weighting kernels use),
 * ieee[i] from the IEEE f32 division.  Host arrays of n entries. */
int pfc_weight_div_check(void* h, const float* e, const float* s, int n,
                         float* fast, float* ieee);

/* Device-side LCG word that drives the resampling offset (see
 * pf_kernels.cu:653-657); set it to replay a resample. */
int pfc_get_lcg(void* h, unsigned long long* lcg);
int pfc_set_lcg(void* h, unsigned long long lcg);

/* Accounting of one handle since creation / the last reset: kernels launched,
 * bytes copied host->device and device->host, host waits on the device. */
typedef struct PfcStats {
    unsigned long long launches;
    unsigned long long h2d_bytes;
    unsigned long long d2h_bytes;
    unsigned long long host_syncs;
} PfcStats;
int pfc_get_stats(void* h, PfcStats* out);
int pfc_reset_stats(void* h);

/* Kernel kinds of the per-kind timing below. */
enum {
    PFC_K_REINIT = 0, PFC_K_PREDICT, PFC_K_WEIGHT, PFC_K_EST, PFC_K_COVS,
    PFC_K_SCAN, PFC_K_GATHER, PFC_K_INJECT, PFC_K_COMMIT, PFC_K_MISC,
    PFC_K_COUNT
};

/* Per-kernel-kind device time: when on, every launch is bracketed by CUDA
 * events on the handle's stream; pfc_profile_read waits for them and returns
 * the accumulated milliseconds and launch counts (PFC_K_COUNT entries each)
 * since the last read. */
int pfc_profile(void* h, int on);
int pfc_profile_read(void* h, double* ms, long long* counts);

/* Weighting kernel variant.  Both perform every rounded operation of the
 * reference expression (src/cuda/pf_kernels.cu:240-269) in its order, so the
 * log-likelihoods are identical: 0 = packed f32x2 arithmetic over two
 * particles for chunks of Cartesian observations (default), 1 = scalar
 * arithmetic throughout. */
int pfc_set_weight_kernel(void* h, int variant);

/* ---------------------------------------------------------------------
 * Global localization, additive.
 * ------------------------------------------------------------------- */

/* n_pos uniform free-space positions x n_yaw yaws theta0 + j*2*pi/n_yaw
 * (theta0 uniform per position); hypothesis index = pos*n_yaw + j. */
int pfgl_generate_yaws(void* h, int n_pos, int n_yaw, unsigned long long seed);
/* Positions [p0, p0 + n_pos) of that same dispersion (hypothesis index on
 * this handle = (pos - p0)*n_yaw + j): one rank's slice of a global
 * hypothesis set, identical to the corresponding rows of pfgl_generate_yaws
 * with n_pos >= p0 + n_pos positions. */
int pfgl_generate_yaws_range(void* h, int p0, int n_pos, int n_yaw,
                             unsigned long long seed);

/* Batched uniform CBGL (no counterpart in the reference): nq queries, query
 * q with its own scan (scans + q*nrays) and the dispersion of
 * pfgl_generate_yaws(n_pos, n_yaw, seeds[q]); every hypothesis scored
 * exhaustively (the CAERs equal pfgl_score's bit for bit), each query's
 * bottom-k (stable by CAER, ties to the lower index) written to
 * out3k/caer_k/idx_k at [q*k, q*k + k) with indices within the query.
 * Needs n_pos*n_yaw <= 65536 and k <= 128; queries are processed in chunks
 * of cap_hyp / (n_pos*n_yaw).  Returns k (clamped to n_pos*n_yaw) or -1. */
int pfgl_localize_batch(void* h, const float* scans, int nq, int nrays, float rmax,
                        float ang_span, int n_pos, int n_yaw,
                        const unsigned long long* seeds, int k, float* out3k,
                        float* caer_k, int* idx_k);

/* Set / read hypotheses directly (3n floats x,y,theta). */
int pfgl_set_hyps(void* h, const float* hyp3n, int n);
int pfgl_get_hyps(void* h, float* hyp3n);

/* CAER of every current hypothesis (n floats) from the last pfgl_score. */
int pfgl_get_caer(void* h, float* caer);

/* DDA cell visits that scoring the current hypotheses with nrays rays over
 * ang_span takes (the work unit of CAER scoring), counted by a separate,
 * untimed kernel that replays the scorer's ray stepping; -1 on error.  No
 * reference counterpart (a measurement aid). */
long long pfgl_count_visits(void* h, int nrays, float ang_span);

/* Bottom-k with scores and indices: out3k may be NULL; caer_k / idx_k may be
 * NULL.  Returns the count written or -1. */
int pfgl_topk_ex(void* h, int k, float* out3k, float* caer_k, int* idx_k);

/* Bottom-k of caller scores (host array of n floats), ordered by
 * (CAER ascending, index ascending); writes min(k,n) indices. */
int pfgl_topk_from_scores(void* h, const float* caer, int n, int k,
                          int* idx_out);

/* Bottom-k of caller scores by the one-block radix select that the fused
 * localizers use (no reference counterpart): n <= 65536 and k <= 128.  Same
 * order as pfgl_topk_from_scores; when dropped_last is nonzero, negative
 * scores (hypotheses a pruned pass dropped) sort after every other one, in
 * index order.  The scores replace the handle's CAERs.  Writes min(k,n)
 * indices; returns that count or -1. */
int pfgl_select_from_scores(void* h, const float* caer, int n, int k,
                            int dropped_last, int* idx_out);

/* Fused global localization over the current hypotheses: raycast + CAER with
 * exact early termination against the running k-th best, and bottom-k
 * selection.  Same results as pfgl_score + pfgl_topk_ex for those k.  CAERs
 * of pruned hypotheses are not computed. */
int pfgl_localize(void* h, const float* scan, int nrays, float rmax,
                  float ang_span, int k, float* out3k, float* caer_k,
                  int* idx_k);

/* Device pointer to the k x (x, y, theta) poses of the last bottom-k
 * (pfgl_topk, pfgl_topk_ex, pfgl_localize); *k receives their count.  The
 * poses are complete when the returning call has returned, and stay valid
 * until the next bottom-k on this handle.  NULL before any bottom-k. */
const float* pfgl_topk_device(void* h, int* k);

/* Occupancy value the device sees for cell (cx,cy): 0 free, 1 occupied. */
int pfgl_cell(void* h, int cx, int cy);

/* Allocation-free bottom-k (no counterpart in the reference).  For callers
 * that must not allocate device memory when they select winners — a
 * localization step inside a fixed-rate control loop, where cudaMalloc /
 * cudaFree can block and synchronise the device, or an application whose
 * device memory all belongs to its own pool allocator.  The caller passes the
 * scores (device array of n floats) and the output (device array of k ints);
 * the sort's working memory is a fixed 1 MiB + 32 KiB array inside the
 * library, held by every GPU that loads the library until the process exits.
 * Writes the indices of the min(k,n) smallest scores ordered by (score,
 * index), as pfgl_topk_from_scores, asynchronously on `stream` (a
 * cudaStream_t; NULL = the legacy default stream).  Returns min(k,n), or -1
 * for n > 65536 or bad arguments.  All calls on a device share the working
 * array, so calls that overlap on the GPU race: issue them on one stream.
 * The first call on each device looks up the array's device address (once);
 * make that first call before any stream capture or real-time section. */
int pfgl_topk_noalloc(const float* d_scores, int n, int k, int* d_idx,
                      void* stream);

/* ------------------------------------------------------------------------
 * Batched particle filters (no counterpart in the reference).  Many
 * independent filters of uneven size advance together: one cycle of every
 * filter (predict + gated weighting + softmax + estimate + ESS-triggered
 * resample with injection + estimate, as pfc_cycle) is one CUDA-graph launch.
 * Filter f of a batch produces the same particles, weights and resampling as
 * the same filter run alone through pfc_cycle with the same seed and inputs;
 * its FP64 estimate sums agree to rounding (different summation tiles).
 * ------------------------------------------------------------------------ */

/* Per-filter input of one cycle: odometry and the slice
 * [obs_off, obs_off + nobs) of the cycle's concatenated observations. */
typedef struct PfcBatchCycle {
    PfcOdom odom;
    int obs_off;
    int nobs;
} PfcBatchCycle;

/* n_filters filters of n[f] particles; seeds[f] (NULL: 42; 0 becomes 42);
 * obs_cap = most observations of one cycle over all filters.  NULL on error. */
void* pfc_batch_create(int n_filters, const int* n, const unsigned* seeds,
                       int obs_cap);
int pfc_batch_destroy(void* b);
/* Per-filter cycle parameters (n_filters entries). */
int pfc_batch_set_params(void* b, const PfcCycleParams* prm);
/* Landmark tables: counts[f] landmarks of filter f, concatenated (3 floats
 * each) in filter order. */
int pfc_batch_upload_landmarks(void* b, const float* xyz, const int* counts);
/* Gaussian priors: pose7 (x,y,z,qw,qx,qy,qz), pos_std3 and rot_std3 per filter. */
int pfc_batch_reinit(void* b, const float* pose7, const float* pos_std3,
                     const float* rot_std3);
/* One cycle of every filter from host inputs: odom[f], nobs[f] and the
 * concatenated observations (filter order).  est_out (may be NULL):
 * n_filters x PFC_EST_LEN records laid out as pfc_cycle's. */
int pfc_batch_cycle(void* b, const PfcOdom* odom, const CObservation* obs,
                    const int* nobs, double* est_out);
/* Same from device-resident inputs (n_filters records, n_obs observations).
 * With est_out == NULL the call returns without waiting; pfc_batch_result
 * then waits and copies the records. */
int pfc_batch_cycle_device(void* b, const PfcBatchCycle* d_cycle,
                           const CObservation* d_obs, int n_obs, double* est_out);
int pfc_batch_result(void* b, double* est_out);
/* 1 (default): cycles run as one CUDA-graph launch; 0: direct launches. */
int pfc_batch_use_graph(void* b, int on);
/* Estimate-pass tile (particles, multiple of 1024) per size bucket
 * (n < 8192, < 32768, < 131072, larger) and the weighting variant. */
int pfc_batch_set_tiles(void* b, const int* est_tile4, int use_packed);
int pfc_batch_get_tiles(void* b, int* est_tile4, int* use_packed);
/* Time the candidate tiles per bucket on the current cloud (best of reps)
 * and keep the fastest; writes the choices. */
int pfc_batch_autotune(void* b, int reps, int* est_tile4, int* use_packed);
int pfc_batch_snapshot(void* b, int f, float* pos3n, float* quat4n);
int pfc_batch_get_weights(void* b, int f, float* w);
int pfc_batch_size(void* b, int f);
void* pfc_batch_stream(void* b);
/* Kernels launched by this handle so far (a graph launch counts its kernels). */
long long pfc_batch_launches(void* b);
/* Test hook for the bounded device waits (no counterpart in the reference).
 * spin_limit: polls before a resampling look-back gives up (0 restores the
 * default of 2^22).  stall_filter: a filter whose first resampling tile
 * publishes its prefix under a stale epoch, a flag no waiter accepts, so the
 * look-backs of its later tiles run out (-1: none).  A wait that runs out
 * sets an error bit: the cycle call (or pfc_batch_result) returns -1 with
 * "look-back wait timed out" in pfc_last_error_message(), and the handle keeps
 * failing from then on (its particles are no longer trustworthy); other
 * handles and the CUDA context are unaffected. */
int pfc_batch_set_wait_test(void* b, int spin_limit, int stall_filter);

/* ------------------------------------------------------------------------
 * Learned proposal for global localization (no counterpart in the
 * reference).  A per-map MLP maps a normalised range scan to a 32-component
 * Gaussian mixture over (x, y, cos yaw, sin yaw); queries sample hypotheses
 * from the mixture and score them with plain CAER, falling back to uniform
 * dispersion when the best CAER exceeds a threshold calibrated on held-out
 * poses.  Network: 384 (360 rays + zero padding) -> 4 x 1024 ReLU -> 384
 * (288 used: 32 logits, 32x4 means, 32x4 log-sigma pre-activations), BF16
 * weights and activations, FP32 accumulation and master weights, trained with
 * Adam by the library's own tcgen05 kernels.  A handle borrows the pfgl
 * handle (map, scorer, stream) it is created on and must be destroyed first.
 * ------------------------------------------------------------------------ */
enum {
    PFGL_LP_IN = 384,      /* padded input width (rays / rmax, then zeros) */
    PFGL_LP_HIDDEN = 1024, /* hidden width (4 hidden layers) */
    PFGL_LP_OUT = 384,     /* padded output width */
    PFGL_LP_COMP = 32,     /* mixture components */
    PFGL_LP_LAYERS = 5
};

/* batch: training minibatch rows (multiple of 128).  Returns NULL on error. */
void* pfgl_learned_create(void* gl, int batch, unsigned long long seed);
int pfgl_learned_destroy(void* lp);
/* Number of f32 parameters in the flattened order W0,b0,...,W4,b4 with
 * W_l row-major [out_l][in_l] over the padded widths. */
long long pfgl_learned_num_params(void);
int pfgl_learned_get_params(void* lp, float* out);
int pfgl_learned_set_params(void* lp, const float* in);
/* Render scans at caller poses with the library's raycaster (the CAER ray
 * geometry) plus N(0, noise_std^2) range noise; out is n x nrays. */
int pfgl_render_scans(void* gl, const float* pose3n, int n, int nrays,
                      float rmax, float ang_span, float noise_std,
                      unsigned long long seed, float* out);
/* Generate n_pairs (scan, pose) training pairs on the device: poses uniform
 * over free cells with yaw uniform in [0, 2 pi), nrays <= 384 rays over
 * ang_span with range noise noise_std. */
int pfgl_learned_make_data(void* lp, long long n_pairs, int nrays, float rmax,
                           float ang_span, float noise_std,
                           unsigned long long seed);
/* Run `steps` Adam steps over the generated pairs (peak learning rate lr,
 * linear warm-up then cosine decay over total_steps).  loss_out (may be
 * NULL) receives the mean loss of each step. */
int pfgl_learned_train(void* lp, int steps, int total_steps, float lr,
                       float* loss_out);
/* Loss and gradients (no update) for caller inputs: x is batch x 384
 * normalised scans (padded), y is batch x 4 targets (x_n, y_n, cos, sin).
 * grad receives pfgl_learned_num_params() floats. */
int pfgl_learned_grad(void* lp, const float* x, const float* y, float* loss,
                      float* grad);
/* Mixture parameters (rows x 288) for rows <= 128 caller inputs (rows x 384). */
int pfgl_learned_forward(void* lp, const float* x, int rows, float* out);
/* Map normalisation: x_n = (x - c[0]) / c[2], y_n = (y - c[1]) / c[3]. */
int pfgl_learned_norm(void* lp, float* c4);
/* Localize one scan: n_samples mixture samples scored with CAER; when the
 * best CAER exceeds the calibrated threshold, n_fallback uniform hypotheses
 * (16 yaws per position) are scored as well and the better list is kept.
 * info (may be NULL): 0 learned, 1 fallback ran and learned kept, 2 fallback
 * result returned.  Returns k written or -1. */
int pfgl_learned_localize(void* lp, const float* scan, int nrays, float rmax,
                          float ang_span, int n_samples, int n_fallback, int k,
                          float* out3k, float* caer_k, int* idx_k, int* info);
/* Learned localization of nq queries in batches (no counterpart in the
 * reference): the scans go through the network as rows of one tiled GEMM
 * per layer, n_samples mixture samples per query are scored exhaustively in
 * one launch across the batch, and each query's bottom-k is selected by its
 * own block; results at [q*k, q*k + k) of out3k/caer_k/idx_k, info[q] as
 * pfgl_learned_localize.  A query whose best CAER exceeds the calibrated
 * threshold falls back to n_fallback uniform hypotheses (n_fallback = 0:
 * never).  Needs n_samples <= 65536 and k <= 128.  Returns k (clamped to
 * n_samples) or -1. */
int pfgl_learned_localize_batch(void* lp, const float* scans, int nq, int nrays,
                                float rmax, float ang_span, int n_samples, int n_fallback,
                                int k, float* out3k, float* caer_k, int* idx_k, int* info);

/* Calibrate the fallback threshold on n_queries held-out poses: the
 * `quantile` of the best CAER over held-out successes (within 0.5 m and
 * 0.1 rad), the queries run through the batched path (one at a time when
 * n_samples exceeds its limit).  Writes the threshold and the held-out
 * success rate. */
int pfgl_learned_calibrate(void* lp, int n_queries, int nrays, float rmax,
                           float ang_span, float noise_std, int n_samples,
                           float quantile, unsigned long long seed,
                           float* tau_out, float* success_out);
int pfgl_learned_set_threshold(void* lp, float tau);

/* 1 (default): a query of up to 65536 samples and k <= 128 is replayed from a
 * CUDA graph captured on first use (again when its sizes, ray geometry or
 * scan buffer change); 0: direct launches.  Both give the same results. */
int pfgl_learned_set_graph(void* lp, int on);
/* Plain tcgen05 GEMM D = A * B^T (A: M x K, B: N x K, bf16 bit patterns,
 * row-major; D: M x N f32) for numerics tests.  M, N multiples of 128, K a
 * multiple of 64. */
int pfgl_learned_gemm(int M, int N, int K, const unsigned short* A,
                      const unsigned short* B, float* D);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* PFC_ABI_H */
