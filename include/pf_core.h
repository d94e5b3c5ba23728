/*
 * pf_core.h — C-ABI of libpf_core.so, the C++ host layer that sits where the
 * reference's Rust crate pf_core sits: it drives libpf_kernels.so through the
 * pfc_* / pfgl_* calls in exactly the order the Rust code does, so tests and
 * benchmarks exercise the drop-in boundary the way the reference's callers do.
 *
 * Mirrors (reference files, paths within the reference project):
 *   ParticleFilter::new/reinitialize/update   crates/pf_core/src/particle_filter.rs:77-124
 *   CudaBackend (Backend impl over pfc_*)      crates/pf_core/src/cuda.rs:97-358
 *   quat_mean (Markley)                         crates/pf_core/src/types.rs:117-143
 *   LandmarkMap (+ text loader)                 crates/pf_core/src/landmark_map.rs:7-80
 *   OccGrid::from_pgm_yaml                      crates/pf_core/src/global_loc.rs:30-130
 *   CudaGlobalLoc::new/localize                 crates/pf_core/src/global_loc.rs:273-341
 */
#ifndef PF_CORE_H
#define PF_CORE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* PfConfig, crates/pf_core/src/config.rs:4-30 (backend is always CUDA). */
typedef struct PfcoreConfig {
    int particle_count;
    double trans_noise[3];
    double rot_noise[3];
    double range_noise;
    double bearing_noise;
    double resample_ess_ratio;
    double random_inject_ratio;
    double gate_sigma;
    unsigned long long seed;
} PfcoreConfig;

/* Observation, crates/pf_core/src/types.rs:58-67 (mode 0 Cartesian,
 * 1 range-bearing). */
typedef struct PfcoreObservation {
    int landmark_id;
    int mode;
    double vector[3];
    double range;
} PfcoreObservation;

/* OdomDelta, crates/pf_core/src/types.rs:69-79 (rotation w,x,y,z). */
typedef struct PfcoreOdom {
    double translation[3];
    double rotation[4];
    double trans_noise[3];
    double rot_noise[3];
} PfcoreOdom;

/* Estimate, crates/pf_core/src/types.rs:92-103 (attitude w,x,y,z; row-major
 * 3x3 covariances). */
typedef struct PfcoreEstimate {
    double position[3];
    double attitude[4];
    double pos_cov[9];
    double att_cov[9];
    double ess;
    int valid;
    int resampled;
} PfcoreEstimate;

/* PfConfig::default() values (config.rs:49-63). */
void pfcore_config_default(PfcoreConfig* cfg);

/* ParticleFilter::new with the CUDA backend; NULL when no device. */
void* pfcore_filter_new(const PfcoreConfig* cfg);
void pfcore_filter_free(void* pf);

/* Landmark map of the filter (ParticleFilter::set_map semantics). */
int pfcore_map_add(void* pf, int id, double x, double y, double z);
int pfcore_map_clear(void* pf);
/* LandmarkMap::load_from_str: lines "id: [x, y, z]" or "id x y z", '#'
 * comments.  Returns the number of landmarks read, or -1 (message in
 * pfcore_last_error). */
int pfcore_map_load_text(void* pf, const char* text);
int pfcore_map_capacity(void* pf);

/* LandmarkMap as a value of its own (crates/pf_core/src/landmark_map.rs:7-80),
 * host only, no device needed.  new/add/has/at/capacity/len_defined/
 * load_from_str keep the reference's meaning; where the reference panics
 * (a negative id in add, an absent id in at) these return -1 with a message
 * in pfcore_last_error.  load_text returns the number of lines read, or -1 at
 * the first bad line, the lines before it staying in the map as in the
 * reference. */
void* pfcore_landmarks_new(void);
void pfcore_landmarks_free(void* map);
int pfcore_landmarks_add(void* map, int id, double x, double y, double z);
int pfcore_landmarks_has(void* map, int id);
int pfcore_landmarks_at(void* map, int id, double out_xyz[3]);
int pfcore_landmarks_capacity(void* map);
int pfcore_landmarks_len_defined(void* map);
int pfcore_landmarks_load_text(void* map, const char* text);
/* ParticleFilter::set_map (crates/pf_core/src/particle_filter.rs:88-90): the
 * filter takes a copy. */
int pfcore_filter_set_map(void* pf, void* map);

/* ParticleFilter::reinitialize: pose = (x,y,z, qw,qx,qy,qz). */
int pfcore_filter_reinitialize(void* pf, const double pose[7],
                               const double pos_std[3],
                               const double rot_std[3]);

/* ParticleFilter::update over the drop-in pfc_* sequence of CudaBackend. */
int pfcore_filter_update(void* pf, const PfcoreOdom* odom,
                         const PfcoreObservation* obs, int nobs,
                         PfcoreEstimate* out);

/* The same cycle through the additive fused entry point (pfc_cycle): one
 * host sync per cycle. */
int pfcore_filter_update_fused(void* pf, const PfcoreOdom* odom,
                               const PfcoreObservation* obs, int nobs,
                               PfcoreEstimate* out);

/* Backend::snapshot (f64 copies; weights as the library reports them). */
int pfcore_filter_snapshot(void* pf, double* pos3n, double* quat4n,
                           double* w);

/* The underlying pfc handle (for additive calls). */
void* pfcore_filter_handle(void* pf);

/* Markley mean of 10 packed moments (types.rs quat_mean semantics). */
void pfcore_quat_mean(const double m10[10], double q_out[4]);

/* ---------------------------------------------------------------- GL */

/* GlParams, crates/pf_core/src/global_loc.rs:236-257. */
typedef struct PfcoreGlParams {
    int hypotheses;
    int rays;
    double rmax;
    double ang_span;
    int topk;
    unsigned long long seed;
} PfcoreGlParams;

typedef struct PfcorePoseHypothesis {
    double x, y, theta, caer;
} PfcorePoseHypothesis;

void pfcore_gl_params_default(PfcoreGlParams* p);

/* CudaGlobalLoc::new over a row-major W*H occupancy grid. */
void* pfcore_gl_new(int w, int h, double res, double ox, double oy,
                    const unsigned char* cells, const PfcoreGlParams* p);
void pfcore_gl_free(void* gl);
int pfcore_gl_free_cells(void* gl);
int pfcore_gl_set_seed(void* gl, unsigned long long seed);
/* CudaGlobalLoc::localize: bottom-k ascending, caer = NaN as in the
 * reference.  Returns the count written (<= topk) or -1. */
int pfcore_gl_localize(void* gl, const float* scan, int nrays,
                       PfcorePoseHypothesis* out);
void* pfcore_gl_handle(void* gl);

/* OccGrid::from_pgm_yaml (ROS map_server P5 PGM + YAML).  Call with
 * cells == NULL to learn w,h; then with a w*h buffer.  0 or -1. */
int pfcore_grid_from_pgm_yaml(const unsigned char* pgm, size_t pgm_len,
                              const char* yaml, int* w, int* h, double* res,
                              double* ox, double* oy, unsigned char* cells);

const char* pfcore_last_error(void);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* PF_CORE_H */
