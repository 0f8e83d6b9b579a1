/*
 * opentm_b200_driver.h -- the optimisation driver around the homogenization path: initial
 * density fields, field symmetrisation, the tensor-matching design loop with its volume
 * governor and convergence test, and the driver's on-disk formats.
 *
 * Reference counterparts:
 *   initDensity                     Framework.cu:63-145
 *   randTri / randTribase_sincos    homogenization/Framework.cuh:106-215, 237-310
 *   symmetrizeField / symmetrize    homogenization/Framework.cuh:218-235,
 *                                   AutoDiff/TensorExpression.h:446-470, .cuh:70-280
 *   ConvergeChecker, VolumeGovernor homogenization/Framework.cuh:312-411
 *   runCustom                       Framework.cu:147-244
 *   runInstance, wrapper_homo       main.cpp:17-62
 *   cfg::HomoConfig                 cmdline.h:12-33, cmdline.cpp:4-35
 *   writeVectors / readVectors      homogenization/utils.h:47-91
 *   Grid_H::writeDensity (binary)   homogenization/grid.cpp:329-345
 *   heat_tensor_t::writeTo(Txt)     homogenization/homoExpression.h:130-146
 *
 * Fields are FP32 device arrays, lexicographic with x fastest and a row pitch of pitchT floats
 * (pitchT <= 0 means nx), like otm_homo_update. The reference draws its random numbers with
 * cuRAND; here value i of stream `seed` is splitmix64(seed * 2^32 + i) mapped to [0, 1) with
 * 53 bits, so a seeded run is reproducible on any machine.
 */
#ifndef OPENTM_B200_DRIVER_H
#define OPENTM_B200_DRIVER_H

#include "opentm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* cfg::Symmetry (cmdline.h:9) */
#define OTM_SYM_REFLECT3 0
#define OTM_SYM_REFLECT6 1
#define OTM_SYM_ROTATE3 2
#define OTM_SYM_ROTATE2 3
#define OTM_SYM_NONE 4

/* cfg::InitWay (cmdline.h:10) */
#define OTM_INIT_RANDOM 0
#define OTM_INIT_RANDCENTER 1
#define OTM_INIT_NOISE 2
#define OTM_INIT_MANUAL 3 /* density read from input_path (binary format below; OpenVDB is not supported) */
#define OTM_INIT_INTERP 4 /* OpenVDB resampling: OTM_ERR_UNSUPPORTED */
#define OTM_INIT_REP_RANDCENTER 5 /* randcenter with the coefficients read from input_path */
#define OTM_INIT_P 6
#define OTM_INIT_G 7
#define OTM_INIT_D 8
#define OTM_INIT_IWP 9
#define OTM_INIT_EXAMPLE 10

/* cfg::Model (cmdline.h:11) */
#define OTM_MODEL_MMA 0
#define OTM_MODEL_OC 1

/* The fields of cfg::HomoConfig that the driver reads, with HomoConfig::init() defaults. */
typedef struct otm_driver_config {
  int reso;                 /* cells per axis of the cubic cell; default 128 (runCustom reads reso[0]) */
  int sym;                  /* OTM_SYM_*; default OTM_SYM_NONE */
  int winit;                /* OTM_INIT_*; default OTM_INIT_IWP */
  int model;                /* OTM_MODEL_*; default OTM_MODEL_OC */
  double vol_ratio;         /* volume of the random initialisers; default 0.3 */
  double heat_ratio[2];     /* conductivity at rho = 1 and rho = 0; default {1, 0} */
  double finthres;          /* relative objective change of the convergence test; default 5e-4 */
  double fem_rel_thres;     /* homogenization solve tolerance; default 0.01 */
  double target_tensor[6];  /* K00, K11, K22, K01, K21, K02 targets; default {0.3, 0.2, 0.1, 0, 0, 0} */
  int max_iter;             /* design iterations; default 500 */
  int init_period;          /* frequencies per axis of the random basis; default 10 (at most 50) */
  uint64_t seed;            /* random stream of the random initialisers; default 0 */
  const char* input_path;   /* OTM_INIT_MANUAL / OTM_INIT_REP_RANDCENTER input; default NULL */
  const char* output_prefix; /* NULL (default): no files; else the run's files are written with
                                this prefix: "coeff" (random basis coefficients), "init_rand"
                                (initial density), "oc_v_log.txt" (appended: MMA seconds and
                                objective per iteration, OC total seconds), "density<reso>" /
                                "density_mma" (final density); densities in the binary format
                                below, where the reference writes OpenVDB */
} otm_driver_config;

typedef struct otm_driver_result {
  int iterations;      /* design iterations evaluated */
  int converged;       /* 1 when the convergence test ended the loop */
  double objective;    /* last objective value (tensor mismatch minus 1e-4) */
  double volume;       /* mean density at exit */
  double volume_bound; /* OC: the governor's volume bound at exit; MMA: 0 */
  float K[9];          /* last K^H (FP32 copy, as heat_tensor_t holds it) */
  double init_seconds; /* setup and initial density (host clock) */
  double loop_seconds; /* the design iterations (host clock; every iteration waits for its K^H) */
} otm_driver_result;

OTM_API otm_status otm_driver_config_init(otm_driver_config* cfg);

/* ---- field symmetrisation (symetrize_tensor_kernel, AutoDiff/TensorExpression.cuh:70-280) ----
 * Every orbit of the symmetry group is set to its mean; with average == 0, REFLECT3 and ROTATE2
 * copy the representative's value instead (REFLECT6 and ROTATE3 always average, as in the
 * reference). REFLECT3 and ROTATE2 take any sizes; REFLECT6 needs a cube and ROTATE3 an
 * even-sized cube (OTM_ERR_UNSUPPORTED otherwise). Deterministic: each orbit is written by one
 * thread. */
OTM_API otm_status otm_symmetrize(const int reso[3], float* field, int pitchT, int sym, int average, void* stream);

/* ---- random trigonometric basis (randTribase_sincos_kernel, Framework.cuh:106-215) ----
 * Number of coefficients: 6 n + 36 n^2, plus 4 (a rotation quaternion) when centered. */
OTM_API size_t otm_randtri_coeff_count(int n_period, int centered);
/* The coefficients randTri draws: U(-1, 1) from stream `seed`. */
OTM_API otm_status otm_randtri_coefficients(uint64_t seed, int n_period, int centered, float* coeffs_host);
/* field = sum of the basis terms at p = (x, y, z) / (reso - 1) (centered: p - 1/2 rotated by the
 * normalised quaternion in the last 4 coefficients); coeffs_host holds otm_randtri_coeff_count. */
OTM_API otm_status otm_randtri_field(const int reso[3], float* field, int pitchT, int n_period,
                                     const float* coeffs_host, int centered, void* stream);

/* ---- initDensity (Framework.cu:63-145) ----
 * Writes the initial density of cfg->winit into rho (cfg->reso^3 cells) on `stream`, including
 * the final symmetrisation and the clamp to [0.1, 1]. For the random-basis forms coeffs_out
 * (optional, otm_randtri_coeff_count values) receives the coefficients used. Blocks until done. */
OTM_API otm_status otm_init_density(const otm_driver_config* cfg, float* rho, int pitchT, float* coeffs_out,
                                    void* stream);

/* ---- ConvergeChecker (Framework.cuh:312-345) ---- */
typedef struct otm_converge_checker {
  double thres;
  double obj[10];
  int p;
} otm_converge_checker;
OTM_API void otm_converge_checker_init(otm_converge_checker* c, double thres);
/* is_converge(iter, obj): 1 when the relative change stayed <= thres for the last 3 steps. */
OTM_API int otm_converge_checker_step(otm_converge_checker* c, int iter, double obj);

/* ---- VolumeGovernor (Framework.cuh:347-411) ---- */
typedef struct otm_volume_governor {
  float low_bound, volume_bound, decrease, decrease_factor, val_last, vibrate;
  int vibrate_count, count;
} otm_volume_governor;
OTM_API void otm_volume_governor_init(otm_volume_governor* g);
OTM_API int otm_volume_governor_check(otm_volume_governor* g, float value, float low_bound, float volfrac, int itn);
OTM_API float otm_volume_governor_decrease(const otm_volume_governor* g); /* get_current_decrease */

/* ---- runCustom (Framework.cu:147-244) ----
 * The tensor-matching design loop on the current device: k = filter(rho)^3 (k0 - kmin) + kmin
 * (Spline4 radius 1.5, not periodic), K^H of k, objective sum (K_ij - t)^2 - 1e-4 over the six
 * targeted entries, its gradient through sensitivity and the filter adjoint, then an OC step
 * (symmetrised fields, filterSens radius 2, volume bound from the governor) or an MMA step
 * (minimise volume subject to objective <= 0). rho0_host (reso^3 values, optional) replaces
 * initDensity; rho_out_host (optional) receives the final density; obj_history (optional,
 * max_iter values) the objective per iteration. */
OTM_API otm_status otm_run_custom(const otm_driver_config* cfg, const float* rho0_host, float* rho_out_host,
                                  double* obj_history, otm_driver_result* result);

/* ---- on-disk formats ---- */
/* Grid_H::writeDensity binary form (grid.cpp:336-344): int32 reso[3], then reso0*reso1*reso2
 * FP32 densities, x fastest. */
OTM_API otm_status otm_write_density_binary(const char* path, const int reso[3], const float* rho_host);
/* Reads that form: reso receives the sizes; with rho_host == NULL only the header is read;
 * OTM_ERR_INVALID_ARGUMENT when capacity (values) is too small or the file is short. */
OTM_API otm_status otm_read_density_binary(const char* path, int reso[3], float* rho_host, size_t capacity);
/* homoutils::writeVectors<float, N> (utils.h:47-59): n_vec vectors of len values, interleaved
 * element by element (record j holds vec[0][j] ... vec[n_vec-1][j]). */
OTM_API otm_status otm_write_vectors(const char* path, int n_vec, size_t len, const float* const* vecs);
/* readVectors<float, N> (utils.h:73-90): *len receives the record count; with vecs == NULL only
 * the count is returned; otherwise up to capacity records are read into each vecs[i]. */
OTM_API otm_status otm_read_vectors(const char* path, int n_vec, size_t* len, float* const* vecs, size_t capacity);
/* heat_tensor_t::writeTo (9 raw FP32 values) or writeToTxt (text = 1: 3 lines of 3 values). */
OTM_API otm_status otm_write_heat_matrix(const char* path, const float K[9], int text);

#ifdef __cplusplus
}
#endif

#endif /* OPENTM_B200_DRIVER_H */
