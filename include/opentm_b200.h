/*
 * opentm_b200.h -- C ABI of the B200-native OpenTM thermal homogenization hot path.
 *
 * Every entry point takes plain pointers and sizes, returns an otm_status, and runs its GPU
 * work on the stream given to it (or the handle's stream). Device arrays are owned by the
 * caller. A handle holds no global device state, so several handles can be used at once; a
 * single handle must not be used from two host threads at the same time.
 *
 * Each declaration names the reference interface it replaces (file:line relative to the
 * OpenTM project root).
 */
#ifndef OPENTM_B200_H
#define OPENTM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OTM_ABI_VERSION 2

#if defined(__GNUC__)
#define OTM_API __attribute__((visibility("default")))
#else
#define OTM_API
#endif

typedef enum otm_status {
  OTM_OK = 0,
  OTM_ERR_INVALID_ARGUMENT = 1, /* bad size, pointer, pitch or option */
  OTM_ERR_UNSUPPORTED = 2,      /* e.g. resolution above 1024 (homogenization/grid.cpp:23-25) */
  OTM_ERR_CUDA = 3,             /* a CUDA runtime call failed; see otm_last_error() */
  OTM_ERR_OUT_OF_MEMORY = 4,
  OTM_ERR_NOT_CONVERGED = 5, /* iteration cap reached (homogenization/MG.cpp:392-399) */
  OTM_ERR_DIVERGED = 6,      /* residual exploded twice ("MG numerical explode", MG.cpp:407) */
  OTM_ERR_NAN = 7,           /* NaN or Inf in an input or an iterate */
  OTM_ERR_BUDGET = 8,        /* a request does not fit the serving memory budget */
  OTM_ERR_STATE = 9,         /* call out of order, e.g. sensitivity before a solve */
  OTM_ERR_TIMEOUT = 10,      /* a bounded wait ran out */
  OTM_ERR_CANCELLED = 11,    /* a serving request was cancelled */
  OTM_ERR_NOT_READY = 12     /* a serving request is still running */
} otm_status;

typedef enum otm_precision {
  OTM_PRECISION_FP32 = 0,       /* plain FP32 multigrid: the drop-in */
  OTM_PRECISION_MIXED_BF16 = 1, /* BF16 fine-level storage in the V-cycle, FP32 smoothing arithmetic,
                                   FP64 solution and exact FP64 residuals */
  OTM_PRECISION_MIXED_FP16 = 2  /* the same with FP16 storage (residual scaled to max 1) */
} otm_precision;

typedef enum otm_smoother {
  OTM_SMOOTHER_COLOR = 0, /* one launch per colour pair over the whole level: the reference's global
                             colour order (homogenization/grid.cu:318-471) */
  OTM_SMOOTHER_TILED = 1  /* fine level in 16 x 16 x 8 shared-memory tiles, one launch per sweep:
                             colour-ordered Gauss-Seidel inside a tile, the tile halo held at the
                             sweep's starting values, consecutive sweeps on two tilings shifted by
                             half a tile; used with the PCG solver, at least 2 sweeps in each leg,
                             and nx, ny multiples of 16 and nz of 8, else the colour passes */
} otm_smoother;

typedef enum otm_solver {
  OTM_SOLVER_PCG = 0,   /* conjugate gradients preconditioned by one symmetric V-cycle */
  OTM_SOLVER_VCYCLE = 1 /* stationary V-cycles as MG_H::solveEquation (homogenization/MG.cpp:80-142) */
} otm_solver;

/* Solver configuration; the fields mirror cfg::HomoConfig (cmdline.h:12-33) where one
 * exists. Fill with otm_config_init() and then override. */
typedef struct otm_config {
  int reso[3];           /* cells per axis; HomoConfig::reso (cmdline.h:171); each <= 1024 */
  double fem_rel_thres;  /* ||f - A u||_2 / (||f||_2 + 1e-10) target; HomoConfig::femRelThres, default 0.01 */
  int max_iter;          /* iteration cap per solve; default 200 (homogenization/MG.cpp:382) */
  int pre_smooth;        /* GS sweeps before restriction; default 1 (MG.h:282) */
  int post_smooth;       /* GS sweeps after prolongation; default 1 */
  int solver;            /* otm_solver; default OTM_SOLVER_PCG */
  int precision;         /* otm_precision; default OTM_PRECISION_FP32 */
  int coarsest_max_dof;  /* coarsen while the level has more unknowns than this; default 64 */
  float power_penal;     /* k_solver = 1e-9 + k^power_penal; Homogenization_H::power_penal, default 1 */
  int warm_start;        /* reuse the previous solutions as initial guesses; default 1 (homogenization.cu:184) */
  int check_every;       /* iterations between host convergence checks; default 4 */
  int use_graphs;        /* capture the iteration loop in a CUDA graph; default 1 */
  int profile;           /* time the first fine-level post-smoothing sweep of every iteration with CUDA
                            events recorded inside the graph; default 0 */
  int cluster_cycle;     /* run the lower levels and the coarsest solve in one thread-block-cluster
                            launch when they fit, from the first level with <= 16^3 unknowns (2) or
                            <= 32^3 (3); 1: 16^3 when the level above it is tile-smoothed, else
                            32^3; 0: per-level kernels only; default 1 */
  int smoother;          /* otm_smoother of the fine level; default OTM_SMOOTHER_TILED */
} otm_config;

typedef struct otm_solve_stats {
  int iterations;         /* PCG iterations or V-cycles of the last solve (all 3 cases together) */
  int refinements;        /* mixed precision: FP64 residual evaluations r = b - A x64 (with the PCG
                             solver the start and every exact residual replacement; with the
                             V-cycle solver one per refinement step), else 0 */
  double rel_res[3];      /* final ||r|| / (||f|| + 1e-10) per load case */
  int status;             /* otm_status of the last solve */
  int levels;             /* multigrid levels */
  int coarsest_reso[3];   /* coarsest level cells per axis */
  int cluster_level;      /* first level of the one-launch cluster cycle, -1 when not used */
  int smoother;           /* otm_smoother the fine level runs with (OTM_SMOOTHER_TILED only with the PCG
                             solver, at least 2 sweeps per leg and nx, ny multiples of 16, nz of 8) */
} otm_solve_stats;

/* Event-timed fine-level smoother sweeps collected while profile != 0. */
typedef struct otm_profile {
  int sweeps;             /* sweeps timed (iterations that ran) */
  double sweep_ms;        /* total milliseconds of those sweeps (launches_per_sweep launches each) */
  double sweep_bytes;     /* algorithmic bytes of one sweep: nv * (4 + 3 * (4 + 4 + 4)) in FP32 */
  int launches_per_sweep; /* kernel launches per sweep */
  int kernel_kind;        /* 0: the timed region is one colour-pair sweep (launches_per_sweep passes);
                             1: it is the tiled post-smoothing leg (prolongation + post_smooth sweeps, one
                             launch per sweep), sweep_bytes then being that leg's algorithmic bytes */
} otm_profile;

/* Pitched 3-D device array, layout-identical to cudaPitchedPtr. */
typedef struct otm_pitched_ptr {
  void* ptr;
  size_t pitch; /* bytes per row */
  size_t xsize; /* bytes of valid data per row */
  size_t ysize; /* rows */
} otm_pitched_ptr;

OTM_API const char* otm_status_string(otm_status s);
/* Message of the last failing call on this host thread ("" if none). */
OTM_API const char* otm_last_error(void);
OTM_API int otm_abi_version(void);

/* Defaults of cfg::HomoConfig::init (cmdline.cpp:4-35) that apply to the solve. */
OTM_API otm_status otm_config_init(otm_config* cfg);

/* ---- Homogenization_H (homogenization/homogenization.h:15-30) ---- */
typedef struct otm_homo otm_homo;

/* Homogenization_H::Homogenization_H / build (homogenization/homogenization.cpp:31-63,
 * MG_H::build homogenization/MG.cpp:13-44): builds the multigrid hierarchy, allocates all
 * device buffers once. */
OTM_API otm_status otm_homo_create(const otm_config* cfg, otm_homo** out);
OTM_API otm_status otm_homo_destroy(otm_homo* h);
/* All later GPU work of the handle runs on this cudaStream_t (NULL = legacy default stream). */
OTM_API otm_status otm_homo_set_stream(otm_homo* h, void* stream);
OTM_API otm_status otm_homo_get_config(const otm_homo* h, otm_config* cfg);
OTM_API otm_status otm_homo_set_tolerance(otm_homo* h, double fem_rel_thres);

/* Homogenization_H::update(float* rho, int pitchT) (homogenization/homogenization.cpp:76-81):
 * imports the conductivity field (device, x fastest, element (x,y,z) at
 * x + (y + z*ny)*pitchT; pitchT <= 0 means nx) and rebuilds the coarse Galerkin operators
 * (MG_H::updateStencils, homogenization/MG.cpp:144-151). */
OTM_API otm_status otm_homo_update(otm_homo* h, const float* k_dev, int pitchT);

/* otm_density_forward followed by otm_homo_update with its k, in fewer passes: the density chain's
 * forward pass (filter, SIMP map; arguments as otm_density_forward, on the handle's stream) writes
 * the conductivities straight into the handle (the conductivity import of Grid_H::update folded
 * into the pow/affine epilogue of the filter, TensorExpression.h:816-843), then the coarse
 * operators are rebuilt. rho_f may be NULL; dk and wsum are written for otm_density_backward. */
OTM_API otm_status otm_homo_update_density(otm_homo* h, const int reso[3], const float* rho, int rho_pitchT,
                                           float* rho_f, float* dk, float* wsum, int weight_type, float radius,
                                           int periodic, float p, float k0, float kmin);

/* MG_H::solveEquation for the 3 load cases at once (homogenization/MG.cpp:80-142 called per
 * case at homogenization/homogenization.cu:182-188); warm-started unless disabled. */
OTM_API otm_status otm_homo_solve(otm_homo* h, otm_solve_stats* stats);

/* Homogenization_H::heatMatrix(double C[3][3]) (homogenization/homogenization.cu:180-252):
 * solves the 3 load cases and returns the effective conductivity tensor, row-major, in the
 * reference's load-case convention, with FP64 accumulation. */
OTM_API otm_status otm_homo_heat_matrix(otm_homo* h, double C[9]);

/* K^H of the current solutions without solving again. */
OTM_API otm_status otm_homo_heat_matrix_nosolve(otm_homo* h, double C[9]);

/* Homogenization_H::Sensitivity(float dC[3][3], float* sens, int pitchT, bool lexiOrder)
 * (homogenization/homogenization.cu:415-479): sens_e = p k^(p-1) sum_{i<=j} E_ij(e)
 * (dC_ij + [i!=j] dC_ji). lexi != 0 writes element (x,y,z) at x + (y + z*ny)*pitchT (the
 * reference's lexiOrder = true layout); lexi == 0 writes it unpitched. */
OTM_API otm_status otm_homo_sensitivity(otm_homo* h, const float dC[9], float* sens_dev, int pitchT, int lexi);

/* otm_homo_heat_matrix and otm_homo_sensitivity(dC) in one element pass (the sensitivity kernel
 * Sensitivity_kernel_opt_2_H fused with the K^H kernel, homogenization/homogenization.cu:13-153,
 * 255-412) for a dC that does not depend on C (a linear objective such as the OC loop's
 * -trace K^H): solves, then one kernel emits C and sens_dev exactly as the two calls would. */
OTM_API otm_status otm_homo_heat_matrix_sensitivity(otm_homo* h, double C[9], const float dC[9], float* sens_dev,
                                                    int pitchT, int lexi);

/* dK^H_ij / dk_e for the 6 unique pairs (00 01 02 11 12 22), 6 unpitched fields of ne floats. */
OTM_API otm_status otm_homo_element_energy(otm_homo* h, float* energy_dev);

/* MG_H::v_cycle(w_SOR, pre, post) (homogenization/MG.cpp:46-71): one V(pre, post) cycle of the
 * handle's hierarchy (built by the last otm_homo_update) applied to the right-hand sides f_dev of
 * the 3 load cases (3 * nv device floats, case-major, x fastest) from a zero correction; the
 * correction is written to u_dev (3 * nv floats). FP32 form only (OTM_ERR_UNSUPPORTED for the
 * 16-bit forms, whose cycle works on scaled residuals); the smoother is Gauss-Seidel (w_SOR = 1). */
OTM_API otm_status otm_homo_v_cycle(otm_homo* h, const float* f_dev, float* u_dev, int pre, int post);

/* One level of the hierarchy (Grid_H, homogenization/grid.h:104-421): level 0 is the root. */
typedef struct otm_level_info {
  int levels;      /* levels of the hierarchy */
  int reso[3];     /* cells (= periodic vertices) per axis of this level */
  int stencil;     /* 1: the level holds assembled 27-point Galerkin stencils; 0: matrix-free */
  int smoother;    /* otm_smoother of the level (the tile kernels or colour passes); -1: solved
                      directly, in one cluster launch or in the single-CTA cycle */
} otm_level_info;
OTM_API otm_status otm_homo_level(const otm_homo* h, int level, otm_level_info* info);

/* The periodic fluctuation chi of load case c (nv floats, x fastest), as kept in
 * Grid_H::uchar_h (homogenization/grid.cpp:200-211). */
OTM_API otm_status otm_homo_get_solution(otm_homo* h, int lcase, float* dst_dev);
OTM_API otm_status otm_homo_set_solution(otm_homo* h, int lcase, const float* src_dev);
/* MG_H::reset_displacement (homogenization/MG.cpp:73-78): zero the kept solutions. */
OTM_API otm_status otm_homo_reset_displacement(otm_homo* h);
OTM_API otm_status otm_homo_get_stats(const otm_homo* h, otm_solve_stats* stats);
/* Profile counters (see otm_config.profile); reset != 0 clears them after reading. */
OTM_API otm_status otm_homo_get_profile(otm_homo* h, otm_profile* prof, int reset);

/* Kernels this library has launched in the process (graph replays count their kernel nodes). */
OTM_API uint64_t otm_launch_count(void);
/* Temporary device buffers the handle-free entry points (OC update and filter, MMA subsolver,
 * server task tables) have taken from the library's scratch memory pool in this process; no
 * reference counterpart (a diagnostic: an entry point that allocates nothing leaves it unchanged). */
OTM_API uint64_t otm_scratch_alloc_count(void);

/* Page-locked host memory for the arrays a caller moves to and from the device every step
 * (the densities and sensitivities of an optimisation loop): allocated with cudaHostAlloc, so
 * host-to-device copies from it run at the link rate (on the B200 systems measured, 53 GB/s for
 * 8 MB, against 16 GB/s from pages pinned after allocation). Free with otm_host_free. */
OTM_API otm_status otm_host_alloc(size_t bytes, void** out);
OTM_API otm_status otm_host_free(void* p);
/* The per-step transfers themselves: one cudaMemcpyAsync on `stream` (asynchronous from
 * page-locked host memory). */
OTM_API otm_status otm_copy_to_device(void* dst_dev, const void* src_host, size_t bytes, void* stream);
OTM_API otm_status otm_copy_to_host(void* dst_host, const void* src_dev, size_t bytes, void* stream);

/* ---- density filter chain (AutoDiff/TensorExpression.h:640-644, 993-1185; .cuh:281-385) ---- */
#define OTM_WEIGHT_SPLINE4 0
#define OTM_WEIGHT_LINEAR 1

/* conv_kernel (AutoDiff/TensorExpression.cuh:304-350): dst = sum w src / sum_valid w, radial
 * weights normalised over the full (2h+1)^3 cube, h = int(radius + 0.5); wsum (optional, may
 * be NULL) receives sum_valid w per voxel. Arrays are pitched like otm_homo_update. */
OTM_API otm_status otm_filter_forward(const int reso[3], const float* src, int src_pitchT, float* dst, int dst_pitchT,
                              float* wsum, int weight_type, float radius, int periodic, void* stream);
/* conv_backward_kernel (AutoDiff/TensorExpression.cuh:353-385): the adjoint, needs the wsum
 * written by the forward pass. */
OTM_API otm_status otm_filter_backward(const int reso[3], const float* g_dst, int g_dst_pitchT, const float* wsum,
                               float* g_src, int g_src_pitchT, int weight_type, float radius, int periodic,
                               void* stream);

/* Fused density chain of runCustom (Framework.cu:163): rho_f = filter(rho);
 * k = (k0 - kmin) rho_f^p + kmin, dk = d k / d rho_f (pow_umker_t, TensorExpression.h:816-843,
 * affine map). k and dk are unpitched (pitchT = nx); wsum as in otm_filter_forward. */
OTM_API otm_status otm_density_forward(const int reso[3], const float* rho, int rho_pitchT, float* rho_f, float* k,
                               float* dk, float* wsum, int weight_type, float radius, int periodic, float p,
                               float k0, float kmin, void* stream);
/* Chain rule back to rho: g_rho = filter^T(g_k * dk) (unarymap_backward + conv_backward_kernel). */
OTM_API otm_status otm_density_backward(const int reso[3], const float* g_k, const float* dk, const float* wsum,
                                float* g_rho, int g_rho_pitchT, int weight_type, float radius, int periodic,
                                void* stream);

/* ---- OCOptimizer (optimization/OCOptimizer.h:7-20) ---- */
/* OCOptimizer::filterSens (optimization/OCOptimizer.cu:134-152): periodic Linear filter
 * s_e <- sum_n w s_n rho_n / (sum_n w * rho_e), in place. */
OTM_API otm_status otm_oc_filter_sens(float* sens, const float* rho, size_t pitchT, const int reso[3], float radius,
                              void* stream);
/* OCOptimizer::update (optimization/OCOptimizer.cu:38-67): <= 20 bisection steps on the OC
 * multiplier, run entirely on the device; iters_out (optional) gets the steps used. */
OTM_API otm_status otm_oc_update(int ne, const float* sens, float* rho, float volratio, float min_rho, float step_limit,
                         float damp, void* stream, int* iters_out);

#ifdef __cplusplus
}
#endif

#endif /* OPENTM_B200_H */
