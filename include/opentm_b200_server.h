/*
 * opentm_b200_server.h -- serving form of the B200 homogenization library: independent
 * homogenization requests of mixed cell sizes, submitted at any time, on one GPU. The reference
 * has no counterpart (it solves one cell per process, homogenization/homogenization.cu:180-252);
 * each request here is the same solve as otm_homo_heat_matrix from a zero initial guess.
 *
 * Two execution forms share this interface:
 *  - handle form (batched = 0, the default): up to `streams` requests run at once, each as one
 *    resident solver handle on its own CUDA stream with the whole Krylov loop as one device-side
 *    graph launch; handles stay resident per stream and cell size for the next request of that
 *    size (destroyed least recently used first when the memory budget needs room). A result is
 *    bitwise the same as otm_homo_heat_matrix of a handle created with the same settings and
 *    warm_start = 0.
 *  - batched form (batched = 1): up to max_active requests keep their multigrid hierarchies
 *    resident, and each scheduling step advances all of them together: the same multigrid
 *    operation on the same level of every running request is one kernel launch, and the Krylov
 *    updates of all requests are one launch each.
 * In both forms requests are admitted first come, first served while their resident state fits
 * the device-memory budget, and per-request reductions use a block partition that depends only
 * on the request's own size, so a result is bitwise the same whether the request runs alone or
 * among others.
 */
#ifndef OPENTM_B200_SERVER_H
#define OPENTM_B200_SERVER_H

#include "opentm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct otm_server otm_server;

typedef struct otm_server_config {
  size_t hbm_budget_bytes; /* admission budget for resident request state; default 150 GB */
  int max_active;          /* requests on the GPU at once; default 64 (at most 256) */
  double fem_rel_thres;    /* relative residual target of every solve; default 1e-6 */
  int max_iter;            /* iteration cap of every solve; default 200 */
  int pre_smooth;          /* = post_smooth; default 2 */
  int iters_per_step;      /* Krylov iterations between scheduling decisions; default 2 */
  float power_penal;       /* k_solver = 1e-9 + k^p; default 1 */
  int batched;             /* 0: handle form (default); 1: batched form */
  int streams;             /* handle form: requests running at once (one stream each); default 8,
                              at most 64, further capped by max_active */
  size_t host_stage_bytes; /* pinned host memory that holds submitted fields until their upload,
                              allocated at create; default 1 GiB; 0 = none. Fields that find it
                              full wait in pageable memory. */
} otm_server_config;

typedef struct otm_request_info {
  int state;             /* 0 queued, 1 running, 2 done, 3 cancelled, 4 failed */
  int status;            /* otm_status of a finished request */
  double submit_s;       /* host clock (seconds) at submit, admission and completion */
  double admit_s;
  double done_s;
  otm_solve_stats stats;
} otm_request_info;

OTM_API otm_status otm_server_config_init(otm_server_config* cfg);
/* cudaStream_t (NULL = legacy default) on which the server orders all its work. */
OTM_API otm_status otm_server_create(const otm_server_config* cfg, void* stream, otm_server** out);
OTM_API otm_status otm_server_destroy(otm_server* s);
/* Queue a solve of one periodic cell: k_host is a host array of reso[0]*reso[1]*reso[2]
 * conductivities (x fastest), copied at submit. Rejects with OTM_ERR_BUDGET a request that
 * could never fit the budget. */
OTM_API otm_status otm_server_submit(otm_server* s, const int reso[3], const float* k_host, int64_t* request_id);
/* One scheduling step: retire finished requests and admit queued ones that fit.
 * Handle form: admitted requests are queued on their streams and the call returns without
 * waiting for the GPU, except that while queued requests wait for a stream or for memory it
 * waits until some running request finishes (OTM_ERR_TIMEOUT after 600 s).
 * Batched form: then advances all running requests by iters_per_step batched iterations and
 * blocks until that work is done. */
OTM_API otm_status otm_server_step(otm_server* s, int* n_running, int* n_queued);
/* OTM_ERR_NOT_READY while queued or running; OTM_OK with K^H (9 doubles, reference load-case
 * convention) once done; the solve's own status if it failed. */
OTM_API otm_status otm_server_poll(otm_server* s, int64_t request_id, double C[9], otm_request_info* info);
/* Cancel a queued request, or a running one: the batched form drops it at the next step and
 * releases its memory; the handle form lets its solve finish, then reports it cancelled. */
OTM_API otm_status otm_server_cancel(otm_server* s, int64_t request_id);
/* Bytes of device memory a request of this size keeps resident while it runs. */
OTM_API size_t otm_server_request_bytes(const int reso[3]);
/* Device bytes currently held by running requests. */
OTM_API size_t otm_server_bytes_in_use(const otm_server* s);
/* Device bytes of all resident request state: running requests plus, in the handle form, the
 * idle handles kept for reuse. Never above hbm_budget_bytes. */
OTM_API size_t otm_server_bytes_resident(const otm_server* s);

#ifdef __cplusplus
}
#endif

#endif /* OPENTM_B200_SERVER_H */
