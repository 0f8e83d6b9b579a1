/*
 * opentm_b200_mma.h -- MMA (method of moving asymptotes) of the B200 library, FP64 on the
 * device. Replaces MMAOptimizer (optimization/mmaOptimizer.h:12-35) and mmasubDevice
 * (optimization/mmaOpt.h:14-19). Uses the types of opentm_b200.h.
 */
#ifndef OPENTM_B200_MMA_H
#define OPENTM_B200_MMA_H

#include "opentm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Largest number of constraints m supported by the device subsolver. */
#define OTM_MMA_MAX_CONSTRAINTS 8

typedef struct otm_mma otm_mma;

/* MMAOptimizer(nconstrain, nvar, a0, a, c, d) (optimization/mmaOptimizer.cu:18-42): a, c, d
 * are replicated over the m constraints. */
OTM_API otm_status otm_mma_create(int m, int n, double a0, double a, double c, double d, otm_mma** out);
OTM_API otm_status otm_mma_destroy(otm_mma* mma);
/* All later GPU work of the optimizer is ordered on this cudaStream_t (NULL = legacy default). */
OTM_API otm_status otm_mma_set_stream(otm_mma* mma, void* stream);
/* MMAOptimizer::setBound(float xmin, float xmax) (optimization/mmaOptimizer.cu:50-54). */
OTM_API otm_status otm_mma_set_bound_scalar(otm_mma* mma, float xmin, float xmax);
/* MMAOptimizer::setBound(float* xmin, float* xmax) (optimization/mmaOptimizer.cu:44-48): device arrays of n. */
OTM_API otm_status otm_mma_set_bound(otm_mma* mma, const float* xmin_dev, const float* xmax_dev);
/* MMAOptimizer::update(itn, x, dfdx, gval, dgdx) (optimization/mmaOptimizer.cu:61-78): x, dfdx and
 * dgdx[i] are FP32 device arrays of n values, gval a host array of m values. x is updated in
 * place; f0val = 1 and move = 1 as in the reference. */
OTM_API otm_status otm_mma_update(otm_mma* mma, int itn, float* x_dev, const float* dfdx_dev,
                                  const float* gval_host, const float* const* dgdx_dev);

/* mmasubDevice (optimization/mmaOpt.h:14-19, mmaOpt.cpp:38-46, mmasub_g mmaOpt.cu:1021-1062) with
 * the same argument order: every array is FP64 device memory; dgdx is pitched with m rows of n
 * values; gval, a, c, d hold m values. Updates xvar, xold1, xold2, low and upp in place. */
OTM_API otm_status otm_mmasub_device(int m, int n, int itn, double* xvar, double* xmin, double* xmax,
                                     double* xold1, double* xold2, double f0val, double* df0dx, double* gval,
                                     otm_pitched_ptr dgdx, double* low, double* upp, double a0, double* a,
                                     double* c, double* d, double move, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* OPENTM_B200_MMA_H */
