/*
 * CPU restatement of the teuk-kokkos linear RK4 right-hand-side path.
 * TEST INFRASTRUCTURE ONLY: the checker for the B200 engine's parity tests,
 * smoke() and the "port" CPU baseline.  Nothing in the product links it.
 *
 * It follows the reference algorithm in its own nodal storage
 * (mode, field, radial, theta), step by step:
 *   evaluate_rhs: SpatialPipeline::evaluate_rhs_at_time, Disabled policy
 *     (include/teuk/spatial_pipeline.hpp:458-515) = first-order angular
 *     Laplacian (angular_coordinator.hpp:151-174), the three full-stage
 *     Teukolsky kernels (full_spatial.hpp:99-398), band projection of P, Q,
 *     psi (spatial_pipeline.hpp:756-766) and zeroed frozen fields (:623-649);
 *   step: device_classical_rk4_step (include/teuk/device_rk4.hpp:84-128).
 * Pinned against the reference compiled from its own headers
 * (oracle/_ref, built by oracle/Makefile) and against the reference tests'
 * known-answer properties (SBP identity, Gauss-Legendre exactness).
 */
#ifndef TEUK_ORACLE_H
#define TEUK_ORACLE_H

#include <stddef.h>

#include "../include/teuk_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_pipeline oracle_pipeline;

const char* oracle_last_error(void);
int oracle_create(const teuk_b200_config* config, oracle_pipeline** out);
int oracle_destroy(oracle_pipeline* p);
int oracle_set_state(oracle_pipeline* p, const double* state, size_t count);
int oracle_get_state(oracle_pipeline* p, double* state, size_t count);
int oracle_evaluate_rhs(oracle_pipeline* p, const double* stage,
                        double* output, size_t count);
int oracle_step(oracle_pipeline* p, double dt, int steps);
int oracle_gauss_legendre(int nodes, double* x, double* weights);
int oracle_sbp_matrix(int disc, int n, double* derivative, double* norm);

#ifdef __cplusplus
}
#endif

#endif
