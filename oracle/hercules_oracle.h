/*
 * hercules_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of the HERCULES time step (single domain,
 * p_row = p_col = 1), used by tests/ and by bench.py's CPU baseline as the
 * checker. It is never linked into or called by the product library.
 *
 * Parity status: UNPINNED against reference runs. The reference (Fortran 90 +
 * MPI + FFTW 3.3.4 + 2DECOMP&FFT) cannot be compiled in this image (no gfortran,
 * no MPI) and ships no golden vectors or tests. The restatement is pinned instead
 * by analytic known-answer tests derived from the reference's own discretisation
 * (tests/test_oracle_kat.py); the fixtures in tests/golden/ (written by this
 * oracle) guard it against regressions.
 */
#ifndef HERCULES_ORACLE_H
#define HERCULES_ORACLE_H
#include "../include/hercules_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_state or_state;

or_state* or_create(const hc_params* p, int* err);
void      or_destroy(or_state* s);
int       or_get_grid(or_state* s, double* dz, double* l_t, double* l_b,
                      double* dz_t, double* dz_b);
int       or_set_field(or_state* s, int id, const double* interior);
int       or_get_field(or_state* s, int id, double* interior);
int       or_initialize(or_state* s);
int       or_step(or_state* s, int nsteps, hc_diag* diag);
void      or_set_threads(int n);
int       or_set_body_force(or_state* s, const double* fx, const double* fy, const double* fz);

/* unit-level entry points used by the known-answer tests */
int or_fft2d(int nx, int ny, int nz, double* c_interleaved, int direction);
int or_helmholtz_u(or_state* s, const double* rhs_interior, double* out_interior,
                   double rk_c);

#ifdef __cplusplus
}
#endif
#endif
