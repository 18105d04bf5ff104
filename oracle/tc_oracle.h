/*
 * tc_oracle.h -- CPU restatement (FP64, plain C + OpenMP) of TC++'s
 * operator-application hot path.  TEST INFRASTRUCTURE ONLY: it is the
 * checker the CUDA library is compared against, and the timed CPU baseline.
 * Nothing in the product (tc_b200/, libtcg_b200.so) links or calls it.
 *
 * Parity status: the reference (masaochi/TC) cannot be built in this
 * environment (no MPI, FFTW3, Eigen3 or Boost), and its own tests pin only
 * end-to-end SCF energies, so this restatement is "parity unpinned" with
 * respect to the reference binary.  It is cross-checked instead against
 * numpy.fft (FFT conventions), against direct G-space sums for plane-wave
 * orbitals (known answers), and against exact algebraic identities.
 *
 * The descriptors are the library's own (include/tcg.h), so the same inputs
 * drive both implementations.
 */
#ifndef TC_ORACLE_H
#define TC_ORACLE_H

#include <stdint.h>
#include "../include/tcg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* 3D complex FFT in place on an interleaved (re,im) grid, x fastest.
 * forward != 0: exp(-iGr)/N ; forward == 0: exp(+iGr) unscaled
 * (plane_wave_basis.cpp:274-289). */
int tco_fft3d(const int32_t nr[3], double *grid, int forward);

/* Jastrow RPA u(G) and TC two-body potential V_2body(G)
 * (jastrow_functions.cpp:6-97).  G Cartesian (bohr^-1). */
double tco_uk(const tcg_system_desc *sys, const double G[3], int s1, int s2);
double tco_tc2body(const tcg_system_desc *sys, const double G[3], int s1, int s2);

/* calc_hamiltonian::{hf2x,hf2h,tc2x,tc2h,tc3a1,tc3b1,tc3a2a4b2b5,
 * tc3a3b3b4b6} restated; arguments as tcg_apply (accumulating into h2 / h3). */
int tco_apply(const tcg_system_desc *sys, const tcg_state_desc *st,
              uint32_t term_mask, const int32_t *nb_apply,
              const double *psi, double *h2, double *h3, const uint8_t *owned);

/* calc_hamiltonian::kinetic / pseudo restated (TCG_TERM_KINETIC,
 * TCG_TERM_PSEUDO), accumulating into h1; pp may be NULL without PSEUDO. */
int tco_apply_h1(const tcg_system_desc *sys, const tcg_pseudo_desc *pp, uint32_t term_mask,
                 const int32_t *nb_apply, const double *psi, double *h1, const uint8_t *owned);

/* BlochStates::set_density, first SCF iteration. */
int tco_density(const tcg_system_desc *sys, const tcg_state_desc *st, double *density_out);

/* Potentials::set_sum_of_Vaux_each on the SCF mesh. */
int tco_sum_of_vaux(const tcg_system_desc *sys, double *alpha_out, double *sum_vaux_out);

/* OpenMP thread count used by the oracle (<= 0: runtime default). */
void tco_set_threads(int n);
int tco_get_threads(void);

/* Timing-sample mode (CPU baseline only): visit every s-th source k-point
 * in the q-sums (results become partial sums); timers of the shared
 * occupied-pair stage, of whole tco_apply calls and of their set-up
 * (R-space occupied orbitals), in seconds. */
void tco_set_qstride(int s);
void tco_timers(double *shared, double *total, double *init);
void tco_reset_timers(void);

const char *tco_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
