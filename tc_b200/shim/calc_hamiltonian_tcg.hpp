// calc_hamiltonian_tcg.hpp -- TC++ drop-in on top of libtcg_b200.so.
//
// calc_hamiltonian_tcg.cpp defines TC++'s six operator routines
// (src/include/calc_hamiltonian.hpp:54-130: hf2x, tc2x, tc3a1, tc3b1,
// tc3a3b3b4b6, tc3a2a4b2b5) with their exact signatures on top of the C-ABI
// of include/tcg.h, plus the helpers below.  Inside TC++ the six routines are
// declared by calc_hamiltonian.hpp; TCG_SHIM_STANDALONE builds the shim
// against tcpp_standin.hpp instead (tests, examples).
#pragma once
#ifdef TCG_SHIM_STANDALONE
#include "tcpp_standin.hpp"
#else
#include "include/header.hpp"
#endif
#include <cstdint>
#include <ostream>

namespace tcg_shim {
using Orbitals = std::vector<std::vector<std::vector<std::vector<Eigen::VectorXcd>>>>;

// Call once per SCF iteration, after BlochStates changed (set_density): the
// occupied orbitals, fillings and density are uploaded again on the next
// routine call.  BlochStates is const across every calc_hamiltonian::all
// call of one block_davidson call (diagonalization_davidson.cpp:228,242,433),
// so between two new_scf_iteration() calls the device copy is reused.
void new_scf_iteration();

// TCG_PREC_FP64 (default: the reference's arithmetic) or TCG_PREC_MIXED.
// Takes effect at the next context creation (call before the first routine).
void set_precision(int32_t precision);

// The whole two- plus three-body block of calc_hamiltonian::all
// (calc_hamiltonian_all.cpp:80-157) in one library call: hf2x for HF,
// tc2x + tc3a1 + tc3b1 + tc3a2a4b2b5 + tc3a3b3b4b6 for TC / BITC.  Accumulates
// into H2phi and H3phi (H3phi is untouched for HF).  One upload of phi and
// one R-space transform of it serve all five terms, where the per-routine
// entry points transform it once per routine.
void apply_two_three_body(const Parallelization &parallelization, const Method &method,
                          const CrystalStructure &crystal_structure, const Symmetry &symmetry,
                          const Potentials &potentials, const Spin &spin, const Kpoints &kpoints,
                          const PlaneWaveBasis &plane_wave_basis, const BlochStates &bloch_states,
                          const Orbitals &phi, Orbitals &H2phi, Orbitals &H3phi);

// Destroy the library context (end of the run).
void release();

// Kernels the library has launched so far (0 without a context).
int64_t launches();
} // namespace tcg_shim

#ifdef TCG_SHIM_STANDALONE
namespace calc_hamiltonian {
using tcg_shim::Orbitals;
void hf2x(const Parallelization &, const Method &, const CrystalStructure &, const Potentials &, const Spin &,
          const Kpoints &, PlaneWaveBasis &, const BlochStates &, const Orbitals &phi, Orbitals &H2phi, std::ostream *);
void tc2x(const Parallelization &, const Method &, const CrystalStructure &, const Potentials &, const Spin &,
          const Kpoints &, PlaneWaveBasis &, const BlochStates &, const Orbitals &phi, Orbitals &H2phi, std::ostream *);
void tc3a1(const Parallelization &, const Method &, const CrystalStructure &, const Potentials &, const Spin &,
           const Kpoints &, PlaneWaveBasis &, const BlochStates &, const Orbitals &phi, Orbitals &H3phi, std::ostream *);
void tc3b1(const Parallelization &, const Method &, const CrystalStructure &, const Potentials &, const Spin &,
           const Kpoints &, PlaneWaveBasis &, const BlochStates &, const Orbitals &phi, Orbitals &H3phi, std::ostream *);
void tc3a3b3b4b6(const Parallelization &, const Method &, const CrystalStructure &, const Potentials &, const Spin &,
                 const Kpoints &, PlaneWaveBasis &, const BlochStates &, const Orbitals &phi, Orbitals &H3phi,
                 std::ostream *);
void tc3a2a4b2b5(const Parallelization &, const Method &, const CrystalStructure &, const Symmetry &,
                 const Potentials &, const Spin &, const Kpoints &, PlaneWaveBasis &, const BlochStates &,
                 const Orbitals &phi, Orbitals &H3phi, std::ostream *);
} // namespace calc_hamiltonian
#endif
