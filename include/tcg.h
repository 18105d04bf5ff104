/*
 * tcg.h -- C-ABI of the B200 operator-application library (libtcg_b200.so).
 *
 * The library applies the exchange / transcorrelated operator terms of a
 * plane-wave HF / TC / BITC calculation to a block of trial orbitals:
 *
 *   H2 psi += hf2x psi                         (HF)
 *   H2 psi += tc2x psi                         (TC, BITC)
 *   H3 psi += (tc3a1 + tc3b1 + tc3a2a4b2b5 + tc3a3b3b4b6) psi   (TC, BITC)
 *
 * It replaces the six routines declared in TC++'s
 * src/include/calc_hamiltonian.hpp:54-130 (hf2x, tc2x, tc3a1, tc3b1,
 * tc3a3b3b4b6, tc3a2a4b2b5).  Those take nested
 * std::vector<...<Eigen::VectorXcd>> containers; here every container is a
 * flat, packed array of interleaved (re, im) doubles -- the memory layout of
 * std::complex<double> / Eigen::VectorXcd -- so the reference's C++ host can
 * pass its buffers after one memcpy per band.
 *
 * Conventions (all follow TC++):
 *  - FFT grid nr[0] x nr[1] x nr[2], x = nr[0] fastest; grid index
 *    i0 + nr0*(i1 + nr1*i2)  (plane_wave_basis.cpp:205-216, :158-161).
 *  - Forward FFT (R -> G) is exp(-iGr) scaled by 1/N; backward (G -> R) is
 *    exp(+iGr) unscaled (plane_wave_basis.cpp:274-289).
 *  - Orbital coefficients are normalised so that sum_G |c_G|^2 = 1.
 *  - Vectors k are fractional (crystal) coordinates; Cartesian = recip^T k,
 *    with recip's rows the reciprocal vectors b_i (bohr^-1, 2pi included,
 *    crystal_structure.hpp:16).
 *  - Spin: nspin = num_independent_spins (1 = unpolarised, 2 = polarised).
 *    density[] always holds two spin channels (bloch_states.hpp).
 *
 * Scope: calc_mode "SCF" with every k-point of non-zero weight (the SCF mesh),
 * no density-matrix mixing (filling_old empty), RPA Jastrow.  In that case
 * TC++'s sum_of_kVaux vanishes for every k (potentials_coulomb.cpp:186-190),
 * so the kVaux-weighted divergence corrections of tc2x / tc3a3b3b4b6 /
 * tc3a2a4b2b5 are identically zero and are not part of this interface.
 *
 * Errors: every entry point returns an int status (TCG_OK = 0).  The library
 * never aborts the process; tcg_last_error() returns a message for the
 * calling thread's most recent failure.
 */
#ifndef TCG_H
#define TCG_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define TCG_OK               0
#define TCG_ERR_ARG          1   /* invalid argument / inconsistent sizes        */
#define TCG_ERR_CUDA         2   /* CUDA runtime error (message has details)     */
#define TCG_ERR_TIMEOUT      3   /* a bounded device-side wait ran out           */
#define TCG_ERR_UNSUPPORTED  4   /* valid input outside the implemented scope    */
#define TCG_ERR_STATE        5   /* call order violated (e.g. apply before set)  */
#define TCG_ERR_NOMEM        6   /* device allocation failed                     */
#define TCG_ERR_NUMERIC      7   /* non-finite value detected in an input        */

/* ---- methods / precision --------------------------------------------- */
#define TCG_METHOD_HF    0
#define TCG_METHOD_TC    1
#define TCG_METHOD_BITC  2

#define TCG_PREC_FP64    0   /* complex128 everywhere                          */
#define TCG_PREC_MIXED   1   /* complex64 FFTs / pair products, FP64 accumulation */

/* ---- term mask ----------------------------------------------------------
 * Bit i selects one of the reference routines.  hf2x and tc2x add to H2,
 * the tc3* terms add to H3 (calc_hamiltonian_all.cpp:80-157). */
#define TCG_TERM_HF2X          (1u << 0)
#define TCG_TERM_TC2X          (1u << 1)
#define TCG_TERM_TC3A1         (1u << 2)
#define TCG_TERM_TC3B1         (1u << 3)
#define TCG_TERM_TC3A2A4B2B5   (1u << 4)
#define TCG_TERM_TC3A3B3B4B6   (1u << 5)
#define TCG_TERMS_HF   (TCG_TERM_HF2X)
#define TCG_TERMS_TC   (TCG_TERM_TC2X | TCG_TERM_TC3A1 | TCG_TERM_TC3B1 | \
                        TCG_TERM_TC3A2A4B2B5 | TCG_TERM_TC3A3B3B4B6)
/* Hartree-type two-body terms (local potentials of the density, added to H2):
 * hf2h (calc_hamiltonian_hf2h.cpp:7-85) for HF, tc2h
 * (calc_hamiltonian_tc2h.cpp:10-235) for TC / BITC. */
#define TCG_TERM_HF2H          (1u << 6)
#define TCG_TERM_TC2H          (1u << 7)
/* One-body terms, applied by tcg_apply_h1 into H1: kinetic
 * (calc_hamiltonian_kinetic.cpp:6-52) and pseudopotential, local + non-local
 * (calc_hamiltonian_pseudo.cpp:6-180; data from tcg_set_pseudo). */
#define TCG_TERM_KINETIC       (1u << 8)
#define TCG_TERM_PSEUDO        (1u << 9)
#define TCG_TERMS_H1   (TCG_TERM_KINETIC | TCG_TERM_PSEUDO)
#define TCG_TERMS_H2   (TCG_TERM_HF2X | TCG_TERM_TC2X | TCG_TERM_HF2H | TCG_TERM_TC2H)

/* ---- static system description (one per run) ----------------------------
 * "nk_all" below is sum_k nsym_k (Kpoints::num_kpoints_all_scf).  Arrays
 * indexed by an "all-k" index a list the equivalent k-points irreducible-
 * major: a = (sum_{k'<ik} nsym_k[k']) + isym, the order of
 * Kpoints::index_all_kscf (kpoints.cpp:82-91). */
typedef struct tcg_system_desc {
    int32_t nr[3];               /* FFT grid (nr1, nr2, nr3)                   */
    double  recip[9];            /* reciprocal vectors b_i as rows (bohr^-1)   */
    double  lattice[9];          /* lattice vectors a_i as rows (bohr)         */
    double  omega;               /* unit-cell volume (bohr^3)                  */
    int32_t calc_method;         /* TCG_METHOD_*                               */
    int32_t nspin;               /* num_independent_spins: 1 or 2              */
    int32_t nk_irr;              /* irreducible SCF k-points                   */
    int32_t num_kpoints;         /* Kpoints::num_kpoints()                     */
    const int32_t *nsym_k;       /* [nk_irr] kvectors_scf[ik].size()            */
    const double  *kvec;         /* [nk_all][3] fractional k                    */
    const uint8_t *time_rev;     /* [nk_all] is_time_reversal_used_at_k         */
    const int32_t *rot_index;    /* [nk_all] index_of_rotation_at_k             */
    int32_t nsymop;              /* Symmetry::num_symmetry_operations           */
    const int32_t *rotation;     /* [nsymop][3][3] U, row-major, crystal coords */
    const double  *translation;  /* [nsymop][3] fractional translations         */
    const int32_t *npw;          /* [nk_irr] num_G_at_k_scf                     */
    const int32_t *gindex;       /* [nspin][nk_all][npw of its ik] Gindex_at_k_scf */
    const double  *phase;        /* [nspin][nk_all][npw] complex phase_factor_at_k */
    double  jastrow_A[4];        /* A_long[s1][s2], row-major (atomic units)   */
    double  jastrow_F[4];        /* F_long[s1][s2]                              */
    int32_t includes_div_correction;
    double  alpha_Vaux;          /* Potentials::alpha_Vaux                      */
    const double *sum_Vaux;      /* [nk_irr] Potentials::sum_of_Vaux_scf        */
} tcg_system_desc;

/* ---- per-SCF-iteration state (BlochStates) --------------------------------
 * phik[s][ik][b] holds num_bands_scf[s] bands of npw[ik] coefficients; the
 * first nocc[s][ik] carry the occupied orbitals summed over in the exchange
 * terms, fillings >= 1e-8 enter the divergence corrections (as TC++). */
typedef struct tcg_state_desc {
    const int32_t *nbands;       /* [nspin] num_bands_scf                       */
    const int32_t *nocc;         /* [nspin][nk_irr] num_occupied_bands          */
    const double  *filling;      /* [nspin][nk_irr][nbands[s]]                  */
    const double  *phik;         /* [nspin][nk_irr][nbands[s]][npw] complex     */
    const double  *phik_left;    /* BITC: same layout (left orbitals); else NULL */
    const double  *density;      /* [2][N] complex, R-space (set_density)       */
} tcg_state_desc;

/* ---- pseudopotential (Potentials, one per run) ---------------------------
 * What calc_hamiltonian::pseudo reads (calc_hamiltonian_pseudo.cpp:6-180):
 * the local potential on the FFT grid and, per irreducible k, the non-local
 * projectors <beta|k+G> of every species as Potentials::projector_nonlocal
 * returns them (without the exp(i G.R_atom) factor, which is applied here). */
typedef struct tcg_pseudo_desc {
    const double  *vloc;            /* [N] Potentials::Vpp_local (real, R space) or NULL */
    int32_t nspecies, natoms;
    const int32_t *species_of_atom; /* [natoms] CrystalStructure::index_of_atoms */
    const double  *atom_pos;        /* [natoms][3] atomic_position_cartesian (bohr) */
    const int32_t *nproj;           /* [nspecies] pseudo_lbeta[is].size()          */
    const int32_t *lbeta;           /* [sum nproj] pseudo_lbeta                     */
    const double  *dij;             /* [sum nproj^2] pseudo_dij[is](i, j) row-major */
    const double  *projector;       /* complex [nk_irr][sum_is sum_ip (2 l + 1)][npw of k]:
                                       projector[is][ip][m] at the isym-0 plane waves of k */
} tcg_pseudo_desc;

/* Opaque context: device copies of the system and state, FFT plans, scratch. */
typedef struct tcg_ctx tcg_ctx;

/* Create a context on the current CUDA device.  precision = TCG_PREC_*.
 * Replaces the per-call setup the reference repeats inside every routine
 * (G-vector tables, Jastrow tables; e.g. calc_hamiltonian_hf2x.cpp:32-37). */
int tcg_ctx_create(const tcg_system_desc *sys, int32_t precision, tcg_ctx **out);
int tcg_ctx_destroy(tcg_ctx *ctx);

/* Upload the occupied orbitals / fillings / density of one SCF iteration.
 * BlochStates is const across all calc_hamiltonian::all calls of one
 * Davidson call (diagonalization_davidson.cpp:228,242,433), so the R-space
 * occupied orbitals are built once here and reused by every apply. */
int tcg_set_state(tcg_ctx *ctx, const tcg_state_desc *st);

/* Redo the per-state work of the last tcg_set_state from the device-resident
 * copy (R-space orbitals, local three-body potentials, and -- on the next
 * apply -- the tc3a2a4b2b5 occupied-pair stage), without a host upload.
 * Equivalent to calling tcg_set_state again with the same arrays. */
int tcg_refresh_state(tcg_ctx *ctx);

/* Apply the selected terms to a block of trial orbitals and ACCUMULATE into
 * h2 / h3 (the reference's "+=" semantics; the caller zeroes them first as
 * calc_hamiltonian_all.cpp:29-49 does).  H2 terms: hf2x, hf2h (HF) or tc2x,
 * tc2h (TC / BITC); H3 terms: the four tc3* routines.
 *   nb_apply : [nspin][nk_irr] bands per (spin, k)  (H2phi[ispin][ik].size())
 *   psi      : [nspin][nk_irr][nb_apply][npw] complex, packed
 *   h2, h3   : same layout as psi; h3 may be NULL for HF, h2 NULL if no
 *              H2 term is selected
 *   owned    : [nspin][nk_irr][nb_apply] bytes; 0 = band owned by another rank
 *              (Parallelization::is_assigned_irreducible_kpoints_all_bands);
 *              NULL = all owned.
 * Host pointers.  Replaces calc_hamiltonian::hf2x / tc2x / tc3a1 / tc3b1 /
 * tc3a2a4b2b5 / tc3a3b3b4b6 (calc_hamiltonian.hpp:54-130). */
int tcg_apply(tcg_ctx *ctx, uint32_t term_mask, const int32_t *nb_apply,
              const double *psi, double *h2, double *h3, const uint8_t *owned);

/* One-body terms (TCG_TERM_KINETIC, TCG_TERM_PSEUDO) applied to psi and
 * ACCUMULATED into h1 (host pointers, layout of tcg_apply).  Replaces
 * calc_hamiltonian::kinetic (calc_hamiltonian_kinetic.cpp:6-52) and
 * calc_hamiltonian::pseudo (calc_hamiltonian_pseudo.cpp:6-180); the
 * pseudopotential needs tcg_set_pseudo first. */
int tcg_apply_h1(tcg_ctx *ctx, uint32_t term_mask, const int32_t *nb_apply,
                 const double *psi, double *h1, const uint8_t *owned);

/* Upload the pseudopotential data (once per run).  Fails with TCG_ERR_ARG
 * if pseudo_dij couples projectors of different l (as the reference). */
int tcg_set_pseudo(tcg_ctx *ctx, const tcg_pseudo_desc *pp);

/* Same as tcg_apply but psi / h2 / h3 are DEVICE pointers (layout as above)
 * and the work is queued on the context's stream without a host sync. */
int tcg_apply_device(tcg_ctx *ctx, uint32_t term_mask, const int32_t *nb_apply,
                     const void *psi_dev, void *h2_dev, void *h3_dev,
                     const uint8_t *owned);

/* Two- and three-body energies of the applied bands, reduced on the device in
 * FP64 (TotalEnergy::calc_total_energy, total_energy.cpp:101-168):
 *   E_n = sum_{s, k, isym, b} f_b e_n(b) / (n N_k),  n = 2, 3,
 *   e_n(b) = <chi_kb | h_n b>  (conjugated for time-reversed images),
 * where chi_kb is band b of the current state's left (BITC) or right
 * orbitals and h2_dev / h3_dev are DEVICE arrays in the packed layout of
 * tcg_apply with nb_apply bands per (spin, k) -- e.g. the outputs of
 * tcg_apply_device with psi = the occupied orbitals.  Either may be NULL
 * (that energy is then 0).  Bands b >= nbands or with zero filling are
 * skipped.  e_out[4] = {Re E2, Im E2, Re E3, Im E3} (host).  The sum runs in a
 * fixed order: repeated calls give identical bits. */
int tcg_energy(tcg_ctx *ctx, const int32_t *nb_apply, const void *h2_dev, const void *h3_dev, double *e_out);

/* Backward pass: energy gradients of the current state (no reference
 * counterpart -- TC++ has no adjoint).  E = E2 + E3 as tcg_energy, with H
 * (the terms of term_mask) applied to the occupied right orbitals and built
 * from those same orbitals and the state's density (for a variational
 * gradient, the density of these orbitals, e.g. from tcg_density).
 *   e_out[4]     E2, E3 (re, im)
 *   dE_dchi_dev  DEVICE [nspin][nk][nbands[s]][npw] complex (the layout of
 *                phik_left) or NULL: dE / d conj(chi_i)(G) = f_i / N_k
 *                (H2 + H3) phi_i(G) for the occupied bands, 0 for the others
 *                (E is a polynomial in conj(chi) and H2, H3 are its
 *                mean-field derivatives).  Needs nsym_k = 1 for every k.
 *   dE_du, dE_dv2  host [nspin][N] complex each, or NULL: the tc2x part of
 *                dE/du(G; s, s) and dE/dV_2body(G; s, s) on the FFT grid,
 *                from pair densities recomputed block by block (never all
 *                stored).  Gamma-only systems, TCG_TERM_TC2X in term_mask.
 * Fails with TCG_ERR_UNSUPPORTED outside these limits. */
int tcg_energy_grad(tcg_ctx *ctx, uint32_t term_mask, double *e_out, void *dE_dchi_dev, double *dE_du,
                    double *dE_dv2);

/* Rayleigh-Ritz step of the block Davidson for one (spin, k) block, on the
 * device in FP64 (Diagonalization::block_davidson,
 * diagonalization_davidson.cpp:462-600):
 *   H_n,sub = Vref^H (H_n V)  for the given n = 1, 2, 3 (ZGEMM),
 *   H_sub = sum_n H_n,sub,  H_sub X = X D  (general complex eigensolve;
 *   ComplexEigenSolver in the reference), eigenpairs sorted by the real part
 *   (sort_eigen, diagonalization_utils.cpp:82-119), X_left = (X^-1)^H,
 *   V_out = V X[:, :nout],  Vl_out = Vref X_left[:, :nout] (if non-NULL),
 *   e_out[3][nout] = diag(L^H H_n,sub X), L = X_left if biortho else X.
 * V, Vref (NULL: V), H1V, H2V, H3V (NULL: absent): DEVICE [ndim][npw]
 * complex, one basis vector after the other; eig_out [ndim] and e_out
 * [3][nout] complex on the host (e_out may be NULL); V_out, Vl_out DEVICE
 * [nout][npw].  `stream` is a cudaStream_t (NULL: default); the call returns
 * after the work finished.  Scratch is allocated and freed per call. */
int tcg_subspace_ritz(int32_t ndim, int32_t npw, int32_t nout, int32_t biortho, const void *V, const void *Vref,
                      const void *H1V, const void *H2V, const void *H3V, double *eig_out, double *e_out,
                      void *V_out, void *Vl_out, void *stream);

/* Gram-Schmidt orthonormalisation of nvec DEVICE vectors V [nvec][npw] in
 * place, in order (Diagonalization::Gram_Schmidt, diagonalization_utils.cpp:
 * 7-28); with Vl non-NULL the bi-orthonormalisation of (V, Vl), <Vl_i|V_j> =
 * delta_ij (Gram_Schmidt_biortho, :30-77).  TCG_ERR_NUMERIC when a vector
 * becomes linearly dependent (norm < 1e-8, 1e-10 bi-orthogonal), as the
 * reference stops there. */
int tcg_gram_schmidt(int32_t nvec, int32_t npw, void *V, void *Vl, void *stream);

/* New trial vectors of one block-Davidson block for one (spin, k), on the
 * device in FP64 (diagonalization_davidson.cpp:283-318 with
 * Diagonalization::make_a_new_trial_vector, diagonalization_utils.cpp:
 * 165-211): for each b < nblock the preconditioned residual
 * -K(|k+G|^2 / t_b) (H1 + H2 + H3 - e_b) phi_b, t_b the kinetic expectation of
 * phi_b, normalised; then orthonormalised against the rows of V in order
 * (the new rows of this call included) and appended as row *nbasis_out of V,
 * unless its norm falls below 1e-8, in which case it is dropped.
 * V: DEVICE [nbasis + nblock][npw] (capacity), rows < nbasis the current
 * orthonormal basis; phi, H1phi, H2phi, H3phi (NULL: absent): DEVICE
 * [nblock][npw]; kG2: DEVICE [npw] |k+G|^2; eig_ref: host complex [nblock],
 * the eigenvalues of the previous iteration.  Returns after the work. */
int tcg_davidson_expand(int32_t nbasis, int32_t nblock, int32_t npw, void *V, const void *phi, const void *H1phi,
                        const void *H2phi, const void *H3phi, const double *kG2, const double *eig_ref,
                        int32_t *nbasis_out, void *stream);

/* Divergence-correction scalars for the SCF mesh (Potentials::set_sum_of_Vaux
 * with set_sum_of_Vaux_each, potentials_coulomb.cpp:60-161), computed on the
 * device.  Writes alpha_Vaux and sum_Vaux[nk_irr]; needs only the geometry
 * and k-point fields of sys (sum_Vaux / alpha_Vaux of sys are ignored). */
int tcg_sum_of_vaux(const tcg_system_desc *sys, double *alpha_out, double *sum_vaux_out);

/* Allocation-free variant of tcg_sum_of_vaux for callers that cannot
 * allocate device memory: an application or framework whose memory pool has
 * reserved the GPU's memory up front (a cudaMalloc would fail or fragment the
 * pool), or code that must not trigger the implicit device-wide
 * synchronisation of cudaMalloc / cudaFree.  No counterpart in the reference
 * (TC++ computes these sums on the host).
 * All arrays are DEVICE pointers: kirr_dev [nk_irr][3] and kall_dev
 * [nk_all][3] fractional k-vectors (irreducible k, full SCF mesh), output
 * sum_vaux_dev [nk_irr]; alpha_out is a host pointer (may be NULL).  The
 * work is queued on `stream` (cudaStream_t as void*, NULL = default); the
 * call then copies a convergence flag to the host and synchronises that
 * stream before it returns.  Scratch is a static device array of 16384
 * (k, q) pairs held by every GPU that loads the library until the process
 * exits; larger nk_irr * nk_all is rejected with TCG_ERR_ARG, as are a
 * non-finite recip or omega.  A k-vector difference that is not finite or
 * beyond +-64 fails with TCG_ERR_NUMERIC.  Set-up: the first call on a device
 * looks the array's device address up (cudaGetSymbolAddress, with that device
 * current) and keeps it for the life of the process, so make that first call
 * before any stream capture begins; after a cudaDeviceReset of that device
 * the kept address is stale and the entry point must not be called again.
 * Every call shares the one array: calls that overlap on the GPU (other
 * threads or streams) race and must be serialised by the caller. */
int tcg_sum_of_vaux_noalloc(const double recip[9], double omega, int32_t nk_irr, int32_t nk_all,
                            const double *kirr_dev, const double *kall_dev, double *sum_vaux_dev,
                            double *alpha_out, void *stream);

/* n_s(r) of the given orbitals (BlochStates::set_density, first iteration,
 * bloch_states_scfloop_filling_density.cpp:256-360), computed on the device;
 * density_out is [2][N] complex.  Fails with TCG_ERR_NUMERIC if an orbital's
 * norm <chi|phi> deviates from 1 by more than 1e-4 (as the reference). */
int tcg_density(tcg_ctx *ctx, const tcg_state_desc *st, double *density_out);

/* Occupied-pair stage of tc3a2a4b2b5 split over ranks.  The stage sums, for
 * every occupied target (q2, i2), intermediates over all occupied sources
 * (q1, i1); the reference splits the q1 bands over MPI ranks and
 * MPI_Allreduces the intermediate grids (calc_hamiltonian_tc3a2a4b2b5.cpp:
 * 214-235, 490-493, 649-659).  Here:
 *   tcg_qp_partial: this rank's share (the sources in nranks contiguous
 *     blocks, block `rank`) into a device buffer of FP64 complex grids;
 *     returns its address and size in bytes.  The caller sums the buffer
 *     over all ranks in place (e.g. ncclAllReduce of bytes/8 doubles, sum)
 *     and synchronises, then calls
 *   tcg_qp_finish: divergence correction, symmetry rotations and the local
 *     potentials on the summed grids; the next tcg_apply uses the result.
 * Every rank must call both with the same state.  Without these calls,
 * tcg_apply computes the whole stage on one rank.  Between the two calls
 * tcg_apply with the tc3a2a4b2b5 bit fails with TCG_ERR_STATE. */
int tcg_qp_partial(tcg_ctx *ctx, int32_t rank, int32_t nranks, void **buf_dev, size_t *bytes);
int tcg_qp_finish(tcg_ctx *ctx);

/* Tuning knob: bytes of pass temporaries one chunk of (target x source)
 * pairs may use (0 = default, 8 GiB).  Smaller chunks keep the temporaries
 * resident in L2; larger ones launch fewer kernels.  No reference
 * counterpart (TC++ has no chunked pair pipeline). */
int tcg_set_tuning(tcg_ctx *ctx, int64_t tmp_budget_bytes);

/* Kernel forms of the pass pipelines (the choices an autotuner explores; no
 * reference counterpart).  xy: 0 = each term's default (split lines on the
 * grids that have them), 1 = one thread per line, 2 = a lane pair per line,
 * 3 = split lines (six threads per line at 36^3, four at 48^3); z: 0 =
 * default, 1 = one thread per z-line, 2 = a lane pair, 3 = split lines with
 * the inputs in shared memory, 4 = split lines with the inputs in registers
 * (3 and 4 need a 36^3 or 48^3 grid).  xy 1 or 2 and z 1 or 2 turn the
 * pruning of band-limited grids off (only the split-line kernels honour it).  Flags, each
 * 0 or 1: prefetch (the inverse XY pass copies the next plane set while it
 * transforms the current one), prune (band-limited grids on the pencils
 * their support meets), fuse (tc2x, tc3a3b3b4b6 and tc3a2a4b2b5's band part
 * share their transforms), qp_sacc / sacc (shared-memory accumulation in the
 * occupied-pair / first-stage inverse XY passes).  min_targets: targets per
 * chunk (0 = default).  tcg_get_forms reads the current choice. */
typedef struct tcg_forms {
    int32_t xy, z, prefetch, prune, fuse, qp_sacc, sacc, min_targets;
} tcg_forms;
int tcg_set_forms(tcg_ctx *ctx, const tcg_forms *forms);
int tcg_get_forms(tcg_ctx *ctx, tcg_forms *forms);

/* Per-kernel timing with CUDA events recorded on the context stream around
 * every launch (off by default; enabling clears earlier records).  No
 * reference counterpart (TC++ times whole phases at 1 s resolution,
 * my_clock.cpp:19-33). */
int tcg_profile(tcg_ctx *ctx, int enable);
/* Aggregate of the recorded launches per "term:pass" tag (pass = xyf, z,
 * xyi; "misc" for the rest): count, device milliseconds and algorithmic
 * bytes (N s per grid and pass; a 3D FFT = 2 N s).  tags: cap x 32 chars. */
int tcg_profile_read(tcg_ctx *ctx, int cap, char *tags, int64_t *count, double *ms, double *bytes, int *ntags);

/* Device stream the context queues work on (cudaStream_t, as void*). */
void *tcg_stream(tcg_ctx *ctx);

/* Number of kernels this context has launched since creation. */
int64_t tcg_launch_count(const tcg_ctx *ctx);

/* Message of the calling thread's last failure ("" if none). */
const char *tcg_last_error(void);

/* Library version string. */
const char *tcg_version(void);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* TCG_H */
