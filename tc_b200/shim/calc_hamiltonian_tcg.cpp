// calc_hamiltonian_tcg.cpp -- TC++'s six operator routines
// (src/include/calc_hamiltonian.hpp:54-130) on top of libtcg_b200.so.
//
// Build inside TC++: add this file (and calc_hamiltonian_tcg.hpp) to src/,
// remove calc_hamiltonian_{hf2x,tc2x,tc3a1,tc3b1,tc3a2a4b2b5,tc3a3b3b4b6}.cpp,
// add <repo>/include to the include path and link -L<repo>/tc_b200 -ltcg_b200.
// Outside TC++ (tests): -DTCG_SHIM_STANDALONE with tcpp_standin.hpp.
//
// What the shim does per call: flatten the nested Eigen containers into the
// packed arrays of include/tcg.h (one memcpy per band), create the device
// context once per run (geometry, k-points, G-vector maps, Jastrow,
// divergence scalars), upload the state once per SCF iteration
// (tcg_shim::new_scf_iteration), apply, and copy the accumulated H phi back.
// A non-zero library status becomes error_messages::stop, as every error of
// the reference does (error_messages.cpp:60-64).
#include "calc_hamiltonian_tcg.hpp"

#include <algorithm>
#include <cstring>

#include "../../include/tcg.h"

namespace tcg_shim {
namespace {

struct Cache {
    tcg_ctx *ctx = nullptr;
    bool real_symmetry = false;     // rotation table from Symmetry (not placeholders)
    long epoch = -1;                // SCF iteration whose state is on the device
    int32_t precision = TCG_PREC_FP64;
};
Cache g;
long g_epoch = 0;

void check(int rc)
{
    if (rc != TCG_OK) error_messages::stop(std::string("libtcg_b200: ") + tcg_last_error());
}

int32_t method_code(const Method &m)
{
    if (m.calc_method() == "HF") return TCG_METHOD_HF;
    if (m.calc_method() == "TC") return TCG_METHOD_TC;
    if (m.calc_method() == "BITC") return TCG_METHOD_BITC;
    error_messages::stop("libtcg_b200 shim: calc_method " + m.calc_method() + " is not supported");
    return -1;
}

void create_context(const Method &method, const CrystalStructure &cs, const Symmetry *sym, const Potentials &pot,
                    const Spin &spin, const Kpoints &kp, const PlaneWaveBasis &pw)
{
    if (method.calc_mode() != "SCF") error_messages::stop("libtcg_b200 shim: only calc_mode SCF is supported");
    const int nspin = spin.num_independent_spins();
    const int nk = kp.num_irreducible_kpoints_scf();
    tcg_system_desc d;
    std::memset(&d, 0, sizeof d);
    for (int i = 0; i < 3; i++) d.nr[i] = pw.size_FFT_grid_vec()[i];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            d.recip[3 * i + j] = cs.reciprocal_vectors()(i, j);   // rows b_i (crystal_structure.hpp:16)
            d.lattice[3 * i + j] = cs.lattice_vectors()(i, j);
        }
    d.omega = cs.unit_cell_volume();
    d.calc_method = method_code(method);
    d.nspin = nspin;
    d.nk_irr = nk;
    d.num_kpoints = kp.num_kpoints();
    std::vector<int32_t> nsym(nk), rot_index, npw(nk), gindex;
    std::vector<double> kvec, phase;
    std::vector<uint8_t> time_rev;
    int max_rot = 0;
    for (int ik = 0; ik < nk; ik++) {
        nsym[ik] = (int32_t)kp.kvectors_scf()[ik].size();
        npw[ik] = pw.num_G_at_k_scf()[ik];
        for (int isym = 0; isym < nsym[ik]; isym++) {
            for (int x = 0; x < 3; x++) kvec.push_back(kp.kvectors_scf()[ik][isym](x));
            time_rev.push_back(kp.is_time_reversal_used_at_k()[ik][isym] ? 1 : 0);
            rot_index.push_back(kp.index_of_rotation_at_k()[ik][isym]);
            max_rot = std::max(max_rot, rot_index.back());
        }
    }
    for (int s = 0; s < nspin; s++)
        for (int ik = 0; ik < nk; ik++)
            for (int isym = 0; isym < nsym[ik]; isym++) {
                const Eigen::VectorXi &gi = pw.Gindex_at_k_scf()[s][ik][isym];
                const Eigen::VectorXcd &ph = pw.phase_factor_at_k()[s][ik][isym];
                gindex.insert(gindex.end(), gi.data(), gi.data() + gi.size());
                const double *p = reinterpret_cast<const double *>(ph.data());
                phase.insert(phase.end(), p, p + 2 * ph.size());
            }
    // rotations: the Symmetry's table, or identity placeholders for the
    // routines that never rotate (their signatures carry no Symmetry)
    std::vector<int32_t> rot;
    std::vector<double> trans;
    if (sym) {
        for (int i = 0; i < sym->num_symmetry_operations(); i++) {
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) rot.push_back(sym->rotation()[i](r, c));
            for (int x = 0; x < 3; x++) trans.push_back(sym->translation()[i](x));
        }
    } else {
        for (int i = 0; i <= max_rot; i++) {
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) rot.push_back(r == c ? 1 : 0);
            for (int x = 0; x < 3; x++) trans.push_back(0.0);
        }
    }
    d.nsym_k = nsym.data();
    d.kvec = kvec.data();
    d.time_rev = time_rev.data();
    d.rot_index = rot_index.data();
    d.nsymop = (int32_t)(rot.size() / 9);
    d.rotation = rot.data();
    d.translation = trans.data();
    d.npw = npw.data();
    d.gindex = gindex.data();
    d.phase = phase.data();
    const auto &A = pot.jastrow.A_long();
    const auto &F = pot.jastrow.F_long();
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            const bool have = d.calc_method != TCG_METHOD_HF && (int)A.size() > i && (int)A[i].size() > j;
            d.jastrow_A[2 * i + j] = have ? A[i][j] : 0.0;
            d.jastrow_F[2 * i + j] = have ? F[i][j] : 1.0;
        }
    d.includes_div_correction = pot.includes_div_correction() ? 1 : 0;
    d.alpha_Vaux = pot.alpha_Vaux();
    d.sum_Vaux = pot.sum_of_Vaux_scf().data();
    if (g.ctx) tcg_ctx_destroy(g.ctx);
    g.ctx = nullptr;
    check(tcg_ctx_create(&d, g.precision, &g.ctx));
    g.real_symmetry = sym != nullptr;
    g.epoch = -1;
}

void ensure_context(const Method &method, const CrystalStructure &cs, const Symmetry *sym, const Potentials &pot,
                    const Spin &spin, const Kpoints &kp, const PlaneWaveBasis &pw)
{
    if (g.ctx && (g.real_symmetry || !sym)) return;
    create_context(method, cs, sym, pot, spin, kp, pw);
}

void ensure_state(const BlochStates &bs, const Method &method)
{
    if (g.epoch == g_epoch) return;
    const bool bitc = method.calc_method() == "BITC";
    const int nspin = (int)bs.num_bands_scf().size();
    std::vector<int32_t> nbands(nspin), nocc;
    std::vector<double> fill, phik, left, dens;
    for (int s = 0; s < nspin; s++) {
        nbands[s] = bs.num_bands_scf()[s];
        const int nk = (int)bs.phik_scf()[s].size();
        for (int ik = 0; ik < nk; ik++) {
            nocc.push_back(bs.num_occupied_bands()[s][ik]);
            for (int b = 0; b < nbands[s]; b++) {
                fill.push_back(bs.filling()[s][ik][b]);
                const Eigen::VectorXcd &v = bs.phik_scf()[s][ik][b][0];
                const double *p = reinterpret_cast<const double *>(v.data());
                phik.insert(phik.end(), p, p + 2 * v.size());
                if (bitc) {
                    const Eigen::VectorXcd &w = bs.phik_left_scf()[s][ik][b][0];
                    const double *q = reinterpret_cast<const double *>(w.data());
                    left.insert(left.end(), q, q + 2 * w.size());
                }
            }
        }
    }
    for (int s = 0; s < 2; s++) {
        const Eigen::VectorXcd &n = bs.density()[std::min<size_t>(s, bs.density().size() - 1)];
        const double *p = reinterpret_cast<const double *>(n.data());
        dens.insert(dens.end(), p, p + 2 * n.size());
    }
    tcg_state_desc st;
    std::memset(&st, 0, sizeof st);
    st.nbands = nbands.data();
    st.nocc = nocc.data();
    st.filling = fill.data();
    st.phik = phik.data();
    st.phik_left = bitc ? left.data() : nullptr;
    st.density = dens.data();
    check(tcg_set_state(g.ctx, &st));
    g.epoch = g_epoch;
}

// flatten phi / H, apply the terms of `mask`, copy the accumulated H back
void run(uint32_t mask, const Parallelization &par, const Orbitals &phi, Orbitals *H2, Orbitals *H3)
{
    std::vector<int32_t> nb;
    std::vector<double> psi, h2, h3;
    std::vector<uint8_t> owned;
    for (size_t s = 0; s < phi.size(); s++)
        for (size_t k = 0; k < phi[s].size(); k++) {
            nb.push_back((int32_t)phi[s][k].size());
            for (size_t j = 0; j < phi[s][k].size(); j++) {
                const Eigen::VectorXcd &v = phi[s][k][j][0];
                const double *p = reinterpret_cast<const double *>(v.data());
                psi.insert(psi.end(), p, p + 2 * v.size());
                if (H2) {
                    const Eigen::VectorXcd &h = (*H2)[s][k][j][0];
                    const double *q = reinterpret_cast<const double *>(h.data());
                    h2.insert(h2.end(), q, q + 2 * h.size());     // accumulate semantics
                }
                if (H3) {
                    const Eigen::VectorXcd &h = (*H3)[s][k][j][0];
                    const double *q = reinterpret_cast<const double *>(h.data());
                    h3.insert(h3.end(), q, q + 2 * h.size());
                }
                owned.push_back(par.is_assigned_irreducible_kpoints_all_bands()[s][k][j] ? 1 : 0);
            }
        }
    check(tcg_apply(g.ctx, mask, nb.data(), psi.data(), H2 ? h2.data() : nullptr, H3 ? h3.data() : nullptr,
                    owned.data()));
    size_t o2 = 0, o3 = 0;
    for (size_t s = 0; s < phi.size(); s++)
        for (size_t k = 0; k < phi[s].size(); k++)
            for (size_t j = 0; j < phi[s][k].size(); j++) {
                if (H2) {
                    Eigen::VectorXcd &h = (*H2)[s][k][j][0];
                    std::memcpy(h.data(), h2.data() + o2, sizeof(double) * 2 * h.size());
                    o2 += 2 * h.size();
                }
                if (H3) {
                    Eigen::VectorXcd &h = (*H3)[s][k][j][0];
                    std::memcpy(h.data(), h3.data() + o3, sizeof(double) * 2 * h.size());
                    o3 += 2 * h.size();
                }
            }
}

} // namespace

void new_scf_iteration() { ++g_epoch; }

void set_precision(int32_t precision) { g.precision = precision; }

void release()
{
    if (g.ctx) tcg_ctx_destroy(g.ctx);
    g.ctx = nullptr;
    g.epoch = -1;
}

int64_t launches() { return g.ctx ? tcg_launch_count(g.ctx) : 0; }

void apply_two_three_body(const Parallelization &par, const Method &method, const CrystalStructure &cs,
                          const Symmetry &sym, const Potentials &pot, const Spin &spin, const Kpoints &kp,
                          const PlaneWaveBasis &pw, const BlochStates &bs, const Orbitals &phi, Orbitals &H2phi,
                          Orbitals &H3phi)
{
    ensure_context(method, cs, &sym, pot, spin, kp, pw);
    ensure_state(bs, method);
    if (method.calc_method() == "HF") run(TCG_TERMS_HF, par, phi, &H2phi, nullptr);
    else run(TCG_TERMS_TC, par, phi, &H2phi, &H3phi);
}

} // namespace tcg_shim

// ------------------------------------------------ the reference's routines --
namespace calc_hamiltonian {
using tcg_shim::Orbitals;

#define TCG_SHIM_ROUTINE(NAME, TERM, SYMPTR, HX)                                                             \
    {                                                                                                        \
        tcg_shim::ensure_context(method, crystal_structure, SYMPTR, potentials, spin, kpoints, plane_wave_basis); \
        tcg_shim::ensure_state(bloch_states, method);                                                        \
        tcg_shim::run(TERM, parallelization, phi, (TERM & (TCG_TERM_HF2X | TCG_TERM_TC2X)) ? &HX : nullptr,   \
                      (TERM & (TCG_TERM_HF2X | TCG_TERM_TC2X)) ? nullptr : &HX);                              \
    }

void hf2x(const Parallelization &parallelization, const Method &method, const CrystalStructure &crystal_structure,
          const Potentials &potentials, const Spin &spin, const Kpoints &kpoints, PlaneWaveBasis &plane_wave_basis,
          const BlochStates &bloch_states, const Orbitals &phi, Orbitals &H2phi, std::ostream *)
TCG_SHIM_ROUTINE(hf2x, TCG_TERM_HF2X, nullptr, H2phi)

void tc2x(const Parallelization &parallelization, const Method &method, const CrystalStructure &crystal_structure,
          const Potentials &potentials, const Spin &spin, const Kpoints &kpoints, PlaneWaveBasis &plane_wave_basis,
          const BlochStates &bloch_states, const Orbitals &phi, Orbitals &H2phi, std::ostream *)
TCG_SHIM_ROUTINE(tc2x, TCG_TERM_TC2X, nullptr, H2phi)

void tc3a1(const Parallelization &parallelization, const Method &method, const CrystalStructure &crystal_structure,
           const Potentials &potentials, const Spin &spin, const Kpoints &kpoints, PlaneWaveBasis &plane_wave_basis,
           const BlochStates &bloch_states, const Orbitals &phi, Orbitals &H3phi, std::ostream *)
TCG_SHIM_ROUTINE(tc3a1, TCG_TERM_TC3A1, nullptr, H3phi)

void tc3b1(const Parallelization &parallelization, const Method &method, const CrystalStructure &crystal_structure,
           const Potentials &potentials, const Spin &spin, const Kpoints &kpoints, PlaneWaveBasis &plane_wave_basis,
           const BlochStates &bloch_states, const Orbitals &phi, Orbitals &H3phi, std::ostream *)
TCG_SHIM_ROUTINE(tc3b1, TCG_TERM_TC3B1, nullptr, H3phi)

void tc3a3b3b4b6(const Parallelization &parallelization, const Method &method,
                 const CrystalStructure &crystal_structure, const Potentials &potentials, const Spin &spin,
                 const Kpoints &kpoints, PlaneWaveBasis &plane_wave_basis, const BlochStates &bloch_states,
                 const Orbitals &phi, Orbitals &H3phi, std::ostream *)
TCG_SHIM_ROUTINE(tc3a3b3b4b6, TCG_TERM_TC3A3B3B4B6, nullptr, H3phi)

void tc3a2a4b2b5(const Parallelization &parallelization, const Method &method,
                 const CrystalStructure &crystal_structure, const Symmetry &symmetry, const Potentials &potentials,
                 const Spin &spin, const Kpoints &kpoints, PlaneWaveBasis &plane_wave_basis,
                 const BlochStates &bloch_states, const Orbitals &phi, Orbitals &H3phi, std::ostream *)
TCG_SHIM_ROUTINE(tc3a2a4b2b5, TCG_TERM_TC3A2A4B2B5, &symmetry, H3phi)

#undef TCG_SHIM_ROUTINE
} // namespace calc_hamiltonian
