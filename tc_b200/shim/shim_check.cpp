// shim_check.cpp -- drives the TC++ shim the way calc_hamiltonian::all does,
// from a system dumped to a binary file, and writes the results.
//
//   shim_check <input.bin> <output.bin>
//
// It rebuilds the reference's nested containers (kvectors_scf[ik][isym],
// Gindex_at_k_scf[s][ik][isym], phik_scf[s][ik][b][0], ...) from the flat
// dump, then
//   1. calls the routines one by one, as calc_hamiltonian_all.cpp:80-157
//      does (hf2x; or tc2x, tc3a1, tc3b1, tc3a2a4b2b5, tc3a3b3b4b6), on
//      zeroed H2phi / H3phi (calc_hamiltonian_all.cpp:29-49);
//   2. calls tcg_shim::apply_two_three_body once on fresh zeroed outputs;
// and writes H2 and H3 of both, packed like the input psi, plus the launch
// count.  Any error ends the program with status 1 and the message on stderr.
// Input layout: written by tests/_shim_io.py (write_system).
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <stdexcept>

#include "calc_hamiltonian_tcg.hpp"
#include "../../include/tcg.h"

namespace {
struct Reader {
    std::ifstream f;
    explicit Reader(const char *path) : f(path, std::ios::binary)
    {
        if (!f) throw std::runtime_error(std::string("cannot open ") + path);
    }
    template <typename X> X one()
    {
        X x;
        f.read(reinterpret_cast<char *>(&x), sizeof x);
        if (!f) throw std::runtime_error("input file truncated");
        return x;
    }
    template <typename X> void many(X *p, size_t n)
    {
        f.read(reinterpret_cast<char *>(p), sizeof(X) * n);
        if (!f) throw std::runtime_error("input file truncated");
    }
};

using tcg_shim::Orbitals;

Orbitals zeros_like(const Orbitals &phi)
{
    Orbitals h = phi;
    for (auto &s : h)
        for (auto &k : s)
            for (auto &b : k) b[0].setZero();
    return h;
}

void write(std::ofstream &o, const Orbitals &h)
{
    for (const auto &s : h)
        for (const auto &k : s)
            for (const auto &b : k) o.write(reinterpret_cast<const char *>(b[0].data()), 16 * b[0].size());
}
} // namespace

int main(int argc, char **argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s <input.bin> <output.bin>\n", argv[0]);
        return 2;
    }
    try {
        Reader r(argv[1]);
        if (r.one<int32_t>() != 0x53474354) throw std::runtime_error("bad magic");
        const int32_t method_i = r.one<int32_t>(), nspin = r.one<int32_t>(), nk = r.one<int32_t>();
        int32_t nr[3];
        r.many(nr, 3);
        const int32_t num_kpoints = r.one<int32_t>(), nsymop = r.one<int32_t>(), precision = r.one<int32_t>();
        Method method;
        method.method = method_i == 0 ? "HF" : (method_i == 1 ? "TC" : "BITC");
        CrystalStructure cs;
        double m9[9];
        r.many(m9, 9);
        for (int i = 0; i < 9; i++) cs.lattice(i / 3, i % 3) = m9[i];
        r.many(m9, 9);
        for (int i = 0; i < 9; i++) cs.recip(i / 3, i % 3) = m9[i];
        cs.volume = r.one<double>();
        Spin spin;
        spin.nspin = nspin;
        Kpoints kp;
        kp.nk_all_weighted = num_kpoints;
        std::vector<int32_t> nsym(nk);
        r.many(nsym.data(), nk);
        kp.kvec.resize(nk);
        kp.rot_index.resize(nk);
        kp.time_rev.resize(nk);
        for (int ik = 0; ik < nk; ik++)
            for (int is = 0; is < nsym[ik]; is++) {
                Eigen::Vector3d v;
                for (int x = 0; x < 3; x++) v(x) = r.one<double>();
                kp.kvec[ik].push_back(v);
                kp.rot_index[ik].push_back(r.one<int32_t>());
                kp.time_rev[ik].push_back(r.one<int32_t>() != 0);
            }
        PlaneWaveBasis pw;
        pw.nr.assign(nr, nr + 3);
        pw.npw.resize(nk);
        r.many(pw.npw.data(), nk);
        pw.gindex.assign(nspin, std::vector<std::vector<Eigen::VectorXi>>(nk));
        pw.phase.assign(nspin, std::vector<std::vector<Eigen::VectorXcd>>(nk));
        for (int s = 0; s < nspin; s++)
            for (int ik = 0; ik < nk; ik++)
                for (int is = 0; is < nsym[ik]; is++) {
                    Eigen::VectorXi gi(pw.npw[ik]);
                    r.many(gi.data(), pw.npw[ik]);
                    Eigen::VectorXcd ph(pw.npw[ik]);
                    r.many(ph.data(), pw.npw[ik]);
                    pw.gindex[s][ik].push_back(gi);
                    pw.phase[s][ik].push_back(ph);
                }
        Symmetry sym;
        for (int i = 0; i < nsymop; i++) {
            Eigen::Matrix3i u;
            for (int e = 0; e < 9; e++) u(e / 3, e % 3) = r.one<int32_t>();
            sym.rot.push_back(u);
        }
        for (int i = 0; i < nsymop; i++) {
            Eigen::Vector3d t;
            for (int x = 0; x < 3; x++) t(x) = r.one<double>();
            sym.trans.push_back(t);
        }
        Potentials pot;
        double A[4], F[4];
        r.many(A, 4);
        r.many(F, 4);
        pot.jastrow.A = {{A[0], A[1]}, {A[2], A[3]}};
        pot.jastrow.F = {{F[0], F[1]}, {F[2], F[3]}};
        pot.div = r.one<int32_t>() != 0;
        pot.alpha = r.one<double>();
        pot.sum_vaux.resize(nk);
        r.many(pot.sum_vaux.data(), nk);
        BlochStates bs;
        bs.nbands.resize(nspin);
        r.many(bs.nbands.data(), nspin);
        bs.nocc.assign(nspin, std::vector<int>(nk));
        for (int s = 0; s < nspin; s++) r.many(bs.nocc[s].data(), nk);
        bs.fill.assign(nspin, std::vector<std::vector<double>>(nk));
        for (int s = 0; s < nspin; s++)
            for (int ik = 0; ik < nk; ik++) {
                bs.fill[s][ik].resize(bs.nbands[s]);
                r.many(bs.fill[s][ik].data(), bs.nbands[s]);
            }
        auto read_orbs = [&](Orbitals &o, const std::vector<int> &nb_of_s_k) {
            o.assign(nspin, std::vector<std::vector<std::vector<Eigen::VectorXcd>>>(nk));
            for (int s = 0; s < nspin; s++)
                for (int ik = 0; ik < nk; ik++)
                    for (int b = 0; b < nb_of_s_k[s * nk + ik]; b++) {
                        Eigen::VectorXcd v(pw.npw[ik]);
                        r.many(v.data(), pw.npw[ik]);
                        o[s][ik].push_back({v});
                    }
        };
        std::vector<int> nbands_sk(nspin * nk);
        for (int s = 0; s < nspin; s++)
            for (int ik = 0; ik < nk; ik++) nbands_sk[s * nk + ik] = bs.nbands[s];
        read_orbs(bs.phik, nbands_sk);
        if (method_i == 2) read_orbs(bs.phik_left, nbands_sk);
        const long N = (long)nr[0] * nr[1] * nr[2];
        for (int s = 0; s < 2; s++) {
            Eigen::VectorXcd d(N);
            r.many(d.data(), N);
            bs.dens.push_back(d);
        }
        std::vector<int> nb_apply(nspin * nk);
        r.many(nb_apply.data(), nspin * nk);
        Orbitals phi;
        read_orbs(phi, nb_apply);
        Parallelization par;
        par.assigned.assign(nspin, std::vector<std::vector<bool>>(nk));
        for (int s = 0; s < nspin; s++)
            for (int ik = 0; ik < nk; ik++)
                for (int b = 0; b < nb_apply[s * nk + ik]; b++) par.assigned[s][ik].push_back(r.one<int32_t>() != 0);

        tcg_shim::set_precision(precision);
        tcg_shim::new_scf_iteration();
        // 1. the routines one by one, as calc_hamiltonian::all calls them
        Orbitals H2 = zeros_like(phi), H3 = zeros_like(phi);
        if (method_i == 0) {
            calc_hamiltonian::hf2x(par, method, cs, pot, spin, kp, pw, bs, phi, H2, nullptr);
        } else {
            calc_hamiltonian::tc2x(par, method, cs, pot, spin, kp, pw, bs, phi, H2, nullptr);
            calc_hamiltonian::tc3a1(par, method, cs, pot, spin, kp, pw, bs, phi, H3, nullptr);
            calc_hamiltonian::tc3b1(par, method, cs, pot, spin, kp, pw, bs, phi, H3, nullptr);
            calc_hamiltonian::tc3a2a4b2b5(par, method, cs, sym, pot, spin, kp, pw, bs, phi, H3, nullptr);
            calc_hamiltonian::tc3a3b3b4b6(par, method, cs, pot, spin, kp, pw, bs, phi, H3, nullptr);
        }
        // 2. the whole block in one call
        Orbitals B2 = zeros_like(phi), B3 = zeros_like(phi);
        tcg_shim::apply_two_three_body(par, method, cs, sym, pot, spin, kp, pw, bs, phi, B2, B3);
        const int64_t launches = tcg_shim::launches();
        tcg_shim::release();
        std::ofstream o(argv[2], std::ios::binary);
        write(o, H2);
        write(o, H3);
        write(o, B2);
        write(o, B3);
        o.write(reinterpret_cast<const char *>(&launches), sizeof launches);
        if (!o) throw std::runtime_error("cannot write the output file");
    } catch (const std::exception &e) {
        std::fprintf(stderr, "shim_check: %s\n", e.what());
        return 1;
    }
    return 0;
}
