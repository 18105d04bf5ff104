// tcpp_standin.hpp -- the few TC++ and Eigen declarations the shim
// (calc_hamiltonian_tcg.cpp) touches, for building and testing it outside a
// TC++ tree.  Inside TC++ the shim includes "include/header.hpp" instead and
// this file is not used.
//
// Every accessor keeps the name, return type and container nesting of the
// reference's headers (src/include/*.hpp); only the members the shim reads
// exist, as plain public data behind the accessors.
#pragma once
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

using Complex = std::complex<double>;    // header.hpp:42

namespace Eigen {
// dense vectors with contiguous storage (the layout the shim copies from)
template <typename S>
class Vec {
public:
    Vec() = default;
    explicit Vec(long n) : v_(n) {}
    long size() const { return (long)v_.size(); }
    void resize(long n) { v_.resize(n); }
    void setZero() { std::fill(v_.begin(), v_.end(), S()); }
    S *data() { return v_.data(); }
    const S *data() const { return v_.data(); }
    S &operator()(long i) { return v_[i]; }
    const S &operator()(long i) const { return v_[i]; }
private:
    std::vector<S> v_;
};
using VectorXcd = Vec<std::complex<double>>;
using VectorXi = Vec<int>;
using VectorXd = Vec<double>;

template <typename S, int R, int C>
class Fixed {
public:
    S &operator()(int i, int j = 0) { return a_[i * C + j]; }
    const S &operator()(int i, int j = 0) const { return a_[i * C + j]; }
private:
    S a_[R * C] = {};
};
using Matrix3d = Fixed<double, 3, 3>;
using Matrix3i = Fixed<int, 3, 3>;
using Vector3d = Fixed<double, 3, 1>;
} // namespace Eigen

namespace error_messages {
// error_messages.hpp:27 -- the reference prints and calls MPI_Abort; the
// stand-in throws so that a driver can report the message and exit non-zero
inline void stop(const std::string &message) { throw std::runtime_error(message); }
} // namespace error_messages

class Parallelization {                              // parallelization.hpp
public:
    std::vector<std::vector<std::vector<bool>>> assigned;
    const std::vector<std::vector<std::vector<bool>>> &is_assigned_irreducible_kpoints_all_bands() const { return assigned; }
};

class Method {                                       // method.hpp:14-15
public:
    std::string method, mode = "SCF";
    const std::string &calc_method() const { return method; }
    const std::string &calc_mode() const { return mode; }
};

class CrystalStructure {                             // crystal_structure.hpp:34-36
public:
    Eigen::Matrix3d lattice, recip;
    double volume = 0;
    const Eigen::Matrix3d &lattice_vectors() const { return lattice; }
    const Eigen::Matrix3d &reciprocal_vectors() const { return recip; }
    double unit_cell_volume() const { return volume; }
};

class Symmetry {                                     // symmetry.hpp:25-30
public:
    std::vector<Eigen::Matrix3i> rot;
    std::vector<Eigen::Vector3d> trans;
    int num_symmetry_operations() const { return (int)rot.size(); }
    const std::vector<Eigen::Matrix3i> &rotation() const { return rot; }
    const std::vector<Eigen::Vector3d> &translation() const { return trans; }
};

class Jastrow {                                      // jastrow.hpp:94-95
public:
    std::vector<std::vector<double>> A, F;
    const std::vector<std::vector<double>> &A_long() const { return A; }
    const std::vector<std::vector<double>> &F_long() const { return F; }
};

class Potentials {                                   // potentials.hpp:71, :80-82
public:
    Jastrow jastrow;
    bool div = true;
    double alpha = 0;
    std::vector<double> sum_vaux;
    bool includes_div_correction() const { return div; }
    double alpha_Vaux() const { return alpha; }
    const std::vector<double> &sum_of_Vaux_scf() const { return sum_vaux; }
};

class Spin {                                         // spin.hpp:21
public:
    int nspin = 1;
    int num_independent_spins() const { return nspin; }
};

class Kpoints {                                      // kpoints.hpp:43-52
public:
    int nk_all_weighted = 0;
    std::vector<std::vector<Eigen::Vector3d>> kvec;
    std::vector<std::vector<int>> rot_index;
    std::vector<std::vector<bool>> time_rev;
    int num_irreducible_kpoints_scf() const { return (int)kvec.size(); }
    int num_kpoints() const { return nk_all_weighted; }
    const std::vector<std::vector<Eigen::Vector3d>> &kvectors_scf() const { return kvec; }
    const std::vector<std::vector<int>> &index_of_rotation_at_k() const { return rot_index; }
    const std::vector<std::vector<bool>> &is_time_reversal_used_at_k() const { return time_rev; }
};

class PlaneWaveBasis {                               // plane_wave_basis.hpp:37-42
public:
    std::vector<int> npw, nr;
    std::vector<std::vector<std::vector<Eigen::VectorXi>>> gindex;
    std::vector<std::vector<std::vector<Eigen::VectorXcd>>> phase;
    const std::vector<int> &num_G_at_k_scf() const { return npw; }
    const std::vector<std::vector<std::vector<Eigen::VectorXi>>> &Gindex_at_k_scf() const { return gindex; }
    const std::vector<std::vector<std::vector<Eigen::VectorXcd>>> &phase_factor_at_k() const { return phase; }
    const std::vector<int> &size_FFT_grid_vec() const { return nr; }
};

class BlochStates {                                  // bloch_states.hpp:65-77
public:
    using Orbs = std::vector<std::vector<std::vector<std::vector<Eigen::VectorXcd>>>>;
    std::vector<int> nbands;
    std::vector<std::vector<int>> nocc;
    std::vector<std::vector<std::vector<double>>> fill;
    Orbs phik, phik_left;
    std::vector<Eigen::VectorXcd> dens;
    const std::vector<int> &num_bands_scf() const { return nbands; }
    const std::vector<std::vector<int>> &num_occupied_bands() const { return nocc; }
    const std::vector<std::vector<std::vector<double>>> &filling() const { return fill; }
    const Orbs &phik_scf() const { return phik; }
    const Orbs &phik_left_scf() const { return phik_left; }
    const std::vector<Eigen::VectorXcd> &density() const { return dens; }
};
