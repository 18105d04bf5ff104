// adjoint.cuh -- gradients of the energy functional (backward pass of the
// apply).
//
// E = sum_{k, i} f_i [e2_i / 2 + e3_i / 3] / N_k,  e_n = <chi_i | H_n phi_i>
// (TotalEnergy::calc_total_energy, total_energy.cpp:101-168), with H built
// from the same occupied orbitals and their density.
//
// * Orbitals.  E is a polynomial in conj(chi) of degree 2 (two-body) and 3
//   (three-body) and H2, H3 are the mean-field derivatives of E2, E3, so
//   dE / d conj(chi_i)(G) = f_i / N_k (H2 + H3) phi_i(G): the forward apply to
//   the occupied orbitals, scaled.
// * Jastrow tables of tc2x (Gamma only).  calc_hamiltonian_tc2x.cpp:255-401
//   make E2 linear in V_2body(G; s, s) and in du_d(G) = G_d u(G; s, s):
//     E2 = c sum_{i,j} f_i f_j sum_G [ V_2body(G) rho_ij(G) rho_ji(-G)
//          + sum_d G_d u(G) (rho^d_ij(G) rho_ji(-G) - rho_ij(G) rho^d_ji(-G)) ],
//   rho_ij = FFT(conj(chi_i) phi_j), rho^d_ij = FFT(conj(chi_i) grad_d phi_j),
//   c = t / (2 N_k) with t the two-body factor -1/(N_k Omega) (halved when
//   unpolarised).  The gradient tables are these sums with V_2body or u
//   removed; the pair densities are recomputed per block of pairs, never
//   stored for all pairs at once.
#pragma once
#include "terms.cuh"

namespace tcg {

// out[q] = conj(A[q]) B[q] of one pair grid (FP64), q over the N points
template <typename T>
__global__ void k_pair_prod64(int N, int npair, const typename C2<T>::t *const *A, const typename C2<T>::t *const *B,
                              double2 *out)
{
    const int pr = blockIdx.y;
    if (pr >= npair) return;
    const typename C2<T>::t *a = A[pr], *b = B[pr];
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < N; p += gridDim.x * blockDim.x)
        out[(size_t)pr * N + p] = cmulc(to64(a[p]), to64(b[p]));
}

struct GradPair {
    int g;              // first of the pair's 8 G-space grids: rho_ij, rho^d_ij (3), rho_ji, rho^d_ji (3)
    double w;           // c f_i f_j (i != j: both orders are held by the 8 grids)
    int both;           // 1: add the (j, i) order too
};

// dV2(G) += w [rho_ij(G) rho_ji(-G) (+ swap)],
// du(G)  += w sum_d G_d [rho^d_ij(G) rho_ji(-G) - rho_ij(G) rho^d_ji(-G) (+ swap)]
static __global__ void k_grad_tc2x(GridDesc g, RecipC rc, int npair, const GradPair *pairs, const double2 *G8,
                                   double2 *dv2, double2 *du)
{
    const double zero[3] = {0, 0, 0};
    const size_t N = g.N;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += gridDim.x * blockDim.x) {
        int x, y, z;
        xyz_of(g, p, x, y, z);
        double G[3];
        gvec(rc.R, g, x, y, z, zero, G);
        const int nx = x == 0 ? 0 : g.n0 - x, ny = y == 0 ? 0 : g.n1 - y, nz = z == 0 ? 0 : g.n2 - z;
        const size_t q = (size_t)nx + (size_t)g.n0 * (ny + (size_t)g.n1 * nz);   // -G
        double2 av = {0, 0}, au = {0, 0};
        for (int k = 0; k < npair; k++) {
            const GradPair P = pairs[k];
            const double2 *r = G8 + (size_t)P.g * N;
            for (int o = 0; o < (P.both ? 2 : 1); o++) {
                const double2 *rij = r + (size_t)(o ? 4 : 0) * N, *rji = r + (size_t)(o ? 0 : 4) * N;
                double2 t = cmul(rij[p], rji[q]);
                av = {av.x + P.w * t.x, av.y + P.w * t.y};
                for (int d = 0; d < 3; d++) {
                    t = csub(cmul(rij[(size_t)(1 + d) * N + p], rji[q]), cmul(rij[p], rji[(size_t)(1 + d) * N + q]));
                    au = {au.x + P.w * G[d] * t.x, au.y + P.w * G[d] * t.y};
                }
            }
        }
        dv2[p] = cadd(dv2[p], av);
        du[p] = cadd(du[p], au);
    }
}

// dE/d conj(chi_b) = fac_b (h2 + h3) for the applied (occupied) bands,
// scattered into the [spin][k][nbands][npw] layout of the orbitals
struct GradBand {
    const double2 *h2, *h3;
    double2 *out;
    double fac;
    int npw;
};
static __global__ void k_grad_orbital(const GradBand *bands)
{
    const GradBand b = bands[blockIdx.y];
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < b.npw; p += gridDim.x * blockDim.x) {
        double2 v = {0, 0};
        if (b.h2) v = cadd(v, b.h2[p]);
        if (b.h3) v = cadd(v, b.h3[p]);
        b.out[p] = cscale(v, b.fac);
    }
}

// two-body Jastrow-table gradients (Gamma only), spin s
template <typename T>
static int grad_tables_tc2x(tcg_ctx *c, int s, double2 *dv2, double2 *du)
{
    PhaseScope ps_(c, "grad:tc2x");
    using V = typename C2<T>::t;
    Host &h = c->h;
    const size_t N = h.N;
    const bool bitc = h.method == TCG_METHOD_BITC;
    const int no = h.nocc[s * h.nk + 0];
    const size_t g0 = h.occ_off[(size_t)s * h.nk_all + 0];
    double tb = -1.0 / (h.num_kpoints * h.omega);
    if (h.nspin == 1) tb /= 2.0;
    const double cfac = tb / (2.0 * h.num_kpoints);
    std::vector<double> f(no);
    for (int i = 0; i < no; i++) f[i] = h.filling[fill_off(h, s, 0) + i];
    std::vector<std::pair<int, int>> pairs;
    for (int i = 0; i < no; i++)
        for (int j = i; j < no; j++) pairs.emplace_back(i, j);
    const V *Rphi = c->Rocc.as<V>(), *Rch = bitc ? c->Rchi.as<V>() : c->Rocc.as<V>(), *Rg = c->Rgrad.as<V>();
    const size_t per = 8 * N * sizeof(double2);
    const size_t blk = std::max<size_t>(1, std::min<size_t>(pairs.size(), ((size_t)1 << 30) / per));
    TRY(c->adjw.ensure(blk * per));
    double2 *G8 = c->adjw.as<double2>();
    const unsigned pblocks = (unsigned)std::min<size_t>(148 * 8, (N + 255) / 256);
    for (size_t b0 = 0; b0 < pairs.size(); b0 += blk) {
        const size_t nb = std::min(blk, pairs.size() - b0);
        std::vector<const V *> A(nb * 8), B(nb * 8);
        std::vector<GradPair> gp(nb);
        for (size_t k = 0; k < nb; k++) {
            const int i = pairs[b0 + k].first, j = pairs[b0 + k].second;
            // rho_ij = conj(chi_i) phi_j, rho^d_ij = conj(chi_i) grad_d phi_j; then (j, i)
            for (int o = 0; o < 2; o++) {
                const int a = o ? j : i, bb = o ? i : j;
                A[k * 8 + 4 * o] = Rch + (g0 + a) * N;
                B[k * 8 + 4 * o] = Rphi + (g0 + bb) * N;
                for (int d = 0; d < 3; d++) {
                    A[k * 8 + 4 * o + 1 + d] = Rch + (g0 + a) * N;
                    B[k * 8 + 4 * o + 1 + d] = Rg + ((g0 + bb) * 3 + d) * N;
                }
            }
            gp[k].g = (int)(8 * k);
            gp[k].w = cfac * f[i] * f[j];
            gp[k].both = i != j;
        }
        TRY(c->items.ensure(nb * 8 * 2 * sizeof(void *) + nb * sizeof(GradPair)));
        const V **dA = c->items.as<const V *>();
        const V **dB = dA + nb * 8;
        GradPair *dP = reinterpret_cast<GradPair *>(dB + nb * 8);
        TCG_CUDA(cudaMemcpyAsync(dA, A.data(), nb * 8 * sizeof(void *), cudaMemcpyHostToDevice, c->stream));
        TCG_CUDA(cudaMemcpyAsync(dB, B.data(), nb * 8 * sizeof(void *), cudaMemcpyHostToDevice, c->stream));
        TCG_CUDA(cudaMemcpyAsync(dP, gp.data(), nb * sizeof(GradPair), cudaMemcpyHostToDevice, c->stream));
        for (size_t q0 = 0; q0 < nb * 8; q0 += 65535)
            TRY(launch(c, k_pair_prod64<T>, dim3((unsigned)std::min<size_t>(64, (N + 255) / 256),
                                                 (unsigned)std::min<size_t>(65535, nb * 8 - q0)),
                       dim3(256), 0, (int)N, (int)std::min<size_t>(65535, nb * 8 - q0), (const V *const *)(dA + q0),
                       (const V *const *)(dB + q0), G8 + q0 * N));
        TCG_CUDA(cudaStreamSynchronize(c->stream));   // c->items is reused by the FFT helper
        std::vector<void *> grids(nb * 8);
        for (size_t q = 0; q < nb * 8; q++) grids[q] = G8 + q * N;
        TRY((fft3_list<double, -1>(c, grids)));
        TCG_CUDA(cudaMemcpyAsync(c->items.p, gp.data(), nb * sizeof(GradPair), cudaMemcpyHostToDevice, c->stream));
        RecipC rc;
        memcpy(rc.R, h.recip, sizeof rc.R);
        TRY(launch(c, k_grad_tc2x, dim3(pblocks), dim3(256), 0, c->gd, rc, (int)nb, (const GradPair *)c->items.p,
                   (const double2 *)G8, dv2, du));
        TCG_CUDA(cudaStreamSynchronize(c->stream));
    }
    return TCG_OK;
}

template <typename T>
static int energy_grad_impl(tcg_ctx *c, uint32_t mask, double *e_out, void *dchi, double *du_out, double *dv2_out)
{
    Host &h = c->h;
    const size_t N = h.N;
    // the occupied right orbitals as the applied block
    std::vector<int32_t> nb((size_t)h.nspin * h.nk);
    size_t n = 0;
    for (int s = 0; s < h.nspin; s++)
        for (int k = 0; k < h.nk; k++) {
            nb[s * h.nk + k] = h.nocc[s * h.nk + k];
            n += (size_t)nb[s * h.nk + k] * h.npw[k];
        }
    TRY(c->gpsi.ensure(std::max<size_t>(16, 3 * n * sizeof(double2))));
    double2 *psi = c->gpsi.as<double2>(), *h2 = psi + n, *h3 = psi + 2 * n;
    size_t o = 0;
    for (int s = 0; s < h.nspin; s++)
        for (int k = 0; k < h.nk; k++) {
            const size_t bytes = (size_t)nb[s * h.nk + k] * h.npw[k] * sizeof(double2);
            if (bytes)
                TCG_CUDA(cudaMemcpyAsync(psi + o, c->phik.as<double2>() + h.orb_off[(size_t)s * h.nk + k], bytes,
                                         cudaMemcpyDeviceToDevice, c->stream));
            o += (size_t)nb[s * h.nk + k] * h.npw[k];
        }
    TCG_CUDA(cudaMemsetAsync(h2, 0, 2 * n * sizeof(double2), c->stream));
    ApplyArgs A{};
    A.mask = mask;
    A.nb = nb.data();
    A.psi = psi;
    A.h2 = h2;
    A.h3 = h3;
    if (n) TRY(apply_impl<T>(c, A));
    TRY(tcg_energy(c, nb.data(), (mask & TCG_TERMS_H2) ? h2 : nullptr, (mask & ~TCG_TERMS_H2) ? h3 : nullptr, e_out));
    if (dchi) {
        size_t norb = 0;
        for (int s = 0; s < h.nspin; s++)
            for (int k = 0; k < h.nk; k++) norb += (size_t)h.nbands[s] * h.npw[k];
        TCG_CUDA(cudaMemsetAsync(dchi, 0, norb * sizeof(double2), c->stream));
        std::vector<GradBand> gb;
        o = 0;
        for (int s = 0; s < h.nspin; s++)
            for (int k = 0; k < h.nk; k++)
                for (int b = 0; b < nb[s * h.nk + k]; b++, o += h.npw[k]) {
                    GradBand x;
                    x.h2 = (mask & TCG_TERMS_H2) ? h2 + o : nullptr;
                    x.h3 = (mask & ~TCG_TERMS_H2) ? h3 + o : nullptr;
                    x.out = (double2 *)dchi + h.orb_off[(size_t)s * h.nk + k] + (size_t)b * h.npw[k];
                    x.fac = h.filling[fill_off(h, s, k) + b] / h.num_kpoints;
                    x.npw = h.npw[k];
                    gb.push_back(x);
                }
        if (!gb.empty()) {
            TRY(c->items.ensure(gb.size() * sizeof(GradBand)));
            TCG_CUDA(cudaMemcpyAsync(c->items.p, gb.data(), gb.size() * sizeof(GradBand), cudaMemcpyHostToDevice,
                                     c->stream));
            for (size_t b0 = 0; b0 < gb.size(); b0 += 65535)
                TRY(launch(c, k_grad_orbital, dim3(4, (unsigned)std::min<size_t>(65535, gb.size() - b0)), dim3(256), 0,
                           (const GradBand *)(c->items.as<GradBand>() + b0)));
            TCG_CUDA(cudaStreamSynchronize(c->stream));
        }
    }
    if (du_out || dv2_out) {
        TRY(c->adjt.ensure((size_t)2 * h.nspin * N * sizeof(double2)));
        double2 *dv2 = c->adjt.as<double2>(), *du = dv2 + (size_t)h.nspin * N;
        TCG_CUDA(cudaMemsetAsync(dv2, 0, (size_t)2 * h.nspin * N * sizeof(double2), c->stream));
        for (int s = 0; s < h.nspin; s++) TRY(grad_tables_tc2x<T>(c, s, dv2 + (size_t)s * N, du + (size_t)s * N));
        if (dv2_out)
            TCG_CUDA(cudaMemcpyAsync(dv2_out, dv2, (size_t)h.nspin * N * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
        if (du_out)
            TCG_CUDA(cudaMemcpyAsync(du_out, du, (size_t)h.nspin * N * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
        TCG_CUDA(cudaStreamSynchronize(c->stream));
    }
    return TCG_OK;
}

} // namespace tcg
