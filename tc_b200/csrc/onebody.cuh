// onebody.cuh -- one-body terms of H phi on the device:
//   kinetic     calc_hamiltonian_kinetic.cpp:6-52   H1 += 1/2 |k+G|^2 phi(G)
//   pseudo      calc_hamiltonian_pseudo.cpp:6-180   non-local (Kleinman-Bylander
//               projectors, D_ij) + local V_loc(r) phi(r)
// The projector values <beta_{ip,m}|k+G> come from the caller
// (Potentials::projector_nonlocal in TC++); the exp(i G.R_atom) factor of
// every atom is applied at tcg_set_pseudo, giving per k a dense block
// B[c][G], c = (atom, projector, m).  Then per band
//   coeff_c = sum_G B_c(G) phi(G),  t = D coeff,  H1(G) += sum_c conj(B_c(G)) t_c,
// with D coupling components of the same atom and m (pseudo_dij).
#pragma once
#include "terms.cuh"

namespace tcg {

struct NLItem {
    const double2 *psi;      // [npw]
    double2 *h;              // [npw] accumulate
    const double2 *B;        // [ncomp][npw]
    int npw;
};

// one block per band; D as CSR over columns: for component c, rows
// dcol[dptr[c] .. dptr[c+1]) with values dval
static __global__ void __launch_bounds__(256) k_nonlocal(const NLItem *items, int ncomp, const int *dptr,
                                                         const int *dcol, const double *dval)
{
    const NLItem it = items[blockIdx.x];
    extern __shared__ double2 sh[];           // [ncomp] coefficients, [ncomp] t, [256] reduction
    double2 *coeff = sh, *tv = sh + ncomp, *red = sh + 2 * ncomp;
    for (int cc = 0; cc < ncomp; cc++) {
        double2 loc = {0, 0};
        const double2 *b = it.B + (size_t)cc * it.npw;
        for (int p = threadIdx.x; p < it.npw; p += blockDim.x) loc = cadd(loc, cmul(b[p], it.psi[p]));
        red[threadIdx.x] = loc;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) red[threadIdx.x] = cadd(red[threadIdx.x], red[threadIdx.x + s]);
            __syncthreads();
        }
        if (threadIdx.x == 0) coeff[cc] = red[0];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int cc = 0; cc < ncomp; cc++) tv[cc] = {0, 0};
        for (int cc = 0; cc < ncomp; cc++)
            for (int e = dptr[cc]; e < dptr[cc + 1]; e++) tv[dcol[e]] = cadd(tv[dcol[e]], cscale(coeff[cc], dval[e]));
    }
    __syncthreads();
    for (int p = threadIdx.x; p < it.npw; p += blockDim.x) {
        double2 hv = it.h[p];
        for (int cc = 0; cc < ncomp; cc++) hv = cadd(hv, cmulc(it.B[(size_t)cc * it.npw + p], tv[cc]));
        it.h[p] = hv;
    }
}

struct KinItem {
    const double2 *psi;
    double2 *h;
    const int *g0;           // [npw] grid index of each plane wave
    double k[3];             // Cartesian k
    int npw;
};

// H1 += 1/2 |k+G|^2 phi (calc_hamiltonian_kinetic.cpp:35-41)
static __global__ void k_kinetic(const KinItem *items, GridDesc g, RecipC rc)
{
    const KinItem it = items[blockIdx.y];
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < it.npw; p += gridDim.x * blockDim.x) {
        int x, y, z;
        xyz_of(g, (size_t)it.g0[p], x, y, z);
        double G[3];
        gvec(rc.R, g, x, y, z, it.k, G);
        const double e = 0.5 * (G[0] * G[0] + G[1] * G[1] + G[2] * G[2]);
        it.h[p] = cadd(it.h[p], cscale(it.psi[p], e));
    }
}

// acc[t] += V(r) phi_t(r), V real (calc_hamiltonian_pseudo.cpp:163-171)
template <typename T>
__global__ void k_local_real(int N, const typename C2<T>::t *Rpsi, const double *Vr, double2 *acc)
{
    const size_t t = blockIdx.y;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < N; p += gridDim.x * blockDim.x)
        acc_add(acc + t * N + p, to64(Rpsi[t * N + p]), Vr[p]);
}

// Upload of the pseudopotential: vloc, B = exp(i G.R_atom) x projector per k,
// and D between components as CSR.
static int set_pseudo(tcg_ctx *c, const tcg_pseudo_desc *pp)
{
    Host &h = c->h;
    if (!pp) return fail(TCG_ERR_ARG, "null pseudopotential descriptor");
    if (pp->nspecies < 0 || pp->natoms < 0) return fail(TCG_ERR_ARG, "negative species / atom count");
    if (pp->natoms > 0 && (!pp->species_of_atom || !pp->atom_pos || !pp->nproj || !pp->lbeta || !pp->dij ||
                           !pp->projector))
        return fail(TCG_ERR_ARG, "missing projector arrays");
    std::vector<int> poff(pp->nspecies + 1, 0), doff(pp->nspecies + 1, 0), coff;
    std::vector<int> spc_first(pp->nspecies + 1, 0);   // first component of a species in one k block
    int nspc = 0;
    for (int is = 0; is < pp->nspecies; is++) {
        if (pp->nproj[is] < 0) return fail(TCG_ERR_ARG, "negative projector count");
        poff[is + 1] = poff[is] + pp->nproj[is];
        doff[is + 1] = doff[is] + pp->nproj[is] * pp->nproj[is];
        spc_first[is] = nspc;
        for (int ip = 0; ip < pp->nproj[is]; ip++) {
            const int l = pp->lbeta[poff[is] + ip];
            if (l < 0 || l > 3) return fail(TCG_ERR_UNSUPPORTED, "projector l outside 0..3");
            coff.push_back(nspc);
            nspc += 2 * l + 1;
        }
    }
    spc_first[pp->nspecies] = nspc;
    for (int ia = 0; ia < pp->natoms; ia++)
        if (pp->species_of_atom[ia] < 0 || pp->species_of_atom[ia] >= pp->nspecies)
            return fail(TCG_ERR_ARG, "species index out of range");
    // components of the atoms: (atom, ip, m) in atom-major order
    std::vector<int> atom_first(pp->natoms + 1, 0);
    for (int ia = 0; ia < pp->natoms; ia++) {
        const int is = pp->species_of_atom[ia];
        atom_first[ia + 1] = atom_first[ia] + spc_first[is + 1] - spc_first[is];
    }
    const int ncomp = atom_first[pp->natoms];
    // D as CSR over columns (atom, jp, m): rows (atom, ip, m) with |D(ip, jp)| > 1e-8
    std::vector<int> dptr(ncomp + 1, 0), dcol;
    std::vector<double> dval;
    for (int ia = 0; ia < pp->natoms; ia++) {
        const int is = pp->species_of_atom[ia], np = pp->nproj[is];
        for (int jp = 0; jp < np; jp++) {
            const int lj = pp->lbeta[poff[is] + jp];
            for (int m = 0; m < 2 * lj + 1; m++) {
                const int col = atom_first[ia] + coff[poff[is] + jp] - spc_first[is] + m;
                for (int ip = 0; ip < np; ip++) {
                    const double D = pp->dij[doff[is] + ip * np + jp];
                    if (!(fabs(D) > 1e-8)) continue;
                    if (pp->lbeta[poff[is] + ip] != lj)
                        return fail(TCG_ERR_ARG, "dij is not diagonal w.r.t. l in pseudopot.");
                    dcol.push_back(atom_first[ia] + coff[poff[is] + ip] - spc_first[is] + m);
                    dval.push_back(D);
                }
                dptr[col + 1] = (int)dcol.size();
            }
        }
    }
    // B per irreducible k (isym 0, spin 0's plane waves; the reference uses
    // Gindex_at_k[ispin][ik][0], identical for both spins)
    std::vector<double2> B;
    h.nl_koff.assign(h.nk + 1, 0);
    const double2 *proj = (const double2 *)pp->projector;
    size_t pin = 0;
    for (int k = 0; k < h.nk; k++) {
        h.nl_koff[k] = B.size();
        const int npw = h.npw[k];
        const size_t o = h.gidx_off[h.kall_off[k]];
        // plane wave -> grid index -> signed Miller index -> Cartesian G (without k)
        for (int ia = 0; ia < pp->natoms; ia++) {
            const int is = pp->species_of_atom[ia];
            const double *R = pp->atom_pos + 3 * ia;
            const int ns = spc_first[is + 1] - spc_first[is];
            for (int cc = 0; cc < ns; cc++) {
                const double2 *src = proj + pin + (size_t)(spc_first[is] + cc) * npw;
                for (int p = 0; p < npw; p++) {
                    const int gi = h.gidx_host[o + p];
                    const int m0 = gi % h.n[0], m1 = (gi / h.n[0]) % h.n[1], m2 = gi / (h.n[0] * h.n[1]);
                    const double mm[3] = {(double)(m0 <= h.n[0] / 2 ? m0 : m0 - h.n[0]),
                                          (double)(m1 <= h.n[1] / 2 ? m1 : m1 - h.n[1]),
                                          (double)(m2 <= h.n[2] / 2 ? m2 : m2 - h.n[2])};
                    double G[3];
                    for (int d = 0; d < 3; d++)
                        G[d] = h.recip[0 * 3 + d] * mm[0] + h.recip[1 * 3 + d] * mm[1] + h.recip[2 * 3 + d] * mm[2];
                    const double arg = G[0] * R[0] + G[1] * R[1] + G[2] * R[2];
                    const double cs = cos(arg), sn = sin(arg);
                    const double2 v = src[p];
                    B.push_back(make_double2(cs * v.x - sn * v.y, cs * v.y + sn * v.x));
                }
            }
        }
        pin += (size_t)nspc * npw;
    }
    h.nl_koff[h.nk] = B.size();
    h.nl_ncomp = ncomp;
    std::vector<unsigned char> dbytes((ncomp + 1 + dcol.size()) * sizeof(int) + dval.size() * sizeof(double) + 16);
    memcpy(dbytes.data(), dptr.data(), (ncomp + 1) * sizeof(int));
    memcpy(dbytes.data() + (ncomp + 1) * sizeof(int), dcol.data(), dcol.size() * sizeof(int));
    const size_t voff = ((ncomp + 1 + dcol.size()) * sizeof(int) + 7) & ~(size_t)7;
    dbytes.resize(voff + dval.size() * sizeof(double) + 8);
    memcpy(dbytes.data() + voff, dval.data(), dval.size() * sizeof(double));
    h.nl_dval_off = voff;
    TRY(up(c->nlB, B.data(), std::max<size_t>(1, B.size()) * sizeof(double2), c->stream));
    TRY(up(c->nlD, dbytes.data(), dbytes.size(), c->stream));
    h.have_vloc = pp->vloc != nullptr;
    if (h.have_vloc) {
        for (int i = 0; i < h.N; i++)
            if (!std::isfinite(pp->vloc[i])) return fail(TCG_ERR_NUMERIC, "non-finite local pseudopotential");
        TRY(up(c->vloc, pp->vloc, (size_t)h.N * sizeof(double), c->stream));
    }
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    h.have_pseudo = true;
    return TCG_OK;
}

template <typename T>
static int apply_h1_impl(tcg_ctx *c, uint32_t mask, const int32_t *nb, const double2 *psi, double2 *h1,
                         const uint8_t *owned)
{
    PhaseScope ps_(c, "ap:h1");
    using V = typename C2<T>::t;
    Host &h = c->h;
    const size_t N = h.N;
    ApplyArgs A{};
    A.mask = mask;
    A.nb = nb;
    A.owned = owned;
    A.psi = psi;
    Targets Tg = make_targets(c, A);
    const size_t nt = Tg.s.size();
    if (nt == 0) return TCG_OK;
    RecipC rc;
    memcpy(rc.R, h.recip, sizeof rc.R);
    if (mask & TCG_TERM_KINETIC) {
        std::vector<KinItem> it(nt);
        for (size_t t = 0; t < nt; t++) {
            it[t].psi = psi + Tg.psi_off[t];
            it[t].h = h1 + Tg.psi_off[t];
            it[t].g0 = c->gidx0.as<int>() + h.g0_off[(size_t)Tg.s[t] * h.nk + Tg.k[t]];
            cart(h, &h.kvec[3 * h.kall_off[Tg.k[t]]], it[t].k);
            it[t].npw = h.npw[Tg.k[t]];
        }
        TRY(c->items.ensure(nt * sizeof(KinItem)));
        TCG_CUDA(cudaMemcpyAsync(c->items.p, it.data(), nt * sizeof(KinItem), cudaMemcpyHostToDevice, c->stream));
        for (size_t b0 = 0; b0 < nt; b0 += 65535)
            TRY(launch(c, k_kinetic, dim3(4, (unsigned)std::min<size_t>(65535, nt - b0)), dim3(256), 0,
                       (const KinItem *)(c->items.as<KinItem>() + b0), c->gd, rc));
        TCG_CUDA(cudaStreamSynchronize(c->stream));   // c->items is reused below
    }
    if ((mask & TCG_TERM_PSEUDO) && h.nl_ncomp > 0) {
        std::vector<NLItem> it(nt);
        for (size_t t = 0; t < nt; t++) {
            it[t].psi = psi + Tg.psi_off[t];
            it[t].h = h1 + Tg.psi_off[t];
            it[t].B = c->nlB.as<double2>() + h.nl_koff[Tg.k[t]];
            it[t].npw = h.npw[Tg.k[t]];
        }
        TRY(c->items.ensure(nt * sizeof(NLItem)));
        TCG_CUDA(cudaMemcpyAsync(c->items.p, it.data(), nt * sizeof(NLItem), cudaMemcpyHostToDevice, c->stream));
        const int nc = h.nl_ncomp;
        const int *dptr = c->nlD.as<int>();
        const double *dval = reinterpret_cast<const double *>(c->nlD.as<char>() + h.nl_dval_off);
        TRY(launch(c, k_nonlocal, dim3((unsigned)nt), dim3(256), (2 * nc + 256) * sizeof(double2),
                   (const NLItem *)c->items.p, nc, dptr, dptr + nc + 1, dval));
        TCG_CUDA(cudaStreamSynchronize(c->stream));
    }
    if ((mask & TCG_TERM_PSEUDO) && h.have_vloc) {
        TRY(c->Rpsi.ensure(nt * N * sizeof(V)));
        std::vector<SphereItem> items;
        for (size_t t = 0; t < nt; t++) {
            const int s = Tg.s[t], k = Tg.k[t], a = h.kall_off[k];
            SphereItem si{};
            si.coef = psi + Tg.psi_off[t];
            si.inv = c->inv.as<int>() + ((size_t)s * h.nk_all + a) * N;
            si.phase = c->phase.as<double2>() + h.gidx_off[(size_t)s * h.nk_all + a];
            si.out = c->Rpsi.as<V>() + t * N;
            items.push_back(si);
        }
        TRY(sphere_to_r<T>(c, items));
        TRY(c->acc1.ensure(nt * N * sizeof(double2)));
        const unsigned pblocks = (unsigned)std::min<size_t>(148 * 8, (nt * N + 255) / 256);
        TRY(launch(c, k_zero, dim3(pblocks), dim3(256), 0, c->acc1.as<double2>(), nt * N));
        for (size_t b0 = 0; b0 < nt; b0 += 65535)
            TRY(launch(c, k_local_real<T>, dim3((unsigned)std::min<size_t>(64, (N + 255) / 256),
                                                (unsigned)std::min<size_t>(65535, nt - b0)),
                       dim3(256), 0, (int)N, (const V *)(c->Rpsi.as<V>() + b0 * N), (const double *)c->vloc.p,
                       c->acc1.as<double2>() + b0 * N));
        TRY(finalize_acc(c, Tg, c->acc1.as<double2>(), h1, 1.0));
    }
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    return TCG_OK;
}

} // namespace tcg
