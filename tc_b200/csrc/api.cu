// api.cu -- C-ABI entry points (include/tcg.h): context life cycle, state
// upload, the apply orchestration and the host-visible helpers.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <mutex>
#include <unordered_set>
#include "ctx.cuh"
#include "passes.cuh"
#include "util.cuh"
#include "terms.cuh"
#include "onebody.cuh"

namespace tcg {

static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

} // namespace tcg

using namespace tcg;

// ================================================================ C-ABI ====
extern "C" const char *tcg_last_error(void) { return tcg::g_err; }
extern "C" const char *tcg_version(void) { return "tcg_b200 0.1 (sm_100a)"; }
extern "C" void *tcg_stream(tcg_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }
extern "C" int64_t tcg_launch_count(const tcg_ctx *ctx) { return ctx ? ctx->launches : 0; }

static int validate_system(const tcg_system_desc *s)
{
    if (!s) return fail(TCG_ERR_ARG, "null system descriptor");
    for (int d = 0; d < 3; d++)
        if (s->nr[d] < 1) return fail(TCG_ERR_ARG, "FFT grid must be positive");
    if (s->nspin != 1 && s->nspin != 2) return fail(TCG_ERR_ARG, "nspin must be 1 or 2");
    if (s->calc_method < TCG_METHOD_HF || s->calc_method > TCG_METHOD_BITC) return fail(TCG_ERR_ARG, "bad calc_method");
    if (s->nk_irr < 1 || s->num_kpoints < 1) return fail(TCG_ERR_ARG, "no k-points");
    if (!s->nsym_k || !s->kvec || !s->time_rev || !s->npw || !s->gindex || !s->phase)
        return fail(TCG_ERR_ARG, "missing k-point / G-vector arrays");
    if (!(s->omega > 0)) return fail(TCG_ERR_ARG, "unit-cell volume must be positive");
    if (s->includes_div_correction && !s->sum_Vaux) return fail(TCG_ERR_ARG, "sum_Vaux required with div correction");
    if (s->nsymop < 0) return fail(TCG_ERR_ARG, "negative nsymop");
    return TCG_OK;
}

// Pencil table of the pruned transforms (36^3 path).  A pair density
// conj(a_q(r)) b_k(r) of two orbitals on the plane-wave spheres of q and k
// has Fourier components G = G1 - G2 with |k + G1| <= R_k and |q + G2| <= R_q,
// so it vanishes outside the ball |G + k - q| < R_k + R_q; for every
// (irreducible k, all-k q) pair the table marks the (x, y) pencils of the grid
// that meet that ball, and lists them first.  Built only when no ball reaches
// past the grid's Miller range (the support would wrap) and the table stays
// under 256 MB.
static int build_prune_table(tcg_ctx *c)
{
    Host &h = c->h;
    c->prune_ok = false;
    const int n0 = h.n[0], n1 = h.n[1], n2 = h.n[2], np = n0 * n1;
    const size_t nent = (size_t)h.nk * h.nk_all;
    if (nent * np * 3 + nent * sizeof(int) + nent * n0 * 8 > ((size_t)256 << 20)) return TCG_OK;
    auto cartv = [&](const double *x, double *v) {
        for (int d = 0; d < 3; d++) v[d] = h.recip[0 * 3 + d] * x[0] + h.recip[1 * 3 + d] * x[1] + h.recip[2 * 3 + d] * x[2];
    };
    auto signed_m = [](int i, int n) { return i <= n / 2 ? i : i - n; };
    // sphere radius of every irreducible k: max |k + G| over its plane waves
    std::vector<double> R(h.nk, 0.0);
    for (int k = 0; k < h.nk; k++) {
        double kc[3];
        cartv(&h.kvec[3 * h.kall_off[k]], kc);
        const size_t o = h.gidx_off[h.kall_off[k]];
        for (int p = 0; p < h.npw[k]; p++) {
            const int gi = h.gidx_host[o + p];
            const double m[3] = {(double)signed_m(gi % n0, n0), (double)signed_m((gi / n0) % n1, n1),
                                 (double)signed_m(gi / np, n2)};
            double G[3];
            cartv(m, G);
            const double r = sqrt((kc[0] + G[0]) * (kc[0] + G[0]) + (kc[1] + G[1]) * (kc[1] + G[1]) +
                                  (kc[2] + G[2]) * (kc[2] + G[2]));
            R[k] = std::max(R[k], r);
        }
    }
    // |a_i| / (2 pi): Miller extent of a Cartesian length
    double alen[3];
    for (int i = 0; i < 3; i++)
        alen[i] = sqrt(h.lattice[3 * i] * h.lattice[3 * i] + h.lattice[3 * i + 1] * h.lattice[3 * i + 1] +
                       h.lattice[3 * i + 2] * h.lattice[3 * i + 2]) / (2.0 * PI_D);
    const double *b1 = &h.recip[0], *b2 = &h.recip[3], *b3 = &h.recip[6];
    const double b33 = b3[0] * b3[0] + b3[1] * b3[1] + b3[2] * b3[2];
    if (n1 > 64) return TCG_OK;                       // column bit masks hold 64 rows
    const size_t bits_off = (nent * np * 3 + nent * sizeof(int) + 7) & ~(size_t)7;
    std::vector<unsigned char> tab(bits_off + nent * n0 * sizeof(unsigned long long));
    unsigned char *mask = tab.data();
    unsigned short *perm = reinterpret_cast<unsigned short *>(tab.data() + nent * np);
    int *nact = reinterpret_cast<int *>(tab.data() + nent * np * 3);
    unsigned long long *bits = reinterpret_cast<unsigned long long *>(tab.data() + bits_off);
    const int zlo = -((n2 - 1) / 2), zhi = n2 / 2;
    for (int ik = 0; ik < h.nk; ik++)
        for (int a = 0; a < h.nk_all; a++) {
            const size_t e = (size_t)ik * h.nk_all + a;
            double kk[3], qq[3], kq[3];
            cartv(&h.kvec[3 * h.kall_off[ik]], kk);
            cartv(&h.kvec[3 * a], qq);
            for (int d = 0; d < 3; d++) kq[d] = kk[d] - qq[d];
            const double Rr = (R[ik] + R[h.ik_of_all[a]]) * (1.0 + 1e-9) + 1e-9;
            // the ball centre -kq in Miller coordinates: m_i = -kq . a_i / (2 pi)
            for (int i = 0; i < 3; i++) {
                const double ci = -(kq[0] * h.lattice[3 * i] + kq[1] * h.lattice[3 * i + 1] + kq[2] * h.lattice[3 * i + 2]) /
                                  (2.0 * PI_D);
                if (fabs(ci) + Rr * alen[i] >= (h.n[i] - 1) / 2.0) return TCG_OK;   // support could wrap
            }
            int na = 0;
            std::vector<int> act, inact;
            for (int y = 0; y < n1; y++)
                for (int x = 0; x < n0; x++) {
                    const int mx = signed_m(x, n0), my = signed_m(y, n1);
                    double P[3];
                    for (int d = 0; d < 3; d++) P[d] = mx * b1[d] + my * b2[d] + kq[d];
                    const double bb = P[0] * b3[0] + P[1] * b3[1] + P[2] * b3[2];
                    const double cc = P[0] * P[0] + P[1] * P[1] + P[2] * P[2] - Rr * Rr;
                    const double disc = bb * bb - b33 * cc;
                    bool on = false;
                    if (disc >= 0) {
                        const double lo = (-bb - sqrt(disc)) / b33 - 1e-9, hi = (-bb + sqrt(disc)) / b33 + 1e-9;
                        const double zl = std::max(ceil(lo), (double)zlo), zh = std::min(floor(hi), (double)zhi);
                        on = zl <= zh;
                    }
                    mask[e * np + x + n0 * y] = on ? 1 : 0;
                    if (on) bits[e * n0 + x] |= 1ull << y;
                    (on ? act : inact).push_back(x + n0 * y);
                    na += on;
                }
            for (size_t i = 0; i < act.size(); i++) perm[e * np + i] = (unsigned short)act[i];
            for (size_t i = 0; i < inact.size(); i++) perm[e * np + act.size() + i] = (unsigned short)inact[i];
            nact[e] = na;
        }
    TRY(up(c->prune_tab, tab.data(), tab.size(), c->stream));
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    c->prune_nact.assign(nact, nact + nent);
    c->prune_ok = true;
    return TCG_OK;
}

extern "C" int tcg_ctx_create(const tcg_system_desc *sys, int32_t precision, tcg_ctx **out)
{
    if (!out) return fail(TCG_ERR_ARG, "null output pointer");
    *out = nullptr;
    TRY(validate_system(sys));
    if (precision != TCG_PREC_FP64 && precision != TCG_PREC_MIXED) return fail(TCG_ERR_ARG, "bad precision");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(TCG_ERR_CUDA, "no CUDA device available");
    }
    tcg_ctx *c = new tcg_ctx();
    c->prec = precision;
    cudaGetDevice(&c->device);
    Host &h = c->h;
    for (int d = 0; d < 3; d++) h.n[d] = sys->nr[d];
    h.N = h.n[0] * h.n[1] * h.n[2];
    memcpy(h.recip, sys->recip, sizeof h.recip);
    memcpy(h.lattice, sys->lattice, sizeof h.lattice);
    h.omega = sys->omega;
    h.method = sys->calc_method;
    h.nspin = sys->nspin;
    h.nk = sys->nk_irr;
    h.num_kpoints = sys->num_kpoints;
    h.nsym_k.assign(sys->nsym_k, sys->nsym_k + h.nk);
    h.npw.assign(sys->npw, sys->npw + h.nk);
    h.kall_off.assign(h.nk + 1, 0);
    for (int k = 0; k < h.nk; k++) {
        if (h.nsym_k[k] < 1) { delete c; return fail(TCG_ERR_ARG, "nsym_k must be >= 1"); }
        if (h.npw[k] < 1) { delete c; return fail(TCG_ERR_ARG, "npw must be >= 1"); }
        h.kall_off[k + 1] = h.kall_off[k] + h.nsym_k[k];
    }
    h.nk_all = h.kall_off[h.nk];
    h.ik_of_all.resize(h.nk_all);
    for (int k = 0; k < h.nk; k++)
        for (int a = h.kall_off[k]; a < h.kall_off[k + 1]; a++) h.ik_of_all[a] = k;
    h.kvec.assign(sys->kvec, sys->kvec + 3 * h.nk_all);
    h.time_rev.assign(sys->time_rev, sys->time_rev + h.nk_all);
    h.nsymop = sys->nsymop;
    if (h.nsymop > 0) {
        if (!sys->rotation || !sys->translation || !sys->rot_index) { delete c; return fail(TCG_ERR_ARG, "missing symmetry arrays"); }
        h.rotation.assign(sys->rotation, sys->rotation + 9 * h.nsymop);
        h.translation.assign(sys->translation, sys->translation + 3 * h.nsymop);
        h.rot_index.assign(sys->rot_index, sys->rot_index + h.nk_all);
        for (int a = 0; a < h.nk_all; a++)
            if (h.rot_index[a] < 0 || h.rot_index[a] >= h.nsymop) { delete c; return fail(TCG_ERR_ARG, "rot_index out of range"); }
    } else {
        for (int a = 0; a < h.nk_all; a++)
            if (h.nsym_k[h.ik_of_all[a]] > 1) { delete c; return fail(TCG_ERR_ARG, "symmetry-expanded k-points need rotations"); }
        h.rotation.assign(9, 0);
        h.rotation[0] = h.rotation[4] = h.rotation[8] = 1;
        h.translation.assign(3, 0.0);
        h.rot_index.assign(h.nk_all, 0);
        h.nsymop = 1;
    }
    memcpy(h.A, sys->jastrow_A, sizeof h.A);
    memcpy(h.F, sys->jastrow_F, sizeof h.F);
    h.A_zero = true;
    for (int i = 0; i < 4; i++)
        if (fabs(h.A[i]) > 1e-8) h.A_zero = false;
    if (!h.A_zero)
        for (int i = 0; i < 4; i++)
            if (!(fabs(h.F[i]) > 1e-8)) { delete c; return fail(TCG_ERR_ARG, "Jastrow F must be non-zero"); }
    h.div = sys->includes_div_correction != 0;
    h.alpha = sys->alpha_Vaux;
    if (h.div) {
        h.sum_vaux.assign(sys->sum_Vaux, sys->sum_Vaux + h.nk);
        if (!(h.alpha > 0)) { delete c; return fail(TCG_ERR_ARG, "alpha_Vaux must be positive"); }
    } else {
        h.sum_vaux.assign(h.nk, 0.0);
    }
    // SCF mesh check: every k-point must lie on the mesh (kVaux = 0)
    int rc = TCG_OK;
    // G maps
    h.gidx_off.resize((size_t)h.nspin * h.nk_all);
    size_t off = 0;
    for (int s = 0; s < h.nspin; s++)
        for (int a = 0; a < h.nk_all; a++) {
            h.gidx_off[(size_t)s * h.nk_all + a] = off;
            off += h.npw[h.ik_of_all[a]];
        }
    const size_t ngi = off;
    h.gidx_host.assign(sys->gindex, sys->gindex + ngi);
    std::vector<int> inv((size_t)h.nspin * h.nk_all * h.N, -1);
    for (int s = 0; s < h.nspin && rc == TCG_OK; s++)
        for (int a = 0; a < h.nk_all && rc == TCG_OK; a++) {
            const size_t o = h.gidx_off[(size_t)s * h.nk_all + a];
            int *im = inv.data() + ((size_t)s * h.nk_all + a) * h.N;
            for (int p = 0; p < h.npw[h.ik_of_all[a]]; p++) {
                const int gi = sys->gindex[o + p];
                if (gi < 0 || gi >= h.N) { rc = fail(TCG_ERR_ARG, "gindex out of range"); break; }
                if (im[gi] >= 0) { rc = fail(TCG_ERR_ARG, "duplicate gindex within one k-point"); break; }
                im[gi] = p;
            }
        }
    if (rc != TCG_OK) { delete c; return rc; }
    // plane-wave -> grid index of every (spin, irreducible k) at isym 0 (one-body terms)
    std::vector<int> g0;
    h.g0_off.resize((size_t)h.nspin * h.nk);
    for (int s = 0; s < h.nspin; s++)
        for (int k = 0; k < h.nk; k++) {
            h.g0_off[(size_t)s * h.nk + k] = g0.size();
            const size_t o = h.gidx_off[(size_t)s * h.nk_all + h.kall_off[k]];
            g0.insert(g0.end(), sys->gindex + o, sys->gindex + o + h.npw[k]);
        }
    // FFT plans
    GridDesc &g = c->gd;
    g.n0 = h.n[0]; g.n1 = h.n[1]; g.n2 = h.n[2]; g.N = h.N;
    for (int d = 0; d < 3; d++)
        if ((rc = make_axis(h.n[d], g.ax[d])) != TCG_OK) { delete c; return rc; }
    {
        const double PI = 3.14159265358979323846;
        std::vector<double2> t64(3 * MAXN);
        std::vector<float2> t32(3 * MAXN);
        for (int d = 0; d < 3; d++)
            for (int j = 0; j < h.n[d]; j++) {
                long double a = 2.0L * (long double)PI * j / h.n[d];
                double cr = (double)cosl(a), ci = -(double)sinl(a);
                t64[d * MAXN + j] = make_double2(cr, ci);
                t32[d * MAXN + j] = make_float2((float)cr, (float)ci);
            }
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            delete c;
            return fail(TCG_ERR_CUDA, "stream creation failed");
        }
        if ((rc = up(c->tw64, t64.data(), t64.size() * sizeof(double2), c->stream)) ||
            (rc = up(c->tw32, t32.data(), t32.size() * sizeof(float2), c->stream)) ||
            (rc = up(c->recip, h.recip, sizeof h.recip, c->stream)) ||
            (rc = up(c->inv, inv.data(), inv.size() * sizeof(int), c->stream)) ||
            (rc = up(c->phase, sys->phase, ngi * sizeof(double2), c->stream)) ||
            (rc = up(c->gidx0, g0.data(), g0.size() * sizeof(int), c->stream))) {
            tcg_ctx_destroy(c);
            return rc;
        }
        g.tw64 = c->tw64.as<const double2>();
        g.tw32 = c->tw32.as<const float2>();
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
        tcg_ctx_destroy(c);
        return fail(TCG_ERR_CUDA, "upload failed");
    }
    if (h.n[0] == h.n[1] && h.n[1] == h.n[2]) {
        const int fastn[] = {12, 16, 24, 32, 36, 40, 48};
        for (int f : fastn)
            if (h.n[0] == f) c->fast_n = f;
    }
    if (getenv("TCG_GENERIC_PASSES")) c->force_generic = true;
    if (getenv("TCG_NO_PRUNE")) c->no_prune = true;
    if (getenv("TCG_SACC")) c->use_sacc = true;
    if (getenv("TCG_NO_QP_SACC")) c->qp_sacc = false;
    if (getenv("TCG_NO_FUSE")) c->no_fuse = true;
    if (split_line_grid(c->fast_n) && (rc = build_prune_table(c)) != TCG_OK) {
        tcg_ctx_destroy(c);
        return rc;
    }
    if (const char *e = getenv("TCG_XY_KERNELS"))   // "line" / "pair": override the per-term choice
        c->xy_kernels = !strcmp(e, "line") ? 1 : (!strcmp(e, "pair") ? 2 : (!strcmp(e, "t6") ? 3 : 0));
    if (getenv("TCG_NO_PREFETCH")) c->no_prefetch = true;
    if (const char *e = getenv("TCG_MIN_TARGETS")) c->min_targets = atoi(e);
    if (const char *e = getenv("TCG_Z_KERNELS"))    // "line" / "split": override the per-term choice
        c->z_kernels = !strcmp(e, "line") ? 1 : (!strcmp(e, "split") ? 2 : (!strcmp(e, "t6") ? 3 : (!strcmp(e, "t6r") ? 4 : 0)));
    *out = c;
    return TCG_OK;
}

extern "C" int tcg_ctx_destroy(tcg_ctx *c)
{
    if (!c) return TCG_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    DBuf *bufs[] = {&c->gpsi, &c->adjw, &c->adjt, &c->prune_tab, &c->VH, &c->V2h, &c->pgw, &c->gidx0, &c->vloc, &c->nlB, &c->nlD, &c->acc1, &c->h1buf,
                    &c->tw64, &c->tw32, &c->recip, &c->inv, &c->phase, &c->phik, &c->chik, &c->fill,
                    &c->Rocc, &c->Rchi, &c->Rgrad, &c->dens, &c->densT, &c->occfill, &c->Vloc, &c->dnu, &c->dnuT,
                    &c->V3a1, &c->V3b1, &c->V3a2, &c->V3b2, &c->Qt, &c->Bt, &c->accP, &c->qtg, &c->div3b6,
                    &c->psi, &c->h2, &c->h3, &c->Rpsi, &c->Rgpsi, &c->acc2, &c->acc3, &c->qsum, &c->tmp,
                    &c->tmp2, &c->aux, &c->ftab, &c->items, &c->meta, &c->rotw, &c->q3b2w,
                    &c->nGw, &c->Ww};
    for (DBuf *b : bufs) b->release();
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return TCG_OK;
}

// upload the orbital / filling part of a state (no R-space work)
static int tcg_set_state_orbitals_only(tcg_ctx *c, const tcg_state_desc *st)
{
    if (!c || !st) return fail(TCG_ERR_ARG, "null argument");
    Host &h = c->h;
    if (!st->nbands || !st->nocc || !st->filling || !st->phik) return fail(TCG_ERR_ARG, "missing state arrays");
    const bool bitc = h.method == TCG_METHOD_BITC;
    if (bitc && !st->phik_left) return fail(TCG_ERR_ARG, "BITC needs phik_left");
    h.have_state = false;
    h.nbands.assign(st->nbands, st->nbands + h.nspin);
    h.nocc.assign(st->nocc, st->nocc + h.nspin * h.nk);
    size_t nfill = 0;
    for (int s = 0; s < h.nspin; s++) {
        if (h.nbands[s] < 0) return fail(TCG_ERR_ARG, "negative nbands");
        nfill += (size_t)h.nk * h.nbands[s];
        for (int k = 0; k < h.nk; k++)
            if (h.nocc[s * h.nk + k] < 0 || h.nocc[s * h.nk + k] > h.nbands[s])
                return fail(TCG_ERR_ARG, "nocc must lie in [0, nbands]");
    }
    h.filling.assign(st->filling, st->filling + nfill);
    for (double f : h.filling)
        if (!std::isfinite(f)) return fail(TCG_ERR_NUMERIC, "non-finite filling");
    h.orb_off.resize((size_t)h.nspin * h.nk);
    size_t off = 0;
    for (int s = 0; s < h.nspin; s++)
        for (int k = 0; k < h.nk; k++) {
            h.orb_off[(size_t)s * h.nk + k] = off;
            off += (size_t)h.nbands[s] * h.npw[k];
        }
    const size_t norb = off;
    for (size_t i = 0; i < 2 * norb; i++)
        if (!std::isfinite(st->phik[i])) return fail(TCG_ERR_NUMERIC, "non-finite orbital coefficient");
    h.occ_off.resize((size_t)h.nspin * h.nk_all);
    size_t g = 0;
    std::vector<double> occfill;
    for (int s = 0; s < h.nspin; s++)
        for (int a = 0; a < h.nk_all; a++) {
            h.occ_off[(size_t)s * h.nk_all + a] = g;
            const int ik = h.ik_of_all[a];
            const int no = h.nocc[s * h.nk + ik];
            for (int i = 0; i < no; i++) {
                size_t fo = 0;
                for (int s2 = 0; s2 < s; s2++) fo += (size_t)h.nk * h.nbands[s2];
                occfill.push_back(h.filling[fo + (size_t)ik * h.nbands[s] + i]);
            }
            g += no;
        }
    h.nocc_grids = g;
    int rc;
    if ((rc = up(c->phik, st->phik, norb * sizeof(double2), c->stream))) return rc;
    if (bitc && (rc = up(c->chik, st->phik_left, norb * sizeof(double2), c->stream))) return rc;
    if ((rc = up(c->fill, h.filling.data(), nfill * sizeof(double), c->stream))) return rc;
    if ((rc = up(c->occfill, occfill.data(), occfill.size() * sizeof(double), c->stream))) return rc;
    return TCG_OK;
}

extern "C" int tcg_set_state(tcg_ctx *c, const tcg_state_desc *st)
{
    if (st && !st->density) return fail(TCG_ERR_ARG, "missing density");
    TRY(tcg_set_state_orbitals_only(c, st));
    Host &h = c->h;
    int rc;
    for (size_t i = 0; i < 4 * (size_t)h.N; i++)
        if (!std::isfinite(st->density[i])) return fail(TCG_ERR_NUMERIC, "non-finite density");
    if ((rc = up(c->dens, st->density, 2 * (size_t)h.N * sizeof(double2), c->stream))) return rc;
    rc = c->prec == TCG_PREC_FP64 ? build_occupied<double>(c) : build_occupied<float>(c);
    if (rc) return rc;
    rc = c->prec == TCG_PREC_FP64 ? state_terms<double>(c) : state_terms<float>(c);
    if (rc) return rc;
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    h.have_state = true;
    return TCG_OK;
}

// Redo all per-state work (R-space occupied orbitals and gradients, local
// three-body potentials; the tc3a2a4b2b5 occupied-pair stage on the next
// apply) from the device-resident state of the last tcg_set_state.
extern "C" int tcg_refresh_state(tcg_ctx *c)
{
    if (!c) return fail(TCG_ERR_ARG, "null context");
    if (!c->h.have_state) return fail(TCG_ERR_STATE, "no state to refresh");
    int rc = c->prec == TCG_PREC_FP64 ? build_occupied<double>(c) : build_occupied<float>(c);
    if (rc) return rc;
    rc = c->prec == TCG_PREC_FP64 ? state_terms<double>(c) : state_terms<float>(c);
    if (rc) return rc;
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    return TCG_OK;
}

static int check_apply(tcg_ctx *c, uint32_t mask, const int32_t *nb)
{
    if (!c || !nb) return fail(TCG_ERR_ARG, "null argument");
    if (!c->h.have_state) return fail(TCG_ERR_STATE, "tcg_set_state must be called before tcg_apply");
    const bool hf = c->h.method == TCG_METHOD_HF;
    if (mask & ~(TCG_TERMS_H2 | TCG_TERMS_TC)) return fail(TCG_ERR_ARG, "unknown term bits (one-body terms: tcg_apply_h1)");
    if (hf && (mask & ~(TCG_TERM_HF2X | TCG_TERM_HF2H))) return fail(TCG_ERR_ARG, "TC terms requested for an HF context");
    if (!hf && (mask & (TCG_TERM_HF2X | TCG_TERM_HF2H))) return fail(TCG_ERR_ARG, "HF terms requested for a TC/BITC context");
    for (int i = 0; i < c->h.nspin * c->h.nk; i++)
        if (nb[i] < 0) return fail(TCG_ERR_ARG, "negative band count");
    return TCG_OK;
}

static size_t psi_count(const tcg_ctx *c, const int32_t *nb)
{
    size_t n = 0;
    for (int s = 0; s < c->h.nspin; s++)
        for (int k = 0; k < c->h.nk; k++) n += (size_t)nb[s * c->h.nk + k] * c->h.npw[k];
    return n;
}

extern "C" int tcg_apply_device(tcg_ctx *c, uint32_t mask, const int32_t *nb, const void *psi, void *h2, void *h3,
                                const uint8_t *owned)
{
    TRY(check_apply(c, mask, nb));
    if (!psi) return fail(TCG_ERR_ARG, "psi is NULL");
    if ((mask & TCG_TERMS_H2) && !h2) return fail(TCG_ERR_ARG, "h2 is NULL");
    if ((mask & ~TCG_TERMS_H2) && !h3) return fail(TCG_ERR_ARG, "h3 is NULL");
    ApplyArgs A{};
    A.mask = mask;
    A.nb = nb;
    A.owned = owned;
    A.psi = (const double2 *)psi;
    A.h2 = (double2 *)h2;
    A.h3 = (double2 *)h3;
    return c->prec == TCG_PREC_FP64 ? apply_impl<double>(c, A) : apply_impl<float>(c, A);
}

extern "C" int tcg_apply(tcg_ctx *c, uint32_t mask, const int32_t *nb, const double *psi, double *h2, double *h3,
                         const uint8_t *owned)
{
    TRY(check_apply(c, mask, nb));
    if (!psi) return fail(TCG_ERR_ARG, "psi is NULL");
    const bool need2 = mask & TCG_TERMS_H2;
    const bool need3 = mask & ~TCG_TERMS_H2;
    if (need2 && !h2) return fail(TCG_ERR_ARG, "h2 is NULL");
    if (need3 && !h3) return fail(TCG_ERR_ARG, "h3 is NULL");
    const size_t n = psi_count(c, nb);
    for (size_t i = 0; i < 2 * n; i++)
        if (!std::isfinite(psi[i])) return fail(TCG_ERR_NUMERIC, "non-finite value in psi");
    const size_t bytes = n * sizeof(double2);
    TRY(c->psi.ensure(bytes));
    TRY(c->h2.ensure(need2 ? bytes : 16));
    TRY(c->h3.ensure(need3 ? bytes : 16));
    TCG_CUDA(cudaMemcpyAsync(c->psi.p, psi, bytes, cudaMemcpyHostToDevice, c->stream));
    if (need2) TCG_CUDA(cudaMemcpyAsync(c->h2.p, h2, bytes, cudaMemcpyHostToDevice, c->stream));
    if (need3) TCG_CUDA(cudaMemcpyAsync(c->h3.p, h3, bytes, cudaMemcpyHostToDevice, c->stream));
    TRY(tcg_apply_device(c, mask, nb, c->psi.p, need2 ? c->h2.p : nullptr, need3 ? c->h3.p : nullptr, owned));
    if (need2) TCG_CUDA(cudaMemcpyAsync(h2, c->h2.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    if (need3) TCG_CUDA(cudaMemcpyAsync(h3, c->h3.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    return TCG_OK;
}

extern "C" int tcg_qp_partial(tcg_ctx *c, int32_t rank, int32_t nranks, void **buf_dev, size_t *bytes)
{
    if (!c || !buf_dev || !bytes) return fail(TCG_ERR_ARG, "null argument");
    if (nranks < 1 || rank < 0 || rank >= nranks) return fail(TCG_ERR_ARG, "rank outside [0, nranks)");
    Host &h = c->h;
    if (!h.have_state) return fail(TCG_ERR_STATE, "tcg_set_state must be called before tcg_qp_partial");
    if (h.method == TCG_METHOD_HF) return fail(TCG_ERR_ARG, "HF contexts have no tc3a2a4b2b5 stage");
    h.qp_ready = false;
    h.qp_pending = false;
    TRY(c->prec == TCG_PREC_FP64 ? qp_partial<double>(c, rank, nranks) : qp_partial<float>(c, rank, nranks));
    const std::vector<size_t> off = qp_acc_offsets(c);
    *buf_dev = c->accP.p;
    *bytes = off[h.nspin] * (size_t)h.N * sizeof(double2);
    h.qp_pending = true;
    return TCG_OK;
}

extern "C" int tcg_qp_finish(tcg_ctx *c)
{
    if (!c) return fail(TCG_ERR_ARG, "null context");
    Host &h = c->h;
    if (!h.qp_pending) return fail(TCG_ERR_STATE, "tcg_qp_finish without a pending tcg_qp_partial");
    h.qp_pending = false;
    return c->prec == TCG_PREC_FP64 ? qp_finish<double>(c) : qp_finish<float>(c);
}

extern "C" int tcg_set_pseudo(tcg_ctx *c, const tcg_pseudo_desc *pp)
{
    if (!c) return fail(TCG_ERR_ARG, "null context");
    c->h.have_pseudo = false;
    return set_pseudo(c, pp);
}

extern "C" int tcg_apply_h1(tcg_ctx *c, uint32_t mask, const int32_t *nb, const double *psi, double *h1,
                            const uint8_t *owned)
{
    if (!c || !nb || !psi || !h1) return fail(TCG_ERR_ARG, "null argument");
    if (mask & ~TCG_TERMS_H1) return fail(TCG_ERR_ARG, "tcg_apply_h1 applies the one-body terms only");
    if ((mask & TCG_TERM_PSEUDO) && !c->h.have_pseudo) return fail(TCG_ERR_STATE, "tcg_set_pseudo must come first");
    for (int i = 0; i < c->h.nspin * c->h.nk; i++)
        if (nb[i] < 0) return fail(TCG_ERR_ARG, "negative band count");
    const size_t n = psi_count(c, nb);
    for (size_t i = 0; i < 2 * n; i++)
        if (!std::isfinite(psi[i])) return fail(TCG_ERR_NUMERIC, "non-finite value in psi");
    const size_t bytes = n * sizeof(double2);
    TRY(c->psi.ensure(std::max<size_t>(16, bytes)));
    TRY(c->h1buf.ensure(std::max<size_t>(16, bytes)));
    TCG_CUDA(cudaMemcpyAsync(c->psi.p, psi, bytes, cudaMemcpyHostToDevice, c->stream));
    TCG_CUDA(cudaMemcpyAsync(c->h1buf.p, h1, bytes, cudaMemcpyHostToDevice, c->stream));
    TRY(c->prec == TCG_PREC_FP64 ? apply_h1_impl<double>(c, mask, nb, c->psi.as<double2>(), c->h1buf.as<double2>(), owned)
                                 : apply_h1_impl<float>(c, mask, nb, c->psi.as<double2>(), c->h1buf.as<double2>(), owned));
    TCG_CUDA(cudaMemcpyAsync(h1, c->h1buf.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    return TCG_OK;
}

extern "C" int tcg_set_tuning(tcg_ctx *c, int64_t tmp_budget_bytes)
{
    if (!c || tmp_budget_bytes < 0) return fail(TCG_ERR_ARG, "bad tuning argument");
    c->tmp_budget = (size_t)tmp_budget_bytes;
    return TCG_OK;
}

extern "C" int tcg_set_forms(tcg_ctx *c, const tcg_forms *f)
{
    if (!c || !f) return fail(TCG_ERR_ARG, "null argument");
    if (f->xy < 0 || f->xy > 3 || f->z < 0 || f->z > 4 || f->min_targets < 0)
        return fail(TCG_ERR_ARG, "bad kernel form");
    if (!split_line_grid(c->fast_n) && (f->xy == 3 || f->z >= 3))
        return fail(TCG_ERR_UNSUPPORTED, "split-line kernel forms need a 36^3 or 48^3 grid");
    c->xy_kernels = f->xy;
    c->z_kernels = f->z;
    c->no_prefetch = !f->prefetch;
    c->no_prune = !f->prune;
    c->no_fuse = !f->fuse;
    c->qp_sacc = f->qp_sacc != 0;
    c->use_sacc = f->sacc != 0;
    c->min_targets = f->min_targets;
    return TCG_OK;
}

extern "C" int tcg_get_forms(tcg_ctx *c, tcg_forms *f)
{
    if (!c || !f) return fail(TCG_ERR_ARG, "null argument");
    f->xy = c->xy_kernels;
    f->z = c->z_kernels;
    f->prefetch = c->no_prefetch ? 0 : 1;
    f->prune = c->no_prune ? 0 : 1;
    f->fuse = c->no_fuse ? 0 : 1;
    f->qp_sacc = c->qp_sacc ? 1 : 0;
    f->sacc = c->use_sacc ? 1 : 0;
    f->min_targets = c->min_targets;
    return TCG_OK;
}

// ------------------------------------------------------ divergence sums --
// one block per (irreducible k, all-k q): shells until the shell sum drops
// below 1e-20 (potentials_coulomb.cpp:118-139), fixed-tree block reduction.
__global__ void k_sum_vaux(int nk_all, const double *kirr, const double *kall, RecipC rc, double alpha,
                           double *partial, int *match, int max_shell)
{
    const int ik = blockIdx.x / nk_all, a = blockIdx.x % nk_all;
    __shared__ double red[256];
    double kq[3];
    bool in_range = true;
    for (int d = 0; d < 3; d++) {
        double v = kirr[3 * ik + d] - kall[3 * a + d];
        // fractional coordinates: a difference that is not finite or beyond
        // +-64 is no k-vector, and the wrap loops below would not end on it
        if (!(fabs(v) < 64.0)) {
            in_range = false;
            v = 0.0;
        }
        while (v < -1e-8) v += 1.0;
        while (v > 1.0 - 1e-8) v -= 1.0;
        kq[d] = v;
    }
    if (!in_range) {  // the same for every thread of the block
        if (threadIdx.x == 0) {
            partial[blockIdx.x] = 0.0;
            match[blockIdx.x] = 2;
        }
        return;
    }
    const bool m = kq[0] * kq[0] + kq[1] * kq[1] + kq[2] * kq[2] < 1e-8;
    double total = 0.0;
    if (!m) {
        double v[3];
        for (int d = 0; d < 3; d++) v[d] = rc.R[0 * 3 + d] * kq[0] + rc.R[1 * 3 + d] * kq[1] + rc.R[2 * 3 + d] * kq[2];
        const double k2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        total += exp(-alpha * k2) / k2;
    }
    int ns = 1;
    for (; ns <= max_shell; ns++) {
        const int w = 2 * ns + 1;
        double loc = 0.0;
        for (int i = threadIdx.x; i < w * w * w; i += blockDim.x) {
            const int gx = i % w - ns, gy = (i / w) % w - ns, gz = i / (w * w) - ns;
            if (gx != ns && -gx != ns && gy != ns && -gy != ns && gz != ns && -gz != ns) continue;
            const double x[3] = {kq[0] + gx, kq[1] + gy, kq[2] + gz};
            double v[3];
            for (int d = 0; d < 3; d++) v[d] = rc.R[0 * 3 + d] * x[0] + rc.R[1 * 3 + d] * x[1] + rc.R[2 * 3 + d] * x[2];
            const double g2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            loc += exp(-alpha * g2) / g2;
        }
        red[threadIdx.x] = loc;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
            __syncthreads();
        }
        const double shell = red[0];
        __syncthreads();
        total += shell;
        if (shell < 1e-20) break;
    }
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = total;
        match[blockIdx.x] = (m ? 1 : 0) | (ns > max_shell ? 2 : 0);
    }
}

extern "C" int tcg_sum_of_vaux(const tcg_system_desc *sys, double *alpha_out, double *sum_out)
{
    if (!sys || !alpha_out || !sum_out || !sys->nsym_k || !sys->kvec) return fail(TCG_ERR_ARG, "null argument");
    if (!(sys->omega > 0) || sys->nk_irr < 1) return fail(TCG_ERR_ARG, "bad geometry");
    const double PI = 3.14159265358979323846;
    double alpha = cbrt(sys->omega) / (2.0 * PI);
    alpha = alpha * alpha;
    const int nk = sys->nk_irr;
    int nk_all = 0;
    std::vector<double> kirr(3 * (size_t)nk);
    for (int k = 0; k < nk; k++) {
        for (int d = 0; d < 3; d++) kirr[3 * k + d] = sys->kvec[3 * nk_all + d];
        nk_all += sys->nsym_k[k];
    }
    RecipC rc;
    memcpy(rc.R, sys->recip, sizeof rc.R);
    DBuf dk, dka, dp, dm;
    int rc_;
    if ((rc_ = dk.ensure(kirr.size() * sizeof(double))) || (rc_ = dka.ensure(3 * (size_t)nk_all * sizeof(double))) ||
        (rc_ = dp.ensure((size_t)nk * nk_all * sizeof(double))) || (rc_ = dm.ensure((size_t)nk * nk_all * sizeof(int))))
        return rc_;
    TCG_CUDA(cudaMemcpy(dk.p, kirr.data(), kirr.size() * sizeof(double), cudaMemcpyHostToDevice));
    TCG_CUDA(cudaMemcpy(dka.p, sys->kvec, 3 * (size_t)nk_all * sizeof(double), cudaMemcpyHostToDevice));
    k_sum_vaux<<<nk * nk_all, 256>>>(nk_all, dk.as<double>(), dka.as<double>(), rc, alpha, dp.as<double>(), dm.as<int>(), 400);
    TCG_CUDA(cudaGetLastError());
    std::vector<double> part((size_t)nk * nk_all);
    std::vector<int> match((size_t)nk * nk_all);
    TCG_CUDA(cudaMemcpy(part.data(), dp.p, part.size() * sizeof(double), cudaMemcpyDeviceToHost));
    TCG_CUDA(cudaMemcpy(match.data(), dm.p, match.size() * sizeof(int), cudaMemcpyDeviceToHost));
    dk.release(); dka.release(); dp.release(); dm.release();
    for (int k = 0; k < nk; k++) {
        double total = 0.0;
        bool m = false;
        for (int a = 0; a < nk_all; a++) {
            const int f = match[(size_t)k * nk_all + a];
            if (f & 2) return fail(TCG_ERR_NUMERIC, "divergence shell sum did not converge (or a k-vector difference is not finite or beyond +-64)");
            m = m || (f & 1);
            total += part[(size_t)k * nk_all + a];
        }
        total *= 4.0 * PI;
        if (m) total -= 4.0 * PI * alpha;
        sum_out[k] = total;
    }
    *alpha_out = alpha;
    return TCG_OK;
}

// ---------------------------------------------------------------- density --
// n_s(r) = sum_{k, isym, i} f |phi(r)|^2  (conj(chi) phi for BITC), /2 when
// unpolarised (bloch_states_scfloop_filling_density.cpp:282-359)
__global__ void k_density(int N, int ngrid, const double2 *phi, const double2 *chi, const double *f, double scale,
                          double2 *out, int bitc)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < N; p += gridDim.x * blockDim.x) {
        double2 acc = {0, 0};
        for (int gi = 0; gi < ngrid; gi++) {
            const double2 a = phi[(size_t)gi * N + p];
            double2 sub;
            if (bitc) sub = cmulc(chi[(size_t)gi * N + p], a);
            else sub = {a.x * a.x + a.y * a.y, 0.0};
            acc = {acc.x + f[gi] * sub.x, acc.y + f[gi] * sub.y};
        }
        out[p] = {acc.x * scale, acc.y * scale};
    }
}
__global__ void k_norms(int N, const double2 *phi, const double2 *chi, double2 *norm, int bitc)
{
    __shared__ double2 red[256];
    const int gi = blockIdx.x;
    double2 loc = {0, 0};
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        const double2 a = phi[(size_t)gi * N + p];
        const double2 sub = bitc ? cmulc(chi[(size_t)gi * N + p], a) : double2{a.x * a.x + a.y * a.y, 0.0};
        loc = cadd(loc, sub);
    }
    red[threadIdx.x] = loc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = cadd(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) norm[gi] = red[0];
}

extern "C" int tcg_density(tcg_ctx *c, const tcg_state_desc *st, double *out)
{
    if (!c || !st || !out) return fail(TCG_ERR_ARG, "null argument");
    TRY(tcg_set_state_orbitals_only(c, st));
    Host &h = c->h;
    const size_t N = h.N;
    const bool bitc = h.method == TCG_METHOD_BITC;
    // FP64 R-space grids of all occupied orbitals (isym-expanded)
    DBuf phi, chi, fl, nrm, dn;
    TRY(phi.ensure(std::max<size_t>(1, h.nocc_grids) * N * sizeof(double2)));
    if (bitc) TRY(chi.ensure(std::max<size_t>(1, h.nocc_grids) * N * sizeof(double2)));
    std::vector<SphereItem> items;
    std::vector<double> f;
    for (int s = 0; s < h.nspin; s++)
        for (int a = 0; a < h.nk_all; a++) {
            const int ik = h.ik_of_all[a];
            for (int i = 0; i < h.nocc[s * h.nk + ik]; i++) {
                SphereItem it{};
                const size_t cof = h.orb_off[(size_t)s * h.nk + ik] + (size_t)i * h.npw[ik];
                it.coef = c->phik.as<double2>() + cof;
                it.inv = c->inv.as<int>() + ((size_t)s * h.nk_all + a) * N;
                it.phase = c->phase.as<double2>() + h.gidx_off[(size_t)s * h.nk_all + a];
                it.tr = h.time_rev[a];
                const size_t grid = h.occ_off[(size_t)s * h.nk_all + a] + i;
                it.out = phi.as<double2>() + grid * N;
                items.push_back(it);
                if (bitc) {
                    it.coef = c->chik.as<double2>() + cof;
                    it.out = chi.as<double2>() + grid * N;
                    items.push_back(it);
                }
                f.push_back(h.filling[fill_off(h, s, ik) + i]);
            }
        }
    TRY(sphere_to_r<double>(c, items));
    TRY(fl.ensure(std::max<size_t>(1, f.size()) * sizeof(double)));
    TRY(nrm.ensure(std::max<size_t>(1, f.size()) * sizeof(double2)));
    TRY(dn.ensure(2 * N * sizeof(double2)));
    if (!f.empty()) TCG_CUDA(cudaMemcpyAsync(fl.p, f.data(), f.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const double scale = h.nspin == 1 ? 0.5 : 1.0;
    for (int s = 0; s < h.nspin; s++) {
        const size_t g0 = h.occ_off[(size_t)s * h.nk_all];
        const size_t g1 = s + 1 < h.nspin ? h.occ_off[(size_t)(s + 1) * h.nk_all] : h.nocc_grids;
        TRY(launch(c, k_density, dim3((unsigned)std::min<size_t>(148 * 8, (N + 255) / 256)), dim3(256), 0, (int)N,
                   (int)(g1 - g0), (const double2 *)(phi.as<double2>() + g0 * N),
                   (const double2 *)(bitc ? chi.as<double2>() + g0 * N : nullptr), (const double *)(fl.as<double>() + g0),
                   scale, dn.as<double2>() + (size_t)s * N, bitc ? 1 : 0));
    }
    if (h.nspin == 1)
        TCG_CUDA(cudaMemcpyAsync(dn.as<double2>() + N, dn.p, N * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
    if (h.nocc_grids)
        TRY(launch(c, k_norms, dim3((unsigned)h.nocc_grids), dim3(256), 0, (int)N, (const double2 *)phi.as<double2>(),
                   (const double2 *)(bitc ? chi.as<double2>() : nullptr), nrm.as<double2>(), bitc ? 1 : 0));
    std::vector<double2> norms(h.nocc_grids);
    TCG_CUDA(cudaMemcpyAsync(out, dn.p, 2 * N * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    if (h.nocc_grids)
        TCG_CUDA(cudaMemcpyAsync(norms.data(), nrm.p, h.nocc_grids * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    for (const double2 &n : norms) {
        const double re = n.x / (double)N - 1.0, im = n.y / (double)N;
        if (std::sqrt(re * re + im * im) > 1e-4) return fail(TCG_ERR_NUMERIC, "normalization breaks");
    }
    return TCG_OK;
}

// ------------------------------------------------------------ energies --
// e_n of one applied band: <chi_b | h_n b> over its plane waves (fixed-order
// tree reduction), one block per (spin, k, band) with a non-zero filling.
struct EnergyBand {
    const double2 *bra;      // left (BITC) or right orbital of the band, G space
    const double2 *h2, *h3;  // applied terms of the band (nullptr: skipped)
    int npw;
};
static __global__ void __launch_bounds__(256) k_band_dots(const EnergyBand *bands, double2 *dots)
{
    const EnergyBand b = bands[blockIdx.x];
    __shared__ double2 red[2][256];
    double2 a2 = {0, 0}, a3 = {0, 0};
    for (int p = threadIdx.x; p < b.npw; p += blockDim.x) {
        const double2 c = b.bra[p];
        if (b.h2) a2 = cadd(a2, cmulc(c, b.h2[p]));
        if (b.h3) a3 = cadd(a3, cmulc(c, b.h3[p]));
    }
    red[0][threadIdx.x] = a2;
    red[1][threadIdx.x] = a3;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[0][threadIdx.x] = cadd(red[0][threadIdx.x], red[0][threadIdx.x + s]);
            red[1][threadIdx.x] = cadd(red[1][threadIdx.x], red[1][threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        dots[2 * blockIdx.x] = red[0][0];
        dots[2 * blockIdx.x + 1] = red[1][0];
    }
}
// E_n = sum_bands f (n_plain e_n + n_tr conj(e_n)) / (n N_k): one thread,
// bands in order, so the sum is reproducible bit for bit
static __global__ void k_energy_sum(int nband, const double2 *dots, const double *w, double inv_nk, double *out)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double2 e2 = {0, 0}, e3 = {0, 0};
    for (int i = 0; i < nband; i++) {
        const double wp = w[2 * i], wt = w[2 * i + 1];   // f * (images without / with time reversal)
        const double2 d2 = dots[2 * i], d3 = dots[2 * i + 1];
        e2.x += (wp + wt) * d2.x; e2.y += (wp - wt) * d2.y;
        e3.x += (wp + wt) * d3.x; e3.y += (wp - wt) * d3.y;
    }
    out[0] = e2.x * inv_nk / 2.0; out[1] = e2.y * inv_nk / 2.0;
    out[2] = e3.x * inv_nk / 3.0; out[3] = e3.y * inv_nk / 3.0;
}

extern "C" int tcg_energy(tcg_ctx *c, const int32_t *nb, const void *h2_dev, const void *h3_dev, double *e_out)
{
    if (!c || !nb || !e_out) return fail(TCG_ERR_ARG, "null argument");
    Host &h = c->h;
    if (!h.have_state) return fail(TCG_ERR_STATE, "tcg_set_state must be called before tcg_energy");
    const bool bitc = h.method == TCG_METHOD_BITC;
    std::vector<EnergyBand> bands;
    std::vector<double> w;
    size_t off = 0;
    for (int s = 0; s < h.nspin; s++)
        for (int k = 0; k < h.nk; k++) {
            if (nb[s * h.nk + k] < 0) return fail(TCG_ERR_ARG, "negative band count");
            int nplain = 0, ntr = 0;
            for (int a = h.kall_off[k]; a < h.kall_off[k + 1]; a++) (h.time_rev[a] ? ntr : nplain)++;
            for (int b = 0; b < nb[s * h.nk + k]; b++, off += h.npw[k]) {
                if (b >= h.nbands[s]) continue;
                const double f = h.filling[fill_off(h, s, k) + b];
                if (f == 0.0) continue;
                EnergyBand e;
                e.bra = (bitc ? c->chik.as<double2>() : c->phik.as<double2>()) + h.orb_off[(size_t)s * h.nk + k] +
                        (size_t)b * h.npw[k];
                e.h2 = h2_dev ? (const double2 *)h2_dev + off : nullptr;
                e.h3 = h3_dev ? (const double2 *)h3_dev + off : nullptr;
                e.npw = h.npw[k];
                bands.push_back(e);
                w.push_back(f * nplain);
                w.push_back(f * ntr);
            }
        }
    if (bands.empty()) {
        for (int i = 0; i < 4; i++) e_out[i] = 0.0;
        return TCG_OK;
    }
    const size_t nbd = bands.size();
    DBuf &buf = c->aux;
    const size_t b0 = 0, b1 = (nbd * sizeof(EnergyBand) + 255) & ~(size_t)255;
    const size_t b2 = b1 + ((nbd * 2 * sizeof(double) + 255) & ~(size_t)255);
    const size_t b3 = b2 + ((nbd * 2 * sizeof(double2) + 255) & ~(size_t)255);
    TRY(buf.ensure(b3 + 4 * sizeof(double)));
    char *base = buf.as<char>();
    TCG_CUDA(cudaMemcpyAsync(base + b0, bands.data(), nbd * sizeof(EnergyBand), cudaMemcpyHostToDevice, c->stream));
    TCG_CUDA(cudaMemcpyAsync(base + b1, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    TRY(launch(c, k_band_dots, dim3((unsigned)nbd), dim3(256), 0, (const EnergyBand *)(base + b0), (double2 *)(base + b2)));
    TRY(launch(c, k_energy_sum, dim3(1), dim3(1), 0, (int)nbd, (const double2 *)(base + b2), (const double *)(base + b1),
               1.0 / h.num_kpoints, (double *)(base + b3)));
    TCG_CUDA(cudaMemcpyAsync(e_out, base + b3, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    return TCG_OK;
}

#include "adjoint.cuh"

extern "C" int tcg_energy_grad(tcg_ctx *c, uint32_t mask, double *e_out, void *dchi, double *du, double *dv2)
{
    if (!c || !e_out) return fail(TCG_ERR_ARG, "null argument");
    Host &h = c->h;
    if (!h.have_state) return fail(TCG_ERR_STATE, "tcg_set_state must be called before tcg_energy_grad");
    TRY(check_apply(c, mask, std::vector<int32_t>((size_t)h.nspin * h.nk, 0).data()));
    if (dchi)
        for (int k = 0; k < h.nk; k++)
            if (h.nsym_k[k] != 1)
                return fail(TCG_ERR_UNSUPPORTED, "orbital gradient needs every k-point irreducible alone (nsym_k = 1)");
    if (du || dv2) {
        if (h.nk_all != 1) return fail(TCG_ERR_UNSUPPORTED, "Jastrow-table gradients are implemented for Gamma-only systems");
        if (!(mask & TCG_TERM_TC2X)) return fail(TCG_ERR_ARG, "Jastrow-table gradients need TCG_TERM_TC2X in the mask");
    }
    return c->prec == TCG_PREC_FP64 ? energy_grad_impl<double>(c, mask, e_out, dchi, du, dv2)
                                    : energy_grad_impl<float>(c, mask, e_out, dchi, du, dv2);
}

// ------------------------------------------------------------- profiling --
extern "C" int tcg_profile(tcg_ctx *c, int enable)
{
    if (!c) return fail(TCG_ERR_ARG, "null context");
    for (auto &r : c->prof_recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    c->prof_recs.clear();
    c->prof = enable != 0;
    return TCG_OK;
}

// Aggregate the recorded launches per tag: for tag i writes count, total
// device milliseconds and algorithmic bytes.  Returns the number of tags via
// *ntags (<= cap).  Tags: "xyf", "z", "xyi", "misc".
extern "C" int tcg_profile_read(tcg_ctx *c, int cap, char *tags /* cap x 32 */, int64_t *count, double *ms,
                                double *bytes, int *ntags)
{
    if (!c || !ntags) return fail(TCG_ERR_ARG, "null argument");
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    std::vector<std::string> names;
    std::vector<int64_t> cnt;
    std::vector<double> tms, tb;
    auto add = [&](const std::string &tag, double e, double by) {
        size_t i = 0;
        for (; i < names.size(); i++)
            if (names[i] == tag) break;
        if (i == names.size()) { names.push_back(tag); cnt.push_back(0); tms.push_back(0); tb.push_back(0); }
        cnt[i]++;
        tms[i] += e;
        tb[i] += by;
    };
    for (size_t k = 0; k < c->prof_recs.size(); k++) {
        const auto &r = c->prof_recs[k];
        float e = 0;
        TCG_CUDA(cudaEventElapsedTime(&e, r.a, r.b));
        add(r.tag, e, r.bytes);
        if (k > 0) {
            // device time between the previous launch's end and this one's start
            // (host work, synchronisation, copies): reported as "idle>tag"
            float gap = 0;
            TCG_CUDA(cudaEventElapsedTime(&gap, c->prof_recs[k - 1].b, r.a));
            add(std::string("idle>") + r.tag, gap, 0.0);
        }
    }
    const int n = (int)std::min<size_t>(names.size(), (size_t)cap);
    for (int i = 0; i < n; i++) {
        if (tags) { memset(tags + 32 * i, 0, 32); strncpy(tags + 32 * i, names[i].c_str(), 31); }
        if (count) count[i] = cnt[i];
        if (ms) ms[i] = tms[i];
        if (bytes) bytes[i] = tb[i];
    }
    *ntags = n;
    return TCG_OK;
}

// ------------------------------------- allocation-free divergence sums --
// Scratch of tcg_sum_of_vaux_noalloc: one partial shell sum and one flag
// word per (irreducible k, mesh q) pair, plus an error word.  File-scope
// device arrays: every GPU that loads the library holds them (about 192 KiB)
// until the process exits; no call allocates.
constexpr int TCG_NOALLOC_MAX_PAIRS = 16384;
static __device__ __align__(256) double g_noalloc_partial[TCG_NOALLOC_MAX_PAIRS];
static __device__ __align__(256) int g_noalloc_flags[TCG_NOALLOC_MAX_PAIRS];
static __device__ __align__(256) int g_noalloc_err[1];

struct NoallocScratch {
    double *partial = nullptr;
    int *flags = nullptr;
    int *err = nullptr;
};
static std::mutex g_noalloc_mu;
static NoallocScratch g_noalloc_dev[64];

// Device addresses of the scratch arrays on the current device.  Host code
// only holds a host-side stand-in for a __device__ array's name, so the
// address is looked up once per device with that device current.
static int noalloc_scratch(NoallocScratch &out)
{
    int dev = 0;
    TCG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(TCG_ERR_UNSUPPORTED, "device index >= 64");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoallocScratch &s = g_noalloc_dev[dev];
    if (!s.partial) {
        NoallocScratch t;
        TCG_CUDA(cudaGetSymbolAddress((void **)&t.partial, g_noalloc_partial));
        TCG_CUDA(cudaGetSymbolAddress((void **)&t.flags, g_noalloc_flags));
        TCG_CUDA(cudaGetSymbolAddress((void **)&t.err, g_noalloc_err));
        s = t;
    }
    out = s;
    return TCG_OK;
}

// sum over the mesh q of one irreducible k, in q order (as tcg_sum_of_vaux)
static __global__ void k_sum_vaux_final(int nk, int nk_all, const double *partial, const int *flags, double alpha,
                                        double *sum_out, int *err)
{
    const double FOURPI = 4.0 * 3.14159265358979323846;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nk) return;
    double total = 0.0;
    int match = 0, bad = 0;
    for (int a = 0; a < nk_all; a++) {
        const int f = flags[(size_t)k * nk_all + a];
        match |= f & 1;
        bad |= f & 2;
        total += partial[(size_t)k * nk_all + a];
    }
    total *= FOURPI;
    if (match) total -= FOURPI * alpha;
    sum_out[k] = total;
    if (bad) atomicOr(err, 1);
}

extern "C" int tcg_sum_of_vaux_noalloc(const double recip[9], double omega, int32_t nk_irr, int32_t nk_all,
                                       const double *kirr_dev, const double *kall_dev, double *sum_vaux_dev,
                                       double *alpha_out, void *stream)
{
    if (!recip || !kirr_dev || !kall_dev || !sum_vaux_dev) return fail(TCG_ERR_ARG, "null argument");
    if (!(omega > 0) || !std::isfinite(omega)) return fail(TCG_ERR_ARG, "unit-cell volume must be positive and finite");
    for (int i = 0; i < 9; i++)
        if (!std::isfinite(recip[i])) return fail(TCG_ERR_ARG, "non-finite reciprocal lattice vector");
    if (nk_irr < 1 || nk_all < 1) return fail(TCG_ERR_ARG, "no k-points");
    if ((int64_t)nk_irr * nk_all > TCG_NOALLOC_MAX_PAIRS)
        return fail(TCG_ERR_ARG, "nk_irr * nk_all exceeds the 16384 (k, q) pairs of the static scratch");
    NoallocScratch sc;
    TRY(noalloc_scratch(sc));
    cudaStream_t st = (cudaStream_t)stream;
    const double PI = 3.14159265358979323846;
    double alpha = cbrt(omega) / (2.0 * PI);
    alpha = alpha * alpha;
    RecipC rc;
    memcpy(rc.R, recip, sizeof rc.R);
    // every partial / flag used below is written by k_sum_vaux before it is
    // read; only the error word has to start at zero
    TCG_CUDA(cudaMemsetAsync(sc.err, 0, sizeof(int), st));
    k_sum_vaux<<<nk_irr * nk_all, 256, 0, st>>>(nk_all, kirr_dev, kall_dev, rc, alpha, sc.partial, sc.flags, 400);
    TCG_CUDA(cudaGetLastError());
    k_sum_vaux_final<<<(nk_irr + 127) / 128, 128, 0, st>>>(nk_irr, nk_all, sc.partial, sc.flags, alpha, sum_vaux_dev,
                                                           sc.err);
    TCG_CUDA(cudaGetLastError());
    int err = 0;
    TCG_CUDA(cudaMemcpyAsync(&err, sc.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    TCG_CUDA(cudaStreamSynchronize(st));
    if (err) return fail(TCG_ERR_NUMERIC, "divergence shell sum did not converge (or a k-vector difference is not finite or beyond +-64)");
    if (alpha_out) *alpha_out = alpha;
    return TCG_OK;
}
