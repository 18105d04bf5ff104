// tc3.cuh -- orchestration of all terms: chunk planning, per-state work
// (occupied grids, local three-body potentials, tc3a2a4b2b5 occupied-pair
// stage) and the per-apply pipelines.
#pragma once
#include "terms.cuh"

namespace tcg {

// ------------------------------------------------------------- utilities --
static __global__ void k_zero(double2 *p, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = {0, 0};
}

static __global__ void k_add(size_t n, const double2 *a, double2 *b)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        b[i] = cadd(b[i], a[i]);
}

// y += a x
static __global__ void k_axpy(size_t n, double a, const double2 *x, double2 *y)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = {y[i].x + a * x[i].x, y[i].y + a * x[i].y};
}

template <typename T>
__global__ void k_to_prec(const double2 *src, typename C2<T>::t *dst, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = from64<typename C2<T>::t>(src[i]);
}

template <typename T>
static __global__ void k_dens_sum(int N, const double2 *dens, typename C2<T>::t *out)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < N; p += gridDim.x * blockDim.x)
        out[p] = from64<typename C2<T>::t>(cadd(dens[p], dens[(size_t)N + p]));
}

// acc[t] += fac * V(r) * phi_t(r)   (local potentials: tc3a1.cpp:101-112 etc.)
template <typename T>
__global__ void k_local(int N, const typename C2<T>::t *Rpsi, const double2 *V, double2 *acc)
{
    const size_t t = blockIdx.y;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < N; p += gridDim.x * blockDim.x)
        acc_add(acc + t * N + p, cmul(V[p], to64(Rpsi[t * N + p])), 1.0);
}

// out = sum_d a_d * b_d  (pointwise, fp64; b in compute precision)
template <typename T>
__global__ void k_dot3(int N, const double2 *a, const typename C2<T>::t *b, double2 *acc, double fac, int nt)
{
    // per target t: acc[t] += fac * sum_d a[t][d] b[d]
    const size_t t = blockIdx.y;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < N; p += gridDim.x * blockDim.x) {
        double2 s = {0, 0};
        for (int d = 0; d < 3; d++) s = cadd(s, cmul(a[(t * 3 + d) * N + p], to64(b[(size_t)d * N + p])));
        acc_add(acc + t * N + p, s, fac);
    }
}

// per-target input part of the combined 3b3 + 3b4 + 3b5 transform (OpTC3X):
// W[t][d] = b3 dnu_d psi_t + b4 qsum[t][d], once per target instead of once
// per (target, source) pair
template <typename T>
__global__ void k_w3x(int N, const typename C2<T>::t *dnu, const typename C2<T>::t *psi, const double2 *qsum,
                      double b3, double b4, typename C2<T>::t *W, int nt)
{
    using V = typename C2<T>::t;
    using S = decltype(V{}.x);
    const size_t t = blockIdx.y;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < N; p += gridDim.x * blockDim.x) {
        const V ps = psi[t * N + p];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const V w = cscale(cmul(dnu[(size_t)d * N + p], ps), (S)b3);
            W[(t * 3 + d) * N + p] = cadd(w, cscale(from64<V>(qsum[(t * 3 + d) * N + p]), (S)b4));
        }
    }
}

// dnu_s[d](G) = sum_{s3} u(G; s, s3) G_d n_{s3}(G)   (tc3a1.cpp:53-70)
static __global__ void k_dnu_g(GridDesc g, RecipC rc, Jastrow J, int s, const double2 *nG, double2 *out)
{
    const double zero[3] = {0, 0, 0};
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += gridDim.x * blockDim.x) {
        int x, y, z;
        xyz_of(g, p, x, y, z);
        double G[3];
        gvec(rc.R, g, x, y, z, zero, G);
        double2 a[3] = {{0, 0}, {0, 0}, {0, 0}};
        for (int js = 0; js < 2; js++) {
            const double u = J.uk(G, s, js);
            const double2 n = nG[(size_t)js * g.N + p];
            for (int d = 0; d < 3; d++) a[d] = cadd(a[d], cscale(n, u * G[d]));
        }
        for (int d = 0; d < 3; d++) out[(size_t)d * g.N + p] = a[d];
    }
}

// V3a1(r) = sum_d dnu_d(r)^2 (complex square, tc3a1.cpp:78-84)
static __global__ void k_square_sum(int N, const double2 *dnu, double2 *V)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < N; p += gridDim.x * blockDim.x) {
        double2 s = {0, 0};
        for (int d = 0; d < 3; d++) s = cadd(s, cmul(dnu[(size_t)d * N + p], dnu[(size_t)d * N + p]));
        V[p] = s;
    }
}

// W_d = dnu_d(r) n(r)  (tc3b1.cpp:77-82)
static __global__ void k_mul_dens(int N, const double2 *dnu, const double2 *n, double2 *W)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < N; p += gridDim.x * blockDim.x)
        for (int d = 0; d < 3; d++) W[(size_t)d * N + p] = cmul(dnu[(size_t)d * N + p], n[p]);
}

// V(G) += sum_{s2} u(G; s1, s2) G . W[s2ref](G)    (tc3b1.cpp:86-101)
// mode 1 (3b2, tc3a2a4b2b5.cpp:927-958): V(G) += fac * sum_d G_d u'(G) W_d(G)
static __global__ void k_gdot(GridDesc g, RecipC rc, Jastrow J, int s1, int nspin, const double2 *W0, const double2 *W1,
                       double2 *V, int mode, int sq)
{
    const double zero[3] = {0, 0, 0};
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += gridDim.x * blockDim.x) {
        int x, y, z;
        xyz_of(g, p, x, y, z);
        double G[3];
        gvec(rc.R, g, x, y, z, zero, G);
        double2 acc = V[p];
        if (mode == 0) {
            for (int s2 = 0; s2 < 2; s2++) {
                const double2 *W = (nspin == 1 || s2 == 0) ? W0 : W1;
                const double u = J.uk(G, s1, s2);
                for (int d = 0; d < 3; d++) acc = cadd(acc, cscale(W[(size_t)d * g.N + p], u * G[d]));
            }
        } else {
            const double u = nspin == 1 ? J.uk(G, s1, 0) + J.uk(G, s1, 1) : J.uk(G, s1, sq);
            double2 t = {0, 0};
            for (int d = 0; d < 3; d++) t = cadd(t, cscale(W0[(size_t)d * g.N + p], G[d] * u));
            acc = cadd(acc, t);
        }
        V[p] = acc;
    }
}

// tG(G) = sum_js 4 pi n_js(G) A_{0,sj} u(G; 0, sj) [G != 0]   (tc3a3b3b4b6.cpp:96-107, 429-451)
static __global__ void k_div3b6_g(GridDesc g, RecipC rc, Jastrow J, double A00, double A01, int s, const double2 *nG,
                           double2 *tG)
{
    const double zero[3] = {0, 0, 0};
    const double FOURPI = 4.0 * 3.14159265358979323846;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += gridDim.x * blockDim.x) {
        int x, y, z;
        xyz_of(g, p, x, y, z);
        double G[3];
        gvec(rc.R, g, x, y, z, zero, G);
        double2 acc = {0, 0};
        for (int js = 0; js < 2; js++) {
            const int sj = s == js ? 0 : 1;
            const double AuG = p == 0 ? 0.0 : J.uk(G, 0, sj) * (sj == 0 ? A00 : A01);
            acc = cadd(acc, cscale(nG[(size_t)js * g.N + p], FOURPI * AuG));
        }
        tG[p] = acc;
    }
}

// 3b6 divergence correction per target (tc3a3b3b4b6.cpp:454-533, if_match)
struct Div3b6Item {
    const double2 *psi;      // G, npw
    double2 *h;              // G, npw
    const void *Rpsi;        // R, compute precision
    double2 *acc;            // R, fp64
    const double2 *phik, *chik;     // G [nb][npw]
    const void *Rphi, *Rchi;        // R [nocc][N] (compute precision)
    const double *fill;
    const double2 *tR;       // R fp64
    double2 t1;              // scalar temp_div_3b6_1
    int npw, nocc;
    double b6;
};

template <typename T>
__global__ void __launch_bounds__(256) k_div3b6(const Div3b6Item *items, int N)
{
    using V = typename C2<T>::t;
    const Div3b6Item it = items[blockIdx.x];
    __shared__ double2 red[256];
    const V *Rpsi = (const V *)it.Rpsi;
    for (int b = 0; b < it.nocc; b++) {
        const double f = it.fill[b];
        if (f < 1e-8) continue;
        const V *chr = (const V *)it.Rchi + (size_t)b * N;
        const V *phr = (const V *)it.Rphi + (size_t)b * N;
        double2 loc = {0, 0};
        for (int p = threadIdx.x; p < it.npw; p += blockDim.x) loc = cadd(loc, cmulc(it.chik[(size_t)b * it.npw + p], it.psi[p]));
        red[threadIdx.x] = loc;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) red[threadIdx.x] = cadd(red[threadIdx.x], red[threadIdx.x + s]);
            __syncthreads();
        }
        const double2 cpi = red[0];
        __syncthreads();
        loc = {0, 0};
        for (int p = threadIdx.x; p < N; p += blockDim.x)
            loc = cadd(loc, cmul(cmulc(to64(chr[p]), to64(Rpsi[p])), it.tR[p]));
        red[threadIdx.x] = loc;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) red[threadIdx.x] = cadd(red[threadIdx.x], red[threadIdx.x + s]);
            __syncthreads();
        }
        const double2 dot2 = cscale(red[0], 1.0 / (double)N);
        __syncthreads();
        const double2 c1 = cscale(cmul(it.t1, cpi), f * it.b6);
        const double2 c2 = cscale(dot2, f * it.b6);
        const double2 *phg = it.phik + (size_t)b * it.npw;
        for (int p = threadIdx.x; p < it.npw; p += blockDim.x) {
            double2 hv = cadd(it.h[p], cmul(c1, phg[p]));
            it.h[p] = cadd(hv, cmul(c2, phg[p]));
        }
        const double2 c3 = cscale(cpi, f * it.b6);
        for (int p = threadIdx.x; p < N; p += blockDim.x) acc_add(it.acc + p, cmul(c3, cmul(it.tR[p], to64(phr[p]))), 1.0);
        __syncthreads();
    }
}

// symmetry rotation of G-space grids (tc3a2a4b2b5.cpp:576-644, 682-764)
struct RotArgs {
    int U[9];
    double t[3];
    double M[9];
    int tr;
};
// scalar: out[idx] += fac * phase * (tr ? conj(in) : in)
static __global__ void k_rot_scalar(GridDesc g, RotArgs ra, const double2 *in, double2 *out, double fac)
{
    const double TWOPI = 2.0 * 3.14159265358979323846;
    const int nr[3] = {g.n0, g.n1, g.n2};
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += gridDim.x * blockDim.x) {
        int x, y, z;
        xyz_of(g, p, x, y, z);
        const int m[3] = {miller(x, g.n0), miller(y, g.n1), miller(z, g.n2)};
        int Gt[3];
        for (int i = 0; i < 3; i++) {
            Gt[i] = ra.U[0 * 3 + i] * m[0] + ra.U[1 * 3 + i] * m[1] + ra.U[2 * 3 + i] * m[2];
            if (ra.tr) Gt[i] = -Gt[i];
            Gt[i] %= nr[i];
            if (Gt[i] < 0) Gt[i] += nr[i];
        }
        const double arg = TWOPI * (ra.t[0] * Gt[0] + ra.t[1] * Gt[1] + ra.t[2] * Gt[2]);
        double sn, cs;
        sincos(arg, &sn, &cs);
        const int idx = Gt[0] + Gt[1] * nr[0] + Gt[2] * nr[0] * nr[1];
        double2 v = in[p];
        if (ra.tr) v.y = -v.y;
        const double2 r = cmul(double2{cs, sn}, v);
        out[idx] = cadd(out[idx], cscale(r, fac));
    }
}
// vector (3 components, Cartesian U^+): out_d[idx] = +-phase * sum_e M[d][e] (tr ? conj(in_e) : in_e)
static __global__ void k_rot_vec(GridDesc g, RotArgs ra, const double2 *in, double2 *out)
{
    const double TWOPI = 2.0 * 3.14159265358979323846;
    const int nr[3] = {g.n0, g.n1, g.n2};
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += gridDim.x * blockDim.x) {
        int x, y, z;
        xyz_of(g, p, x, y, z);
        const int m[3] = {miller(x, g.n0), miller(y, g.n1), miller(z, g.n2)};
        int Gt[3];
        for (int i = 0; i < 3; i++) {
            Gt[i] = ra.U[0 * 3 + i] * m[0] + ra.U[1 * 3 + i] * m[1] + ra.U[2 * 3 + i] * m[2];
            if (ra.tr) Gt[i] = -Gt[i];
            Gt[i] %= nr[i];
            if (Gt[i] < 0) Gt[i] += nr[i];
        }
        const double arg = TWOPI * (ra.t[0] * Gt[0] + ra.t[1] * Gt[1] + ra.t[2] * Gt[2]);
        double sn, cs;
        sincos(arg, &sn, &cs);
        const double2 ph = {cs, sn};
        const int idx = Gt[0] + Gt[1] * nr[0] + Gt[2] * nr[0] * nr[1];
        double2 v[3];
        for (int e = 0; e < 3; e++) {
            v[e] = in[(size_t)e * g.N + p];
            if (ra.tr) v[e].y = -v[e].y;
        }
        for (int d = 0; d < 3; d++) {
            double2 s = {0, 0};
            for (int e = 0; e < 3; e++) s = cadd(s, cscale(v[e], ra.M[d * 3 + e]));
            s = cmul(ph, s);
            if (ra.tr) s = cscale(s, -1.0);
            out[(size_t)d * g.N + idx] = s;
        }
    }
}

// B = -conj(Q) for TC (tc3a2a4b2b5.cpp:662)
static __global__ void k_negconj(size_t n, const double2 *Q, double2 *B)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        B[i] = {-Q[i].x, Q[i].y};
}

// qsum3b2[d] += f2 * Bt_d(r) * phi_q2sym(r)  (tc3a2a4b2b5.cpp:811-815)
template <typename T>
__global__ void k_qsum3b2(int N, const double2 *Bt, const typename C2<T>::t *phi, double2 *q, double f2)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < N; p += gridDim.x * blockDim.x)
        for (int d = 0; d < 3; d++) acc_add(q + (size_t)d * N + p, cmul(Bt[(size_t)d * N + p], to64(phi[p])), f2);
}

// 3a2 divergence correction (tc3a2a4b2b5.cpp:496-573) for one q2 target:
// T_xr(0)  -= 4pi A_x (A_x dcorr + u(0; sq, x)) f1 phiphi(0) phij(0)
// T_xr(G)  -= 4pi A_x f1 u(G; sq, x) (phiphi(G) phij(0) + phiphi(0) phij(G))
template <typename T>
__global__ void k_div3a2(GridDesc g, RecipC rc, Jastrow J, int sq, int nspin, int ni, const typename C2<T>::t *pf,
                         const double *f1, double A0, double A1, double dcorr, double2 *Tq)
{
    using V = typename C2<T>::t;
    const double zero[3] = {0, 0, 0};
    const double FOURPI = 4.0 * 3.14159265358979323846;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += gridDim.x * blockDim.x) {
        int x, y, z;
        xyz_of(g, p, x, y, z);
        double G[3];
        gvec(rc.R, g, x, y, z, zero, G);
        for (int i1 = 0; i1 < ni; i1++) {
            const V *pp = pf + (size_t)i1 * 2 * g.N;     // [2][N]: phiphi, phij
            const double2 a0 = to64(pp[0]), b0 = to64(pp[g.N]);
            const double2 ap = to64(pp[p]), bp = to64(pp[g.N + p]);
            for (int xs = 0; xs < 2; xs++) {
                const int xr = nspin == 1 ? 0 : xs;
                const double Ax = xs == 0 ? A0 : A1;
                double2 *t = Tq + (size_t)xr * g.N + p;
                if (p == 0) {
                    const double c = FOURPI * Ax * (Ax * dcorr + J.uk(zero, sq, xs)) * f1[i1];
                    *t = csub(*t, cscale(cmul(a0, b0), c));
                } else {
                    const double c = FOURPI * Ax * f1[i1] * J.uk(G, sq, xs);
                    *t = csub(*t, cscale(cadd(cmul(ap, b0), cmul(a0, bp)), c));
                }
            }
        }
    }
}

// ------------------------------------------------ Hartree-type two-body --
// V_H(G) = 4 pi n(G) / |G|^2 with V_H(0) = 0, in place on n_0 + n_1 in G
// (calc_hamiltonian_hf2h.cpp:40-50)
static __global__ void k_hartree_g(GridDesc g, RecipC rc, double2 *V)
{
    const double zero[3] = {0, 0, 0};
    const double FOURPI = 4.0 * 3.14159265358979323846;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += gridDim.x * blockDim.x) {
        if (p == 0) { V[0] = {0, 0}; continue; }
        int x, y, z;
        xyz_of(g, p, x, y, z);
        double G[3];
        gvec(rc.R, g, x, y, z, zero, G);
        const double f = FOURPI / (G[0] * G[0] + G[1] * G[1] + G[2] * G[2]);
        V[p] = {V[p].x * f, V[p].y * f};
    }
}

// tc2h [2b_h2]: out_d(r) = sum over the occupied grids of one spin of
// f conj(chi(r)) grad_d phi(r), grids in order (calc_hamiltonian_tc2h.cpp:53-136)
template <typename T>
__global__ void k_phiq_gphiq(int N, int ngrid, const typename C2<T>::t *chi, const typename C2<T>::t *grad,
                             const double *fill, double2 *out)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < N; p += gridDim.x * blockDim.x) {
        double2 a[3] = {{0, 0}, {0, 0}, {0, 0}};
        for (int gi = 0; gi < ngrid; gi++) {
            const double2 c = to64(chi[(size_t)gi * N + p]);
            const double f = fill[gi];
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const double2 v = cmulc(c, to64(grad[((size_t)gi * 3 + d) * N + p]));
                a[d] = {a[d].x + f * v.x, a[d].y + f * v.y};
            }
        }
#pragma unroll
        for (int d = 0; d < 3; d++) out[(size_t)d * N + p] = a[d];
    }
}

// tc2h potential of spin s in G (calc_hamiltonian_tc2h.cpp:146-180):
// V(G) = sum_js [ V_2body(G; s, js) n_js(G) + u(G; s, js) G . pg[js'](G) / spin_factor ]
static __global__ void k_tc2h_g(GridDesc g, RecipC rc, Jastrow J, int s, int nspin, const double2 *nG,
                                const double2 *pg, double2 *V)
{
    const double zero[3] = {0, 0, 0};
    const double spin_factor = nspin == 1 ? 2.0 : 1.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += gridDim.x * blockDim.x) {
        int x, y, z;
        xyz_of(g, p, x, y, z);
        double G[3];
        gvec(rc.R, g, x, y, z, zero, G);
        double2 acc = {0, 0};
        for (int js = 0; js < 2; js++) {
            const int jr = nspin == 1 ? 0 : js;
            const double2 n = nG[(size_t)js * g.N + p];
            const double v2 = J.tc2body(G, s, js), u = J.uk(G, s, js);
            acc = {acc.x + v2 * n.x, acc.y + v2 * n.y};
            for (int d = 0; d < 3; d++) {
                const double2 q = pg[((size_t)jr * 3 + d) * g.N + p];
                acc = {acc.x + u * G[d] * q.x / spin_factor, acc.y + u * G[d] * q.y / spin_factor};
            }
        }
        V[p] = acc;
    }
}

// acc[t] += a (V(r) phi_t(r) - sum_d grad_d phi_t(r) W_d(r))   (tc2h.cpp:211-222;
// hf2h.cpp:70-73 with W absent)
template <typename T>
__global__ void k_local_h2(int N, const typename C2<T>::t *Rpsi, const typename C2<T>::t *Rgpsi, const double2 *Vr,
                           const double2 *W, double a, double2 *acc)
{
    const size_t t = blockIdx.y;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < N; p += gridDim.x * blockDim.x) {
        double2 v = cmul(Vr[p], to64(Rpsi[t * N + p]));
        if (W)
            for (int d = 0; d < 3; d++) v = csub(v, cmul(to64(Rgpsi[(t * 3 + d) * N + p]), W[(size_t)d * N + p]));
        acc_add(acc + t * N + p, v, a);
    }
}

// ------------------------------------------------------- chunk planning --
struct ChunkPlan {
    int t0, nt, s0, ns, nTB, nSB;
    size_t meta_off;         // byte offset in the meta arena
    const int *tb, *sb;
    const double *kq;
    const int *pent;         // [nTB*nSB] pencil-table entry of each (target k, source q) pair
    double pfrac;            // mean active-pencil fraction over the chunk's items
};

// Plan (target range x source range) chunks; kq = tcart[tkey] - scart[skey].
// items <= max_items; targets per chunk >= min_t when possible.
static int plan_chunks(tcg_ctx *c, DBuf &meta, int ntg, const std::vector<int> &tkey, const std::vector<double> &tc,
                       int nsrc, const std::vector<int> &skey, const std::vector<double> &sc, size_t max_items,
                       int min_t, std::vector<ChunkPlan> &out)
{
    out.clear();
    if (ntg == 0 || nsrc == 0) return TCG_OK;
    int nt_c = std::min(ntg, std::max(1, min_t));
    if ((size_t)nt_c > max_items) nt_c = (int)std::max<size_t>(1, max_items);
    int ns_c = (int)std::max<size_t>(1, std::min<size_t>(nsrc, max_items / nt_c));
    // grow the target range if all sources fit
    if (ns_c == nsrc) nt_c = (int)std::min<size_t>(ntg, std::max<size_t>(nt_c, max_items / nsrc));
    std::vector<unsigned char> host;
    for (int t0 = 0; t0 < ntg; t0 += nt_c)
        for (int s0 = 0; s0 < nsrc; s0 += ns_c) {
            ChunkPlan p{};
            p.t0 = t0;
            p.nt = std::min(nt_c, ntg - t0);
            p.s0 = s0;
            p.ns = std::min(ns_c, nsrc - s0);
            std::vector<int> tb(p.nt), sb(p.ns), tk, sk;
            for (int i = 0; i < p.nt; i++) {
                const int key = tkey[t0 + i];
                if (tk.empty() || tk.back() != key) {
                    auto f = std::find(tk.begin(), tk.end(), key);
                    if (f == tk.end()) { tk.push_back(key); tb[i] = (int)tk.size() - 1; }
                    else tb[i] = (int)(f - tk.begin());
                } else tb[i] = (int)tk.size() - 1;
            }
            for (int i = 0; i < p.ns; i++) {
                const int key = skey[s0 + i];
                if (sk.empty() || sk.back() != key) {
                    auto f = std::find(sk.begin(), sk.end(), key);
                    if (f == sk.end()) { sk.push_back(key); sb[i] = (int)sk.size() - 1; }
                    else sb[i] = (int)(f - sk.begin());
                } else sb[i] = (int)sk.size() - 1;
            }
            p.nTB = (int)tk.size();
            p.nSB = (int)sk.size();
            std::vector<double> kq((size_t)p.nTB * p.nSB * 3);
            for (int a = 0; a < p.nTB; a++)
                for (int b = 0; b < p.nSB; b++) {
                    // tkey / skey index the Cartesian vector tables
                    int ti = -1, si = -1;
                    for (int i = 0; i < p.nt && ti < 0; i++) if (tb[i] == a) ti = t0 + i;
                    for (int i = 0; i < p.ns && si < 0; i++) if (sb[i] == b) si = s0 + i;
                    for (int d = 0; d < 3; d++) kq[((size_t)a * p.nSB + b) * 3 + d] = tc[3 * ti + d] - sc[3 * si + d];
                }
            // append to the meta arena (8-byte aligned blocks)
            auto append = [&](const void *src, size_t bytes) {
                size_t o = (host.size() + 7) & ~(size_t)7;
                host.resize(o + bytes);
                memcpy(host.data() + o, src, bytes);
                return o;
            };
            // pencil-table entry of each pair: target key (irreducible k) x source key (all-k)
            std::vector<int> pent((size_t)p.nTB * p.nSB);
            for (int a = 0; a < p.nTB; a++)
                for (int b = 0; b < p.nSB; b++) pent[(size_t)a * p.nSB + b] = tk[a] * c->h.nk_all + sk[b];
            p.pfrac = 1.0;
            if (c->prune_ok) {
                double sum = 0;
                for (int i = 0; i < p.nt; i++)
                    for (int j = 0; j < p.ns; j++) sum += c->prune_nact[pent[(size_t)tb[i] * p.nSB + sb[j]]];
                p.pfrac = sum / ((double)p.nt * p.ns * c->h.n[0] * c->h.n[1]);
            }
            p.meta_off = append(kq.data(), kq.size() * sizeof(double));
            size_t otb = append(tb.data(), tb.size() * sizeof(int));
            size_t osb = append(sb.data(), sb.size() * sizeof(int));
            size_t ope = append(pent.data(), pent.size() * sizeof(int));
            // stash offsets in the pointer fields; resolved after upload
            p.kq = reinterpret_cast<const double *>(p.meta_off);
            p.tb = reinterpret_cast<const int *>(otb);
            p.sb = reinterpret_cast<const int *>(osb);
            p.pent = reinterpret_cast<const int *>(ope);
            out.push_back(p);
        }
    TRY(meta.ensure(host.size() + 8));
    TCG_CUDA(cudaMemcpyAsync(meta.p, host.data(), host.size(), cudaMemcpyHostToDevice, c->stream));
    char *base = meta.as<char>();
    for (auto &p : out) {
        p.kq = reinterpret_cast<const double *>(base + (size_t)p.kq);
        p.tb = reinterpret_cast<const int *>(base + (size_t)p.tb);
        p.sb = reinterpret_cast<const int *>(base + (size_t)p.sb);
        p.pent = reinterpret_cast<const int *>(base + (size_t)p.pent);
    }
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    return TCG_OK;
}

// targets per chunk: the XYI pass runs one CTA per (target, plane group)
// and loops over the chunk's sources.  c->min_targets > 0 (TCG_MIN_TARGETS)
// overrides the default of ~12 waves of CTAs.
static int min_targets(const tcg_ctx *c)
{
    if (c->min_targets > 0) return c->min_targets;
    const int n2 = c->h.n[2];
    return std::max(1, (148 * 3 * 12 * 4 + n2 - 1) / n2);
}

// chunk budget: tmp slots bytes <= c->tmp_budget
static size_t max_items_for(const tcg_ctx *c, int nslots, size_t vbytes)
{
    const size_t per = (size_t)nslots * c->h.N * vbytes;
    const size_t budget = c->tmp_budget ? c->tmp_budget : ((size_t)8 << 30);
    return std::min<size_t>(65535, std::max<size_t>(1, budget / per));   // grid.y limit
}

// Algorithmic bytes per pass launch: a 3D FFT of N points moves 2 N s bytes
// (one read + one write of the grid); each of the two passes of a
// transform is credited half of it, N s per grid.
// Fast-path launcher, defined in fast_launch.cuh and instantiated per grid
// size in fast_inst.cu (one translation unit per N).
template <typename T, int N, class Op>
int run_chunk_fast(tcg_ctx *c, const Op &op, int items, int nt, bool do_xyf, bool do_xyi);

// Algorithmic bytes per pass launch: a 3D FFT of N points moves 2 N s bytes
// (one read + one write of the grid); each of the two passes of a
// transform is credited half of it, N s per grid.

// Algorithmic bytes per pass launch: a 3D FFT of N points moves 2 N s bytes
// (one read + one write of the grid); each of the two passes of a
// transform is credited half of it, N s per grid.
template <typename T, class Op>
static int run_chunk(tcg_ctx *c, const Op &op, int items, int nt, bool do_xyf = true, bool do_xyi = true)
{
    using V = typename C2<T>::t;
    const GridDesc &g = c->gd;
    if (c->fast_n && !c->force_generic) {
        switch (c->fast_n) {
        case 12: return run_chunk_fast<T, 12, Op>(c, op, items, nt, do_xyf, do_xyi);
        case 16: return run_chunk_fast<T, 16, Op>(c, op, items, nt, do_xyf, do_xyi);
        case 24: return run_chunk_fast<T, 24, Op>(c, op, items, nt, do_xyf, do_xyi);
        case 32: return run_chunk_fast<T, 32, Op>(c, op, items, nt, do_xyf, do_xyi);
        case 36: return run_chunk_fast<T, 36, Op>(c, op, items, nt, do_xyf, do_xyi);
        case 40: return run_chunk_fast<T, 40, Op>(c, op, items, nt, do_xyf, do_xyi);
        case 48: return run_chunk_fast<T, 48, Op>(c, op, items, nt, do_xyf, do_xyi);
        default: break;
        }
    }
    const int ntiles = (g.n0 * g.n1 + ZTC - 1) / ZTC;
    const double gb = (double)g.N * sizeof(V);
    if (do_xyf) TRY(launch_tagged(c, tagname(Op::NAME, "xyf"), (double)items * Op::NF * gb, k_xyf<T, Op>, dim3(g.n2, items), dim3(256), smem_xy<V>(g), op));
    TRY(launch_tagged(c, tagname(Op::NAME, "z"), (double)items * (Op::NF + (Op::ZINV ? Op::NB : 0)) * gb, k_z<T, Op>, dim3(ntiles, items), dim3(256),
                      smem_z<V>(g, Op::NF), op));
    if (do_xyi) {
        int nref = 0;
        if (Op::REFWD) nref = Op::NB - 1;
        TRY(launch_tagged(c, tagname(Op::NAME, "xyi"), (double)items * (Op::NB + nref) * gb, k_xyi<T, Op>, dim3(g.n2, nt), dim3(256),
                          sizeof(V) * (3 * MAXN + (Op::GS + 2) * (size_t)g.n0 * g.n1), op));
    }
    return TCG_OK;
}

template <typename T, class Op>
static void op_common(tcg_ctx *c, Op &op, const ChunkPlan &p, int nsl, int ntab)
{
    using V = typename C2<T>::t;
    op.g = c->gd;
    op.tmp = c->tmp.as<V>();
    op.nsl = nsl;
    op.ns = p.ns;
    op.m.tb = p.tb;
    op.m.sb = p.sb;
    op.m.kq = p.kq;
    op.m.tab = c->aux.as<double>();
    op.m.ftab = c->ftab.as<float4>();
    op.m.nSB = p.nSB;
    op.m.ntab = ntab;
    op.m.nrec = c->ftab_nrec;
    // pruning: 36^3 or 48^3 grid, table built, split-line Z and inverse XY
    // passes (k_z_t6 / k_z_t6r read only the active pencils, k_xyi_t6 zeroes
    // the others; the forward XY pass may write more than the active ones)
    const int np = c->h.n[0] * c->h.n[1];
    op.m.np = np;
    op.m.prune = (c->prune_ok && !c->no_prune && split_line_grid(c->fast_n) && !c->force_generic &&
                  (c->xy_kernels == 0 || c->xy_kernels == 3) && (c->z_kernels == 0 || c->z_kernels >= 3) &&
                  (Op::BLI | Op::BLO) != 0) ? 1 : 0;
    op.m.pent = p.pent;
    op.m.pfrac = op.m.prune ? p.pfrac : 1.0;
    const size_t nent = (size_t)c->h.nk * c->h.nk_all;
    op.m.pmask = c->prune_tab.as<const unsigned char>();
    op.m.pperm = reinterpret_cast<const unsigned short *>(c->prune_tab.as<const unsigned char>() + nent * np);
    op.m.pnact = reinterpret_cast<const int *>(c->prune_tab.as<const unsigned char>() + nent * np * 3);
    op.m.pbits = reinterpret_cast<const unsigned long long *>(
        c->prune_tab.as<const unsigned char>() + ((nent * np * 3 + nent * sizeof(int) + 7) & ~(size_t)7));
    memcpy(op.rc.R, c->h.recip, sizeof op.rc.R);
    op.invN = 1.0 / (double)c->h.N;
}

// Jastrow tables of one chunk: FP64 columns for the FP64 path, FP32
// coefficient records (nrec per grid point) for the mixed path
template <typename T>
static int gen_tables(tcg_ctx *c, const ChunkPlan &p, int mode, int s, int nrec = 1)
{
    const int npair = p.nTB * p.nSB;
    RecipC rc;
    memcpy(rc.R, c->h.recip, sizeof rc.R);
    if constexpr (sizeof(T) == 4) {
        TRY(c->ftab.ensure((size_t)npair * c->h.N * nrec * sizeof(float4)));
        c->ftab_nrec = nrec;
        return launch(c, k_ftables, dim3(148 * 4), dim3(256), 0, c->gd, rc, make_jastrow(c->h), mode, s, nrec, npair,
                      p.kq, 1.0 / (double)c->h.N, c->ftab.as<float4>());
    } else {
        const int ntab = mode == TAB_U_SS ? 1 : 2;
        TRY(c->aux.ensure((size_t)npair * c->h.N * ntab * sizeof(double)));
        return launch(c, k_tables, dim3(148 * 4), dim3(256), 0, c->gd, rc, make_jastrow(c->h), mode, s, npair, p.kq,
                      c->aux.as<double>());
    }
}

// forward transform + gather: h += fac * FFT(acc)
static int finalize_acc(tcg_ctx *c, const Targets &T, double2 *acc, double2 *hout, double fac)
{
    PhaseScope ps_(c, "ap:final");
    const GridDesc &g = c->gd;
    const Host &h = c->h;
    const size_t nt = T.s.size();
    if (nt == 0) return TCG_OK;
    const size_t N = h.N;
    std::vector<void *> grids(nt);
    std::vector<GatherItem> gi(nt);
    for (size_t t = 0; t < nt; t++) {
        grids[t] = acc + t * N;
        gi[t].grid = acc + t * N;
        gi[t].inv = c->inv.as<int>() + ((size_t)T.s[t] * h.nk_all + h.kall_off[T.k[t]]) * N;
        gi[t].h = hout + T.psi_off[t];
        gi[t].fac = make_double2(fac / (double)N, 0.0);
    }
    TRY(c->items.ensure(nt * (sizeof(void *) + sizeof(GatherItem))));
    // the items first: GatherItem holds a double2 (16-byte aligned), the
    // pointer array after them (8-byte aligned whatever nt is)
    GatherItem *d_gi = c->items.as<GatherItem>();
    void **d_grids = reinterpret_cast<void **>(d_gi + nt);
    TCG_CUDA(cudaMemcpyAsync(d_grids, grids.data(), nt * sizeof(void *), cudaMemcpyHostToDevice, c->stream));
    TCG_CUDA(cudaMemcpyAsync(d_gi, gi.data(), nt * sizeof(GatherItem), cudaMemcpyHostToDevice, c->stream));
    const int ntiles = (g.n0 * g.n1 + ZTC - 1) / ZTC;
    for (size_t b0 = 0; b0 < nt; b0 += 65535) {
        const unsigned nb = (unsigned)std::min<size_t>(65535, nt - b0);
        GridRefs gr;
        gr.dev = d_grids + b0;
        TRY(launch(c, k_xy_inplace<double, -1>, dim3(g.n2, nb), dim3(256), smem_xy<double2>(g), g, gr));
        TRY(launch(c, k_gather_z, dim3(ntiles, nb), dim3(256), smem_z<double2>(g, 0), g, (const GatherItem *)(d_gi + b0)));
    }
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    return TCG_OK;
}

// --------------------------------------------------------- div (2-body) --
struct DivItem {
    const double2 *psi;
    double2 *h;
    const double2 *phik, *chik;
    const double *fill;
    int npw, nb;
    double dc;
};

// h += sum_b fill_b dc <chi_kb|psi> phi_kb   (hf2x.cpp:150-200, tc2x.cpp:409-511)
static __global__ void __launch_bounds__(256) k_div_2x(const DivItem *items)
{
    const DivItem it = items[blockIdx.x];
    __shared__ double2 red[256];
    for (int b = 0; b < it.nb; b++) {
        const double f = it.fill[b];
        if (f < 1e-8) continue;
        const double2 *chi = it.chik + (size_t)b * it.npw;
        const double2 *phi = it.phik + (size_t)b * it.npw;
        double2 loc = {0, 0};
        for (int p = threadIdx.x; p < it.npw; p += blockDim.x) loc = cadd(loc, cmulc(chi[p], it.psi[p]));
        red[threadIdx.x] = loc;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) red[threadIdx.x] = cadd(red[threadIdx.x], red[threadIdx.x + s]);
            __syncthreads();
        }
        double2 prod = cscale(cscale(red[0], it.dc), f);
        __syncthreads();
        for (int p = threadIdx.x; p < it.npw; p += blockDim.x) it.h[p] = cadd(it.h[p], cmul(prod, phi[p]));
        __syncthreads();
    }
}

static size_t fill_off(const Host &h, int s, int k)
{
    size_t fo = 0;
    for (int s2 = 0; s2 < s; s2++) fo += (size_t)h.nk * h.nbands[s2];
    return fo + (size_t)k * h.nbands[s];
}

static int div_2x(tcg_ctx *c, const Targets &T, const ApplyArgs &A, double2 *hout)
{
    PhaseScope ps_(c, "ap:div2x");
    const Host &h = c->h;
    if (!h.div) return TCG_OK;
    const size_t nt = T.s.size();
    if (nt == 0) return TCG_OK;
    std::vector<DivItem> di(nt);
    const bool bitc = h.method == TCG_METHOD_BITC;
    for (size_t t = 0; t < nt; t++) {
        const int s = T.s[t], k = T.k[t];
        double dc = 1.0 / std::sqrt(PI_D * h.alpha);
        dc -= h.sum_vaux[k] / (h.num_kpoints * h.omega);
        dc *= -1;
        if (h.nspin == 1) dc /= 2.0;
        DivItem &d = di[t];
        d.psi = A.psi + T.psi_off[t];
        d.h = hout + T.psi_off[t];
        d.phik = c->phik.as<double2>() + h.orb_off[(size_t)s * h.nk + k];
        d.chik = (bitc ? c->chik.as<double2>() : c->phik.as<double2>()) + h.orb_off[(size_t)s * h.nk + k];
        d.fill = c->fill.as<double>() + fill_off(h, s, k);
        d.npw = h.npw[k];
        d.nb = h.nbands[s];
        d.dc = dc;
    }
    TRY(c->items.ensure(nt * sizeof(DivItem)));
    TCG_CUDA(cudaMemcpyAsync(c->items.p, di.data(), nt * sizeof(DivItem), cudaMemcpyHostToDevice, c->stream));
    TRY(launch(c, k_div_2x, dim3((unsigned)nt), dim3(256), 0, (const DivItem *)c->items.p));
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    return TCG_OK;
}

// ------------------------------------------------------ source / target --
// Occupied sources of spin s: all (a, i) in Rocc order.
struct Sources {
    size_t base;                  // first grid index in Rocc
    std::vector<int> key;         // all-k index a
    std::vector<double> cartq;    // [n][3]
};
static Sources sources_of(const tcg_ctx *c, int s)
{
    const Host &h = c->h;
    Sources S;
    S.base = h.occ_off[(size_t)s * h.nk_all];
    for (int a = 0; a < h.nk_all; a++) {
        double q[3];
        cart(h, &h.kvec[3 * a], q);
        for (int i = 0; i < h.nocc[s * h.nk + h.ik_of_all[a]]; i++) {
            S.key.push_back(a);
            S.cartq.insert(S.cartq.end(), q, q + 3);
        }
    }
    return S;
}

// targets of one spin: contiguous range of T
struct TRange {
    int t0, n;
    std::vector<int> key;
    std::vector<double> cartk;
};
static TRange targets_of(const tcg_ctx *c, const Targets &T, int s)
{
    const Host &h = c->h;
    TRange R{0, 0, {}, {}};
    int first = -1;
    for (size_t t = 0; t < T.s.size(); t++)
        if (T.s[t] == s) {
            if (first < 0) first = (int)t;
            R.n++;
            R.key.push_back(T.k[t]);
            double k[3];
            cart(h, &h.kvec[3 * h.kall_off[T.k[t]]], k);
            R.cartk.insert(R.cartk.end(), k, k + 3);
        }
    R.t0 = first < 0 ? 0 : first;
    return R;
}

// ================================================================= terms ==
template <typename T>
static int run_hf2x(tcg_ctx *c, const Targets &Tg, double2 *acc)
{
    PhaseScope ps_(c, "ap:2x");
    using V = typename C2<T>::t;
    const Host &h = c->h;
    const size_t N = h.N;
    for (int s = 0; s < h.nspin; s++) {
        TRange TR = targets_of(c, Tg, s);
        Sources S = sources_of(c, s);
        std::vector<ChunkPlan> plan;
        TRY(plan_chunks(c, c->meta, TR.n, TR.key, TR.cartk, (int)S.key.size(), S.key, S.cartq,
                        max_items_for(c, 1, sizeof(V)), min_targets(c), plan));
        for (const ChunkPlan &p : plan) {
            TRY(c->tmp.ensure((size_t)p.nt * p.ns * N * sizeof(V)));
            OpHF2X<T> op;
            op_common<T>(c, op, p, 1, 0);
            op.Rpsi = c->Rpsi.as<V>() + (size_t)(TR.t0 + p.t0) * N;
            op.Rocc = c->Rocc.as<V>() + (S.base + p.s0) * N;
            op.acc = acc + (size_t)(TR.t0 + p.t0) * N;
            op.fill = c->occfill.as<double>() + S.base + p.s0;
            TRY((run_chunk<T, OpHF2X<T>>(c, op, p.nt * p.ns, p.nt)));
        }
    }
    return TCG_OK;
}

template <typename T>
static int run_tc2x(tcg_ctx *c, const Targets &Tg, double2 *acc)
{
    PhaseScope ps_(c, "ap:2x");
    using V = typename C2<T>::t;
    const Host &h = c->h;
    const size_t N = h.N;
    const bool bitc = h.method == TCG_METHOD_BITC;
    for (int s = 0; s < h.nspin; s++) {
        TRange TR = targets_of(c, Tg, s);
        Sources S = sources_of(c, s);
        std::vector<ChunkPlan> plan;
        TRY(plan_chunks(c, c->meta, TR.n, TR.key, TR.cartk, (int)S.key.size(), S.key, S.cartq,
                        max_items_for(c, 4, sizeof(V)), min_targets(c), plan));
        for (const ChunkPlan &p : plan) {
            TRY(c->tmp.ensure((size_t)p.nt * p.ns * 4 * N * sizeof(V)));
            TRY(gen_tables<T>(c, p, TAB_TC2X, s));
            OpTC2X<T> op;
            op_common<T>(c, op, p, 4, 2);
            op.Rpsi = c->Rpsi.as<V>() + (size_t)(TR.t0 + p.t0) * N;
            op.Rgpsi = c->Rgpsi.as<V>() + (size_t)(TR.t0 + p.t0) * 3 * N;
            op.Rocc = c->Rocc.as<V>() + (S.base + p.s0) * N;
            op.Rchi = (bitc ? c->Rchi.as<V>() : c->Rocc.as<V>()) + (S.base + p.s0) * N;
            op.Rgrad = c->Rgrad.as<V>() + (S.base + p.s0) * 3 * N;
            op.acc = acc + (size_t)(TR.t0 + p.t0) * N;
            op.fill = c->occfill.as<double>() + S.base + p.s0;
            TRY((run_chunk<T, OpTC2X<T>>(c, op, p.nt * p.ns, p.nt)));
        }
    }
    return TCG_OK;
}

// tc3a3b3b4b6 stages A (first q loop) and B (3b6), EQ: equal Jastrow channels
template <typename T, bool EQ>
static int tc3_stage_ab(tcg_ctx *c, const Targets &Tg, const TRange &TR, const Sources &S, int s, double b3, double b6,
                        double2 *acc, double2 *qsum)
{
    using V = typename C2<T>::t;
    using OA = OpTC3A<T, EQ>;
    using OB = OpTC3B<T, EQ>;
    const Host &h = c->h;
    const size_t N = h.N;
    const bool bitc = h.method == TCG_METHOD_BITC;
    const V *dnuT = c->dnuT.as<V>() + (size_t)s * 3 * N;
    const int nsl = OA::NB, n2 = OB::NF;
    std::vector<ChunkPlan> plan;
    TRY(plan_chunks(c, c->meta, TR.n, TR.key, TR.cartk, (int)S.key.size(), S.key, S.cartq,
                    max_items_for(c, nsl + n2, sizeof(V)), min_targets(c), plan));
    for (const ChunkPlan &p : plan) {
        const size_t items = (size_t)p.nt * p.ns;
        TRY(c->tmp.ensure(items * nsl * N * sizeof(V)));
        TRY(c->tmp2.ensure(items * n2 * N * sizeof(V)));
        TRY(gen_tables<T>(c, p, TAB_U_SX, s, EQ ? 1 : 2));
        OA a;
        op_common<T>(c, a, p, nsl, 2);
        a.Rpsi = c->Rpsi.as<V>() + (size_t)(TR.t0 + p.t0) * N;
        a.Rocc = c->Rocc.as<V>() + (S.base + p.s0) * N;
        a.Rchi = (bitc ? c->Rchi.as<V>() : c->Rocc.as<V>()) + (S.base + p.s0) * N;
        a.dnu = dnuT;
        a.densT = c->densT.as<V>() + (EQ ? 2 * N : 0);
        a.acc = acc + (size_t)(TR.t0 + p.t0) * N;
        a.qsum = qsum + (size_t)(TR.t0 + p.t0) * 3 * N;
        a.fill = c->occfill.as<double>() + S.base + p.s0;
        a.tmp2 = c->tmp2.as<V>();
        a.s = s;
        a.b3 = b3;
        a.sacc_on = c->use_sacc ? 1 : 0;
        a.sacc_n = OA::SACC;
        TRY((run_chunk<T, OA>(c, a, (int)items, p.nt)));
        OB b;
        op_common<T>(c, b, p, nsl, 2);
        b.Rocc = a.Rocc;
        b.acc = a.acc;
        b.tmp2 = a.tmp2;
        b.b6 = b6;
        b.s = s;
        TRY((run_chunk<T, OB>(c, b, (int)items, p.nt, false, true)));
    }
    return TCG_OK;
}

// factor of the 3a4 band part of tc3a2a4b2b5 (tc3a2a4b2b5.cpp:34-48); 3b5's is its negative
static double band_fa4(const Host &h)
{
    const double Nk = h.num_kpoints, Om = h.omega;
    const double base = 1.0 / (Nk * Nk * Om * Om);
    return h.nspin == 1 ? base / 4.0 : base;
}

// tc2x together with stages A and B of tc3a3b3b4b6 for spin s with equal
// Jastrow channels (OpTC2X3 + OpTC3B): tc2x's sum goes to acc2 (the H2
// accumulator), 3a3 / 3b4's to qsum, 3b6 (and, with band, 3a4) to acc (H3);
// 3b3 runs later in OpTC3X
template <typename T>
static int tc2x_tc3_stage_ab(tcg_ctx *c, const TRange &TR, const Sources &S, int s, double b3, double b6,
                             double2 *acc2, double2 *acc, double2 *qsum, bool band)
{
    using V = typename C2<T>::t;
    using OX = OpTC2X3<T>;
    using OB = OpTC3B<T, true>;
    const Host &h = c->h;
    const size_t N = h.N;
    const bool bitc = h.method == TCG_METHOD_BITC;
    const int nsl = OX::NB, n2 = OB::NF;
    std::vector<ChunkPlan> plan;
    TRY(plan_chunks(c, c->meta, TR.n, TR.key, TR.cartk, (int)S.key.size(), S.key, S.cartq,
                    max_items_for(c, nsl + n2, sizeof(V)), min_targets(c), plan));
    for (const ChunkPlan &p : plan) {
        const size_t items = (size_t)p.nt * p.ns;
        TRY(c->tmp.ensure(items * nsl * N * sizeof(V)));
        TRY(c->tmp2.ensure(items * n2 * N * sizeof(V)));
        TRY(gen_tables<T>(c, p, TAB_TC2X, s));
        OX x;
        op_common<T>(c, x, p, nsl, 2);
        x.Rpsi = c->Rpsi.as<V>() + (size_t)(TR.t0 + p.t0) * N;
        x.Rgpsi = c->Rgpsi.as<V>() + (size_t)(TR.t0 + p.t0) * 3 * N;
        x.Rocc = c->Rocc.as<V>() + (S.base + p.s0) * N;
        x.Rchi = (bitc ? c->Rchi.as<V>() : c->Rocc.as<V>()) + (S.base + p.s0) * N;
        x.Rgrad = c->Rgrad.as<V>() + (S.base + p.s0) * 3 * N;
        x.acc = acc2 + (size_t)(TR.t0 + p.t0) * N;
        x.fill = c->occfill.as<double>() + S.base + p.s0;
        x.densT = c->densT.as<V>() + 2 * N;
        x.qsum = qsum + (size_t)(TR.t0 + p.t0) * 3 * N;
        x.tmp2 = c->tmp2.as<V>();
        x.band = band ? 1 : 0;
        x.Qt = c->Qt.as<V>() + (S.base + p.s0) * 3 * N;
        x.acc3 = acc + (size_t)(TR.t0 + p.t0) * N;
        x.fa4 = band_fa4(h);
        x.sacc_on = c->use_sacc ? 1 : 0;
        x.sacc_n = band ? 4 : 3;
        TRY((run_chunk<T, OX>(c, x, (int)items, p.nt)));
        // 3b6B reads du from 3a3b6A's table layout (TAB_U_SX, one record for equal channels)
        TRY(gen_tables<T>(c, p, TAB_U_SX, s, 1));
        OB b;
        op_common<T>(c, b, p, nsl, 2);
        b.Rocc = x.Rocc;
        b.acc = acc + (size_t)(TR.t0 + p.t0) * N;
        b.tmp2 = x.tmp2;
        b.b6 = b6;
        b.s = s;
        TRY((run_chunk<T, OB>(c, b, (int)items, p.nt, false, true)));
    }
    return TCG_OK;
}

// equal Jastrow channels of spin s: u(G; 0, s) == u(G; 1, s)
static bool eq_channels(const Host &h, int s)
{
    return h.A[0 * 2 + s] == h.A[1 * 2 + s] && h.F[0 * 2 + s] == h.F[1 * 2 + s];
}

// tc2x runs fused with tc3a3b3b4b6 (tc2x_tc3_stage_ab) when both are applied
// and every spin has equal Jastrow channels (any grid and kernel form)
static bool fuse_tc2x_tc3(const tcg_ctx *c, uint32_t mask)
{
    const Host &h = c->h;
    if (c->no_fuse || !(mask & TCG_TERM_TC2X) || !(mask & TCG_TERM_TC3A3B3B4B6)) return false;
    for (int s = 0; s < h.nspin; s++)
        if (!eq_channels(h, s)) return false;
    return true;
}

template <typename T>
static int run_tc3a3b3b4b6(tcg_ctx *c, const Targets &Tg, const ApplyArgs &A, double2 *acc, double2 *acc2_fused,
                           bool band_fused)
{
    PhaseScope ps_(c, "ap:tc3");
    using V = typename C2<T>::t;
    const Host &h = c->h;
    const size_t N = h.N;
    const bool bitc = h.method == TCG_METHOD_BITC;
    const double Nk = h.num_kpoints, Om = h.omega;
    const double base = 1.0 / (Nk * Nk * Om * Om);
    double a3 = -base, b3 = base, b4 = -base, b6 = base;
    if (h.nspin == 1) { a3 /= 2.0; b3 /= 2.0; b4 /= 4.0; b6 /= 2.0; }
    const size_t nt_all = Tg.s.size();
    TRY(c->qsum.ensure(nt_all * 3 * N * sizeof(double2)));
    double2 *qsum = c->qsum.as<double2>();
    TRY(launch(c, k_zero, dim3(148 * 8), dim3(256), 0, qsum, nt_all * 3 * N));
    for (int s = 0; s < h.nspin; s++) {
        TRange TR = targets_of(c, Tg, s);
        Sources S = sources_of(c, s);
        if (TR.n == 0) continue;
        const V *dnuT = c->dnuT.as<V>() + (size_t)s * 3 * N;
        // stages A + B (with tc2x when acc2_fused is given)
        const bool eq = eq_channels(h, s);
        if (acc2_fused) TRY((tc2x_tc3_stage_ab<T>(c, TR, S, s, b3, b6, acc2_fused, acc, qsum, band_fused)));
        else if (eq) TRY((tc3_stage_ab<T, true>(c, Tg, TR, S, s, b3, b6, acc, qsum)));
        else TRY((tc3_stage_ab<T, false>(c, Tg, TR, S, s, b3, b6, acc, qsum)));
        // 3a3: acc += a3 sum_d qsum_d dnu_d  (:629-641)
        TRY(launch(c, k_dot3<T>, dim3((unsigned)((N + 255) / 256), TR.n), dim3(256), 0, (int)N,
                   (const double2 *)(qsum + (size_t)TR.t0 * 3 * N), dnuT, acc + (size_t)TR.t0 * N, a3, TR.n));
        // 3b6 divergence correction (:394-535)
        if (h.div && !h.A_zero) {
            std::vector<Div3b6Item> di;
            for (int i = 0; i < TR.n; i++) {
                const int t = TR.t0 + i, k = Tg.k[t];
                const size_t og = h.occ_off[(size_t)s * h.nk_all + h.kall_off[k]];
                Div3b6Item it{};
                it.psi = A.psi + Tg.psi_off[t];
                it.h = A.h3 + Tg.psi_off[t];
                it.Rpsi = c->Rpsi.as<V>() + (size_t)t * N;
                it.acc = acc + (size_t)t * N;
                it.phik = c->phik.as<double2>() + h.orb_off[(size_t)s * h.nk + k];
                it.chik = (bitc ? c->chik.as<double2>() : c->phik.as<double2>()) + h.orb_off[(size_t)s * h.nk + k];
                it.Rphi = c->Rocc.as<V>() + og * N;
                it.Rchi = (bitc ? c->Rchi.as<V>() : c->Rocc.as<V>()) + og * N;
                it.fill = c->fill.as<double>() + fill_off(h, s, k);
                it.tR = c->div3b6.as<double2>() + (size_t)s * N;
                it.t1 = c->t1_3b6[(size_t)s * h.nk + k];
                it.npw = h.npw[k];
                it.nocc = h.nocc[s * h.nk + k];
                it.b6 = b6;
                di.push_back(it);
            }
            TRY(c->items.ensure(di.size() * sizeof(Div3b6Item)));
            TCG_CUDA(cudaMemcpyAsync(c->items.p, di.data(), di.size() * sizeof(Div3b6Item), cudaMemcpyHostToDevice, c->stream));
            TRY(launch(c, k_div3b6<T>, dim3((unsigned)di.size()), dim3(256), 0, (const Div3b6Item *)c->items.p, (int)N));
            TCG_CUDA(cudaStreamSynchronize(c->stream));
        }
        // stage C: 3b4 (:651-770); after the fused first stage also 3b3 and,
        // with band_fused, tc3a2a4b2b5's 3b5 (OpTC3X)
        std::vector<ChunkPlan> plan;
        TRY(plan_chunks(c, c->meta, TR.n, TR.key, TR.cartk, (int)S.key.size(), S.key, S.cartq,
                        max_items_for(c, 3, sizeof(V)), min_targets(c), plan));
        if (acc2_fused) {   // the targets' part of the combined input, qsum now complete
            TRY(c->w3x.ensure((size_t)TR.n * 3 * N * sizeof(V)));
            TRY(launch(c, k_w3x<T>, dim3((unsigned)((N + 255) / 256), TR.n), dim3(256), 0, (int)N, dnuT,
                       (const V *)(c->Rpsi.as<V>() + (size_t)TR.t0 * N), (const double2 *)(qsum + (size_t)TR.t0 * 3 * N),
                       b3, b4, c->w3x.as<V>(), TR.n));
        }
        for (const ChunkPlan &p : plan) {
            const size_t items = (size_t)p.nt * p.ns;
            TRY(c->tmp.ensure(items * 3 * N * sizeof(V)));
            TRY(gen_tables<T>(c, p, TAB_U_SS, s));
            if (acc2_fused) {
                OpTC3X<T> op;
                op_common<T>(c, op, p, 3, 1);
                op.Rpsi = c->Rpsi.as<V>() + (size_t)(TR.t0 + p.t0) * N;
                op.Rocc = c->Rocc.as<V>() + (S.base + p.s0) * N;
                op.Rchi = (bitc ? c->Rchi.as<V>() : c->Rocc.as<V>()) + (S.base + p.s0) * N;
                op.W = c->w3x.as<V>() + (size_t)p.t0 * 3 * N;
                op.Bt = band_fused ? c->Bt.as<V>() + (S.base + p.s0) * 3 * N : nullptr;
                op.acc = acc + (size_t)(TR.t0 + p.t0) * N;
                op.fill = c->occfill.as<double>() + S.base + p.s0;
                op.b5 = -band_fa4(h);
                TRY((run_chunk<T, OpTC3X<T>>(c, op, (int)items, p.nt)));
                continue;
            }
            OpTC3C<T> op;
            op_common<T>(c, op, p, 3, 1);
            op.Rocc = c->Rocc.as<V>() + (S.base + p.s0) * N;
            op.Rchi = (bitc ? c->Rchi.as<V>() : c->Rocc.as<V>()) + (S.base + p.s0) * N;
            op.qsum = qsum + (size_t)(TR.t0 + p.t0) * 3 * N;
            op.acc = acc + (size_t)(TR.t0 + p.t0) * N;
            op.fill = c->occfill.as<double>() + S.base + p.s0;
            op.b4 = b4;
            TRY((run_chunk<T, OpTC3C<T>>(c, op, (int)items, p.nt)));
        }
    }
    return TCG_OK;
}

// occupied-pair chunks of tc3a2a4b2b5 for spin sq, sources [lo, hi) of S
template <typename T, bool BITC, bool EQ>
static int qp_pairs(tcg_ctx *c, int sq, int ntq, const std::vector<int> &tkey, const std::vector<double> &tcart,
                    const Sources &S0, int lo, int hi, double2 *accP, int nacc)
{
    using V = typename C2<T>::t;
    using OQ = OpQP<T, BITC, EQ>;
    const Host &h = c->h;
    const size_t N = h.N;
    const int nsl = OQ::NB;
    if (hi <= lo) return TCG_OK;
    Sources S;
    S.base = S0.base + lo;
    S.key.assign(S0.key.begin() + lo, S0.key.begin() + hi);
    S.cartq.assign(S0.cartq.begin() + 3 * (size_t)lo, S0.cartq.begin() + 3 * (size_t)hi);
    std::vector<ChunkPlan> plan;
    TRY(plan_chunks(c, c->meta, ntq, tkey, tcart, (int)S.key.size(), S.key, S.cartq, max_items_for(c, nsl, sizeof(V)),
                    min_targets(c), plan));
    for (const ChunkPlan &p : plan) {
        const size_t items = (size_t)p.nt * p.ns;
        TRY(c->tmp.ensure(items * nsl * N * sizeof(V)));
        TRY(gen_tables<T>(c, p, TAB_U_QX, sq, EQ ? 1 : 2));
        OQ op;
        op_common<T>(c, op, p, nsl, 2);
        op.Rq2 = c->qtg.as<V>() + (size_t)p.t0 * N;
        op.Rq2c = BITC ? c->qtg.as<V>() + (size_t)(ntq + p.t0) * N : op.Rq2;
        op.Rocc = c->Rocc.as<V>() + (S.base + p.s0) * N;
        op.Rchi = (BITC ? c->Rchi.as<V>() : c->Rocc.as<V>()) + (S.base + p.s0) * N;
        op.acc = accP + (size_t)p.t0 * nacc * N;
        op.fill = c->occfill.as<double>() + S.base + p.s0;
        op.nacc = nacc;
        op.nspin = h.nspin;
        op.sq = sq;
        // the chunk's sources summed in FP32 shared-memory planes, one FP64
        // red.add per accumulator point at the end (in place of one per source)
        op.sacc_on = c->qp_sacc ? 1 : 0;
        op.sacc_n = nacc;
        TRY((run_chunk<T, OQ>(c, op, (int)items, p.nt)));
    }
    return TCG_OK;
}

// ------------------------------------ tc3a2a4b2b5: per-state occupied stage --
// Targets of spin sq: (iq2 irreducible, i2), with their grid index in Rocc.
struct QPTargets {
    std::vector<int> key, grid;
    std::vector<double> cart;
};
static QPTargets qp_targets(const tcg_ctx *c, int sq)
{
    const Host &h = c->h;
    QPTargets Q;
    for (int iq2 = 0; iq2 < h.nk; iq2++) {
        double q[3];
        cart(h, &h.kvec[3 * h.kall_off[iq2]], q);
        for (int i = 0; i < h.nocc[sq * h.nk + iq2]; i++) {
            Q.key.push_back(iq2);
            Q.grid.push_back((int)(h.occ_off[(size_t)sq * h.nk_all + h.kall_off[iq2]] + i));
            Q.cart.insert(Q.cart.end(), q, q + 3);
        }
    }
    return Q;
}

// Offsets (in grids of N points) of each spin's accumulators in accP:
// [sq][target][nacc][N], nacc = nspin + 6 (3a2 per spin, 3a4 x3, 3b5 x3).
static std::vector<size_t> qp_acc_offsets(const tcg_ctx *c)
{
    const Host &h = c->h;
    const int nacc = h.nspin + 6;
    std::vector<size_t> off(h.nspin + 1, 0);
    for (int sq = 0; sq < h.nspin; sq++) {
        size_t ntq = 0;
        for (int iq2 = 0; iq2 < h.nk; iq2++) ntq += h.nocc[sq * h.nk + iq2];
        off[sq + 1] = off[sq] + ntq * nacc;
    }
    return off;
}

// First half of the occupied-pair stage (tc3a2a4b2b5.cpp:210-443): the sums
// over the occupied sources (q1, i1) of the intermediates of every target
// (q2, i2), accumulated in c->accP.  Sources are split into nranks contiguous
// blocks and only block `rank` is summed, so that the ranks' partial buffers
// add up to the whole stage (the reference splits the q1 bands over MPI ranks
// and MPI_Allreduces these grids, :214-235, :490-493, :649-659).
template <typename T>
static int qp_partial(tcg_ctx *c, int rank, int nranks)
{
    PhaseScope ps_(c, "st:qp");
    Host &h = c->h;
    const size_t N = h.N;
    const int ns = h.nspin;
    const bool bitc = h.method == TCG_METHOD_BITC;
    const int nacc = ns + 6;
    const std::vector<size_t> aoff = qp_acc_offsets(c);
    TRY(c->accP.ensure(std::max<size_t>(1, aoff[ns]) * N * sizeof(double2)));
    TRY(launch(c, k_zero, dim3(148 * 8), dim3(256), 0, c->accP.as<double2>(), aoff[ns] * N));
    using V = typename C2<T>::t;
    for (int sq = 0; sq < ns; sq++) {
        const QPTargets Q = qp_targets(c, sq);
        const int ntq = (int)Q.key.size();
        if (ntq == 0) continue;
        Sources S = sources_of(c, sq);
        const int nsrc = (int)S.key.size();
        const int lo = (int)((int64_t)nsrc * rank / nranks), hi = (int)((int64_t)nsrc * (rank + 1) / nranks);
        // target grids are not contiguous in Rocc (isym > 0 grids in between):
        // gather them into a contiguous copy
        TRY(c->qtg.ensure((size_t)ntq * 2 * N * sizeof(V)));
        for (int i = 0; i < ntq; i++) {
            TCG_CUDA(cudaMemcpyAsync(c->qtg.as<V>() + (size_t)i * N, c->Rocc.as<V>() + (size_t)Q.grid[i] * N,
                                     N * sizeof(V), cudaMemcpyDeviceToDevice, c->stream));
            const V *chsrc = bitc ? c->Rchi.as<V>() : c->Rocc.as<V>();
            TCG_CUDA(cudaMemcpyAsync(c->qtg.as<V>() + (size_t)(ntq + i) * N, chsrc + (size_t)Q.grid[i] * N,
                                     N * sizeof(V), cudaMemcpyDeviceToDevice, c->stream));
        }
        double2 *accP = c->accP.as<double2>() + aoff[sq] * N;
        const bool eqq = h.A[sq * 2 + 0] == h.A[sq * 2 + 1] && h.F[sq * 2 + 0] == h.F[sq * 2 + 1];
        if (bitc && eqq) TRY((qp_pairs<T, true, true>(c, sq, ntq, Q.key, Q.cart, S, lo, hi, accP, nacc)));
        else if (bitc) TRY((qp_pairs<T, true, false>(c, sq, ntq, Q.key, Q.cart, S, lo, hi, accP, nacc)));
        else if (eqq) TRY((qp_pairs<T, false, true>(c, sq, ntq, Q.key, Q.cart, S, lo, hi, accP, nacc)));
        else TRY((qp_pairs<T, false, false>(c, sq, ntq, Q.key, Q.cart, S, lo, hi, accP, nacc)));
    }
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    return TCG_OK;
}

// Second half, on the summed c->accP: G = 0 divergence correction of 3a2,
// rotation of the intermediates to every equivalent q2, the 3a2 / 3b2 local
// potentials and the rotated Qt / Bt grids of the band part
// (tc3a2a4b2b5.cpp:496-817, :922-958).
template <typename T>
static int qp_finish(tcg_ctx *c)
{
    PhaseScope ps_(c, "st:qp");
    using V = typename C2<T>::t;
    Host &h = c->h;
    const size_t N = h.N;
    const int ns = h.nspin;
    const bool bitc = h.method == TCG_METHOD_BITC;
    const double Nk = h.num_kpoints, Om = h.omega;
    const int nacc = ns + 6;
    const Jastrow J = make_jastrow(h);
    RecipC rc;
    memcpy(rc.R, h.recip, sizeof rc.R);
    const GridDesc &g = c->gd;
    const unsigned pblocks = (unsigned)std::min<size_t>(148 * 8, (N + 255) / 256);
    const std::vector<size_t> aoff = qp_acc_offsets(c);
    TRY(c->Qt.ensure(h.nocc_grids * 3 * N * sizeof(V)));
    TRY(c->Bt.ensure(h.nocc_grids * 3 * N * sizeof(V)));
    TRY(c->V3a2.ensure((size_t)ns * N * sizeof(double2)));
    TRY(c->V3b2.ensure((size_t)ns * N * sizeof(double2)));
    TRY(launch(c, k_zero, dim3(pblocks), dim3(256), 0, c->V3a2.as<double2>(), (size_t)ns * N));
    TRY(launch(c, k_zero, dim3(pblocks), dim3(256), 0, c->V3b2.as<double2>(), (size_t)ns * N));
    DBuf &rot = c->rotw;              // fp64 work: 6 grids
    TRY(rot.ensure(6 * N * sizeof(double2)));
    DBuf &q3b2 = c->q3b2w;
    TRY(q3b2.ensure(3 * N * sizeof(double2)));
    for (int sq = 0; sq < ns; sq++) {
        TRY(launch(c, k_zero, dim3(pblocks), dim3(256), 0, q3b2.as<double2>(), 3 * N));
        const QPTargets Q = qp_targets(c, sq);
        const std::vector<int> &tkey = Q.key, &tgrid = Q.grid;
        const int ntq = (int)tkey.size();
        if (ntq == 0) continue;
        double2 *accP = c->accP.as<double2>() + aoff[sq] * N;
        // B = -conj(Q) for TC, then forward FFTs of all accumulators
        if (!bitc)
            for (int i = 0; i < ntq; i++)
                TRY(launch(c, k_negconj, dim3(pblocks), dim3(256), 0, 3 * N,
                           (const double2 *)(accP + ((size_t)i * nacc + ns) * N), accP + ((size_t)i * nacc + ns + 3) * N));
        {
            std::vector<void *> grids;
            for (int i = 0; i < ntq; i++)
                for (int sl = 0; sl < nacc; sl++) grids.push_back(accP + ((size_t)i * nacc + sl) * N);
            TRY((fft3_list<double, -1>(c, grids)));
        }
        // 3a2 divergence correction: pair transforms at q1 = q2 (:496-573)
        if (h.div && !h.A_zero) {
            for (int iq2 = 0; iq2 < h.nk; iq2++) {
                const int no = h.nocc[sq * h.nk + iq2];
                if (no == 0) continue;
                const size_t g0 = h.occ_off[(size_t)sq * h.nk_all + h.kall_off[iq2]];
                const int items = no * no;
                std::vector<int> idx(4 * (size_t)items);
                for (int i2 = 0; i2 < no; i2++)
                    for (int i1 = 0; i1 < no; i1++) {
                        const int it = i2 * no + i1;
                        idx[0 * items + it] = (int)(g0 + i1);   // chi_q1 (bra of phiphi)
                        idx[1 * items + it] = (int)(g0 + i2);   // phi_q2
                        idx[2 * items + it] = (int)(g0 + i2);   // chi_q2 (bra of phij)
                        idx[3 * items + it] = (int)(g0 + i1);   // phi_q1
                    }
                TRY(c->aux.ensure(idx.size() * sizeof(int)));
                TCG_CUDA(cudaMemcpyAsync(c->aux.p, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
                TRY(c->tmp.ensure((size_t)items * 2 * N * sizeof(V)));
                OpPairFwd<T> op;
                op.m = ChunkMeta{};
                op.g = g;
                op.tmp = c->tmp.as<V>();
                op.nsl = 2;
                op.ns = 1;
                memcpy(op.rc.R, h.recip, sizeof op.rc.R);
                op.invN = 1.0 / (double)N;
                const V *chi = bitc ? c->Rchi.as<V>() : c->Rocc.as<V>();
                op.A0 = chi; op.B0 = c->Rocc.as<V>(); op.A1 = chi; op.B1 = c->Rocc.as<V>();
                op.ia0 = c->aux.as<int>();
                op.ib0 = op.ia0 + items;
                op.ia1 = op.ia0 + 2 * items;
                op.ib1 = op.ia0 + 3 * items;
                TRY((run_chunk<T, OpPairFwd<T>>(c, op, items, 0, true, false)));
                const double dcorr = 1.0 / std::sqrt(PI_D * h.alpha) * Nk * Om - h.sum_vaux[iq2];
                for (int i2 = 0; i2 < no; i2++) {
                    int tq = -1;
                    for (int i = 0; i < ntq; i++)
                        if (tgrid[i] == (int)(g0 + i2)) tq = i;
                    TRY(launch(c, k_div3a2<T>, dim3(pblocks), dim3(256), 0, g, rc, J, sq, ns, no,
                               (const V *)(c->tmp.as<V>() + (size_t)i2 * no * 2 * N),
                               c->occfill.as<double>() + g0, h.A[sq * 2 + 0], h.A[sq * 2 + 1], dcorr,
                               accP + (size_t)tq * nacc * N));
                }
                TCG_CUDA(cudaStreamSynchronize(c->stream));
            }
        }
        // rotations to every equivalent q2, 3a2 / 3b2 accumulation, Qt / Bt (:576-644, :668-817)
        std::vector<double> hfill((size_t)ntq);
        for (int i = 0; i < ntq; i++) {
            const int iq2 = tkey[i];
            const int i2 = tgrid[i] - (int)h.occ_off[(size_t)sq * h.nk_all + h.kall_off[iq2]];
            hfill[i] = h.filling[fill_off(h, sq, iq2) + i2];
        }
        for (int i = 0; i < ntq; i++) {
            const int iq2 = tkey[i];
            const int i2 = tgrid[i] - (int)h.occ_off[(size_t)sq * h.nk_all + h.kall_off[iq2]];
            const double f2 = hfill[i];
            for (int isym = 0; isym < h.nsym_k[iq2]; isym++) {
                const int a2 = h.kall_off[iq2] + isym;
                RotArgs ra;
                const int *U = &h.rotation[9 * h.rot_index[a2]];
                memcpy(ra.U, U, sizeof ra.U);
                memcpy(ra.t, &h.translation[3 * h.rot_index[a2]], sizeof ra.t);
                ra.tr = h.time_rev[a2];
                // Udag_cart = recip^T U^T lattice / (2 pi)  (:688-690)
                double T1[9];
                for (int r = 0; r < 3; r++)
                    for (int q = 0; q < 3; q++) {
                        double s_ = 0;
                        for (int k = 0; k < 3; k++) s_ += h.recip[k * 3 + r] * (double)U[q * 3 + k];
                        T1[r * 3 + q] = s_;
                    }
                for (int r = 0; r < 3; r++)
                    for (int q = 0; q < 3; q++) {
                        double s_ = 0;
                        for (int k = 0; k < 3; k++) s_ += T1[r * 3 + k] * h.lattice[k * 3 + q];
                        ra.M[r * 3 + q] = s_ / (2 * PI_D);
                    }
                for (int s = 0; s < ns; s++)
                    TRY(launch(c, k_rot_scalar, dim3(pblocks), dim3(256), 0, g, ra,
                               (const double2 *)(accP + ((size_t)i * nacc + s) * N), c->V3a2.as<double2>() + (size_t)s * N, f2));
                double2 *R = rot.as<double2>();
                TRY(launch(c, k_rot_vec, dim3(pblocks), dim3(256), 0, g, ra,
                           (const double2 *)(accP + ((size_t)i * nacc + ns) * N), R));
                TRY(launch(c, k_rot_vec, dim3(pblocks), dim3(256), 0, g, ra,
                           (const double2 *)(accP + ((size_t)i * nacc + ns + 3) * N), R + 3 * N));
                std::vector<void *> grids;
                for (int d = 0; d < 6; d++) grids.push_back(R + (size_t)d * N);
                TRY((fft3_list<double, +1>(c, grids)));
                const size_t gq = h.occ_off[(size_t)sq * h.nk_all + a2] + i2;
                TRY(launch(c, k_qsum3b2<T>, dim3(pblocks), dim3(256), 0, (int)N, (const double2 *)(R + 3 * N),
                           (const V *)(c->Rocc.as<V>() + gq * N), q3b2.as<double2>(), f2));
                TRY(launch(c, k_to_prec<T>, dim3(pblocks), dim3(256), 0, (const double2 *)R, c->Qt.as<V>() + gq * 3 * N, 3 * N));
                TRY(launch(c, k_to_prec<T>, dim3(pblocks), dim3(256), 0, (const double2 *)(R + 3 * N),
                           c->Bt.as<V>() + gq * 3 * N, 3 * N));
            }
        }
        // 3b2 local potential (:922-958): V3b2[s](r) += IFFT[ sum_d G_d u' FFT(qsum3b2_d) ]
        {
            std::vector<void *> grids;
            for (int d = 0; d < 3; d++) grids.push_back(q3b2.as<double2>() + (size_t)d * N);
            TRY((fft3_list<double, -1>(c, grids)));
            for (int s = 0; s < ns; s++) {
                double2 *Vg = rot.as<double2>();
                TRY(launch(c, k_zero, dim3(pblocks), dim3(256), 0, Vg, N));
                TRY(launch(c, k_gdot, dim3(pblocks), dim3(256), 0, g, rc, J, s, ns, (const double2 *)q3b2.as<double2>(),
                           (const double2 *)nullptr, Vg, 1, sq));
                std::vector<void *> gv{Vg};
                TRY((fft3_list<double, +1>(c, gv)));
                TRY(launch(c, k_add, dim3(pblocks), dim3(256), 0, N, (const double2 *)Vg, c->V3b2.as<double2>() + (size_t)s * N));
            }
        }
    }
    {
        std::vector<void *> grids;
        for (int s = 0; s < ns; s++) grids.push_back(c->V3a2.as<double2>() + (size_t)s * N);
        TRY((fft3_list<double, +1>(c, grids)));
    }
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    h.qp_ready = true;
    return TCG_OK;
}

template <typename T>
static int qp_stage(tcg_ctx *c)
{
    TRY(qp_partial<T>(c, 0, 1));
    return qp_finish<T>(c);
}



template <typename T>
static int run_tc3a2a4b2b5_band(tcg_ctx *c, const Targets &Tg, double2 *acc)
{
    PhaseScope ps_(c, "ap:band");
    using V = typename C2<T>::t;
    const Host &h = c->h;
    const size_t N = h.N;
    const bool bitc = h.method == TCG_METHOD_BITC;
    const double fa4 = band_fa4(h), fb5 = -fa4;
    for (int s = 0; s < h.nspin; s++) {
        TRange TR = targets_of(c, Tg, s);
        Sources S = sources_of(c, s);
        std::vector<ChunkPlan> plan;
        TRY(plan_chunks(c, c->meta, TR.n, TR.key, TR.cartk, (int)S.key.size(), S.key, S.cartq,
                        max_items_for(c, 4, sizeof(V)), min_targets(c), plan));
        for (const ChunkPlan &p : plan) {
            TRY(c->tmp.ensure((size_t)p.nt * p.ns * 4 * N * sizeof(V)));
            TRY(gen_tables<T>(c, p, TAB_U_SS, s));
            OpBand<T> op;
            op_common<T>(c, op, p, 4, 1);
            op.Rpsi = c->Rpsi.as<V>() + (size_t)(TR.t0 + p.t0) * N;
            op.Rocc = c->Rocc.as<V>() + (S.base + p.s0) * N;
            op.Rchi = (bitc ? c->Rchi.as<V>() : c->Rocc.as<V>()) + (S.base + p.s0) * N;
            op.Qt = c->Qt.as<V>() + (S.base + p.s0) * 3 * N;
            op.Bt = c->Bt.as<V>() + (S.base + p.s0) * 3 * N;
            op.acc = acc + (size_t)(TR.t0 + p.t0) * N;
            op.fill = c->occfill.as<double>() + S.base + p.s0;
            op.fa4 = fa4;
            op.fb5 = fb5;
            TRY((run_chunk<T, OpBand<T>>(c, op, p.nt * p.ns, p.nt)));
        }
    }
    return TCG_OK;
}

// ----------------------------------------------- per-state work (set_state) --
template <typename T>
static int build_occupied(tcg_ctx *c)
{
    PhaseScope ps_(c, "st:occupied");
    using V = typename C2<T>::t;
    Host &h = c->h;
    const bool bitc = h.method == TCG_METHOD_BITC;
    const size_t N = h.N;
    TRY(c->Rocc.ensure(std::max<size_t>(1, h.nocc_grids) * N * sizeof(V)));
    if (bitc) TRY(c->Rchi.ensure(std::max<size_t>(1, h.nocc_grids) * N * sizeof(V)));
    const bool grad = h.method != TCG_METHOD_HF;
    if (grad) TRY(c->Rgrad.ensure(std::max<size_t>(1, h.nocc_grids) * 3 * N * sizeof(V)));
    std::vector<SphereItem> items;
    for (int s = 0; s < h.nspin; s++)
        for (int a = 0; a < h.nk_all; a++) {
            const int ik = h.ik_of_all[a];
            const size_t go = h.gidx_off[(size_t)s * h.nk_all + a];
            double qc[3];
            cart(h, &h.kvec[3 * a], qc);
            for (int i = 0; i < h.nocc[s * h.nk + ik]; i++) {
                SphereItem it{};
                const size_t cof = h.orb_off[(size_t)s * h.nk + ik] + (size_t)i * h.npw[ik];
                it.coef = c->phik.as<double2>() + cof;
                it.inv = c->inv.as<int>() + ((size_t)s * h.nk_all + a) * N;
                it.phase = c->phase.as<double2>() + go;
                it.tr = h.time_rev[a];
                it.mode = 0;
                memcpy(it.kc, qc, sizeof qc);
                const size_t grid = h.occ_off[(size_t)s * h.nk_all + a] + i;
                it.out = c->Rocc.as<V>() + grid * N;
                items.push_back(it);
                if (grad)
                    for (int d = 0; d < 3; d++) {
                        SphereItem gi = it;
                        gi.mode = 1 + d;                          // (q+G)_d phi_q(G) (tc2x.cpp:342-346)
                        gi.out = c->Rgrad.as<V>() + (grid * 3 + d) * N;
                        items.push_back(gi);
                    }
                if (bitc) {
                    SphereItem ci = it;
                    ci.coef = c->chik.as<double2>() + cof;
                    ci.out = c->Rchi.as<V>() + grid * N;
                    items.push_back(ci);
                }
            }
        }
    return sphere_to_r<T>(c, items);
}

template <typename T>
static int state_terms(tcg_ctx *c)
{
    PhaseScope ps_(c, "st:local");
    using V = typename C2<T>::t;
    Host &h = c->h;
    h.qp_ready = false;
    h.qp_pending = false;
    const size_t N = h.N;
    const int ns = h.nspin;
    const GridDesc &g = c->gd;
    const Jastrow J = make_jastrow(h);
    RecipC rc;
    memcpy(rc.R, h.recip, sizeof rc.R);
    const unsigned pblocks = (unsigned)std::min<size_t>(148 * 8, (N + 255) / 256);
    if (h.method == TCG_METHOD_HF) {
        // Hartree potential of hf2h (calc_hamiltonian_hf2h.cpp:40-51)
        TRY(c->VH.ensure(N * sizeof(double2)));
        TRY(launch(c, k_zero, dim3(pblocks), dim3(256), 0, c->VH.as<double2>(), N));
        TRY(launch(c, k_add, dim3(pblocks), dim3(256), 0, N, (const double2 *)c->dens.as<double2>(), c->VH.as<double2>()));
        TRY(launch(c, k_add, dim3(pblocks), dim3(256), 0, N, (const double2 *)(c->dens.as<double2>() + N),
                   c->VH.as<double2>()));
        std::vector<void *> gv{c->VH.p};
        TRY((fft3_list<double, -1>(c, gv)));
        TRY(launch(c, k_hartree_g, dim3(pblocks), dim3(256), 0, g, rc, c->VH.as<double2>()));
        TRY((fft3_list<double, +1>(c, gv)));
        TCG_CUDA(cudaStreamSynchronize(c->stream));
        return TCG_OK;
    }
    // density in G
    DBuf &nG = c->nGw;
    TRY(nG.ensure(2 * N * sizeof(double2)));
    TCG_CUDA(cudaMemcpyAsync(nG.p, c->dens.p, 2 * N * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
    {
        std::vector<void *> gr{nG.as<double2>(), nG.as<double2>() + N};
        TRY((fft3_list<double, -1>(c, gr)));
    }
    // compute-precision density [n_0, n_1, n_0 + n_1] (3b6 re-forward of tc3a3b3b4b6)
    TRY(c->densT.ensure(3 * N * sizeof(V)));
    TRY(launch(c, k_to_prec<T>, dim3(pblocks), dim3(256), 0, (const double2 *)c->dens.as<double2>(), c->densT.as<V>(), 2 * N));
    TRY(launch(c, k_dens_sum<T>, dim3(pblocks), dim3(256), 0, (int)N, (const double2 *)c->dens.as<double2>(),
               c->densT.as<V>() + 2 * N));
    TRY(c->dnu.ensure((size_t)ns * 3 * N * sizeof(double2)));
    TRY(c->dnuT.ensure((size_t)ns * 3 * N * sizeof(V)));
    TRY(c->V3a1.ensure((size_t)ns * N * sizeof(double2)));
    TRY(c->V3b1.ensure((size_t)ns * N * sizeof(double2)));
    DBuf &W = c->Ww;
    TRY(W.ensure((size_t)ns * 3 * N * sizeof(double2)));
    for (int s = 0; s < ns; s++) {
        double2 *dn = c->dnu.as<double2>() + (size_t)s * 3 * N;
        TRY(launch(c, k_dnu_g, dim3(pblocks), dim3(256), 0, g, rc, J, s, (const double2 *)nG.as<double2>(), dn));
        std::vector<void *> gr{dn, dn + N, dn + 2 * N};
        TRY((fft3_list<double, +1>(c, gr)));
        TRY(launch(c, k_to_prec<T>, dim3(pblocks), dim3(256), 0, (const double2 *)dn, c->dnuT.as<V>() + (size_t)s * 3 * N, 3 * N));
        TRY(launch(c, k_square_sum, dim3(pblocks), dim3(256), 0, (int)N, (const double2 *)dn, c->V3a1.as<double2>() + (size_t)s * N));
        double2 *w = W.as<double2>() + (size_t)s * 3 * N;
        TRY(launch(c, k_mul_dens, dim3(pblocks), dim3(256), 0, (int)N, (const double2 *)dn,
                   (const double2 *)(c->dens.as<double2>() + (size_t)s * N), w));
        std::vector<void *> gw{w, w + N, w + 2 * N};
        TRY((fft3_list<double, -1>(c, gw)));
    }
    for (int s1 = 0; s1 < ns; s1++) {
        double2 *V3 = c->V3b1.as<double2>() + (size_t)s1 * N;
        TRY(launch(c, k_zero, dim3(pblocks), dim3(256), 0, V3, N));
        TRY(launch(c, k_gdot, dim3(pblocks), dim3(256), 0, g, rc, J, s1, ns, (const double2 *)W.as<double2>(),
                   (const double2 *)(W.as<double2>() + (ns > 1 ? 3 * N : 0)), V3, 0, 0));
        std::vector<void *> gv{V3};
        TRY((fft3_list<double, +1>(c, gv)));
    }
    // tc2h potential (calc_hamiltonian_tc2h.cpp:53-186); its [2b_h1] dnu is the
    // tc3a1 dnu above (same spin sum of u(G; s, js) G_d n_js(G))
    TRY(c->V2h.ensure((size_t)ns * N * sizeof(double2)));
    TRY(c->pgw.ensure((size_t)ns * 3 * N * sizeof(double2)));
    for (int s = 0; s < ns; s++) {
        const size_t g0 = h.occ_off[(size_t)s * h.nk_all];
        const size_t g1 = s + 1 < ns ? h.occ_off[(size_t)(s + 1) * h.nk_all] : h.nocc_grids;
        double2 *pg = c->pgw.as<double2>() + (size_t)s * 3 * N;
        const V *chi = (h.method == TCG_METHOD_BITC ? c->Rchi.as<V>() : c->Rocc.as<V>()) + g0 * N;
        TRY(launch(c, k_phiq_gphiq<T>, dim3(pblocks), dim3(256), 0, (int)N, (int)(g1 - g0), chi,
                   (const V *)(c->Rgrad.as<V>() + g0 * 3 * N), (const double *)(c->occfill.as<double>() + g0), pg));
        std::vector<void *> gp{pg, pg + N, pg + 2 * N};
        TRY((fft3_list<double, -1>(c, gp)));
    }
    for (int s = 0; s < ns; s++) {
        double2 *V2 = c->V2h.as<double2>() + (size_t)s * N;
        TRY(launch(c, k_tc2h_g, dim3(pblocks), dim3(256), 0, g, rc, J, s, ns, (const double2 *)nG.as<double2>(),
                   (const double2 *)c->pgw.as<double2>(), V2));
        std::vector<void *> gv{V2};
        TRY((fft3_list<double, +1>(c, gv)));
    }
    // tc3a3b3b4b6 3b6 divergence pieces: tR_s(r), t1[s][k]
    TRY(c->div3b6.ensure((size_t)ns * N * sizeof(double2)));
    c->t1_3b6.assign((size_t)ns * h.nk, make_double2(0, 0));
    if (h.div && !h.A_zero) {
        std::vector<double2> n0(2);
        TCG_CUDA(cudaMemcpyAsync(&n0[0], nG.as<double2>(), sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
        TCG_CUDA(cudaMemcpyAsync(&n0[1], nG.as<double2>() + N, sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
        TCG_CUDA(cudaStreamSynchronize(c->stream));
        const double FOURPI = 4.0 * PI_D, Nk = h.num_kpoints, Om = h.omega;
        for (int s = 0; s < ns; s++) {
            double2 *tg = c->div3b6.as<double2>() + (size_t)s * N;
            TRY(launch(c, k_div3b6_g, dim3(pblocks), dim3(256), 0, g, rc, J, h.A[0], h.A[1], s, (const double2 *)nG.as<double2>(), tg));
            std::vector<void *> gv{tg};
            TRY((fft3_list<double, +1>(c, gv)));
            for (int k = 0; k < h.nk; k++) {
                const double dcorr = 1.0 / std::sqrt(PI_D * h.alpha) * Nk * Om - h.sum_vaux[k];
                double2 t1 = {0, 0};
                for (int js = 0; js < 2; js++) {
                    const double A = h.A[s * 2 + js];
                    // u(0; s, js) = -4 pi A F^2 (jastrow_functions.cpp:61-65)
                    const double u0 = -FOURPI * A * (h.F[s * 2 + js] * h.F[s * 2 + js]);
                    const double Adc = dcorr * A + u0;
                    t1.x += FOURPI * Adc * A * n0[js].x;
                    t1.y += FOURPI * Adc * A * n0[js].y;
                }
                c->t1_3b6[(size_t)s * h.nk + k] = t1;
            }
        }
    }
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    return TCG_OK;
}

// ==================================================================== apply ==
template <typename T>
static int apply_impl(tcg_ctx *c, const ApplyArgs &A)
{
    PhaseScope ps_(c, "ap:setup");
    using V = typename C2<T>::t;
    Host &h = c->h;
    const size_t N = h.N;
    Targets Tg = make_targets(c, A);
    const size_t nt = Tg.s.size();
    if (nt == 0) return TCG_OK;
    const bool need_grad = (A.mask & (TCG_TERM_TC2X | TCG_TERM_TC2H)) != 0;
    TRY(c->Rpsi.ensure(nt * N * sizeof(V)));
    if (need_grad) TRY(c->Rgpsi.ensure(nt * 3 * N * sizeof(V)));
    {
        std::vector<SphereItem> items;
        for (size_t t = 0; t < nt; t++) {
            const int s = Tg.s[t], k = Tg.k[t];
            const int a = h.kall_off[k];
            SphereItem it{};
            it.coef = A.psi + Tg.psi_off[t];
            it.inv = c->inv.as<int>() + ((size_t)s * h.nk_all + a) * N;
            it.phase = c->phase.as<double2>() + h.gidx_off[(size_t)s * h.nk_all + a];
            it.tr = 0;   // isym 0, time reversal not used (hf2x.cpp:60-63)
            it.mode = 0;
            cart(h, &h.kvec[3 * a], it.kc);
            it.out = c->Rpsi.as<V>() + t * N;
            items.push_back(it);
            if (need_grad)
                for (int d = 0; d < 3; d++) {
                    SphereItem gi = it;
                    gi.mode = 1 + d;   // (k+G)_d phi_j(G) (tc2x.cpp:287-297)
                    gi.out = c->Rgpsi.as<V>() + (t * 3 + d) * N;
                    items.push_back(gi);
                }
        }
        TRY(sphere_to_r<T>(c, items));
    }
    const unsigned pblocks = (unsigned)std::min<size_t>(148 * 8, (nt * N + 255) / 256);
    // ---- two-body terms (H2): exchange (hf2x / tc2x) and Hartree (hf2h / tc2h)
    // accumulate in one R-space grid per band, scaled by the exchange
    // factor tbf; the Hartree terms' own factor 1/(N_k Omega) enters as a / tbf
    // tc2x fused with tc3a3b3b4b6: its sum is made in the H3 block below and
    // the H2 accumulator finalised after it
    const bool fused = !(A.mask & TCG_TERM_HF2X) && fuse_tc2x_tc3(c, A.mask);
    double tbf = 1.0 / (h.num_kpoints * h.omega);
    const bool exch = (A.mask & (TCG_TERM_HF2X | TCG_TERM_TC2X)) != 0;
    if (A.mask & TCG_TERMS_H2) {
        TRY(c->acc2.ensure(nt * N * sizeof(double2)));
        TRY(launch(c, k_zero, dim3(pblocks), dim3(256), 0, c->acc2.as<double2>(), nt * N));
        if (A.mask & TCG_TERM_HF2X) {
            tbf = -4.0 * PI_D / (h.num_kpoints * h.omega);
            TRY(run_hf2x<T>(c, Tg, c->acc2.as<double2>()));
        } else if (A.mask & TCG_TERM_TC2X) {
            tbf = -1.0 / (h.num_kpoints * h.omega);
            if (!fused) TRY(run_tc2x<T>(c, Tg, c->acc2.as<double2>()));
        }
        if (exch && h.nspin == 1) tbf /= 2.0;
        if (A.mask & (TCG_TERM_HF2H | TCG_TERM_TC2H)) {
            PhaseScope ps_h(c, "ap:2h");
            const double a = (1.0 / (h.num_kpoints * h.omega)) / tbf;
            const bool tc = (A.mask & TCG_TERM_TC2H) != 0;
            for (int s = 0; s < h.nspin; s++) {
                TRange TR = targets_of(c, Tg, s);
                if (TR.n == 0) continue;
                const double2 *Vr = tc ? c->V2h.as<double2>() + (size_t)s * N : c->VH.as<double2>();
                const double2 *W = tc ? c->dnu.as<double2>() + (size_t)s * 3 * N : nullptr;
                TRY(launch(c, k_local_h2<T>, dim3((unsigned)std::min<size_t>(64, (N + 255) / 256), TR.n), dim3(256), 0,
                           (int)N, (const V *)(c->Rpsi.as<V>() + (size_t)TR.t0 * N),
                           (const V *)(tc ? c->Rgpsi.as<V>() + (size_t)TR.t0 * 3 * N : nullptr), Vr, W, a,
                           c->acc2.as<double2>() + (size_t)TR.t0 * N));
            }
        }
        if (!fused) {
            TRY(finalize_acc(c, Tg, c->acc2.as<double2>(), A.h2, tbf));
            if (exch) TRY(div_2x(c, Tg, A, A.h2));
        }
    }
    // ---- three-body terms (H3)
    const uint32_t m3 = A.mask & ~TCG_TERMS_H2;
    if (m3) {
        TRY(c->acc3.ensure(nt * N * sizeof(double2)));
        double2 *acc = c->acc3.as<double2>();
        TRY(launch(c, k_zero, dim3(pblocks), dim3(256), 0, acc, nt * N));
        if ((m3 & TCG_TERM_TC3A2A4B2B5) && h.qp_pending)
            return fail(TCG_ERR_STATE, "tcg_qp_partial was called: sum its buffer and call tcg_qp_finish first");
        if ((m3 & TCG_TERM_TC3A2A4B2B5) && !h.qp_ready) TRY(qp_stage<T>(c));
        // local potentials: tc3a1, tc3b1, and the 3a2 / 3b2 parts of tc3a2a4b2b5
        const double Nk = h.num_kpoints, Om = h.omega;
        const double base = 1.0 / (Nk * Nk * Om * Om);
        TRY(c->Vloc.ensure((size_t)h.nspin * N * sizeof(double2)));
        bool any_local = false;
        for (int s = 0; s < h.nspin; s++) {
            double2 *Vl = c->Vloc.as<double2>() + (size_t)s * N;
            TRY(launch(c, k_zero, dim3(pblocks), dim3(256), 0, Vl, N));
            if (m3 & TCG_TERM_TC3A1) { TRY(launch(c, k_axpy, dim3(pblocks), dim3(256), 0, N, 0.5 * base, (const double2 *)(c->V3a1.as<double2>() + (size_t)s * N), Vl)); any_local = true; }
            if (m3 & TCG_TERM_TC3B1) { TRY(launch(c, k_axpy, dim3(pblocks), dim3(256), 0, N, -1.0 * base, (const double2 *)(c->V3b1.as<double2>() + (size_t)s * N), Vl)); any_local = true; }
            if (m3 & TCG_TERM_TC3A2A4B2B5) {
                double fa2 = -0.5 * base, fb2 = base;
                if (h.nspin == 1) { fa2 /= 4.0; fb2 /= 4.0; }
                TRY(launch(c, k_axpy, dim3(pblocks), dim3(256), 0, N, fa2, (const double2 *)(c->V3a2.as<double2>() + (size_t)s * N), Vl));
                TRY(launch(c, k_axpy, dim3(pblocks), dim3(256), 0, N, fb2, (const double2 *)(c->V3b2.as<double2>() + (size_t)s * N), Vl));
                any_local = true;
            }
        }
        if (any_local)
            for (int s = 0; s < h.nspin; s++) {
                TRange TR = targets_of(c, Tg, s);
                if (TR.n == 0) continue;
                TRY(launch(c, k_local<T>, dim3((unsigned)std::min<size_t>(64, (N + 255) / 256), TR.n), dim3(256), 0, (int)N,
                           (const V *)(c->Rpsi.as<V>() + (size_t)TR.t0 * N), (const double2 *)(c->Vloc.as<double2>() + (size_t)s * N),
                           acc + (size_t)TR.t0 * N));
            }
        // with tc2x fused into tc3a3b3b4b6, the 3a4 band part of tc3a2a4b2b5 joins them
        const bool band_fused = fused && (m3 & TCG_TERM_TC3A2A4B2B5);
        if ((m3 & TCG_TERM_TC3A2A4B2B5) && !band_fused) TRY(run_tc3a2a4b2b5_band<T>(c, Tg, acc));
        if (m3 & TCG_TERM_TC3A3B3B4B6)
            TRY(run_tc3a3b3b4b6<T>(c, Tg, A, acc, fused ? c->acc2.as<double2>() : nullptr, band_fused));
        TRY(finalize_acc(c, Tg, acc, A.h3, 1.0));
    }
    if (fused) {
        TRY(finalize_acc(c, Tg, c->acc2.as<double2>(), A.h2, tbf));
        if (exch) TRY(div_2x(c, Tg, A, A.h2));
    }
    TCG_CUDA(cudaStreamSynchronize(c->stream));
    return TCG_OK;
}

} // namespace tcg
