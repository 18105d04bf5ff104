/*
 * tc_oracle.c -- FP64 CPU restatement of TC++'s operator-application hot
 * path.  TEST INFRASTRUCTURE: the checker for libtcg_b200.so and the timed
 * CPU baseline; never linked into the product.  Parity unpinned against the
 * reference binary (see tc_oracle.h).
 *
 * Every routine follows the loop structure, factors and G=0 branches of the
 * reference file cited above it.  Two deliberate differences, neither of
 * which changes the mathematics:
 *  - R-space occupied orbitals phi_q(r), chi_q(r), grad phi_q(r) are built
 *    once per call instead of once per (k, j, q) (the reference recomputes
 *    them, e.g. calc_hamiltonian_tc2x.cpp:306-347);
 *  - OpenMP parallelises over (k, j) band-applies (or occupied (q2, i2)
 *    targets) with each task accumulating privately in the reference's
 *    order, so results are deterministic run to run.
 * The FFT is an own mixed-radix Cooley-Tukey (FFTW is the reference's,
 * plane_wave_basis.cpp:175-198), exp(-iGr)/N forward, exp(+iGr) backward.
 */
#include <complex.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "tc_oracle.h"

typedef double complex cplx;
static const double PI = 3.14159265358979323846;
#define FOURPI (4.0 * PI)

static __thread char g_err[512];
static int g_threads = 0;
/* Timing-sample mode for the CPU baseline: q-loops over the all-k sources
 * visit only every g_qstride-th k-point (the results are then partial sums,
 * used for timing only); g_t_shared accumulates the wall time of the
 * occupied-pair stage of tc3a2a4b2b5, g_t_total of tco_apply. */
static int g_qstride = 1;
static double g_t_shared = 0.0, g_t_total = 0.0, g_t_init = 0.0;
static double now_s(void)
{
#ifdef _OPENMP
    return omp_get_wtime();
#else
    return 0.0;
#endif
}
void tco_set_qstride(int s) { g_qstride = s > 0 ? s : 1; }
void tco_timers(double *shared, double *total, double *init)
{
    if (shared) *shared = g_t_shared;
    if (total) *total = g_t_total;
    if (init) *init = g_t_init;
}
void tco_reset_timers(void) { g_t_shared = g_t_total = g_t_init = 0.0; }
#define QSKIP(a) ((a) % g_qstride != 0)

static int fail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}
const char *tco_last_error(void) { return g_err; }
void tco_set_threads(int n) { g_threads = n; }
int tco_get_threads(void)
{
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

/* ======================================================================
 * Mixed-radix FFT (own implementation; stands in for FFTW3)
 * ====================================================================== */
typedef struct {
    int n, nf, f[40];
    cplx *w; /* w[j] = exp(-2 pi i j / n) */
} plan1d;

static void plan_init(plan1d *p, int n)
{
    p->n = n;
    p->nf = 0;
    int m = n;
    while (m % 4 == 0) { p->f[p->nf++] = 4; m /= 4; }
    while (m % 2 == 0) { p->f[p->nf++] = 2; m /= 2; }
    for (int q = 3; m > 1; q += 2)
        while (m % q == 0) { p->f[p->nf++] = q; m /= q; }
    p->w = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    for (int j = 0; j < n; j++) {
        double a = 2.0 * PI * (double)j / (double)n;
        p->w[j] = cos(a) - I * sin(a);
    }
}
static void plan_free(plan1d *p) { free(p->w); }

/* decimation-in-time: X[k + m s] = sum_r W_p^{rs} (W_n^{rk} Y_r[k]) */
static void fft_rec(const cplx *in, int is, cplx *out, int n, const int *f,
                    const plan1d *P, int wstep, int sign)
{
    if (n == 1) { out[0] = in[0]; return; }
    const int p = f[0], m = n / p, N = P->n;
    for (int r = 0; r < p; r++)
        fft_rec(in + (size_t)r * is, is * p, out + (size_t)r * m, m, f + 1, P, wstep * p, sign);
    cplx t[64], wp[64];
    for (int j = 0; j < p; j++) {
        cplx w = P->w[(size_t)j * (N / p)];
        wp[j] = sign < 0 ? w : conj(w);
    }
    for (int k = 0; k < m; k++) {
        for (int r = 0; r < p; r++) {
            cplx w = P->w[(size_t)r * k * wstep];
            t[r] = out[(size_t)r * m + k] * (sign < 0 ? w : conj(w));
        }
        if (p == 2) {
            out[k] = t[0] + t[1];
            out[k + m] = t[0] - t[1];
        } else if (p == 4) {
            cplx a0 = t[0] + t[2], a1 = t[0] - t[2];
            cplx b0 = t[1] + t[3], b1 = (t[1] - t[3]) * (sign < 0 ? -I : I);
            out[k] = a0 + b0;
            out[k + m] = a1 + b1;
            out[k + 2 * m] = a0 - b0;
            out[k + 3 * m] = a1 - b1;
        } else {
            for (int s = 0; s < p; s++) {
                cplx acc = 0;
                for (int r = 0; r < p; r++) acc += t[r] * wp[(r * s) % p];
                out[k + (size_t)m * s] = acc;
            }
        }
    }
}

typedef struct {
    int nr[3], N;
    plan1d p[3];
} fft3;

static void fft3_init(fft3 *F, const int32_t nr[3])
{
    for (int d = 0; d < 3; d++) { F->nr[d] = nr[d]; plan_init(&F->p[d], nr[d]); }
    F->N = nr[0] * nr[1] * nr[2];
}
static void fft3_free(fft3 *F) { for (int d = 0; d < 3; d++) plan_free(&F->p[d]); }

/* forward: exp(-iGr)/N ; backward: exp(+iGr) */
static void fft3_exec(const fft3 *F, cplx *a, int forward)
{
    const int n0 = F->nr[0], n1 = F->nr[1], n2 = F->nr[2];
    const int sign = forward ? -1 : +1;
    int nmax = n0 > n1 ? n0 : n1;
    if (n2 > nmax) nmax = n2;
    cplx bin[256], bout[256];
    cplx *in = bin, *out = bout;
    if (nmax > 256) { in = malloc(sizeof(cplx) * nmax); out = malloc(sizeof(cplx) * nmax); }
    for (int r = 0; r < n1 * n2; r++) {
        cplx *row = a + (size_t)r * n0;
        memcpy(in, row, sizeof(cplx) * n0);
        fft_rec(in, 1, out, n0, F->p[0].f, &F->p[0], 1, sign);
        memcpy(row, out, sizeof(cplx) * n0);
    }
    for (int i2 = 0; i2 < n2; i2++)
        for (int i0 = 0; i0 < n0; i0++) {
            cplx *base = a + (size_t)i2 * n0 * n1 + i0;
            for (int i1 = 0; i1 < n1; i1++) in[i1] = base[(size_t)i1 * n0];
            fft_rec(in, 1, out, n1, F->p[1].f, &F->p[1], 1, sign);
            for (int i1 = 0; i1 < n1; i1++) base[(size_t)i1 * n0] = out[i1];
        }
    for (int i1 = 0; i1 < n1; i1++)
        for (int i0 = 0; i0 < n0; i0++) {
            cplx *base = a + (size_t)i1 * n0 + i0;
            for (int i2 = 0; i2 < n2; i2++) in[i2] = base[(size_t)i2 * n0 * n1];
            fft_rec(in, 1, out, n2, F->p[2].f, &F->p[2], 1, sign);
            for (int i2 = 0; i2 < n2; i2++) base[(size_t)i2 * n0 * n1] = out[i2];
        }
    if (forward) {
        const double s = 1.0 / (double)F->N;
        for (int i = 0; i < F->N; i++) a[i] *= s;
    }
    if (nmax > 256) { free(in); free(out); }
}

int tco_fft3d(const int32_t nr[3], double *grid, int forward)
{
    if (!nr || !grid || nr[0] < 1 || nr[1] < 1 || nr[2] < 1) return fail(TCG_ERR_ARG, "bad grid");
    fft3 F;
    fft3_init(&F, nr);
    fft3_exec(&F, (cplx *)grid, forward);
    fft3_free(&F);
    return TCG_OK;
}

/* ======================================================================
 * Jastrow (RPA), jastrow_functions.cpp:6-97, jastrow_initialize.cpp:86-110
 * ====================================================================== */
static int jastrow_A_zero(const tcg_system_desc *s)
{
    /* Jastrow::set_A_long (jastrow_initialize.cpp:15-22) */
    for (int i = 0; i < 4; i++)
        if (fabs(s->jastrow_A[i]) > 1e-8) return 0;
    return 1;
}

double tco_uk(const tcg_system_desc *sys, const double G[3], int s1, int s2)
{
    if (jastrow_A_zero(sys)) return 0.0; /* Jastrow::uk: no RPA, no polynomial */
    const double A = sys->jastrow_A[s1 * 2 + s2], F = sys->jastrow_F[s1 * 2 + s2];
    const double FourPI_A = FOURPI * A, F2 = F * F;
    const double G2 = G[0] * G[0] + G[1] * G[1] + G[2] * G[2];
    if (G2 < 1e-12) return -FourPI_A * F2;
    return FourPI_A / (G2 * (G2 * F2 + 1));
}

double tco_tc2body(const tcg_system_desc *sys, const double G[3], int s1, int s2)
{
    const double G2 = G[0] * G[0] + G[1] * G[1] + G[2] * G[2];
    if (jastrow_A_zero(sys)) return G2 > 1e-12 ? FOURPI / G2 : 0.0;
    const double A = sys->jastrow_A[s1 * 2 + s2], F = sys->jastrow_F[s1 * 2 + s2];
    const double FourPI_A = FOURPI * A, F2 = F * F;
    const double PI_AAFinv2 = PI * A * A * (1.0 / F2);
    if (G2 < 1e-12) return -2 * PI_AAFinv2 * F;
    const double G1 = sqrt(G2), FG1 = F * G1, F2G2 = F2 * G2;
    return FOURPI / G2 - FourPI_A / (1 + F2G2)
           + (PI_AAFinv2 / G1) * (PI * F2G2 + (4 + 2 * F2G2) * atan(FG1 / 2) - (4 + 4 * F2G2) * atan(FG1));
}

/* ======================================================================
 * Context: offsets, G tables, occupied R-space orbitals
 * ====================================================================== */
typedef struct {
    const tcg_system_desc *sys;
    const tcg_state_desc *st;
    int n0, n1, n2, N, nspin, nk, nk_all;
    int is_bitc;
    fft3 F;
    int *kall_off;      /* [nk+1] */
    int *ik_of_all;     /* [nk_all] */
    size_t *gidx_off;   /* [nspin*nk_all] */
    size_t *orb_off;    /* [nspin*nk] offset (complex units) of band 0 in phik */
    double (*Gv)[3];    /* [N] Cartesian G of grid point (get_Gvector) */
    int (*Gm)[3];       /* [N] signed Miller indices */
    cplx **phiq;        /* [nspin*nk_all] -> nocc grids (R) */
    cplx **chiq;        /* BITC left orbitals (R); == phiq otherwise */
} octx;

static size_t gidx_offset(const octx *c, int s, int a) { return c->gidx_off[(size_t)s * c->nk_all + a]; }

static void get_G(const octx *c, int ipw, int m[3])
{
    int i1 = ipw % c->n0, i2 = (ipw / c->n0) % c->n1, i3 = ipw / (c->n0 * c->n1);
    m[0] = i1 <= c->n0 / 2 ? i1 : i1 - c->n0;
    m[1] = i2 <= c->n1 / 2 ? i2 : i2 - c->n1;
    m[2] = i3 <= c->n2 / 2 ? i3 : i3 - c->n2;
}

/* Cartesian v = recip^T x */
static void cart(const tcg_system_desc *s, const double x[3], double v[3])
{
    for (int d = 0; d < 3; d++)
        v[d] = s->recip[0 * 3 + d] * x[0] + s->recip[1 * 3 + d] * x[1] + s->recip[2 * 3 + d] * x[2];
}

/* PlaneWaveBasis::get_orbital_FFTgrid (plane_wave_basis.cpp:221-271), SCF mode */
static void scatter(const octx *c, int s, int a, const cplx *coef, cplx *grid)
{
    const int ik = c->ik_of_all[a];
    const int npw = c->sys->npw[ik];
    const int32_t *gi = c->sys->gindex + gidx_offset(c, s, a);
    const cplx *ph = (const cplx *)c->sys->phase + gidx_offset(c, s, a);
    memset(grid, 0, sizeof(cplx) * c->N);
    if (c->sys->time_rev[a]) {
        for (int p = 0; p < npw; p++) grid[gi[p]] = conj(coef[p]) * ph[p];
    } else {
        for (int p = 0; p < npw; p++) grid[gi[p]] = coef[p] * ph[p];
    }
}

static const cplx *phik_band(const octx *c, int s, int ik, int b)
{
    return (const cplx *)c->st->phik + c->orb_off[(size_t)s * c->nk + ik] + (size_t)b * c->sys->npw[ik];
}
static const cplx *chik_band(const octx *c, int s, int ik, int b)
{
    const double *base = c->is_bitc ? c->st->phik_left : c->st->phik;
    return (const cplx *)base + c->orb_off[(size_t)s * c->nk + ik] + (size_t)b * c->sys->npw[ik];
}
static double fill(const octx *c, int s, int ik, int b)
{
    size_t off = 0;
    for (int s2 = 0; s2 < s; s2++) off += (size_t)c->nk * c->st->nbands[s2];
    return c->st->filling[off + (size_t)ik * c->st->nbands[s] + b];
}
static int nocc(const octx *c, int s, int ik) { return c->st->nocc[s * c->nk + ik]; }

static cplx *gnew(const octx *c) { return (cplx *)calloc((size_t)c->N, sizeof(cplx)); }

static int ctx_init(octx *c, const tcg_system_desc *sys, const tcg_state_desc *st, int need_orbitals)
{
    memset(c, 0, sizeof *c);
    c->sys = sys;
    c->st = st;
    c->n0 = sys->nr[0]; c->n1 = sys->nr[1]; c->n2 = sys->nr[2];
    c->N = c->n0 * c->n1 * c->n2;
    c->nspin = sys->nspin;
    c->nk = sys->nk_irr;
    c->is_bitc = sys->calc_method == TCG_METHOD_BITC;
    if (c->nspin < 1 || c->nspin > 2 || c->nk < 1 || c->N < 1) return fail(TCG_ERR_ARG, "bad system sizes");
    if (c->is_bitc && st && !st->phik_left) return fail(TCG_ERR_ARG, "BITC needs phik_left");
    c->kall_off = malloc(sizeof(int) * (c->nk + 1));
    c->kall_off[0] = 0;
    for (int k = 0; k < c->nk; k++) c->kall_off[k + 1] = c->kall_off[k] + sys->nsym_k[k];
    c->nk_all = c->kall_off[c->nk];
    c->ik_of_all = malloc(sizeof(int) * c->nk_all);
    for (int k = 0; k < c->nk; k++)
        for (int a = c->kall_off[k]; a < c->kall_off[k + 1]; a++) c->ik_of_all[a] = k;
    c->gidx_off = malloc(sizeof(size_t) * c->nspin * c->nk_all);
    size_t off = 0;
    for (int s = 0; s < c->nspin; s++)
        for (int a = 0; a < c->nk_all; a++) {
            c->gidx_off[(size_t)s * c->nk_all + a] = off;
            off += sys->npw[c->ik_of_all[a]];
        }
    for (size_t i = 0; i < off; i++)
        if (sys->gindex[i] < 0 || sys->gindex[i] >= c->N) return fail(TCG_ERR_ARG, "gindex out of range");
    c->Gv = malloc(sizeof(double[3]) * c->N);
    c->Gm = malloc(sizeof(int[3]) * c->N);
    for (int ipw = 0; ipw < c->N; ipw++) {
        int m[3];
        get_G(c, ipw, m);
        double x[3] = {m[0], m[1], m[2]};
        cart(sys, x, c->Gv[ipw]);
        memcpy(c->Gm[ipw], m, sizeof m);
    }
    fft3_init(&c->F, sys->nr);
    if (st) {
        c->orb_off = malloc(sizeof(size_t) * c->nspin * c->nk);
        off = 0;
        for (int s = 0; s < c->nspin; s++)
            for (int k = 0; k < c->nk; k++) {
                c->orb_off[(size_t)s * c->nk + k] = off;
                off += (size_t)st->nbands[s] * sys->npw[k];
            }
    }
    if (st && need_orbitals) {
        const int nsa = c->nspin * c->nk_all;
        c->phiq = calloc(nsa, sizeof(cplx *));
        c->chiq = calloc(nsa, sizeof(cplx *));
        for (int s = 0; s < c->nspin; s++)
            for (int a = 0; a < c->nk_all; a++) {
                int ik = c->ik_of_all[a], no = nocc(c, s, ik);
                c->phiq[s * c->nk_all + a] = malloc(sizeof(cplx) * (size_t)c->N * (no > 0 ? no : 1));
                c->chiq[s * c->nk_all + a] = c->is_bitc ? malloc(sizeof(cplx) * (size_t)c->N * (no > 0 ? no : 1))
                                                        : c->phiq[s * c->nk_all + a];
            }
        int total = c->nspin * c->nk_all;
#pragma omp parallel for schedule(dynamic, 1) num_threads(tco_get_threads())
        for (int sa = 0; sa < total; sa++) {
            int s = sa / c->nk_all, a = sa % c->nk_all, ik = c->ik_of_all[a];
            for (int i = 0; i < nocc(c, s, ik); i++) {
                cplx *g = c->phiq[sa] + (size_t)i * c->N;
                scatter(c, s, a, phik_band(c, s, ik, i), g);
                fft3_exec(&c->F, g, 0);
                if (c->is_bitc) {
                    g = c->chiq[sa] + (size_t)i * c->N;
                    scatter(c, s, a, chik_band(c, s, ik, i), g);
                    fft3_exec(&c->F, g, 0);
                }
            }
        }
    }
    return TCG_OK;
}

static void ctx_free(octx *c)
{
    if (c->phiq) {
        for (int i = 0; i < c->nspin * c->nk_all; i++) {
            if (c->is_bitc) free(c->chiq[i]);
            free(c->phiq[i]);
        }
        free(c->phiq);
        free(c->chiq);
    }
    free(c->kall_off); free(c->ik_of_all); free(c->gidx_off); free(c->orb_off);
    free(c->Gv); free(c->Gm);
    fft3_free(&c->F);
}

static const cplx *Rphi(const octx *c, int s, int a, int i) { return c->phiq[s * c->nk_all + a] + (size_t)i * c->N; }
static const cplx *Rchi(const octx *c, int s, int a, int i) { return c->chiq[s * c->nk_all + a] + (size_t)i * c->N; }

/* psi-like packed arrays */
typedef struct {
    const int32_t *nb;
    size_t *off; /* [nspin*nk] */
} packing;

static void pack_init(packing *p, const octx *c, const int32_t *nb)
{
    p->nb = nb;
    p->off = malloc(sizeof(size_t) * c->nspin * c->nk);
    size_t off = 0;
    for (int s = 0; s < c->nspin; s++)
        for (int k = 0; k < c->nk; k++) {
            p->off[s * c->nk + k] = off;
            off += (size_t)nb[s * c->nk + k] * c->sys->npw[k];
        }
}
static size_t pk(const packing *p, const octx *c, int s, int k, int b)
{
    return p->off[s * c->nk + k] + (size_t)b * c->sys->npw[k];
}

/* zeroth isym of irreducible k */
static int a0(const octx *c, int ik) { return c->kall_off[ik]; }

/* gather H(ipw) += f * grid(Gindex(ipw)) at (s, ik, isym 0) */
static void gather_add(const octx *c, int s, int ik, const cplx *grid, cplx fac, cplx *h)
{
    const int32_t *gi = c->sys->gindex + gidx_offset(c, s, a0(c, ik));
    for (int p = 0; p < c->sys->npw[ik]; p++) h[p] += fac * grid[gi[p]];
}

static cplx dotc(const cplx *a, const cplx *b, int n) /* Eigen a.dot(b) = sum conj(a) b */
{
    cplx acc = 0;
    for (int i = 0; i < n; i++) acc += conj(a[i]) * b[i];
    return acc;
}

typedef struct { int s, ik, j; } task;

static int make_tasks(const octx *c, const packing *P, const uint8_t *owned, task **out)
{
    int n = 0;
    for (int s = 0; s < c->nspin; s++)
        for (int k = 0; k < c->nk; k++) n += P->nb[s * c->nk + k];
    task *t = malloc(sizeof(task) * (n > 0 ? n : 1));
    int m = 0, flat = 0;
    for (int s = 0; s < c->nspin; s++)
        for (int k = 0; k < c->nk; k++)
            for (int j = 0; j < P->nb[s * c->nk + k]; j++, flat++) {
                if (owned && !owned[flat]) continue;
                t[m].s = s; t[m].ik = k; t[m].j = j; m++;
            }
    *out = t;
    return m;
}

/* div_corr of hf2x / tc2x (calc_hamiltonian_hf2x.cpp:150-163) */
static double div_corr_2x(const octx *c, int ik)
{
    double d = 1.0 / sqrt(PI * c->sys->alpha_Vaux);
    d -= c->sys->sum_Vaux[ik] / (c->sys->num_kpoints * c->sys->omega);
    d *= -1;
    if (c->nspin == 1) d /= 2.0;
    return d;
}

/* ======================================================================
 * hf2x -- calc_hamiltonian_hf2x.cpp:8-205
 * ====================================================================== */
static void run_hf2x(const octx *c, const packing *P, const task *T, int nt, const cplx *psi, cplx *h2)
{
    double tbf = -FOURPI / (c->sys->num_kpoints * c->sys->omega);
    if (c->nspin == 1) tbf /= 2.0;
#pragma omp parallel for schedule(dynamic, 1) num_threads(tco_get_threads())
    for (int t = 0; t < nt; t++) {
        const int s = T[t].s, ik = T[t].ik, j = T[t].j, N = c->N;
        cplx *phij = gnew(c), *phiqj = gnew(c), *Hsub = gnew(c);
        double *V = malloc(sizeof(double) * N);
        const cplx *psij = psi + pk(P, c, s, ik, j);
        const double *kref = c->sys->kvec + 3 * a0(c, ik);
        scatter(c, s, a0(c, ik), psij, phij);
        fft3_exec(&c->F, phij, 0);
        for (int a = 0; a < c->nk_all; a++) {
            const int iq = c->ik_of_all[a];
            if (nocc(c, s, iq) == 0 || QSKIP(a)) continue;
            double dk[3], kq[3];
            for (int d = 0; d < 3; d++) dk[d] = kref[d] - c->sys->kvec[3 * a + d];
            cart(c->sys, dk, kq);
            for (int ipw = 0; ipw < N; ipw++) {
                double x = kq[0] + c->Gv[ipw][0], y = kq[1] + c->Gv[ipw][1], z = kq[2] + c->Gv[ipw][2];
                double tmp = x * x + y * y + z * z;
                V[ipw] = tmp < 1e-8 ? 0.0 : 1.0 / tmp;
            }
            for (int ib = 0; ib < nocc(c, s, iq); ib++) {
                const cplx *phiq = Rphi(c, s, a, ib);
                for (int i = 0; i < N; i++) phiqj[i] = conj(phiq[i]) * phij[i];
                fft3_exec(&c->F, phiqj, 1);
                for (int i = 0; i < N; i++) phiqj[i] *= V[i];
                fft3_exec(&c->F, phiqj, 0);
                const double filq = fill(c, s, iq, ib);
                for (int i = 0; i < N; i++) Hsub[i] += filq * phiqj[i] * phiq[i];
            }
        }
        fft3_exec(&c->F, Hsub, 1);
        cplx *h = h2 + pk(P, c, s, ik, j);
        gather_add(c, s, ik, Hsub, tbf, h);
        if (c->sys->includes_div_correction) {
            const double dc = div_corr_2x(c, ik);
            const int npw = c->sys->npw[ik];
            for (int b = 0; b < c->st->nbands[s]; b++) {
                const double fb = fill(c, s, ik, b);
                if (fb < 1e-8) continue;
                const cplx *pk_ = phik_band(c, s, ik, b);
                cplx prod = dotc(pk_, psij, npw);
                prod *= fb * dc;
                for (int p = 0; p < npw; p++) h[p] += prod * pk_[p];
            }
        }
        free(phij); free(phiqj); free(Hsub); free(V);
    }
}

/* ======================================================================
 * tc2x -- calc_hamiltonian_tc2x.cpp:11-516 (SCF mesh: kVaux = 0)
 * ====================================================================== */
static void run_tc2x(const octx *c, const packing *P, const task *T, int nt, const cplx *psi, cplx *h2)
{
    double tbf = -1.0 / (c->sys->num_kpoints * c->sys->omega);
    if (c->nspin == 1) tbf /= 2.0;
    /* grad phi_q(r) for every occupied (s, a, i): IFFT[(q+G)_d phi_q(G)] */
    const int nsa = c->nspin * c->nk_all;
    cplx **gradq = calloc(nsa, sizeof(cplx *));
    for (int sa = 0; sa < nsa; sa++) {
        int s = sa / c->nk_all, a = sa % c->nk_all, no = nocc(c, s, c->ik_of_all[a]);
        gradq[sa] = malloc(sizeof(cplx) * (size_t)c->N * 3 * (no > 0 ? no : 1));
    }
#pragma omp parallel for schedule(dynamic, 1) num_threads(tco_get_threads())
    for (int sa = 0; sa < nsa; sa++) {
        int s = sa / c->nk_all, a = sa % c->nk_all, iq = c->ik_of_all[a];
        double qv[3];
        cart(c->sys, c->sys->kvec + 3 * a, qv);
        cplx *g = gnew(c);
        for (int ib = 0; ib < nocc(c, s, iq); ib++) {
            scatter(c, s, a, phik_band(c, s, iq, ib), g);
            for (int d = 0; d < 3; d++) {
                cplx *o = gradq[sa] + ((size_t)ib * 3 + d) * c->N;
                for (int i = 0; i < c->N; i++) o[i] = (qv[d] + c->Gv[i][d]) * g[i];
                fft3_exec(&c->F, o, 0);
            }
        }
        free(g);
    }

#pragma omp parallel for schedule(dynamic, 1) num_threads(tco_get_threads())
    for (int t = 0; t < nt; t++) {
        const int s = T[t].s, ik = T[t].ik, j = T[t].j, N = c->N;
        cplx *phij = gnew(c), *phiqj = gnew(c), *Hsub = gnew(c), *temp = gnew(c);
        cplx *gphij[3], *pgp[3];
        for (int d = 0; d < 3; d++) { gphij[d] = gnew(c); pgp[d] = gnew(c); }
        double *V2 = malloc(sizeof(double) * N), *duk[3];
        for (int d = 0; d < 3; d++) duk[d] = malloc(sizeof(double) * N);
        const cplx *psij = psi + pk(P, c, s, ik, j);
        double kvect[3];
        cart(c->sys, c->sys->kvec + 3 * a0(c, ik), kvect);
        scatter(c, s, a0(c, ik), psij, phij);
        for (int i = 0; i < N; i++)
            for (int d = 0; d < 3; d++) gphij[d][i] = (kvect[d] + c->Gv[i][d]) * phij[i];
        for (int d = 0; d < 3; d++) fft3_exec(&c->F, gphij[d], 0);
        fft3_exec(&c->F, phij, 0);
        for (int a = 0; a < c->nk_all; a++) {
            const int iq = c->ik_of_all[a];
            if (nocc(c, s, iq) == 0 || QSKIP(a)) continue;
            double qv[3], kq[3];
            cart(c->sys, c->sys->kvec + 3 * a, qv);
            for (int d = 0; d < 3; d++) kq[d] = kvect[d] - qv[d];
            for (int i = 0; i < N; i++) {
                double G[3] = {kq[0] + c->Gv[i][0], kq[1] + c->Gv[i][1], kq[2] + c->Gv[i][2]};
                V2[i] = tco_tc2body(c->sys, G, s, s);
                double u = tco_uk(c->sys, G, s, s);
                for (int d = 0; d < 3; d++) duk[d][i] = G[d] * u;
            }
            for (int ib = 0; ib < nocc(c, s, iq); ib++) {
                const cplx *phiq = Rphi(c, s, a, ib), *chiq = Rchi(c, s, a, ib);
                const cplx *gq = gradq[s * c->nk_all + a] + (size_t)ib * 3 * N;
                for (int i = 0; i < N; i++) phiqj[i] = conj(chiq[i]) * phij[i];
                fft3_exec(&c->F, phiqj, 1);
                for (int d = 0; d < 3; d++) {
                    for (int i = 0; i < N; i++) pgp[d][i] = phiqj[i] * duk[d][i];
                    fft3_exec(&c->F, pgp[d], 0);
                }
                const double filq = fill(c, s, iq, ib);
                memset(temp, 0, sizeof(cplx) * N);
                for (int d = 0; d < 3; d++)
                    for (int i = 0; i < N; i++) temp[i] += pgp[d][i] * gq[(size_t)d * N + i];
                for (int i = 0; i < N; i++) Hsub[i] -= filq * temp[i];
                for (int d = 0; d < 3; d++) {
                    for (int i = 0; i < N; i++) pgp[d][i] = conj(chiq[i]) * gphij[d][i];
                    fft3_exec(&c->F, pgp[d], 1);
                }
                for (int i = 0; i < N; i++) phiqj[i] *= V2[i];
                for (int d = 0; d < 3; d++)
                    for (int i = 0; i < N; i++) phiqj[i] += pgp[d][i] * duk[d][i];
                fft3_exec(&c->F, phiqj, 0);
                for (int i = 0; i < N; i++) Hsub[i] += filq * phiqj[i] * phiq[i];
            }
        }
        fft3_exec(&c->F, Hsub, 1);
        cplx *h = h2 + pk(P, c, s, ik, j);
        gather_add(c, s, ik, Hsub, tbf, h);
        if (c->sys->includes_div_correction) {
            const double dc = div_corr_2x(c, ik);
            const int npw = c->sys->npw[ik];
            for (int b = 0; b < c->st->nbands[s]; b++) {
                const double fb = fill(c, s, ik, b);
                if (fb < 1e-8) continue;
                cplx prod = dotc(chik_band(c, s, ik, b), psij, npw);
                prod *= dc;
                prod *= fb;
                const cplx *pk_ = phik_band(c, s, ik, b);
                for (int p = 0; p < npw; p++) h[p] += prod * pk_[p];
            }
        }
        free(phij); free(phiqj); free(Hsub); free(temp); free(V2);
        for (int d = 0; d < 3; d++) { free(gphij[d]); free(pgp[d]); free(duk[d]); }
    }
    for (int sa = 0; sa < nsa; sa++) free(gradq[sa]);
    free(gradq);
}

/* ======================================================================
 * local three-body potentials: tc3a1 (calc_hamiltonian_tc3a1.cpp:8-117)
 * and tc3b1 (calc_hamiltonian_tc3b1.cpp:8-135)
 * ====================================================================== */
static const cplx *dens(const octx *c, int s) { return (const cplx *)c->st->density + (size_t)s * c->N; }

/* dnu[d](r) = IFFT[ sum_{s3} u(G; s, s3) G_d n_s3(G) ] */
static void make_dnu(const octx *c, int s, cplx *dnu[3])
{
    const int N = c->N;
    cplx *orb = gnew(c);
    for (int d = 0; d < 3; d++) memset(dnu[d], 0, sizeof(cplx) * N);
    for (int js = 0; js < 2; js++) {
        memcpy(orb, dens(c, js), sizeof(cplx) * N);
        fft3_exec(&c->F, orb, 1);
        for (int i = 0; i < N; i++) {
            double u = tco_uk(c->sys, c->Gv[i], s, js);
            for (int d = 0; d < 3; d++) dnu[d][i] += u * c->Gv[i][d] * orb[i];
        }
    }
    for (int d = 0; d < 3; d++) fft3_exec(&c->F, dnu[d], 0);
    free(orb);
}

static void apply_local(const octx *c, const packing *P, const task *T, int nt, const cplx *psi,
                        cplx *h3, cplx *const *V, double factor)
{
#pragma omp parallel for schedule(dynamic, 1) num_threads(tco_get_threads())
    for (int t = 0; t < nt; t++) {
        const int s = T[t].s, ik = T[t].ik, j = T[t].j;
        cplx *o = gnew(c);
        scatter(c, s, a0(c, ik), psi + pk(P, c, s, ik, j), o);
        fft3_exec(&c->F, o, 0);
        for (int i = 0; i < c->N; i++) o[i] *= V[s][i];
        fft3_exec(&c->F, o, 1);
        gather_add(c, s, ik, o, factor, h3 + pk(P, c, s, ik, j));
        free(o);
    }
}

static void run_tc3a1(const octx *c, const packing *P, const task *T, int nt, const cplx *psi, cplx *h3)
{
    const double Nk = c->sys->num_kpoints, Om = c->sys->omega;
    const double f = 0.5 / (Nk * Nk * Om * Om);
    cplx *V[2] = {0, 0};
    for (int s = 0; s < c->nspin; s++) {
        cplx *dnu[3];
        for (int d = 0; d < 3; d++) dnu[d] = gnew(c);
        make_dnu(c, s, dnu);
        V[s] = gnew(c);
        for (int d = 0; d < 3; d++)
            for (int i = 0; i < c->N; i++) V[s][i] += dnu[d][i] * dnu[d][i];
        for (int d = 0; d < 3; d++) free(dnu[d]);
    }
    apply_local(c, P, T, nt, psi, h3, V, f);
    for (int s = 0; s < c->nspin; s++) free(V[s]);
}

static void run_tc3b1(const octx *c, const packing *P, const task *T, int nt, const cplx *psi, cplx *h3)
{
    const double Nk = c->sys->num_kpoints, Om = c->sys->omega;
    const double f = -1.0 / (Nk * Nk * Om * Om);
    const int N = c->N;
    cplx *dnu[2][3] = {{0}};
    for (int s2 = 0; s2 < c->nspin; s2++) {
        for (int d = 0; d < 3; d++) dnu[s2][d] = gnew(c);
        make_dnu(c, s2, dnu[s2]);
        for (int d = 0; d < 3; d++) {
            const cplx *n2 = dens(c, s2);
            for (int i = 0; i < N; i++) dnu[s2][d][i] *= n2[i];
            fft3_exec(&c->F, dnu[s2][d], 1);
        }
    }
    cplx *V[2] = {0, 0};
    for (int s1 = 0; s1 < c->nspin; s1++) {
        V[s1] = gnew(c);
        for (int s2 = 0; s2 < 2; s2++) {
            int s2r = c->nspin == 1 ? 0 : s2;
            for (int i = 0; i < N; i++) {
                double u = tco_uk(c->sys, c->Gv[i], s1, s2);
                for (int d = 0; d < 3; d++) V[s1][i] += u * c->Gv[i][d] * dnu[s2r][d][i];
            }
        }
        fft3_exec(&c->F, V[s1], 0);
    }
    apply_local(c, P, T, nt, psi, h3, V, f);
    for (int s = 0; s < c->nspin; s++) {
        free(V[s]);
        for (int d = 0; d < 3; d++) free(dnu[s][d]);
    }
}

/* ======================================================================
 * Hartree-type two-body terms: hf2h (calc_hamiltonian_hf2h.cpp:7-85) and
 * tc2h (calc_hamiltonian_tc2h.cpp:10-235)
 * ====================================================================== */
static void run_hf2h(const octx *c, const packing *P, const task *T, int nt, const cplx *psi, cplx *h2)
{
    const double f = 1.0 / (c->sys->num_kpoints * c->sys->omega);   /* :32 */
    cplx *V = gnew(c);
    for (int i = 0; i < c->N; i++) V[i] = dens(c, 0)[i] + dens(c, 1)[i];   /* :40 */
    fft3_exec(&c->F, V, 1);
    V[0] = 0.0;                                                               /* :42 */
    for (int i = 1; i < c->N; i++) {
        const double *G = c->Gv[i];
        V[i] *= FOURPI / (G[0] * G[0] + G[1] * G[1] + G[2] * G[2]);
    }
    fft3_exec(&c->F, V, 0);
    cplx *Vs[2] = {V, V};
    apply_local(c, P, T, nt, psi, h2, Vs, f);                                /* :64-80 */
    free(V);
}

static void run_tc2h(const octx *c, const packing *P, const task *T, int nt, const cplx *psi, cplx *h2)
{
    const int N = c->N, ns = c->nspin;
    const double f = 1.0 / (c->sys->num_kpoints * c->sys->omega);         /* :28 */
    /* [2b_h2] phiq_gphiq[s][d] = sum_q f conj(chi_q(r)) grad_d phi_q(r), to G (:53-140) */
    cplx *pg[2][3] = {{0}};
    cplx *orb = gnew(c), *gr = gnew(c);
    for (int s = 0; s < ns; s++) {
        for (int d = 0; d < 3; d++) pg[s][d] = gnew(c);
        for (int a = 0; a < c->nk_all; a++) {
            const int ik = c->ik_of_all[a];
            double q[3];
            cart(c->sys, c->sys->kvec + 3 * a, q);
            for (int i = 0; i < nocc(c, s, ik); i++) {
                const double fq = fill(c, s, ik, i);
                scatter(c, s, a, phik_band(c, s, ik, i), orb);
                const cplx *chr = Rchi(c, s, a, i);
                for (int d = 0; d < 3; d++) {
                    for (int p = 0; p < N; p++) gr[p] = (q[d] + c->Gv[p][d]) * orb[p];
                    fft3_exec(&c->F, gr, 0);
                    for (int p = 0; p < N; p++) pg[s][d][p] += fq * conj(chr[p]) * gr[p];
                }
            }
        }
        for (int d = 0; d < 3; d++) fft3_exec(&c->F, pg[s][d], 1);
    }
    /* [2a_h + 2b_h2] V_2body[s], [2b_h1] dnu[s][d] (:142-186) */
    cplx *V[2] = {0, 0}, *dn[2][3] = {{0}};
    const double spin_factor = ns == 1 ? 2.0 : 1.0;
    for (int s = 0; s < ns; s++) {
        V[s] = gnew(c);
        for (int d = 0; d < 3; d++) dn[s][d] = gnew(c);
        for (int js = 0; js < 2; js++) {
            const int jr = ns == 1 ? 0 : js;
            memcpy(orb, dens(c, js), sizeof(cplx) * N);
            fft3_exec(&c->F, orb, 1);
            for (int p = 0; p < N; p++) {
                const double *G = c->Gv[p];
                V[s][p] += tco_tc2body(c->sys, G, s, js) * orb[p];
                const double u = tco_uk(c->sys, G, s, js);
                for (int d = 0; d < 3; d++) {
                    V[s][p] += u * G[d] * pg[jr][d][p] / spin_factor;
                    dn[s][d][p] += u * G[d] * orb[p];
                }
            }
        }
        fft3_exec(&c->F, V[s], 0);
        for (int d = 0; d < 3; d++) fft3_exec(&c->F, dn[s][d], 0);
    }
    free(orb);
    free(gr);
    /* per band: V_2body phi - sum_d grad_d phi dnu_d (:188-233) */
#pragma omp parallel for schedule(dynamic, 1) num_threads(tco_get_threads())
    for (int t = 0; t < nt; t++) {
        const int s = T[t].s, ik = T[t].ik, j = T[t].j;
        double k[3];
        cart(c->sys, c->sys->kvec + 3 * a0(c, ik), k);
        cplx *o = gnew(c), *g = gnew(c), *vo = gnew(c);
        scatter(c, s, a0(c, ik), psi + pk(P, c, s, ik, j), o);
        for (int d = 0; d < 3; d++) {
            for (int p = 0; p < N; p++) g[p] = (k[d] + c->Gv[p][d]) * o[p];
            fft3_exec(&c->F, g, 0);
            for (int p = 0; p < N; p++) vo[p] -= g[p] * dn[s][d][p];
        }
        fft3_exec(&c->F, o, 0);
        for (int p = 0; p < N; p++) vo[p] += V[s][p] * o[p];
        fft3_exec(&c->F, vo, 1);
        gather_add(c, s, ik, vo, f, h2 + pk(P, c, s, ik, j));
        free(o); free(g); free(vo);
    }
    for (int s = 0; s < ns; s++) {
        free(V[s]);
        for (int d = 0; d < 3; d++) { free(dn[s][d]); free(pg[s][d]); }
    }
}

/* ======================================================================
 * one-body terms: kinetic (calc_hamiltonian_kinetic.cpp:6-52) and
 * pseudopotential (calc_hamiltonian_pseudo.cpp:6-180)
 * ====================================================================== */
static void run_kinetic(const octx *c, const packing *P, const task *T, int nt, const cplx *psi, cplx *h1)
{
    for (int t = 0; t < nt; t++) {
        const int s = T[t].s, ik = T[t].ik, j = T[t].j;
        double k[3];
        cart(c->sys, c->sys->kvec + 3 * a0(c, ik), k);
        const int32_t *gi = c->sys->gindex + gidx_offset(c, s, a0(c, ik));
        const cplx *ps = psi + pk(P, c, s, ik, j);
        cplx *h = h1 + pk(P, c, s, ik, j);
        for (int p = 0; p < c->sys->npw[ik]; p++) {
            double kg2 = 0;
            for (int d = 0; d < 3; d++) kg2 += (k[d] + c->Gv[gi[p]][d]) * (k[d] + c->Gv[gi[p]][d]);
            h[p] += 0.5 * kg2 * ps[p];                                  /* :38-41 */
        }
    }
}

static int run_pseudo(const octx *c, const tcg_pseudo_desc *pp, const packing *P, const task *T, int nt,
                      const cplx *psi, cplx *h1)
{
    /* component offsets (species, projector) -> first m, and per-k offsets */
    for (int is = 0; is < pp->nspecies; is++)
        if (pp->nproj[is] > 64) return fail(TCG_ERR_UNSUPPORTED, "more than 64 projectors per species");
    int ncomp = 0, *coff = malloc(sizeof(int) * 64 * (pp->nspecies > 0 ? pp->nspecies : 1));
    int *poff = malloc(sizeof(int) * (pp->nspecies + 1)), *doff = malloc(sizeof(int) * (pp->nspecies + 1));
    poff[0] = doff[0] = 0;
    for (int is = 0; is < pp->nspecies; is++) {
        poff[is + 1] = poff[is] + pp->nproj[is];
        doff[is + 1] = doff[is] + pp->nproj[is] * pp->nproj[is];
        for (int ip = 0; ip < pp->nproj[is]; ip++) {
            coff[64 * is + ip] = ncomp;
            ncomp += 2 * pp->lbeta[poff[is] + ip] + 1;
        }
    }
    size_t *koff = malloc(sizeof(size_t) * (c->nk + 1));
    koff[0] = 0;
    for (int k = 0; k < c->nk; k++) koff[k + 1] = koff[k] + (size_t)ncomp * c->sys->npw[k];
    int bad = 0;
    for (int t = 0; t < nt && !bad; t++) {
        const int s = T[t].s, ik = T[t].ik, j = T[t].j;
        const int npw = c->sys->npw[ik];
        const int32_t *gi = c->sys->gindex + gidx_offset(c, s, a0(c, ik));
        const cplx *ps = psi + pk(P, c, s, ik, j);
        cplx *h = h1 + pk(P, c, s, ik, j);
        const cplx *proj = (const cplx *)pp->projector + koff[ik];
        cplx *ph = malloc(sizeof(cplx) * npw);
        /* (1/2) non-local part (:120-160) */
        for (int ia = 0; ia < pp->natoms && !bad; ia++) {
            const int is = pp->species_of_atom[ia];
            const double *R = pp->atom_pos + 3 * ia;
            for (int p = 0; p < npw; p++) {
                const double *G = c->Gv[gi[p]];   /* G without k (:130-134) */
                const double arg = G[0] * R[0] + G[1] * R[1] + G[2] * R[2];
                ph[p] = cos(arg) + I * sin(arg);
            }
            for (int jp = 0; jp < pp->nproj[is]; jp++) {
                const int lb = pp->lbeta[poff[is] + jp];
                for (int im = 0; im < 2 * lb + 1; im++) {
                    const cplx *pj = proj + (size_t)(coff[64 * is + jp] + im) * npw;
                    cplx coeff = 0;
                    for (int p = 0; p < npw; p++) coeff += ph[p] * pj[p] * ps[p];
                    for (int ip = 0; ip < pp->nproj[is]; ip++) {
                        const double D = pp->dij[doff[is] + ip * pp->nproj[is] + jp];
                        if (fabs(D) > 1e-8) {
                            if (pp->lbeta[poff[is] + ip] != lb) { bad = 1; break; }
                            const cplx *pi = proj + (size_t)(coff[64 * is + ip] + im) * npw;
                            for (int p = 0; p < npw; p++) h[p] += D * coeff * conj(ph[p] * pi[p]);
                        }
                    }
                }
            }
        }
        free(ph);
        /* (2/2) local part (:163-175) */
        if (pp->vloc && !bad) {
            cplx *o = gnew(c);
            scatter(c, s, a0(c, ik), ps, o);
            fft3_exec(&c->F, o, 0);
            for (int p = 0; p < c->N; p++) o[p] *= pp->vloc[p];
            fft3_exec(&c->F, o, 1);
            gather_add(c, s, ik, o, 1.0, h);
            free(o);
        }
    }
    free(coff); free(poff); free(doff); free(koff);
    return bad ? fail(TCG_ERR_ARG, "dij is not diagonal w.r.t. l in pseudopot.") : TCG_OK;
}

/* ======================================================================
 * tc3a3b3b4b6 -- calc_hamiltonian_tc3a3b3b4b6.cpp:11-863 (kVaux = 0)
 * ====================================================================== */
static int kpoint_on_mesh(const octx *c, int ik)
{
    /* calc_hamiltonian_tc3a3b3b4b6.cpp:396-410 (all weights non-zero) */
    const double *kr = c->sys->kvec + 3 * a0(c, ik);
    for (int a = 0; a < c->nk_all; a++) {
        double kq[3];
        for (int d = 0; d < 3; d++) {
            kq[d] = kr[d] - c->sys->kvec[3 * a + d];
            while (kq[d] < -1e-8) kq[d] += 1.0;
            while (kq[d] > 1.0 - 1e-8) kq[d] -= 1.0;
        }
        if (kq[0] * kq[0] + kq[1] * kq[1] + kq[2] * kq[2] < 1e-8) return 1;
    }
    return 0;
}

static void run_tc3a3b3b4b6(const octx *c, const packing *P, const task *T, int nt, const cplx *psi, cplx *h3)
{
    const double Nk = c->sys->num_kpoints, Om = c->sys->omega;
    const double base = 1.0 / (Nk * Nk * Om * Om);
    double a3 = -base, b3 = base, b4 = -base, b6 = base;
    if (c->nspin == 1) { a3 /= 2.0; b3 /= 2.0; b4 /= 4.0; b6 /= 2.0; }
    const int N = c->N;
    const int do_div = c->sys->includes_div_correction && !jastrow_A_zero(c->sys);
    double *AuG[2] = {0, 0};
    if (do_div)
        for (int js = 0; js < 2; js++) {
            AuG[js] = calloc(N, sizeof(double));
            for (int i = 1; i < N; i++) AuG[js][i] = tco_uk(c->sys, c->Gv[i], 0, js);
            for (int i = 0; i < N; i++) AuG[js][i] = AuG[js][i] * c->sys->jastrow_A[0 * 2 + js];
        }
    cplx *dnu_s[2][3] = {{0}};
    for (int s = 0; s < c->nspin; s++) {
        for (int d = 0; d < 3; d++) dnu_s[s][d] = gnew(c);
        make_dnu(c, s, dnu_s[s]);
    }
    cplx *nG[2];
    for (int js = 0; js < 2; js++) {
        nG[js] = gnew(c);
        memcpy(nG[js], dens(c, js), sizeof(cplx) * N);
        fft3_exec(&c->F, nG[js], 1);
    }

#pragma omp parallel for schedule(dynamic, 1) num_threads(tco_get_threads())
    for (int t = 0; t < nt; t++) {
        const int s = T[t].s, ik = T[t].ik, j = T[t].j;
        cplx *const *dnu = dnu_s[s];
        cplx *phij = gnew(c), *Hsub = gnew(c), *phiphi = gnew(c), *orb = gnew(c), *orb2 = gnew(c);
        cplx *dnu_phi[3], *qsum[3];
        double *du[2][3];
        for (int d = 0; d < 3; d++) {
            dnu_phi[d] = gnew(c); qsum[d] = gnew(c);
            du[0][d] = malloc(sizeof(double) * N); du[1][d] = malloc(sizeof(double) * N);
        }
        const cplx *psij = psi + pk(P, c, s, ik, j);
        cplx *h = h3 + pk(P, c, s, ik, j);
        double kvect[3];
        cart(c->sys, c->sys->kvec + 3 * a0(c, ik), kvect);
        scatter(c, s, a0(c, ik), psij, phij);
        fft3_exec(&c->F, phij, 0);
        for (int d = 0; d < 3; d++)
            for (int i = 0; i < N; i++) dnu_phi[d][i] = dnu[d][i] * phij[i];

        /* first q loop: 3b3, 3b6, qsum for 3a3 / 3b4 (:192-368) */
        for (int a = 0; a < c->nk_all; a++) {
            const int iq = c->ik_of_all[a];
            if (nocc(c, s, iq) == 0 || QSKIP(a)) continue;
            double qv[3], kq[3];
            cart(c->sys, c->sys->kvec + 3 * a, qv);
            for (int d = 0; d < 3; d++) kq[d] = kvect[d] - qv[d];
            for (int i = 0; i < N; i++) {
                double G[3] = {kq[0] + c->Gv[i][0], kq[1] + c->Gv[i][1], kq[2] + c->Gv[i][2]};
                double uk0 = tco_uk(c->sys, G, 0, s), uk1 = tco_uk(c->sys, G, 1, s);
                for (int d = 0; d < 3; d++) { du[0][d][i] = G[d] * uk0; du[1][d][i] = G[d] * uk1; }
            }
            for (int ib = 0; ib < nocc(c, s, iq); ib++) {
                const cplx *phiq = Rphi(c, s, a, ib), *chiq = Rchi(c, s, a, ib);
                for (int i = 0; i < N; i++) phiphi[i] = conj(chiq[i]) * phij[i];
                fft3_exec(&c->F, phiphi, 1);
                memset(orb2, 0, sizeof(cplx) * N);
                for (int d = 0; d < 3; d++) {
                    for (int i = 0; i < N; i++) orb[i] = dnu_phi[d][i] * conj(chiq[i]);
                    fft3_exec(&c->F, orb, 1);
                    for (int i = 0; i < N; i++) orb2[i] += du[s][d][i] * orb[i];
                }
                fft3_exec(&c->F, orb2, 0);
                const double filq = fill(c, s, iq, ib);
                for (int i = 0; i < N; i++) Hsub[i] += (filq * b3) * orb2[i] * phiq[i];
                for (int i = 0; i < N; i++) phiphi[i] *= filq;
                memset(orb2, 0, sizeof(cplx) * N);
                for (int s2 = 0; s2 < 2; s2++)
                    for (int d = 0; d < 3; d++) {
                        for (int i = 0; i < N; i++) orb[i] = phiphi[i] * du[s2][d][i];
                        fft3_exec(&c->F, orb, 0);
                        if (s2 == s)
                            for (int i = 0; i < N; i++) qsum[d][i] += orb[i] * phiq[i];
                        const cplx *n2 = dens(c, s2);
                        for (int i = 0; i < N; i++) orb[i] *= n2[i];
                        fft3_exec(&c->F, orb, 1);
                        for (int i = 0; i < N; i++) orb2[i] += orb[i] * du[s2][d][i];
                    }
                fft3_exec(&c->F, orb2, 0);
                for (int i = 0; i < N; i++) Hsub[i] += b6 * orb2[i] * phiq[i];
            }
        }
        fft3_exec(&c->F, Hsub, 1);
        gather_add(c, s, ik, Hsub, 1.0, h);

        /* 3b6 divergence correction (:394-535), if_match branch */
        if (do_div) {
            const int if_match = kpoint_on_mesh(c, ik);
            const double dcorr = 1.0 / sqrt(PI * c->sys->alpha_Vaux) * Nk * Om - c->sys->sum_Vaux[ik];
            cplx t1 = 0;
            cplx *tG = gnew(c), *tR = gnew(c);
            for (int js = 0; js < 2; js++) {
                double Adc = dcorr * c->sys->jastrow_A[s * 2 + js];
                const double zero[3] = {0, 0, 0};
                if (if_match) Adc += tco_uk(c->sys, zero, s, js);
                t1 += FOURPI * Adc * c->sys->jastrow_A[s * 2 + js] * nG[js][0];
                const int sj = s == js ? 0 : 1;
                if (if_match)
                    for (int i = 0; i < N; i++) tG[i] += FOURPI * nG[js][i] * AuG[sj][i];
            }
            memcpy(tR, tG, sizeof(cplx) * N);
            fft3_exec(&c->F, tR, 0);
            memset(Hsub, 0, sizeof(cplx) * N);
            const int npw = c->sys->npw[ik];
            for (int b = 0; b < c->st->nbands[s]; b++) {
                const double fb = fill(c, s, ik, b);
                if (fb < 1e-8) continue;
                const cplx *pkr = phik_band(c, s, ik, b);
                cplx *phiq = orb, *chiq = orb2;
                scatter(c, s, a0(c, ik), pkr, phiq);
                fft3_exec(&c->F, phiq, 0);
                if (c->is_bitc) {
                    scatter(c, s, a0(c, ik), chik_band(c, s, ik, b), chiq);
                    fft3_exec(&c->F, chiq, 0);
                }
                const cplx *chir = c->is_bitc ? chiq : phiq;
                for (int i = 0; i < N; i++) phiphi[i] = chir[i] * conj(phij[i]);
                fft3_exec(&c->F, phiphi, 1);
                const cplx cpi = conj(phiphi[0]);
                cplx add = fb * b6 * t1 * cpi;
                for (int p = 0; p < npw; p++) h[p] += add * pkr[p];
                const int sign = if_match ? 1 : -1;
                add = sign * fb * b6 * dotc(phiphi, tG, N);
                for (int p = 0; p < npw; p++) h[p] += add * pkr[p];
                const cplx cf = fb * cpi * b6;
                for (int i = 0; i < N; i++) Hsub[i] += cf * tR[i] * phiq[i];
            }
            fft3_exec(&c->F, Hsub, 1);
            gather_add(c, s, ik, Hsub, 1.0, h);
            free(tG); free(tR);
        }

        /* 3a3 (:629-642) */
        memset(orb, 0, sizeof(cplx) * N);
        for (int d = 0; d < 3; d++)
            for (int i = 0; i < N; i++) orb[i] += qsum[d][i] * dnu[d][i];
        fft3_exec(&c->F, orb, 1);
        gather_add(c, s, ik, orb, a3, h);

        /* second q loop: 3b4 (:664-767) */
        memset(Hsub, 0, sizeof(cplx) * N);
        for (int a = 0; a < c->nk_all; a++) {
            const int iq = c->ik_of_all[a];
            if (nocc(c, s, iq) == 0 || QSKIP(a)) continue;
            double qv[3], kq[3];
            cart(c->sys, c->sys->kvec + 3 * a, qv);
            for (int d = 0; d < 3; d++) kq[d] = kvect[d] - qv[d];
            for (int i = 0; i < N; i++) {
                double G[3] = {kq[0] + c->Gv[i][0], kq[1] + c->Gv[i][1], kq[2] + c->Gv[i][2]};
                double u = tco_uk(c->sys, G, s, s);
                for (int d = 0; d < 3; d++) du[0][d][i] = G[d] * u;
            }
            for (int ib = 0; ib < nocc(c, s, iq); ib++) {
                const cplx *phiq = Rphi(c, s, a, ib), *chiq = Rchi(c, s, a, ib);
                memset(phiphi, 0, sizeof(cplx) * N);
                for (int d = 0; d < 3; d++) {
                    for (int i = 0; i < N; i++) orb[i] = conj(chiq[i]) * qsum[d][i];
                    fft3_exec(&c->F, orb, 1);
                    for (int i = 0; i < N; i++) phiphi[i] += orb[i] * du[0][d][i];
                }
                fft3_exec(&c->F, phiphi, 0);
                const double filq = fill(c, s, iq, ib);
                for (int i = 0; i < N; i++) Hsub[i] += filq * phiphi[i] * phiq[i];
            }
        }
        fft3_exec(&c->F, Hsub, 1);
        gather_add(c, s, ik, Hsub, b4, h);

        free(phij); free(Hsub); free(phiphi); free(orb); free(orb2);
        for (int d = 0; d < 3; d++) { free(dnu_phi[d]); free(qsum[d]); free(du[0][d]); free(du[1][d]); }
    }
    for (int s = 0; s < c->nspin; s++)
        for (int d = 0; d < 3; d++) free(dnu_s[s][d]);
    for (int js = 0; js < 2; js++) { free(nG[js]); free(AuG[js]); }
}

/* ======================================================================
 * tc3a2a4b2b5 -- calc_hamiltonian_tc3a2a4b2b5.cpp:11-1300 (kVaux = 0)
 * ====================================================================== */

/* symmetry transformation of a G-space grid (iq2, 0) -> (iq2, isymq2)
 * (:576-644, :668-764): out[ipw_trans] (+)= phase * (M x)(ipw) or its
 * time-reversed (conjugated, negated) form.  ncomp = 1 (scalar, M unused)
 * or 3 (vector, M = U^+ in Cartesian). */
static void sym_rotate(const octx *c, int a, const double M[9], int ncomp, cplx *const *in, cplx *const *out)
{
    const int ind = c->sys->rot_index[a];
    const int32_t *U = c->sys->rotation + 9 * ind;
    const double *tr = c->sys->translation + 3 * ind;
    const int tr_used = c->sys->time_rev[a];
    const int nr[3] = {c->n0, c->n1, c->n2};
    for (int k = 0; k < ncomp; k++) memset(out[k], 0, sizeof(cplx) * c->N);
    for (int ipw = 0; ipw < c->N; ipw++) {
        const int *Gv = c->Gm[ipw];
        int Gt[3];
        for (int i = 0; i < 3; i++) {
            Gt[i] = U[0 * 3 + i] * Gv[0] + U[1 * 3 + i] * Gv[1] + U[2 * 3 + i] * Gv[2]; /* U^T G */
            if (tr_used) Gt[i] = -Gt[i];
            while (Gt[i] < 0) Gt[i] += nr[i];
            while (Gt[i] >= nr[i]) Gt[i] -= nr[i];
        }
        const double arg = 2 * PI * (tr[0] * Gt[0] + tr[1] * Gt[1] + tr[2] * Gt[2]);
        const cplx phase = cos(arg) + I * sin(arg);
        const int it = Gt[0] + Gt[1] * nr[0] + Gt[2] * nr[0] * nr[1];
        if (ncomp == 1) {
            if (tr_used) out[0][it] += phase * conj(in[0][ipw]);
            else out[0][it] += phase * in[0][ipw];
        } else {
            for (int d = 0; d < 3; d++) {
                if (tr_used)
                    out[d][it] -= phase * (M[d * 3 + 0] * conj(in[0][ipw]) + M[d * 3 + 1] * conj(in[1][ipw])
                                           + M[d * 3 + 2] * conj(in[2][ipw]));
                else
                    out[d][it] += phase * (M[d * 3 + 0] * in[0][ipw] + M[d * 3 + 1] * in[1][ipw]
                                           + M[d * 3 + 2] * in[2][ipw]);
            }
        }
    }
}

/* Udag_cart = recip^T * U^T * lattice / (2 pi)  (:688-690) */
static void udag_cart(const octx *c, int a, double M[9])
{
    const int32_t *U = c->sys->rotation + 9 * c->sys->rot_index[a];
    double T1[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double acc = 0;
            for (int k = 0; k < 3; k++) acc += c->sys->recip[k * 3 + i] * (double)U[j * 3 + k]; /* R^T[i][k] * Udag[k][j] */
            T1[i * 3 + j] = acc;
        }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double acc = 0;
            for (int k = 0; k < 3; k++) acc += T1[i * 3 + k] * c->sys->lattice[k * 3 + j];
            M[i * 3 + j] = acc / (2 * PI);
        }
}

static void run_tc3a2a4b2b5(const octx *c, const packing *P, const task *T, int nt, const cplx *psi, cplx *h3)
{
    const double Nk = c->sys->num_kpoints, Om = c->sys->omega;
    const double base = 1.0 / (Nk * Nk * Om * Om);
    double fa2 = -0.5 * base, fa4 = base, fb2 = base, fb5 = -base;
    if (c->nspin == 1) { fa2 /= 4.0; fa4 /= 4.0; fb2 /= 4.0; fb5 /= 4.0; }
    const int N = c->N, ns = c->nspin, bitc = c->is_bitc;
    const int do_div = c->sys->includes_div_correction && !jastrow_A_zero(c->sys);
    const int nthr = tco_get_threads();

    double *uG[2][2] = {{0}};
    for (int s1 = 0; s1 < ns; s1++)
        for (int s2 = 0; s2 < 2; s2++) {
            uG[s1][s2] = malloc(sizeof(double) * N);
            for (int i = 0; i < N; i++) uG[s1][s2][i] = tco_uk(c->sys, c->Gv[i], s1, s2);
        }
    cplx *V3a2[2] = {0, 0};
    for (int s = 0; s < ns; s++) V3a2[s] = gnew(c);

    for (int sq = 0; sq < ns; sq++) {
        cplx *qsum3b2[3];
        for (int d = 0; d < 3; d++) qsum3b2[d] = gnew(c);
        for (int iq2 = 0; iq2 < c->nk; iq2++) {
            const int no2 = nocc(c, sq, iq2);
            if (no2 == 0 || QSKIP(iq2)) continue;
            const double t_sh0 = now_s();
            double q2v[3];
            cart(c->sys, c->sys->kvec + 3 * a0(c, iq2), q2v);
            /* occupied-pair stage (:210-443): accumulators per (i2, part) */
            /* the visited source k-points (all of them, or every qstride-th in the
             * timing-sample mode), split evenly over the parts */
            int *alist = malloc(sizeof(int) * c->nk_all), nal = 0;
            for (int a1 = 0; a1 < c->nk_all; a1++)
                if (nocc(c, sq, c->ik_of_all[a1]) > 0 && !QSKIP(a1)) alist[nal++] = a1;
            const int nparts = nal == 0 ? 1 : (nthr < nal ? nthr : nal);
            const int nacc = ns + 3 + (bitc ? 3 : 0);
            cplx *acc = calloc((size_t)no2 * nparts * nacc * N, sizeof(cplx));
            if (!acc) { free(alist); return; }
#pragma omp parallel for collapse(2) schedule(dynamic, 1) num_threads(nthr)
            for (int i2 = 0; i2 < no2; i2++)
                for (int part = 0; part < nparts; part++) {
                    cplx *A = acc + ((size_t)i2 * nparts + part) * nacc * N;
                    cplx *q3a2[2] = {A, ns > 1 ? A + N : A};
                    cplx *q3a4 = A + (size_t)ns * N, *q3b5 = A + (size_t)(ns + 3) * N;
                    const int abeg = (int)((long)nal * part / nparts);
                    const int aend = (int)((long)nal * (part + 1) / nparts);
                    const cplx *phiq2 = Rphi(c, sq, a0(c, iq2), i2), *chiq2 = Rchi(c, sq, a0(c, iq2), i2);
                    cplx *phiphi = gnew(c), *phij = gnew(c), *orb = gnew(c), *orb2 = gnew(c);
                    double *du[2][3];
                    for (int x = 0; x < 2; x++)
                        for (int d = 0; d < 3; d++) du[x][d] = malloc(sizeof(double) * N);
                    for (int ia = abeg; ia < aend; ia++) {
                        const int a1 = alist[ia];
                        const int iq1 = c->ik_of_all[a1];
                        double q1v[3], qq[3];
                        cart(c->sys, c->sys->kvec + 3 * a1, q1v);
                        for (int d = 0; d < 3; d++) qq[d] = q2v[d] - q1v[d];
                        for (int i = 0; i < N; i++) {
                            double G[3] = {qq[0] + c->Gv[i][0], qq[1] + c->Gv[i][1], qq[2] + c->Gv[i][2]};
                            double uk0 = tco_uk(c->sys, G, sq, 0), uk1 = tco_uk(c->sys, G, sq, 1);
                            for (int d = 0; d < 3; d++) { du[0][d][i] = G[d] * uk0; du[1][d][i] = G[d] * uk1; }
                        }
                        for (int i1 = 0; i1 < nocc(c, sq, iq1); i1++) {
                            const cplx *phiq1 = Rphi(c, sq, a1, i1), *chiq1 = Rchi(c, sq, a1, i1);
                            for (int i = 0; i < N; i++) phiphi[i] = conj(chiq1[i]) * phiq2[i];
                            fft3_exec(&c->F, phiphi, 1);
                            if (bitc) {
                                for (int i = 0; i < N; i++) phij[i] = conj(phiq1[i]) * chiq2[i];
                                fft3_exec(&c->F, phij, 1);
                            }
                            const double f1 = fill(c, sq, iq1, i1);
                            for (int x = 0; x < 2; x++) {
                                const int xr = ns == 1 ? 0 : x;
                                for (int d = 0; d < 3; d++) {
                                    for (int i = 0; i < N; i++) orb[i] = du[x][d][i] * phiphi[i];
                                    fft3_exec(&c->F, orb, 0);
                                    if (bitc) {
                                        for (int i = 0; i < N; i++) orb2[i] = du[x][d][i] * phij[i];
                                        fft3_exec(&c->F, orb2, 0);
                                        for (int i = 0; i < N; i++) q3a2[xr][i] -= f1 * orb[i] * conj(orb2[i]);
                                    } else {
                                        for (int i = 0; i < N; i++) {
                                            double re = creal(orb[i]), im = cimag(orb[i]);
                                            q3a2[xr][i] -= f1 * (re * re + im * im);
                                        }
                                    }
                                    if (x == sq) {
                                        cplx *o4 = q3a4 + (size_t)d * N;
                                        for (int i = 0; i < N; i++) o4[i] += f1 * orb[i] * phiq1[i];
                                        if (bitc) {
                                            cplx *o5 = q3b5 + (size_t)d * N;
                                            for (int i = 0; i < N; i++) o5[i] -= f1 * conj(orb2[i]) * conj(chiq1[i]);
                                        }
                                    }
                                }
                            }
                        }
                    }
                    free(phiphi); free(phij); free(orb); free(orb2);
                    for (int x = 0; x < 2; x++)
                        for (int d = 0; d < 3; d++) free(du[x][d]);
                }
            g_t_shared += now_s() - t_sh0;
            /* reduce parts in fixed order into part 0 */
            for (int i2 = 0; i2 < no2; i2++) {
                cplx *A0 = acc + ((size_t)i2 * nparts) * nacc * N;
                for (int part = 1; part < nparts; part++) {
                    const cplx *Ap = acc + ((size_t)i2 * nparts + part) * nacc * N;
                    for (size_t i = 0; i < (size_t)nacc * N; i++) A0[i] += Ap[i];
                }
            }

            for (int i2 = 0; i2 < no2; i2++) {
                cplx *A = acc + ((size_t)i2 * nparts) * nacc * N;
                const double f2 = fill(c, sq, iq2, i2);
                const cplx *phiq2 = Rphi(c, sq, a0(c, iq2), i2), *chiq2 = Rchi(c, sq, a0(c, iq2), i2);
                /* 3a2 (:487-644) */
                cplx *Tq[2] = {0, 0};
                for (int s = 0; s < ns; s++) {
                    Tq[s] = gnew(c);
                    memcpy(Tq[s], A + (size_t)s * N, sizeof(cplx) * N);
                    fft3_exec(&c->F, Tq[s], 1);
                }
                if (do_div) {
                    const double dcorr = 1.0 / sqrt(PI * c->sys->alpha_Vaux) * Nk * Om - c->sys->sum_Vaux[iq2];
                    cplx *phiphi = gnew(c), *phij = gnew(c);
                    for (int i1 = 0; i1 < no2; i1++) {
                        const cplx *phiq1 = Rphi(c, sq, a0(c, iq2), i1), *chiq1 = Rchi(c, sq, a0(c, iq2), i1);
                        for (int i = 0; i < N; i++) phiphi[i] = conj(chiq1[i]) * phiq2[i];
                        fft3_exec(&c->F, phiphi, 1);
                        for (int i = 0; i < N; i++) phij[i] = conj(chiq2[i]) * phiq1[i];
                        fft3_exec(&c->F, phij, 1);
                        const double f1 = fill(c, sq, iq2, i1);
                        for (int x = 0; x < 2; x++) {
                            const int xr = ns == 1 ? 0 : x;
                            const double Ax = c->sys->jastrow_A[sq * 2 + x];
                            const double zero[3] = {0, 0, 0};
                            Tq[xr][0] -= FOURPI * Ax * (Ax * dcorr + tco_uk(c->sys, zero, sq, x)) * f1 * phiphi[0] * phij[0];
                            const double ct = FOURPI * Ax * f1;
                            for (int i = 1; i < N; i++)
                                Tq[xr][i] -= ct * uG[sq][x][i] * (phiphi[i] * phij[0] + phiphi[0] * phij[i]);
                        }
                    }
                    free(phiphi); free(phij);
                }
                for (int isym = 0; isym < c->sys->nsym_k[iq2]; isym++) {
                    const int a2 = a0(c, iq2) + isym;
                    for (int s = 0; s < ns; s++) {
                        cplx *R = gnew(c);
                        sym_rotate(c, a2, NULL, 1, &Tq[s], &R);
                        for (int i = 0; i < N; i++) V3a2[s][i] += f2 * R[i];
                        free(R);
                    }
                }
                for (int s = 0; s < ns; s++) free(Tq[s]);

                /* 3a4, b2, b5 (:646-918) */
                cplx *Q[3], *B[3];
                for (int d = 0; d < 3; d++) {
                    Q[d] = gnew(c); B[d] = gnew(c);
                    memcpy(Q[d], A + (size_t)(ns + d) * N, sizeof(cplx) * N);
                    if (bitc) memcpy(B[d], A + (size_t)(ns + 3 + d) * N, sizeof(cplx) * N);
                    else for (int i = 0; i < N; i++) B[d][i] = -conj(Q[d][i]);
                    fft3_exec(&c->F, Q[d], 1);
                    fft3_exec(&c->F, B[d], 1);
                }
                for (int isym = 0; isym < c->sys->nsym_k[iq2]; isym++) {
                    const int a2 = a0(c, iq2) + isym;
                    double M[9];
                    udag_cart(c, a2, M);
                    cplx *Qt[3], *Bt[3];
                    for (int d = 0; d < 3; d++) { Qt[d] = gnew(c); Bt[d] = gnew(c); }
                    sym_rotate(c, a2, M, 3, Q, Qt);
                    sym_rotate(c, a2, M, 3, B, Bt);
                    for (int d = 0; d < 3; d++) { fft3_exec(&c->F, Qt[d], 0); fft3_exec(&c->F, Bt[d], 0); }
                    double q2s[3];
                    cart(c->sys, c->sys->kvec + 3 * a2, q2s);
                    cplx *phiq2s = gnew(c), *chiq2s = bitc ? gnew(c) : phiq2s;
                    scatter(c, sq, a2, phik_band(c, sq, iq2, i2), phiq2s);
                    fft3_exec(&c->F, phiq2s, 0);
                    if (bitc) {
                        scatter(c, sq, a2, chik_band(c, sq, iq2, i2), chiq2s);
                        fft3_exec(&c->F, chiq2s, 0);
                    }
                    for (int d = 0; d < 3; d++)
                        for (int i = 0; i < N; i++) qsum3b2[d][i] += f2 * Bt[d][i] * phiq2s[i];
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthr)
                    for (int t = 0; t < nt; t++) {
                        if (T[t].s != sq) continue;
                        const int ik = T[t].ik, j = T[t].j;
                        double kv[3], kq[3];
                        cart(c->sys, c->sys->kvec + 3 * a0(c, ik), kv);
                        for (int d = 0; d < 3; d++) kq[d] = kv[d] - q2s[d];
                        double *du0[3];
                        for (int d = 0; d < 3; d++) du0[d] = malloc(sizeof(double) * N);
                        for (int i = 0; i < N; i++) {
                            double G[3] = {kq[0] + c->Gv[i][0], kq[1] + c->Gv[i][1], kq[2] + c->Gv[i][2]};
                            double u = tco_uk(c->sys, G, sq, sq);
                            for (int d = 0; d < 3; d++) du0[d][i] = G[d] * u;
                        }
                        cplx *phij = gnew(c), *phiphi = gnew(c), *orb = gnew(c), *orb2 = gnew(c);
                        scatter(c, sq, a0(c, ik), psi + pk(P, c, sq, ik, j), phij);
                        fft3_exec(&c->F, phij, 0);
                        for (int i = 0; i < N; i++) phiphi[i] = conj(chiq2s[i]) * phij[i];
                        fft3_exec(&c->F, phiphi, 1);
                        for (int i = 0; i < N; i++) phiphi[i] *= f2 * fa4;
                        for (int d = 0; d < 3; d++) {
                            for (int i = 0; i < N; i++) orb[i] = phiphi[i] * du0[d][i];
                            fft3_exec(&c->F, orb, 0);
                            for (int i = 0; i < N; i++) orb2[i] += Qt[d][i] * orb[i];
                        }
                        memset(phiphi, 0, sizeof(cplx) * N);
                        for (int d = 0; d < 3; d++) {
                            for (int i = 0; i < N; i++) orb[i] = Bt[d][i] * phij[i];
                            fft3_exec(&c->F, orb, 1);
                            for (int i = 0; i < N; i++) phiphi[i] += orb[i] * du0[d][i];
                        }
                        fft3_exec(&c->F, phiphi, 0);
                        for (int i = 0; i < N; i++) orb2[i] += fb5 * f2 * phiphi[i] * phiq2s[i];
                        fft3_exec(&c->F, orb2, 1);
                        gather_add(c, sq, ik, orb2, 1.0, h3 + pk(P, c, sq, ik, j));
                        free(phij); free(phiphi); free(orb); free(orb2);
                        for (int d = 0; d < 3; d++) free(du0[d]);
                    }
                    for (int d = 0; d < 3; d++) { free(Qt[d]); free(Bt[d]); }
                    free(phiq2s);
                    if (bitc) free(chiq2s);
                }
                for (int d = 0; d < 3; d++) { free(Q[d]); free(B[d]); }
            }
            free(acc);
            free(alist);
        }
        /* 3b2 (:922-992) */
        for (int d = 0; d < 3; d++) fft3_exec(&c->F, qsum3b2[d], 1);
        for (int s = 0; s < ns; s++) {
            cplx *V = gnew(c);
            for (int i = 0; i < N; i++) {
                double u = ns == 1 ? uG[s][0][i] + uG[s][1][i] : uG[s][sq][i];
                for (int d = 0; d < 3; d++) V[i] += (c->Gv[i][d] * u) * qsum3b2[d][i];
            }
            fft3_exec(&c->F, V, 0);
            cplx *Vs[2] = {V, V};
            packing Ps = *P;
            /* apply to bands of spin s only */
            int mt = 0;
            task *Ts = malloc(sizeof(task) * (nt > 0 ? nt : 1));
            for (int t = 0; t < nt; t++)
                if (T[t].s == s) Ts[mt++] = T[t];
            apply_local(c, &Ps, Ts, mt, psi, h3, Vs, fb2);
            free(Ts);
            free(V);
        }
        for (int d = 0; d < 3; d++) free(qsum3b2[d]);
    }
    /* 3a2 (:995-1034) */
    for (int s = 0; s < ns; s++) fft3_exec(&c->F, V3a2[s], 0);
    apply_local(c, P, T, nt, psi, h3, V3a2, fa2);
    for (int s = 0; s < ns; s++) free(V3a2[s]);
    for (int s1 = 0; s1 < ns; s1++)
        for (int s2 = 0; s2 < 2; s2++) free(uG[s1][s2]);
}

/* ======================================================================
 * public entry points
 * ====================================================================== */
static int check_inputs(const tcg_system_desc *sys, const tcg_state_desc *st)
{
    if (!sys || !st) return fail(TCG_ERR_ARG, "null descriptor");
    if (!sys->nsym_k || !sys->kvec || !sys->npw || !sys->gindex || !sys->phase || !sys->time_rev)
        return fail(TCG_ERR_ARG, "missing k-point arrays");
    if (!st->nbands || !st->nocc || !st->filling || !st->phik || !st->density)
        return fail(TCG_ERR_ARG, "missing state arrays");
    if (sys->includes_div_correction && !sys->sum_Vaux) return fail(TCG_ERR_ARG, "missing sum_Vaux");
    return TCG_OK;
}

int tco_apply(const tcg_system_desc *sys, const tcg_state_desc *st, uint32_t mask, const int32_t *nb_apply,
              const double *psi, double *h2, double *h3, const uint8_t *owned)
{
    int rc = check_inputs(sys, st);
    if (rc) return rc;
    if (!nb_apply || !psi) return fail(TCG_ERR_ARG, "missing psi");
    const int is_hf = sys->calc_method == TCG_METHOD_HF;
    if (mask & ~(TCG_TERMS_TC | TCG_TERMS_H2)) return fail(TCG_ERR_ARG, "unknown term bits");
    if (is_hf && (mask & ~(TCG_TERM_HF2X | TCG_TERM_HF2H))) return fail(TCG_ERR_ARG, "TC terms requested for HF");
    if (!is_hf && (mask & (TCG_TERM_HF2X | TCG_TERM_HF2H))) return fail(TCG_ERR_ARG, "HF terms requested for TC/BITC");
    if ((mask & TCG_TERMS_H2) && !h2) return fail(TCG_ERR_ARG, "h2 is NULL");
    if ((mask & ~TCG_TERMS_H2) && !h3) return fail(TCG_ERR_ARG, "h3 is NULL");
    if (sys->nsymop > 0 && (!sys->rotation || !sys->translation || !sys->rot_index))
        return fail(TCG_ERR_ARG, "missing symmetry arrays");
    const double t0 = now_s();
    octx c;
    rc = ctx_init(&c, sys, st, 1);
    if (rc) { ctx_free(&c); return rc; }
    g_t_init += now_s() - t0;
    packing P;
    pack_init(&P, &c, nb_apply);
    task *T;
    int nt = make_tasks(&c, &P, owned, &T);
    const cplx *ps = (const cplx *)psi;
    if (mask & TCG_TERM_HF2X) run_hf2x(&c, &P, T, nt, ps, (cplx *)h2);
    if (mask & TCG_TERM_HF2H) run_hf2h(&c, &P, T, nt, ps, (cplx *)h2);
    if (mask & TCG_TERM_TC2H) run_tc2h(&c, &P, T, nt, ps, (cplx *)h2);
    if (mask & TCG_TERM_TC2X) run_tc2x(&c, &P, T, nt, ps, (cplx *)h2);
    if (mask & TCG_TERM_TC3A1) run_tc3a1(&c, &P, T, nt, ps, (cplx *)h3);
    if (mask & TCG_TERM_TC3B1) run_tc3b1(&c, &P, T, nt, ps, (cplx *)h3);
    if (mask & TCG_TERM_TC3A2A4B2B5) run_tc3a2a4b2b5(&c, &P, T, nt, ps, (cplx *)h3);
    if (mask & TCG_TERM_TC3A3B3B4B6) run_tc3a3b3b4b6(&c, &P, T, nt, ps, (cplx *)h3);
    free(T);
    free(P.off);
    ctx_free(&c);
    g_t_total += now_s() - t0;
    return TCG_OK;
}

int tco_apply_h1(const tcg_system_desc *sys, const tcg_pseudo_desc *pp, uint32_t mask, const int32_t *nb_apply,
                 const double *psi, double *h1, const uint8_t *owned)
{
    if (!sys || !nb_apply || !psi || !h1) return fail(TCG_ERR_ARG, "null argument");
    if (mask & ~TCG_TERMS_H1) return fail(TCG_ERR_ARG, "only one-body terms here");
    if ((mask & TCG_TERM_PSEUDO) && !pp) return fail(TCG_ERR_ARG, "pseudopotential data missing");
    octx c;
    int rc = ctx_init(&c, sys, NULL, 0);
    if (rc) { ctx_free(&c); return rc; }
    packing P;
    pack_init(&P, &c, nb_apply);
    task *T;
    int nt = make_tasks(&c, &P, owned, &T);
    const cplx *ps = (const cplx *)psi;
    if (mask & TCG_TERM_KINETIC) run_kinetic(&c, &P, T, nt, ps, (cplx *)h1);
    if (mask & TCG_TERM_PSEUDO) rc = run_pseudo(&c, pp, &P, T, nt, ps, (cplx *)h1);
    free(T);
    free(P.off);
    ctx_free(&c);
    return rc;
}

/* BlochStates::set_density (bloch_states_scfloop_filling_density.cpp:256-360) */
int tco_density(const tcg_system_desc *sys, const tcg_state_desc *st, double *out)
{
    int rc = check_inputs(sys, st);
    if (rc) return rc;
    octx c;
    rc = ctx_init(&c, sys, st, 0);
    if (rc) { ctx_free(&c); return rc; }
    const int N = c.N;
    cplx *dn = (cplx *)out;
    int bad = 0;
    for (int s = 0; s < c.nspin; s++) {
        cplx *tmp = dn + (size_t)s * N;
        memset(tmp, 0, sizeof(cplx) * N);
        cplx *orb = gnew(&c), *left = gnew(&c);
        for (int ik = 0; ik < c.nk; ik++)
            for (int isym = 0; isym < sys->nsym_k[ik]; isym++)
                for (int b = 0; b < nocc(&c, s, ik); b++) {
                    const int a = a0(&c, ik) + isym;
                    scatter(&c, s, a, phik_band(&c, s, ik, b), orb);
                    fft3_exec(&c.F, orb, 0);
                    if (c.is_bitc) {
                        scatter(&c, s, a, chik_band(&c, s, ik, b), left);
                        fft3_exec(&c.F, left, 0);
                        for (int i = 0; i < N; i++) left[i] = conj(left[i]) * orb[i];
                    } else {
                        for (int i = 0; i < N; i++) {
                            double re = creal(orb[i]), im = cimag(orb[i]);
                            left[i] = re * re + im * im;
                        }
                    }
                    cplx sum = 0;
                    for (int i = 0; i < N; i++) sum += left[i];
                    if (cabs(sum / (double)N - 1.0) > 1e-4) bad = 1;
                    const double f = fill(&c, s, ik, b);
                    for (int i = 0; i < N; i++) tmp[i] += f * left[i];
                }
        if (c.nspin == 1)
            for (int i = 0; i < N; i++) tmp[i] /= 2.0;
        free(orb); free(left);
    }
    if (c.nspin == 1) memcpy(dn + N, dn, sizeof(cplx) * N);
    ctx_free(&c);
    if (bad) return fail(TCG_ERR_NUMERIC, "normalization breaks");
    return TCG_OK;
}

/* Potentials::set_sum_of_Vaux_each (potentials_coulomb.cpp:60-161) */
int tco_sum_of_vaux(const tcg_system_desc *sys, double *alpha_out, double *sum_out)
{
    if (!sys || !alpha_out || !sum_out) return fail(TCG_ERR_ARG, "null argument");
    double alpha = cbrt(sys->omega) / (2.0 * PI);
    alpha = alpha * alpha;
    int nk_all = 0;
    for (int k = 0; k < sys->nk_irr; k++) nk_all += sys->nsym_k[k];
    int off = 0;
    for (int ik = 0; ik < sys->nk_irr; ik++) {
        const double *kr = sys->kvec + 3 * off;
        off += sys->nsym_k[ik];
        double total = 0.0;
        int if_match = 0;
        for (int a = 0; a < nk_all; a++) {
            double kq[3];
            for (int d = 0; d < 3; d++) {
                kq[d] = kr[d] - sys->kvec[3 * a + d];
                while (kq[d] < -1e-8) kq[d] += 1.0;
                while (kq[d] > 1.0 - 1e-8) kq[d] -= 1.0;
            }
            const int m = kq[0] * kq[0] + kq[1] * kq[1] + kq[2] * kq[2] < 1e-8;
            if (m) if_match = 1;
            if (!m) {
                double v[3];
                for (int d = 0; d < 3; d++)
                    v[d] = sys->recip[0 * 3 + d] * kq[0] + sys->recip[1 * 3 + d] * kq[1] + sys->recip[2 * 3 + d] * kq[2];
                double k2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
                total += exp(-alpha * k2) / k2;
            }
            for (int ns = 1;; ns++) {
                double shell = 0.0;
                for (int gx = -ns; gx <= ns; gx++)
                    for (int gy = -ns; gy <= ns; gy++)
                        for (int gz = -ns; gz <= ns; gz++) {
                            if (gx != ns && -gx != ns && gy != ns && -gy != ns && gz != ns && -gz != ns) continue;
                            double x[3] = {kq[0] + gx, kq[1] + gy, kq[2] + gz}, v[3];
                            for (int d = 0; d < 3; d++)
                                v[d] = sys->recip[0 * 3 + d] * x[0] + sys->recip[1 * 3 + d] * x[1] + sys->recip[2 * 3 + d] * x[2];
                            double g2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
                            shell += exp(-alpha * g2) / g2;
                        }
                total += shell;
                if (shell < 1e-20) break;
            }
        }
        total *= FOURPI;
        if (if_match) total -= FOURPI * alpha;
        sum_out[ik] = total;
    }
    *alpha_out = alpha;
    return TCG_OK;
}
