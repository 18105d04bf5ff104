// terms.cuh -- operator terms on top of the pass kernels.
//
//   hf2x         calc_hamiltonian_hf2x.cpp:8-205
//   tc2x         calc_hamiltonian_tc2x.cpp:11-516   (SCF mesh: kVaux = 0)
//   tc3a1, tc3b1 calc_hamiltonian_tc3a1.cpp:8-117, tc3b1.cpp:8-135
//   tc3a3b3b4b6  calc_hamiltonian_tc3a3b3b4b6.cpp:11-863
//   tc3a2a4b2b5  calc_hamiltonian_tc3a2a4b2b5.cpp:11-1300
//
// Every exchange-like sum  sum_{q,i} f_qi X_qi(r) IFFT[K(k-q+G) FFT[Y_qi(r) Z_kj(r)]]
// runs as chunks of (target bands) x (occupied sources) through the three
// fused passes (passes.cuh).  All R-space contributions to H2 psi (resp.
// H3 psi) of one band are summed in one FP64 accumulator and transformed /
// gathered onto the sphere once at the end.  Work that depends only on the
// occupied orbitals (R-space orbitals and gradients, the local three-body
// potentials of tc3a1 / tc3b1 / tc3a2 / tc3b2, and the occupied-pair stage of
// tc3a2a4b2b5 with its symmetry-rotated intermediates) is done once per
// tcg_set_state: TC++ recomputes it inside every calc_hamiltonian::all call,
// although BlochStates is constant across the calls of one Davidson step.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include "ctx.cuh"
#include "passes.cuh"
#include "util.cuh"
#include "jastrow.cuh"

namespace tcg {

struct ApplyArgs {
    uint32_t mask;
    const int32_t *nb;
    const uint8_t *owned;
    const double2 *psi;
    double2 *h2, *h3;
};

constexpr double PI_D = 3.14159265358979323846;

struct RecipC {
    double R[9];
};

static inline void cart(const Host &h, const double *x, double *v)
{
    for (int d = 0; d < 3; d++) v[d] = h.recip[0 * 3 + d] * x[0] + h.recip[1 * 3 + d] * x[1] + h.recip[2 * 3 + d] * x[2];
}

__device__ __forceinline__ void gvec(const double *R, const GridDesc &g, int x, int y, int z, const double *q, double *G)
{
    const int m0 = miller(x, g.n0), m1 = miller(y, g.n1), m2 = miller(z, g.n2);
#pragma unroll
    for (int d = 0; d < 3; d++) G[d] = q[d] + R[0 * 3 + d] * m0 + R[1 * 3 + d] * m1 + R[2 * 3 + d] * m2;
}

__device__ __forceinline__ void xyz_of(const GridDesc &g, size_t p, int &x, int &y, int &z)
{
    x = (int)(p % g.n0);
    y = (int)((p / g.n0) % g.n1);
    z = (int)(p / ((size_t)g.n0 * g.n1));
}

__device__ __forceinline__ void acc_add(double2 *a, double2 v, double f) { *a = {a->x + f * v.x, a->y + f * v.y}; }
// fire-and-forget accumulation (red.global.add.f64): no load / store
// round trip per update.  Every accumulator element is updated by one thread
// only, so the updates of an element keep their program order and the sum
// is deterministic.
__device__ __forceinline__ void acc_red(double2 *a, double2 v, double f)
{
    atomicAdd(&a->x, f * v.x);
    atomicAdd(&a->y, f * v.y);
}

// ---------------------------------------------------------------- sphere --
template <typename T>
static int sphere_to_r(tcg_ctx *c, const std::vector<SphereItem> &items)
{
    using V = typename C2<T>::t;
    const GridDesc &g = c->gd;
    if (items.empty()) return TCG_OK;
    const int nz_tiles = (g.n0 * g.n1 + ZTC - 1) / ZTC;
    const size_t n = items.size();
    std::vector<void *> outs(n);
    for (size_t i = 0; i < n; i++) outs[i] = items[i].out;
    TRY(c->items.ensure(n * (sizeof(SphereItem) + sizeof(void *))));
    SphereItem *d_items = c->items.as<SphereItem>();
    void **d_outs = reinterpret_cast<void **>(d_items + n);
    TCG_CUDA(cudaMemcpyAsync(d_items, items.data(), n * sizeof(SphereItem), cudaMemcpyHostToDevice, c->stream));
    TCG_CUDA(cudaMemcpyAsync(d_outs, outs.data(), n * sizeof(void *), cudaMemcpyHostToDevice, c->stream));
    for (size_t b0 = 0; b0 < n; b0 += 65535) {
        const unsigned nb = (unsigned)std::min<size_t>(65535, n - b0);
        TRY(launch(c, k_sphere_z<T>, dim3(nz_tiles, nb), dim3(256), smem_z<V>(g, 0), g,
                   (const SphereItem *)(d_items + b0), c->recip.as<const double>()));
        GridRefs gr;
        gr.dev = d_outs + b0;
        TRY(launch(c, k_xy_inplace<T, +1>, dim3(g.n2, nb), dim3(256), smem_xy<V>(g), g, gr));
    }
    TCG_CUDA(cudaStreamSynchronize(c->stream));   // c->items is reused by the next caller
    return TCG_OK;
}

// In-place full 3D FFT of a list of grids (DIR -1: forward with 1/N).
template <typename T, int DIR>
static int fft3_list(tcg_ctx *c, const std::vector<void *> &grids)
{
    using V = typename C2<T>::t;
    const GridDesc &g = c->gd;
    if (grids.empty()) return TCG_OK;
    const size_t n = grids.size();
    const int ntiles = (g.n0 * g.n1 + ZTC - 1) / ZTC;
    const double scale = DIR < 0 ? 1.0 / (double)g.N : 1.0;
    if (n <= 8) {   // pointers by value: nothing to upload, nothing to wait for
        GridRefs gr;
        for (size_t i = 0; i < n; i++) gr.inl[i] = grids[i];
        TRY(launch(c, k_xy_inplace<T, DIR>, dim3(g.n2, (unsigned)n), dim3(256), smem_xy<V>(g), g, gr));
        return launch(c, k_z_inplace<T, DIR>, dim3(ntiles, (unsigned)n), dim3(256), smem_z<V>(g, 0), g, gr, scale);
    }
    TRY(c->items.ensure(n * sizeof(void *)));
    void **d = c->items.as<void *>();
    TCG_CUDA(cudaMemcpyAsync(d, grids.data(), n * sizeof(void *), cudaMemcpyHostToDevice, c->stream));
    for (size_t b0 = 0; b0 < n; b0 += 65535) {
        const unsigned nb = (unsigned)std::min<size_t>(65535, n - b0);
        GridRefs gr;
        gr.dev = d + b0;
        TRY(launch(c, k_xy_inplace<T, DIR>, dim3(g.n2, nb), dim3(256), smem_xy<V>(g), g, gr));
        TRY(launch(c, k_z_inplace<T, DIR>, dim3(ntiles, nb), dim3(256), smem_z<V>(g, 0), g, gr, scale));
    }
    TCG_CUDA(cudaStreamSynchronize(c->stream));   // c->items is reused by the next caller
    return TCG_OK;
}

// --------------------------------------------------------------- targets --
struct Targets {
    std::vector<int> s, k, j;
    std::vector<size_t> psi_off;            // complex offset of the band in psi
    std::vector<int> blk;                   // block starts (equal (s,k)) + end
};

static Targets make_targets(const tcg_ctx *c, const ApplyArgs &A)
{
    const Host &h = c->h;
    Targets T;
    size_t off = 0, flat = 0;
    for (int s = 0; s < h.nspin; s++)
        for (int k = 0; k < h.nk; k++) {
            bool opened = false;
            for (int j = 0; j < A.nb[s * h.nk + k]; j++, flat++, off += h.npw[k]) {
                if (A.owned && !A.owned[flat]) continue;
                if (!opened) { T.blk.push_back((int)T.s.size()); opened = true; }
                T.s.push_back(s);
                T.k.push_back(k);
                T.j.push_back(j);
                T.psi_off.push_back(off);
            }
        }
    T.blk.push_back((int)T.s.size());
    return T;
}

// ============================================================ op plumbing ==
// Common chunk description shared by the ops: targets tj in [0, nt),
// sources si in [0, ns), item = tj * ns + si.  Each target belongs to a
// target block tb (equal k) and each source to a source block sb (equal
// all-k index); per (tb, sb) a kq vector and a Jastrow table row exist.
struct ChunkMeta {
    const int *tb;          // [nt]
    const int *sb;          // [ns]
    const double *kq;       // [nTB*nSB][3]
    const double *tab;      // [nTB*nSB][N][ntab]            (FP64 path)
    const float4 *ftab;     // [nTB*nSB][N][nrec] coefficients (mixed path)
    int nSB, ntab, nrec;
    // pruning of band-limited grids (prune != 0): per pair its entry in the
    // context's pencil table; pmask[entry][x + n0 y] = 1 where the pair
    // density's support meets pencil (x, y); pperm lists the active pencils
    // first, pnact counts them
    const int *pent;        // [nTB*nSB]
    const unsigned char *pmask;
    const unsigned short *pperm;
    const int *pnact;
    const unsigned long long *pbits;   // [entry][x]: bit y set where pencil (x, y) is active
    int np, prune;
    double pfrac;           // mean active-pencil fraction of the chunk's items (host accounting)
};

template <typename T>
struct OpBase {
    using V = typename C2<T>::t;
    static constexpr bool ZINV = true, REFWD = false;
    static constexpr int GS = 1;
    static constexpr int ZMINB = 3;          // min resident CTAs of the fast Z pass (register cap)
    static constexpr bool ZSPLIT = true;     // fast Z pass: z-lines split over lane pairs
    // fast XY passes: one thread per line (measured fastest for every term on
    // 36^3 once the plane copies were made division-free) or lines split over
    // lane pairs (half the registers, one shuffle per element)
    static constexpr bool XYF_PAIR = false, XYI_PAIR = false;
    // forward XY pass in split lines by default also in FP32 where a whole
    // line per thread spills (48^3)
    static constexpr bool XYF_SPLIT48 = false;
    // split-line inverse XY pass at 36^3: resident CTAs per SM beyond the
    // default four (a register cap the op's work fits without spilling)
    static constexpr int XYI_MINB_EXTRA = 0;
    // the same for the register-resident split-line Z pass (k_z_t6r)
    static constexpr int ZR_MINB_EXTRA = 0;
    // split-line Z pass in shared memory (k_z_t6): the input plane that holds
    // the inverse transform of each output, valid when every output after the
    // first reads input 0 only in zmix (-1: a plane of its own)
    static constexpr int ZO_ALIAS = -1;
    static constexpr int Z_MINB_EXTRA = 0;    // k_z_t6 as XYI_MINB_EXTRA
    // split-line Z pass (36^3, 48^3): transformed inputs kept in registers
    // (one exchange per transform, fewer resident CTAs); measured faster for
    // three inputs
    static constexpr bool ZREG = false;
    GridDesc g;
    V *tmp;
    int nsl;                // tmp slots per item
    int ns;                 // sources in the chunk
    ChunkMeta m;
    RecipC rc;
    double invN;
    __device__ V *tmp_grid(int item, int f) const { return tmp + ((size_t)item * nsl + f) * g.N; }
    __device__ V *zin_grid(int item, int f) const { return tmp_grid(item, f); }
    __device__ V *out_grid(int item, int o) const { return tmp_grid(item, o); }
    __device__ V *xyi_grid(int item, int b) const { return tmp_grid(item, b); }
    __device__ void xyf_begin(int) const {}
    __device__ void z_begin(int) const {}
    __device__ void xyi_end(int, int) const {}
    __device__ int nsrc(int) const { return ns; }
    __device__ int item_of(int tj, int si) const { return tj * ns + si; }
    __device__ bool refwd_want(int) const { return false; }
    __device__ V refwd_load(int, int, int, size_t, V v) const { return v; }
    __device__ V *refwd_grid(int, int) const { return nullptr; }
    __device__ V xyf_load(int, int, int, int, int, size_t) const { return czero<V>(); }
    // register accumulation (fast XYI path, FP32): grids b with regacc_grid(b)
    // contribute xyi_term(...) to a per-thread column sum flushed once per
    // chunk with xyi_flush; the other grids go through xyi_accum.
    static constexpr bool REGACC = false;
    static constexpr bool BOUTER = false;    // one register accumulator per output grid (xyi_flush_b)
    // RACC_EXTRA: besides the register sum, every output also goes to
    // xyi_extra(tj, item, b, p, v) (other accumulators of the op)
    static constexpr bool RACC_EXTRA = false;
    __device__ void xyi_extra(int, int, int, size_t, const V *) const {}
    // split-line inverse XY pass (k_xyi_t6), FP32: SACC > 0 accumulates the chunk's
    // sources in SACC shared-memory planes per CTA (xyi_sterm picks the slot
    // of output b, -1 for none) and adds them to the FP64 accumulators once
    // at the end (xyi_sflush), instead of one FP64 red.add per source
    static constexpr int SACC = 0;           // most slots an op uses (compile-time bound)
    int sacc_on = 0;                         // runtime switch of the SACC path
    int sacc_n = 0;                          // slots in use when on (<= SACC; sizes the shared memory)
    __device__ int xyi_slot(int) const { return -1; }
    __device__ V xyi_sterm(int, int, int, size_t, V v) const { return v; }
    __device__ void xyi_sflush(int, int, size_t, V) const {}
    // SACC_GROUP: the op defines xyi_sgroup(tj, item, b0, p, vals[GS], add),
    // the contributions of an output group to the slots (add(slot, value));
    // otherwise output b0 goes to slot xyi_slot(b0) as xyi_sterm (sacc_group)
    static constexpr bool SACC_GROUP = false;
    __device__ bool regacc_grid(int) const { return false; }
    __device__ V xyi_term(int, int, int, size_t, const V *v) const { return v[0]; }
    __device__ void xyi_flush(int, size_t, V) const {}
    __device__ int pair_id(int item) const { return m.tb[item / ns] * m.nSB + m.sb[item % ns]; }
    __device__ const double *kq_of(int item) const { return m.kq + 3 * pair_id(item); }
    __device__ const double *tab_of(int item) const { return m.tab + (size_t)pair_id(item) * g.N * m.ntab; }
    // mixed path: record r of the coefficient table at grid point p
    __device__ float4 fco(int item, size_t p, int r) const
    {
        return __ldg(&m.ftab[((size_t)pair_id(item) * g.N + p) * m.nrec + r]);
    }
    static constexpr bool FT = sizeof(T) == 4;   // mixed path: FP32 coefficient tables
    __device__ static float comp(const float4 &c, int d) { return d == 0 ? c.x : (d == 1 ? c.y : (d == 2 ? c.z : c.w)); }
    __device__ size_t pidx(int x, int y, int z) const { return (size_t)x + (size_t)g.n0 * (y + (size_t)g.n1 * z); }
    // Band-limited inputs (bit f of BLI) and outputs (bit o of BLO): pair
    // densities conj(a_q) b_k of two orbitals of the plane-wave spheres of q
    // and k, and G-space multiples of them, vanish outside the ball
    // |G + k - q| < R_k + R_q.  With m.prune set, the pass kernels skip
    // their pencils outside it (XYF stores, Z loads / transforms / stores,
    // XYI loads read as zero); values there are zero up to round-off.
    static constexpr unsigned BLI = 0, BLO = 0;
    __device__ int pent_of(int item) const { return m.pent[pair_id(item)]; }
    __device__ bool pact(int item, int xy) const { return m.pmask[(size_t)pent_of(item) * m.np + xy] != 0; }
    // active rows y of column x of the item's pair (bit y)
    __device__ unsigned long long pcol(int item, int x) const { return m.pbits[(size_t)pent_of(item) * g.n0 + x]; }
};

// =================================================================== hf2x ==
template <typename T>
struct OpHF2X : OpBase<T> {
    using V = typename C2<T>::t;
    static constexpr const char *NAME = "hf2x";
    static constexpr unsigned BLI = 1, BLO = 1;           // conj(phi_q) psi_k and its multiple
    static constexpr bool REGACC = true;
    __device__ bool regacc_grid(int) const { return true; }
    __device__ V xyi_term(int, int item, int, size_t p, const V *v) const
    {
        const int si = item % this->ns;
        return cscale(cmul(v[0], __ldg(&Rocc[(size_t)si * this->g.N + p])), (decltype(v[0].x))fill[si]);
    }
    __device__ void xyi_flush(int tj, size_t p, V s) const { acc_red(acc + (size_t)tj * this->g.N + p, to64(s), 1.0); }
    static constexpr int NF = 1, NB = 1;
    const V *Rpsi, *Rocc;     // chunk's first target / source
    double2 *acc;
    const double *fill;
    __device__ V xyf_load(int item, int, int, int, int, size_t p) const
    {
        const int tj = item / this->ns, si = item % this->ns;
        return cmulc(__ldg(&Rocc[(size_t)si * this->g.N + p]), __ldg(&Rpsi[(size_t)tj * this->g.N + p]));
    }
    __device__ V zmix(int item, int, int x, int y, int z, const V *in) const
    {
        double G[3];
        gvec(this->rc.R, this->g, x, y, z, this->kq_of(item), G);
        const double t = G[0] * G[0] + G[1] * G[1] + G[2] * G[2];
        const double v = t < 1e-8 ? 0.0 : this->invN / t;   // 1/|k-q+G|^2 (hf2x.cpp:93-104), 1/N folded in
        return cscale(in[0], (decltype(in[0].x))v);
    }
    __device__ void xyi_accum(int tj, int item, int, size_t p, const V *v) const
    {
        const int si = item % this->ns;
        acc_red(acc + (size_t)tj * this->g.N + p, to64(cmul(v[0], __ldg(&Rocc[(size_t)si * this->g.N + p]))), fill[si]);
    }
};

// =================================================================== tc2x ==
template <typename T>
struct OpTC2X : OpBase<T> {
    using V = typename C2<T>::t;
    static constexpr const char *NAME = "tc2x";
    static constexpr unsigned BLI = 0xF, BLO = 0xF;       // conj(chi_q) psi_k, conj(chi_q) grad psi_k
    static constexpr bool ZSPLIT = false;     // one thread per z-line measured faster here
    static constexpr int ZO_ALIAS = 1;        // outputs 1-3 read input 0 only (zmix)
    static constexpr int Z_MINB_EXTRA = 1;    // five CTAs of 38 KB at 36^3
    static constexpr bool REGACC = true;
    __device__ bool regacc_grid(int) const { return true; }
    __device__ V xyi_term(int, int item, int b, size_t p, const V *v) const
    {
        const size_t N = this->g.N;
        const int si = item % this->ns;
        const V o = b == 0 ? __ldg(&Rocc[(size_t)si * N + p]) : __ldg(&Rgrad[((size_t)si * 3 + (b - 1)) * N + p]);
        return cscale(cmul(v[0], o), (decltype(v[0].x))(b == 0 ? fill[si] : -fill[si]));
    }
    __device__ void xyi_flush(int tj, size_t p, V s) const { acc_red(acc + (size_t)tj * this->g.N + p, to64(s), 1.0); }
    static constexpr int NF = 4, NB = 4;
    const V *Rpsi, *Rgpsi;        // [nt][N], [nt][3][N]
    const V *Rocc, *Rchi, *Rgrad; // [ns][N], [ns][N], [ns][3][N]
    double2 *acc;
    const double *fill;
    __device__ V xyf_load(int item, int f, int, int, int, size_t p) const
    {
        const size_t N = this->g.N;
        const int tj = item / this->ns, si = item % this->ns;
        const V chi = __ldg(&Rchi[(size_t)si * N + p]);
        const V rhs = f == 0 ? __ldg(&Rpsi[(size_t)tj * N + p]) : __ldg(&Rgpsi[((size_t)tj * 3 + (f - 1)) * N + p]);
        return cmulc(chi, rhs);     // tc2x.cpp:350, :374
    }
    __device__ V zmix(int item, int o, int x, int y, int z, const V *in) const
    {
        using S = decltype(in[0].x);
        if constexpr (OpBase<T>::FT) {
            const float4 c = this->fco(item, this->pidx(x, y, z), 0);
            if (o == 0) {
                V r = cscale(in[0], c.x);
                r = cadd(r, cscale(in[1], c.y));
                r = cadd(r, cscale(in[2], c.z));
                return cadd(r, cscale(in[3], c.w));
            }
            return cscale(in[0], this->comp(c, o));
        }
        double G[3];
        gvec(this->rc.R, this->g, x, y, z, this->kq_of(item), G);
        const size_t p = (size_t)x + (size_t)this->g.n0 * (y + (size_t)this->g.n1 * z);
        const double *tab = this->tab_of(item);
        const double u = tab[2 * p + 1] * this->invN;
        if (o == 0) {   // [2a_x] rho V_2body + [2b_x2] sum_d rho_d du_d   (tc2x.cpp:378-386)
            V r = cscale(in[0], (S)(tab[2 * p] * this->invN));
#pragma unroll
            for (int d = 0; d < 3; d++) r = cadd(r, cscale(in[1 + d], (S)(G[d] * u)));
            return r;
        }
        return cscale(in[0], (S)(G[o - 1] * u));   // [2b_x1] rho du_d (tc2x.cpp:354-358)
    }
    __device__ void xyi_accum(int tj, int item, int b, size_t p, const V *v) const
    {
        const size_t N = this->g.N;
        const int si = item % this->ns;
        const V o = b == 0 ? __ldg(&Rocc[(size_t)si * N + p]) : __ldg(&Rgrad[((size_t)si * 3 + (b - 1)) * N + p]);
        acc_red(acc + (size_t)tj * N + p, to64(cmul(v[0], o)), b == 0 ? fill[si] : -fill[si]);
    }
};

// Jastrow tables per (tb, sb): modes select the columns
enum TabMode { TAB_TC2X = 0, TAB_U_SX = 1, TAB_U_SS = 2, TAB_U_QX = 3 };
// TAB_TC2X : [V_2body(s,s), u(s,s)]                         (tc2x.cpp:266-276)
// TAB_U_SX : [u(G; 0, s), u(G; 1, s)]                        (tc3a3b3b4b6.cpp:208-217)
// TAB_U_SS : [u(G; s, s)]                                    (tc3a3b3b4b6.cpp:679-686)
// TAB_U_QX : [u(G; s, 0), u(G; s, 1)]                        (tc3a2a4b2b5.cpp:244-253)
static __global__ void k_tables(GridDesc g, RecipC rc, Jastrow J, int mode, int s, int npair, const double *kq, double *tab)
{
    const int ntab = mode == TAB_U_SS ? 1 : 2;
    const size_t total = (size_t)npair * g.N;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int pr = (int)(i / g.N);
        const size_t p = i % g.N;
        int x, y, z;
        xyz_of(g, p, x, y, z);
        double G[3];
        gvec(rc.R, g, x, y, z, kq + 3 * pr, G);
        double *o = tab + i * ntab;
        if (mode == TAB_TC2X) { o[0] = J.tc2body(G, s, s); o[1] = J.uk(G, s, s); }
        else if (mode == TAB_U_SX) { o[0] = J.uk(G, 0, s); o[1] = J.uk(G, 1, s); }
        else if (mode == TAB_U_SS) { o[0] = J.uk(G, s, s); }
        else { o[0] = J.uk(G, s, 0); o[1] = J.uk(G, s, 1); }
    }
}

// FP32 coefficient tables of the mixed path, evaluated in FP64 and rounded
// once; G = k - q + G_p, all include the 1/N of the forward transform:
//   TAB_TC2X : {V_2body(s,s), G_0 u, G_1 u, G_2 u} / N       with u = u(G; s, s)
//   TAB_U_SX : record r = {G_d u(G; x_r, s)} / N, x_r = r (nrec 2) or s (nrec 1)
//   TAB_U_SS : {G_d u(G; s, s)} / N
//   TAB_U_QX : record r = {G_d u(G; s, x_r)} / N, x_r = r (nrec 2) or s (nrec 1)
static __global__ void k_ftables(GridDesc g, RecipC rc, Jastrow J, int mode, int s, int nrec, int npair,
                                 const double *kq, double invN, float4 *tab)
{
    const size_t total = (size_t)npair * g.N;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int pr = (int)(i / g.N);
        const size_t p = i % g.N;
        int x, y, z;
        xyz_of(g, p, x, y, z);
        double G[3];
        gvec(rc.R, g, x, y, z, kq + 3 * pr, G);
        float4 *o = tab + i * nrec;
        if (mode == TAB_TC2X) {
            const double u = J.uk(G, s, s) * invN;
            o[0] = make_float4((float)(J.tc2body(G, s, s) * invN), (float)(G[0] * u), (float)(G[1] * u),
                               (float)(G[2] * u));
            continue;
        }
        for (int r = 0; r < nrec; r++) {
            const int xr = nrec == 1 ? s : r;
            double u;
            if (mode == TAB_U_SX) u = J.uk(G, xr, s);
            else if (mode == TAB_U_QX) u = J.uk(G, s, xr);
            else u = J.uk(G, s, s);
            u *= invN;
            o[r] = make_float4((float)(G[0] * u), (float)(G[1] * u), (float)(G[2] * u), 0.f);
        }
    }
}

// ======================================================= tc3a3b3b4b6 ops ==
// stage A: first q loop (tc3a3b3b4b6.cpp:192-368).
// EQ: u(G; 0, s) == u(G; 1, s) (same Jastrow A, F for both spins of x2), so
// the spin sum of the 3b6 chain collapses by linearity,
//   sum_x du_d FFT[n_x IFFT[phiphi du_d]] = du_d FFT[(n_0 + n_1) IFFT[phiphi du_d]],
// and only three P grids (x = s) are needed instead of six.
template <typename T, bool EQ = false>
struct OpTC3A : OpBase<T> {
    using V = typename C2<T>::t;
    static constexpr const char *NAME = "3a3b6A";
    static constexpr int NX = EQ ? 1 : 2;     // spin branches of x2 carried
    static constexpr int NF = 4, NB = 1 + 3 * NX;
    static constexpr int ZO_ALIAS = 1;        // outputs 1.. read input 0 only (zmix)
    // input 0 = conj(chi_q) psi_k and outputs 1.. = its multiples; inputs 1-3
    // carry dnu (their products alias over the whole grid), output 0 mixes them
    static constexpr unsigned BLI = 1, BLO = ((1u << NB) - 1) & ~1u;
    static constexpr bool REFWD = true;
    static constexpr bool ZSPLIT = false;    // one thread per z-line measured faster here
    // accumulation through xyi_accum (FP64 red.add per source), so that the
    // prefetching XYI kernel can transform the re-forwarded planes in place;
    // with REGACC the per-output FP32 column sums over the chunk's sources
    // (b = 0 -> acc, b = 1 + 3 xs + d -> qsum[d] when xs == s) are used instead
    static constexpr bool REGACC = false, BOUTER = true;
    __device__ bool regacc_grid(int b) const { return b == 0 || EQ || (b - 1) / 3 == s; }
    __device__ V xyi_term(int, int item, int b, size_t p, const V *v) const
    {
        const int si = item % this->ns;
        const V t = cmul(v[0], __ldg(&Rocc[(size_t)si * this->g.N + p]));
        return b == 0 ? cscale(t, (decltype(t.x))(fill[si] * b3)) : t;
    }
    __device__ void xyi_flush_b(int tj, int b, size_t p, V sum) const
    {
        const size_t N = this->g.N;
        if (b == 0) acc_red(acc + (size_t)tj * N + p, to64(sum), 1.0);
        else acc_red(qsum + ((size_t)tj * 3 + (b - 1) % 3) * N + p, to64(sum), 1.0);
    }
    const V *Rpsi, *Rocc, *Rchi;  // [nt][N], [ns][N]
    const V *dnu;                 // [3][N] of the targets' spin
    const V *densT;               // [2][N] density (EQ: [0] = n_0 + n_1), compute precision
    double2 *acc, *qsum;          // [nt][N], [nt][3][N]
    const double *fill;
    V *tmp2;                      // [items][3 NX][N]
    int s;
    double b3;
    __device__ V xyf_load(int item, int f, int, int, int, size_t p) const
    {
        const size_t N = this->g.N;
        const int tj = item / this->ns, si = item % this->ns;
        const V chi = __ldg(&Rchi[(size_t)si * N + p]);
        V rhs = __ldg(&Rpsi[(size_t)tj * N + p]);
        if (f > 0) rhs = cmul(__ldg(&dnu[(size_t)(f - 1) * N + p]), rhs);   // dnu_phi (:236)
        return cmulc(chi, rhs);
    }
    __device__ V zmix(int item, int o, int x, int y, int z, const V *in) const
    {
        using S = decltype(in[0].x);
        if constexpr (OpBase<T>::FT) {
            const size_t p = this->pidx(x, y, z);
            if (o == 0) {
                const float4 c = this->fco(item, p, EQ ? 0 : s);
                V r = cscale(in[1], c.x);
                r = cadd(r, cscale(in[2], c.y));
                return cadd(r, cscale(in[3], c.z));
            }
            const int xs = EQ ? s : (o - 1) / 3, d = (o - 1) % 3;
            const float4 c = this->fco(item, p, EQ ? 0 : xs);
            return cscale(in[0], (float)fill[item % this->ns] * this->comp(c, d));
        }
        double G[3];
        gvec(this->rc.R, this->g, x, y, z, this->kq_of(item), G);
        const size_t p = (size_t)x + (size_t)this->g.n0 * (y + (size_t)this->g.n1 * z);
        const double *tab = this->tab_of(item) + 2 * p;
        if (o == 0) {   // [3b3] sum_d du[s]_d FFT(dnu_phi_d conj chi) (:286-295)
            const double u = tab[s] * this->invN;
            V r = cscale(in[1], (S)(G[0] * u));
            r = cadd(r, cscale(in[2], (S)(G[1] * u)));
            return cadd(r, cscale(in[3], (S)(G[2] * u)));
        }
        const int xs = EQ ? s : (o - 1) / 3, d = (o - 1) % 3;   // phiphi f du[xs]_d (:306-314)
        const double f = fill[item % this->ns];
        return cscale(in[0], (S)(f * G[d] * tab[xs] * this->invN));
    }
    __device__ void xyi_accum(int tj, int item, int b, size_t p, const V *v) const
    {
        const size_t N = this->g.N;
        const int si = item % this->ns;
        const V phq = __ldg(&Rocc[(size_t)si * N + p]);
        if (b == 0) {
            acc_red(acc + (size_t)tj * N + p, to64(cmul(v[0], phq)), fill[si] * b3);
        } else {
            const int xs = EQ ? s : (b - 1) / 3, d = (b - 1) % 3;
            if (xs == s) acc_red(qsum + ((size_t)tj * 3 + d) * N + p, to64(cmul(v[0], phq)), 1.0);
        }
    }
    __device__ bool refwd_want(int b) const { return b > 0; }
    __device__ V refwd_load(int, int, int b, size_t p, V v) const
    {
        const int xs = EQ ? 0 : (b - 1) / 3;
        return cmul(v, __ldg(&densT[(size_t)xs * this->g.N + p]));   // orbital * n_s2 (:332)
    }
    // shared-memory accumulation (k_xyi_t6, FP32): slot 0 = acc, 1 + d = qsum_d
    static constexpr int SACC = 4;
    __device__ int xyi_slot(int b) const
    {
        if (b == 0) return 0;
        const int xs = EQ ? s : (b - 1) / 3;
        return xs == s ? 1 + (b - 1) % 3 : -1;
    }
    __device__ V xyi_sterm(int, int item, int b, size_t p, V v) const
    {
        const int si = item % this->ns;
        const V t = cmul(v, __ldg(&Rocc[(size_t)si * this->g.N + p]));
        return b == 0 ? cscale(t, (decltype(t.x))(fill[si] * b3)) : t;
    }
    __device__ void xyi_sflush(int tj, int slot, size_t p, V sum) const
    {
        const size_t N = this->g.N;
        if (slot == 0) acc_red(acc + (size_t)tj * N + p, to64(sum), 1.0);
        else acc_red(qsum + ((size_t)tj * 3 + (slot - 1)) * N + p, to64(sum), 1.0);
    }
    __device__ V *refwd_grid(int item, int b) const { return tmp2 + ((size_t)item * 3 * NX + (b - 1)) * this->g.N; }
};

// stage B: [3b6] sum_{s2,d} FFT(.) du[s2]_d -> IFFT x phi_q (:333-348)
template <typename T, bool EQ = false>
struct OpTC3B : OpBase<T> {
    using V = typename C2<T>::t;
    static constexpr const char *NAME = "3b6B";
    static constexpr bool ZREG = true;
    static constexpr int ZR_MINB_EXTRA = EQ ? 2 : 0;   // 64 registers without spills for one spin channel
    static constexpr int NX = EQ ? 1 : 2;
    static constexpr int NF = 3 * NX, NB = 1;
    static constexpr bool REGACC = true;
    __device__ bool regacc_grid(int) const { return true; }
    __device__ V xyi_term(int, int item, int, size_t p, const V *v) const
    {
        const int si = item % this->ns;
        return cscale(cmul(v[0], __ldg(&Rocc[(size_t)si * this->g.N + p])), (decltype(v[0].x))b6);
    }
    __device__ void xyi_flush(int tj, size_t p, V s) const { acc_red(acc + (size_t)tj * this->g.N + p, to64(s), 1.0); }
    const V *Rocc;
    double2 *acc;
    V *tmp2;
    double b6;
    int s;
    __device__ V *zin_grid(int item, int f) const { return tmp2 + ((size_t)item * NF + f) * this->g.N; }
    __device__ V zmix(int item, int, int x, int y, int z, const V *in) const
    {
        using S = decltype(in[0].x);
        if constexpr (OpBase<T>::FT) {
            const size_t p = this->pidx(x, y, z);
            V r = czero<V>();
#pragma unroll
            for (int xs = 0; xs < NX; xs++) {
                const float4 c = this->fco(item, p, xs);
                r = cadd(r, cscale(in[3 * xs], c.x));
                r = cadd(r, cscale(in[3 * xs + 1], c.y));
                r = cadd(r, cscale(in[3 * xs + 2], c.z));
            }
            return r;
        }
        double G[3];
        gvec(this->rc.R, this->g, x, y, z, this->kq_of(item), G);
        const size_t p = (size_t)x + (size_t)this->g.n0 * (y + (size_t)this->g.n1 * z);
        const double *tab = this->tab_of(item) + 2 * p;
        V r = czero<V>();
#pragma unroll
        for (int xs = 0; xs < NX; xs++) {
            const double u = tab[EQ ? s : xs] * this->invN;
#pragma unroll
            for (int d = 0; d < 3; d++) r = cadd(r, cscale(in[3 * xs + d], (S)(G[d] * u)));
        }
        return r;
    }
    __device__ void xyi_accum(int tj, int item, int, size_t p, const V *v) const
    {
        const int si = item % this->ns;
        acc_red(acc + (size_t)tj * this->g.N + p, to64(cmul(v[0], __ldg(&Rocc[(size_t)si * this->g.N + p]))), b6);
    }
};

// stage C: [3b4] second q loop (:664-767)
template <typename T>
struct OpTC3C : OpBase<T> {
    using V = typename C2<T>::t;
    static constexpr const char *NAME = "3b4C";
    static constexpr bool ZREG = true;
    static constexpr bool REGACC = true;
    __device__ bool regacc_grid(int) const { return true; }
    __device__ V xyi_term(int, int item, int, size_t p, const V *v) const
    {
        const int si = item % this->ns;
        return cscale(cmul(v[0], __ldg(&Rocc[(size_t)si * this->g.N + p])), (decltype(v[0].x))(b4 * fill[si]));
    }
    __device__ void xyi_flush(int tj, size_t p, V s) const { acc_red(acc + (size_t)tj * this->g.N + p, to64(s), 1.0); }
    static constexpr int NF = 3, NB = 1;
    const V *Rocc, *Rchi;
    const double2 *qsum;      // [nt][3][N]
    double2 *acc;
    const double *fill;
    double b4;
    __device__ V xyf_load(int item, int f, int, int, int, size_t p) const
    {
        const size_t N = this->g.N;
        const int tj = item / this->ns, si = item % this->ns;
        return cmulc(__ldg(&Rchi[(size_t)si * N + p]), from64<V>(__ldg(&qsum[((size_t)tj * 3 + f) * N + p])));
    }
    __device__ V zmix(int item, int, int x, int y, int z, const V *in) const
    {
        using S = decltype(in[0].x);
        if constexpr (OpBase<T>::FT) {
            const float4 c = this->fco(item, this->pidx(x, y, z), 0);
            V r = cscale(in[0], c.x);
            r = cadd(r, cscale(in[1], c.y));
            return cadd(r, cscale(in[2], c.z));
        }
        double G[3];
        gvec(this->rc.R, this->g, x, y, z, this->kq_of(item), G);
        const size_t p = (size_t)x + (size_t)this->g.n0 * (y + (size_t)this->g.n1 * z);
        const double u = this->tab_of(item)[p] * this->invN;
        V r = cscale(in[0], (S)(G[0] * u));
        r = cadd(r, cscale(in[1], (S)(G[1] * u)));
        return cadd(r, cscale(in[2], (S)(G[2] * u)));
    }
    __device__ void xyi_accum(int tj, int item, int, size_t p, const V *v) const
    {
        const int si = item % this->ns;
        acc_red(acc + (size_t)tj * this->g.N + p, to64(cmul(v[0], __ldg(&Rocc[(size_t)si * this->g.N + p]))), b4 * fill[si]);
    }
};

// 3b3 (tc3a3b3b4b6.cpp:284-302), 3b4 (:651-770) and 3b5 (tc3a2a4b2b5.cpp:
// 882-894) each transform three grids, contract them with du_d(G) =
// (k - q + G)_d u(G; s, s) and multiply the inverse transform by phi_q f_q:
// by linearity one transform of the sum of their scaled inputs,
//   in_d = conj(chi_q) (b3 dnu_d psi_k + b4 qsum_d[k]) + b5 Bt_d[q] psi_k,
// gives all three (b5 = 0 without tc3a2a4b2b5).  Runs in the second q loop,
// after the first has completed qsum.
template <typename T>
struct OpTC3X : OpBase<T> {
    using V = typename C2<T>::t;
    static constexpr const char *NAME = "3bX";
    static constexpr int NF = 3, NB = 1;
    static constexpr bool ZREG = true;
    static constexpr bool XYF_SPLIT48 = true;    // measured faster at 48^3 (three operand grids per point)
    static constexpr int ZR_MINB_EXTRA = 2;      // 64 registers without spills
    static constexpr bool REGACC = true;
    __device__ bool regacc_grid(int) const { return true; }
    const V *Rpsi, *Rocc, *Rchi;  // [nt][N], [ns][N], [ns][N]
    const V *W;                   // [nt][3][N] per-target part b3 dnu_d psi + b4 qsum_d (k_w3x)
    const V *Bt;                  // [ns][3][N] or null (b5 = 0)
    double2 *acc;
    const double *fill;
    double b5;
    __device__ V xyf_load(int item, int f, int, int, int, size_t p) const
    {
        using S = decltype(V{}.x);
        const size_t N = this->g.N;
        const int tj = item / this->ns, si = item % this->ns;
        V r = cmulc(__ldg(&Rchi[(size_t)si * N + p]), __ldg(&W[((size_t)tj * 3 + f) * N + p]));
        if (Bt) r = cadd(r, cscale(cmul(__ldg(&Bt[((size_t)si * 3 + f) * N + p]), __ldg(&Rpsi[(size_t)tj * N + p])), (S)b5));
        return r;
    }
    __device__ V zmix(int item, int, int x, int y, int z, const V *in) const
    {
        using S = decltype(in[0].x);
        if constexpr (OpBase<T>::FT) {
            const float4 c = this->fco(item, this->pidx(x, y, z), 0);
            V r = cscale(in[0], c.x);
            r = cadd(r, cscale(in[1], c.y));
            return cadd(r, cscale(in[2], c.z));
        }
        double G[3];
        gvec(this->rc.R, this->g, x, y, z, this->kq_of(item), G);
        const size_t p = (size_t)x + (size_t)this->g.n0 * (y + (size_t)this->g.n1 * z);
        const double u = this->tab_of(item)[p] * this->invN;
        V r = cscale(in[0], (S)(G[0] * u));
        r = cadd(r, cscale(in[1], (S)(G[1] * u)));
        return cadd(r, cscale(in[2], (S)(G[2] * u)));
    }
    __device__ V xyi_term(int, int item, int, size_t p, const V *v) const
    {
        const int si = item % this->ns;
        return cscale(cmul(v[0], __ldg(&Rocc[(size_t)si * this->g.N + p])), (decltype(v[0].x))fill[si]);
    }
    __device__ void xyi_flush(int tj, size_t p, V s) const { acc_red(acc + (size_t)tj * this->g.N + p, to64(s), 1.0); }
    __device__ void xyi_accum(int tj, int item, int, size_t p, const V *v) const
    {
        const int si = item % this->ns;
        acc_red(acc + (size_t)tj * this->g.N + p, to64(cmul(v[0], __ldg(&Rocc[(size_t)si * this->g.N + p]))), fill[si]);
    }
};

// ======================================================= tc3a2a4b2b5 ops ==
// occupied-pair stage (tc3a2a4b2b5.cpp:210-443): targets (q2, i2), sources (q1, i1).
// EQ: u(G; sq, 0) == u(G; sq, 1), so both branches x2 = 0, 1 give the same
// orbital grids; one branch is transformed and its 3a2 contribution is
// added to both spin slots (twice into slot 0 when unpolarised).
template <typename T, bool BITC, bool EQ = false>
struct OpQP : OpBase<T> {
    using V = typename C2<T>::t;
    static constexpr const char *NAME = "qp";
    static constexpr int NX = EQ ? 1 : 2;
    static constexpr int NF = BITC ? 2 : 1, NB = (BITC ? 6 : 3) * NX, GS = BITC ? 2 : 1;
    static constexpr unsigned BLI = (1u << NF) - 1, BLO = (1u << NB) - 1;   // pair densities of occupied orbitals
    const V *Rq2, *Rq2c;          // targets phi_q2(r), chi_q2(r)  [nt][N]
    const V *Rocc, *Rchi;         // sources phi_q1, chi_q1        [ns][N]
    double2 *acc;                 // [nt][nacc][N]: 3a2[nspin], 3a4[3], 3b5[3]
    const double *fill;           // sources
    int nacc, nspin, sq;
    __device__ V xyf_load(int item, int f, int, int, int, size_t p) const
    {
        const size_t N = this->g.N;
        const int tj = item / this->ns, si = item % this->ns;
        if (f == 0) return cmulc(__ldg(&Rchi[(size_t)si * N + p]), __ldg(&Rq2[(size_t)tj * N + p]));   // (:359)
        return cmulc(__ldg(&Rocc[(size_t)si * N + p]), __ldg(&Rq2c[(size_t)tj * N + p]));              // (:365)
    }
    __device__ V zmix(int item, int o, int x, int y, int z, const V *in) const
    {
        using S = decltype(in[0].x);
        if constexpr (OpBase<T>::FT) {
            int xs, d, w;
            if (BITC) { w = o & 1; xs = (o >> 1) / 3; d = (o >> 1) % 3; }
            else { w = 0; xs = o / 3; d = o % 3; }
            const float4 c = this->fco(item, this->pidx(x, y, z), EQ ? 0 : xs);
            return cscale(in[w], this->comp(c, d));
        }
        double G[3];
        gvec(this->rc.R, this->g, x, y, z, this->kq_of(item), G);
        const size_t p = (size_t)x + (size_t)this->g.n0 * (y + (size_t)this->g.n1 * z);
        const double *tab = this->tab_of(item) + 2 * p;
        int xs, d, w;
        if (BITC) { w = o & 1; xs = (o >> 1) / 3; d = (o >> 1) % 3; }
        else { w = 0; xs = o / 3; d = o % 3; }
        if (EQ) xs = sq;
        return cscale(in[w], (S)(G[d] * tab[xs] * this->invN));   // du[x]_d * phiphi (:378, :385)
    }
    // shared-memory accumulation (k_xyi_t6, FP32): slot a = accumulator a of
    // the target (3a2 per spin, 3a4_d, 3b5_d), the same sums as xyi_accum
    static constexpr int SACC = 8;
    static constexpr bool SACC_GROUP = true;
    template <class F>
    __device__ void xyi_sgroup(int, int item, int b, size_t p, const V *v, F &&add) const
    {
        using S = decltype(v[0].x);
        const size_t N = this->g.N;
        const int si = item % this->ns;
        const S f1 = (S)fill[si];
        int xs, d;
        if (BITC) { xs = (b >> 1) / 3; d = (b >> 1) % 3; }
        else { xs = b / 3; d = b % 3; }
        if (EQ) xs = sq;
        const V o1 = v[0];
        V c3a2;
        if constexpr (BITC) c3a2 = cmulc(v[1], o1);
        else c3a2 = V{o1.x * o1.x + o1.y * o1.y, (S)0};
        if (EQ) {
            if (nspin == 1) add(0, cscale(c3a2, -2 * f1));
            else { add(0, cscale(c3a2, -f1)); add(1, cscale(c3a2, -f1)); }
        } else {
            add(nspin == 1 ? 0 : xs, cscale(c3a2, -f1));
        }
        if (xs == sq) {
            add(nspin + d, cscale(cmul(v[0], __ldg(&Rocc[(size_t)si * N + p])), f1));
            if constexpr (BITC)
                add(nspin + 3 + d, cscale(cmul(cconj(v[1]), cconj(__ldg(&Rchi[(size_t)si * N + p]))), -f1));
        }
    }
    __device__ void xyi_sflush(int tj, int slot, size_t p, V sum) const
    {
        acc_red(acc + ((size_t)tj * nacc + slot) * this->g.N + p, to64(sum), 1.0);
    }
    __device__ void xyi_accum(int tj, int item, int b, size_t p, const V *v) const
    {
        const size_t N = this->g.N;
        const int si = item % this->ns;
        const double f1 = fill[si];
        int xs, d;
        if (BITC) { xs = (b >> 1) / 3; d = (b >> 1) % 3; }
        else { xs = b / 3; d = b % 3; }
        if (EQ) xs = sq;
        double2 *A = acc + (size_t)tj * nacc * N;
        const double2 o1 = to64(v[0]);
        const double2 c3a2 = BITC ? cmulc(to64(v[1]), o1) : double2{o1.x * o1.x + o1.y * o1.y, 0.0};
        if (EQ) {
            // both x2 branches: slot 0 twice (unpolarised) or slots 0 and 1
            if (nspin == 1) acc_red(A + p, c3a2, -2.0 * f1);
            else { acc_red(A + p, c3a2, -f1); acc_red(A + (size_t)N + p, c3a2, -f1); }
        } else {
            const int xr = nspin == 1 ? 0 : xs;
            acc_red(A + (size_t)xr * N + p, c3a2, -f1);   // (:392-394 BITC, :404-406 TC)
        }
        if (xs == sq) {
            acc_red(A + (size_t)(nspin + d) * N + p, to64(cmul(v[0], __ldg(&Rocc[(size_t)si * N + p]))), f1);
            if (BITC) {
                const double2 cc = to64(cmul(cconj(v[BITC ? 1 : 0]), cconj(__ldg(&Rchi[(size_t)si * N + p]))));
                acc_red(A + (size_t)(nspin + 3 + d) * N + p, cc, -f1);               // (:428-430)
            }
        }
    }
};

// ----------------------------------------- tc2x fused with tc3a3b3b4b6 --
// tc2x and the first q loop of tc3a3b3b4b6 run over the same (target kj,
// source qi) pairs with the same pair density rho = conj(chi_qi) psi_kj.  With
// equal Jastrow channels for the targets' spin the transforms
// w_d = IFFT[rho G_d u(G; s, s)] are tc2x's 2b_x1 grids (tc2x.cpp:353-369) and,
// times the filling, 3a3b6A's outputs 1-3 (tc3a3b3b4b6.cpp:305-349).  OpTC2X3
// is tc2x with those three outputs also summed into qsum_d (3a3 / 3b4) and
// re-forwarded times the density (3b6, for OpTC3B), and with band != 0 also
// the 3a4 band part of tc3a2a4b2b5.  It reads tc2x's coefficient tables
// (TAB_TC2X: V_2body / N and G_d u(s, s) / N), which equal 3a3b6A's for equal
// channels.  The remaining parts that end in sum_d du_d(G) FFT[.] times phi_q
// (3b3, 3b4, 3b5) run as one transform in OpTC3X.
template <typename T>
struct OpTC2X3 : OpTC2X<T> {
    using V = typename C2<T>::t;
    static constexpr const char *NAME = "2x3A";
    static constexpr bool REFWD = true;
    static constexpr bool RACC_EXTRA = true;
    static constexpr int XYI_MINB_EXTRA = 1;     // 56 registers, no spills: 2x3A:xyi 638 -> 586 ms on C3
    const V *densT;               // [N] n_0 + n_1 (compute precision)
    double2 *qsum;                // [nt][3][N]
    V *tmp2;                      // [items][3][N] re-forwarded grids
    // band part of tc3a2a4b2b5 (band != 0): its outputs 0-2 are f a4 w_d too
    // (tc3a2a4b2b5.cpp:867-875), summed times the rotated intermediate Qt_d
    const V *Qt;                  // [ns][3][N]
    double2 *acc3;                // [nt][N] H3 accumulator
    double fa4;
    int band;
    __device__ bool refwd_want(int b) const { return b > 0; }
    __device__ V refwd_load(int, int item, int, size_t p, V v) const
    {
        const int si = item % this->ns;
        return cscale(cmul(v, __ldg(&densT[p])), (decltype(v.x))this->fill[si]);   // f orbital * n (:332)
    }
    __device__ V *refwd_grid(int item, int b) const { return tmp2 + ((size_t)item * 3 + (b - 1)) * this->g.N; }
    // qsum_d += f w_d phi_q (:305-328); tc2x's own sum goes through the registers
    __device__ void xyi_extra(int tj, int item, int b, size_t p, const V *v) const
    {
        if (b == 0) return;
        const size_t N = this->g.N;
        const int si = item % this->ns;
        acc_red(qsum + ((size_t)tj * 3 + (b - 1)) * N + p, to64(cmul(v[0], __ldg(&this->Rocc[(size_t)si * N + p]))),
                this->fill[si]);
        if (band)
            acc_red(acc3 + (size_t)tj * N + p, to64(cmul(__ldg(&Qt[((size_t)si * 3 + (b - 1)) * N + p]), v[0])),
                    this->fill[si] * fa4);
    }
    __device__ void xyi_accum(int tj, int item, int b, size_t p, const V *v) const
    {
        OpTC2X<T>::xyi_accum(tj, item, b, p, v);
        xyi_extra(tj, item, b, p, v);
    }
    // optional shared-memory accumulation of the extra sums (k_xyi_t6, FP32;
    // tc2x's own sum stays in registers): slots 0-2 qsum_d, 3 the band part
    static constexpr int SACC = 4;
    static constexpr bool SACC_GROUP = true;
    template <class F>
    __device__ void xyi_sgroup(int, int item, int b, size_t p, const V *v, F &&add) const
    {
        if (b == 0) return;
        const int si = item % this->ns;
        using S = decltype(v[0].x);
        const S f = (S)this->fill[si];
        add(b - 1, cscale(cmul(v[0], __ldg(&this->Rocc[(size_t)si * this->g.N + p])), f));
        if (band) add(3, cscale(cmul(__ldg(&Qt[((size_t)si * 3 + (b - 1)) * this->g.N + p]), v[0]), (S)(f * fa4)));
    }
    __device__ void xyi_sflush(int tj, int slot, size_t p, V sum) const
    {
        const size_t N = this->g.N;
        if (slot < 3) acc_red(qsum + ((size_t)tj * 3 + slot) * N + p, to64(sum), 1.0);
        else acc_red(acc3 + (size_t)tj * N + p, to64(sum), 1.0);
    }
};

// forward transform of pair products (3a2 divergence correction, :544-550)
template <typename T>
struct OpPairFwd : OpBase<T> {
    using V = typename C2<T>::t;
    static constexpr const char *NAME = "pairfwd";
    static constexpr int NF = 2, NB = 2;
    static constexpr bool ZINV = false;
    const V *A0, *B0, *A1, *B1;   // item i: conj(A0_i) B0_i, conj(A1_i) B1_i, pointers per item via strides
    const int *ia0, *ib0, *ia1, *ib1;   // per item grid indices; results: tmp slots 0, 1 (G space)
    __device__ V xyf_load(int item, int f, int, int, int, size_t p) const
    {
        const size_t N = this->g.N;
        if (f == 0) return cmulc(A0[(size_t)ia0[item] * N + p], B0[(size_t)ib0[item] * N + p]);
        return cmulc(A1[(size_t)ia1[item] * N + p], B1[(size_t)ib1[item] * N + p]);
    }
    __device__ V zmix(int, int o, int, int, int, const V *in) const
    {
        return cscale(in[o], (decltype(in[0].x))this->invN);
    }
    __device__ void xyi_accum(int, int, int, size_t, const V *) const {}
};

// band part of 3a4 / 3b5 (:848-911): targets (k, j), sources (q2sym, i2)
template <typename T>
struct OpBand : OpBase<T> {
    using V = typename C2<T>::t;
    static constexpr const char *NAME = "band";
    // input 0 = conj(chi_q2) psi_k and outputs 0-2 = its multiples; inputs 1-3
    // carry the rotated intermediates Bt (whole grid), output 3 mixes them
    static constexpr unsigned BLI = 1, BLO = 7;
    static constexpr bool ZSPLIT = false;     // one thread per z-line measured faster here
    static constexpr bool REGACC = true;
    __device__ bool regacc_grid(int) const { return true; }
    __device__ V xyi_term(int, int item, int b, size_t p, const V *v) const
    {
        const size_t N = this->g.N;
        const int si = item % this->ns;
        if (b < 3) return cmul(__ldg(&Qt[((size_t)si * 3 + b) * N + p]), v[0]);
        return cscale(cmul(v[0], __ldg(&Rocc[(size_t)si * N + p])), (decltype(v[0].x))(fb5 * fill[si]));
    }
    __device__ void xyi_flush(int tj, size_t p, V s) const { acc_red(acc + (size_t)tj * this->g.N + p, to64(s), 1.0); }
    static constexpr int NF = 4, NB = 4;
    const V *Rpsi;                // [nt][N]
    const V *Rocc, *Rchi;         // phi_q2sym, chi_q2sym [ns][N]
    const V *Qt, *Bt;             // rotated intermediates [ns][3][N]
    double2 *acc;
    const double *fill;           // f2 per source
    double fa4, fb5;
    __device__ V xyf_load(int item, int f, int, int, int, size_t p) const
    {
        const size_t N = this->g.N;
        const int tj = item / this->ns, si = item % this->ns;
        const V phj = __ldg(&Rpsi[(size_t)tj * N + p]);
        if (f == 0) return cmulc(__ldg(&Rchi[(size_t)si * N + p]), phj);   // (:865)
        return cmul(__ldg(&Bt[((size_t)si * 3 + (f - 1)) * N + p]), phj);   // (:885)
    }
    __device__ V zmix(int item, int o, int x, int y, int z, const V *in) const
    {
        using S = decltype(in[0].x);
        if constexpr (OpBase<T>::FT) {
            const float4 c = this->fco(item, this->pidx(x, y, z), 0);
            if (o < 3) return cscale(in[0], (float)(fill[item % this->ns] * fa4) * this->comp(c, o));
            V r = cscale(in[1], c.x);
            r = cadd(r, cscale(in[2], c.y));
            return cadd(r, cscale(in[3], c.z));
        }
        double G[3];
        gvec(this->rc.R, this->g, x, y, z, this->kq_of(item), G);
        const size_t p = (size_t)x + (size_t)this->g.n0 * (y + (size_t)this->g.n1 * z);
        const double u = this->tab_of(item)[p] * this->invN;
        if (o < 3) {    // f2 a4 phiphi du0_d  (:867-872)
            const double f2 = fill[item % this->ns];
            return cscale(in[0], (S)(f2 * fa4 * G[o] * u));
        }
        V r = cscale(in[1], (S)(G[0] * u));     // sum_d FFT(Bt_d phi_j) du0_d (:882-890)
        r = cadd(r, cscale(in[2], (S)(G[1] * u)));
        return cadd(r, cscale(in[3], (S)(G[2] * u)));
    }
    __device__ void xyi_accum(int tj, int item, int b, size_t p, const V *v) const
    {
        const size_t N = this->g.N;
        const int si = item % this->ns;
        double2 *a = acc + (size_t)tj * N + p;
        if (b < 3) acc_red(a, to64(cmul(__ldg(&Qt[((size_t)si * 3 + b) * N + p]), v[0])), 1.0);    // (:875)
        else acc_red(a, to64(cmul(v[0], __ldg(&Rocc[(size_t)si * N + p]))), fb5 * fill[si]);      // (:894)
    }
};

} // namespace tcg

#include "tc3.cuh"
