// fft.cuh -- batched 3D FFT building blocks for sm_100a.
//
// A 3D transform of an n0 x n1 x n2 grid (x fastest, TC++'s layout,
// plane_wave_basis.cpp:205-216) is split into two passes over HBM/L2:
//   * XY pass: one CTA owns one z-plane (n1 rows x n0 columns) of one grid,
//     transforms along x then y entirely in shared memory;
//   * Z pass : one CTA owns TC consecutive (x,y) columns of all n2 planes
//     (TC contiguous elements per plane -> coalesced), transforms along z.
// Both passes call user hooks for the element loads / stores, so pair
// products, Coulomb / Jastrow kernel multiplies and the accumulation into
// H psi are fused into the FFT prologue / epilogue instead of separate
// sweeps over the grid.
//
// 1D transforms are self-sorting Stockham, mixed radix {2,3,4,5,8 + generic
// prime}, ping-ponging between two shared-memory buffers (one barrier per
// radix stage).  Twiddles are computed in FP64 on the host and staged in
// shared memory (w[j] = exp(-2 pi i j / n)); the FP32 path rounds them once.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tcg {

constexpr int MAXN = 128;       // max grid length per axis
constexpr int MAXST = 12;       // max radix stages per axis

struct Axis {
    int n, nst;
    int R[MAXST];
};

struct GridDesc {
    int n0, n1, n2, N;
    Axis ax[3];
    const double2 *tw64;        // [3][MAXN] device twiddles, fp64
    const float2 *tw32;         // [3][MAXN] device twiddles, fp32
};

// ---------------------------------------------------------------- complex --
template <typename T> struct C2;
template <> struct C2<double> { using t = double2; };
template <> struct C2<float> { using t = float2; };

template <typename V> __device__ __forceinline__ V cadd(V a, V b) { return {a.x + b.x, a.y + b.y}; }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { return {a.x - b.x, a.y - b.y}; }
template <typename V> __device__ __forceinline__ V cmul(V a, V b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
// conj(a) * b
template <typename V> __device__ __forceinline__ V cmulc(V a, V b) { return {a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x}; }
template <typename V, typename S> __device__ __forceinline__ V cscale(V a, S s) { return {a.x * s, a.y * s}; }
template <typename V> __device__ __forceinline__ V cconj(V a) { return {a.x, -a.y}; }
// i * s * a  (s = +-1)
template <typename V> __device__ __forceinline__ V cmuli(V a, int s) { return s > 0 ? V{-a.y, a.x} : V{a.y, -a.x}; }

__device__ __forceinline__ double2 to64(double2 a) { return a; }
__device__ __forceinline__ double2 to64(float2 a) { return {(double)a.x, (double)a.y}; }
template <typename V> __device__ __forceinline__ V from64(double2 a);
template <> __device__ __forceinline__ double2 from64<double2>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 from64<float2>(double2 a) { return {(float)a.x, (float)a.y}; }
template <typename V> __device__ __forceinline__ V czero() { return {0, 0}; }

// ------------------------------------------------------------ radix DFTs --
// DIR = -1 forward (exp(-i...)), +1 backward.
template <typename V, int DIR> __device__ __forceinline__ void dft2(V *v)
{
    V a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}
template <typename V, int DIR> __device__ __forceinline__ void dft3(V *v)
{
    using S = decltype(v[0].x);
    const S h = (S)0.86602540378443864676;   // sin(2 pi / 3)
    V a = v[0], b = v[1], c = v[2];
    V t1 = cadd(b, c);
    V t2 = {a.x - (S)0.5 * t1.x, a.y - (S)0.5 * t1.y};
    V t3 = cmuli(cscale(csub(b, c), h), DIR);
    v[0] = cadd(a, t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
}
template <typename V, int DIR> __device__ __forceinline__ void dft4(V *v)
{
    V a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    V b0 = cadd(v[1], v[3]), b1 = cmuli(csub(v[1], v[3]), DIR);
    v[0] = cadd(a0, b0);
    v[1] = cadd(a1, b1);
    v[2] = csub(a0, b0);
    v[3] = csub(a1, b1);
}
template <typename V, int DIR> __device__ __forceinline__ void dft5(V *v)
{
    using S = decltype(v[0].x);
    const S c1 = (S)0.30901699437494742410, c2 = (S)-0.80901699437494742410;   // cos(2pi/5), cos(4pi/5)
    const S s1 = (S)0.95105651629515357212, s2 = (S)0.58778525229247312917;    // sin(2pi/5), sin(4pi/5)
    V a = v[0];
    V t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    V t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    V m1 = {a.x + c1 * t1.x + c2 * t2.x, a.y + c1 * t1.y + c2 * t2.y};
    V m2 = {a.x + c2 * t1.x + c1 * t2.x, a.y + c2 * t1.y + c1 * t2.y};
    V n1 = cmuli(V{s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y}, DIR);
    V n2 = cmuli(V{s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y}, DIR);
    v[0] = cadd(a, cadd(t1, t2));
    v[1] = cadd(m1, n1);
    v[4] = csub(m1, n1);
    v[2] = cadd(m2, n2);
    v[3] = csub(m2, n2);
}
template <typename V, int DIR> __device__ __forceinline__ void dft8(V *v)
{
    using S = decltype(v[0].x);
    const S r = (S)0.70710678118654752440;   // 1/sqrt(2)
    // radix-2 x radix-4 split: even / odd halves
    V e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    dft4<V, DIR>(e);
    dft4<V, DIR>(o);
    // twiddles w8^k, k = 0..3 : 1, (1 + DIR i) r, DIR i, (-1 + DIR i) r
    V o1 = {r * (o[1].x - DIR * o[1].y), r * (o[1].y + DIR * o[1].x)};
    V o2 = cmuli(o[2], DIR);
    V o3 = {r * (-o[3].x - DIR * o[3].y), r * (-o[3].y + DIR * o[3].x)};
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
}

// One Stockham stage with compile-time radix R on B sequences of length n
// (element stride es, sequence stride ss).  src -> dst.
template <typename V, int R, int DIR>
__device__ __forceinline__ void stage(const V *__restrict__ src, V *__restrict__ dst, const V *tw, int n,
                                      int Ns, int B, int es, int ss, bool seq_fast)
{
    const int m = n / R;
    const int items = B * m;
    const int wstep = n / (Ns * R);
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        int seq, j;
        if (seq_fast) { seq = it % B; j = it / B; }
        else { j = it % m; seq = it / m; }
        const V *s = src + seq * ss;
        V *d = dst + seq * ss;
        const int k = j % Ns;
        V v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = s[(j + r * m) * es];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; r++) {
                V w = tw[k * r * wstep];
                if (DIR > 0) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        if (R == 2) dft2<V, DIR>(v);
        else if (R == 3) dft3<V, DIR>(v);
        else if (R == 4) dft4<V, DIR>(v);
        else if (R == 5) dft5<V, DIR>(v);
        else if (R == 8) dft8<V, DIR>(v);
        const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) d[(idxD + r * Ns) * es] = v[r];
    }
}

// generic prime radix via the twiddle table
template <typename V, int DIR>
__device__ __forceinline__ void stage_generic(const V *__restrict__ src, V *__restrict__ dst, const V *tw, int n,
                                              int R, int Ns, int B, int es, int ss, bool seq_fast)
{
    const int m = n / R;
    const int items = B * m;
    const int wstep = n / (Ns * R);
    const int rstep = n / R;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        int seq, j;
        if (seq_fast) { seq = it % B; j = it / B; }
        else { j = it % m; seq = it / m; }
        const V *s = src + seq * ss;
        V *d = dst + seq * ss;
        const int k = j % Ns;
        V v[16];
        for (int r = 0; r < R; r++) {
            V x = s[(j + r * m) * es];
            if (Ns > 1 && r > 0) {
                V w = tw[k * r * wstep];
                if (DIR > 0) w.y = -w.y;
                x = cmul(x, w);
            }
            v[r] = x;
        }
        const int idxD = (j / Ns) * Ns * R + k;
        for (int q = 0; q < R; q++) {
            V acc = czero<V>();
            for (int r = 0; r < R; r++) {
                V w = tw[((r * q) % R) * rstep];
                if (DIR > 0) w.y = -w.y;
                acc = cadd(acc, cmul(v[r], w));
            }
            d[(idxD + q * Ns) * es] = acc;
        }
    }
}

// Full 1D transform along one axis of data held in smem buffer a (scratch
// b).  Returns the buffer holding the result (a or b).
template <typename V, int DIR>
__device__ V *fft_axis(V *a, V *b, const V *tw, const Axis &ax, int B, int es, int ss, bool seq_fast)
{
    int Ns = 1;
    for (int st = 0; st < ax.nst; st++) {
        const int R = ax.R[st];
        switch (R) {
        case 2: stage<V, 2, DIR>(a, b, tw, ax.n, Ns, B, es, ss, seq_fast); break;
        case 3: stage<V, 3, DIR>(a, b, tw, ax.n, Ns, B, es, ss, seq_fast); break;
        case 4: stage<V, 4, DIR>(a, b, tw, ax.n, Ns, B, es, ss, seq_fast); break;
        case 5: stage<V, 5, DIR>(a, b, tw, ax.n, Ns, B, es, ss, seq_fast); break;
        case 8: stage<V, 8, DIR>(a, b, tw, ax.n, Ns, B, es, ss, seq_fast); break;
        default: stage_generic<V, DIR>(a, b, tw, ax.n, R, Ns, B, es, ss, seq_fast); break;
        }
        __syncthreads();
        V *t = a; a = b; b = t;
        Ns *= R;
    }
    return a;
}

// Stage the three axes' twiddles into shared memory (3 x MAXN).
template <typename V> __device__ __forceinline__ const V *twsrc(const GridDesc &g);
template <> __device__ __forceinline__ const double2 *twsrc<double2>(const GridDesc &g) { return g.tw64; }
template <> __device__ __forceinline__ const float2 *twsrc<float2>(const GridDesc &g) { return g.tw32; }

template <typename V>
__device__ __forceinline__ void load_twiddles(const GridDesc &g, V *tws, int axes_mask)
{
    const V *src = twsrc<V>(g);
    for (int d = 0; d < 3; d++) {
        if (!(axes_mask & (1 << d))) continue;
        for (int i = threadIdx.x; i < g.ax[d].n; i += blockDim.x) tws[d * MAXN + i] = src[d * MAXN + i];
    }
}

// XY transform of one plane held in smem (a, scratch b); returns result buffer.
template <typename V, int DIR>
__device__ __forceinline__ V *fft_plane(V *a, V *b, const V *tws, const GridDesc &g)
{
    V *r = fft_axis<V, DIR>(a, b, tws + 0 * MAXN, g.ax[0], g.n1, 1, g.n0, false);
    V *o = (r == a) ? b : a;
    return fft_axis<V, DIR>(r, o, tws + 1 * MAXN, g.ax[1], g.n0, g.n0, 1, true);
}

// Z transform of a tile of TCc columns x n2 planes (element (z, c) at z*TCc + c).
template <typename V, int DIR>
__device__ __forceinline__ V *fft_zcols(V *a, V *b, const V *tws, const GridDesc &g, int TCc)
{
    return fft_axis<V, DIR>(a, b, tws + 2 * MAXN, g.ax[2], TCc, TCc, 1, true);
}

// signed Miller index of grid coordinate i along an axis of length n
// (PlaneWaveBasis::get_Gvector, plane_wave_basis.cpp:205-216)
__device__ __forceinline__ int miller(int i, int n) { return i <= n / 2 ? i : i - n; }

} // namespace tcg
