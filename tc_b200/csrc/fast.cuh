// fast.cuh -- compile-time-size pass kernels for cubic grids N^3.
//
// Each 1D transform of length N is held by ONE thread in registers and run
// as a fully unrolled mixed-radix Stockham (all indices compile-time; no
// integer division, no barrier inside a line).  Shared memory only
// transposes planes between the x and y sweeps:
//   XY pass: P planes per CTA, thread (plane, line); global -> smem
//            (coalesced) -> row FFT (registers) -> smem -> column FFT
//            (registers) -> global straight from registers (coalesced: the
//            threads of a plane hold consecutive columns x).
//   Z pass : one thread per (x, y) pencil, loaded from / stored to global
//            straight from registers (consecutive threads = consecutive x);
//            the NF transformed inputs are staged in shared memory for the
//            G-space combination, each output is inverse-transformed in
//            registers and stored.
// Rows of a shared plane are padded to N+1 elements (odd stride for even N)
// so that the row sweeps are free of bank conflicts.
// Both XY passes also exist with each line split over a lane pair
// (k_xyf_pair / k_xyi_pair: N/2 values per thread, one radix-2 step through
// shuffles); each term picks one form per pass (Op::XYF_PAIR, Op::XYI_PAIR).
#pragma once
#include "fft.cuh"

namespace tcg {
namespace fast {

// ------------------------------------------------------ radix schedule --
__host__ __device__ constexpr int radix_at(int n, int s)
{
    // greedy: 8s, 4s, 2s, then odd primes; s-th radix
    int m = n, k = 0;
    while (m % 8 == 0) { if (k == s) return 8; m /= 8; k++; }
    while (m % 4 == 0) { if (k == s) return 4; m /= 4; k++; }
    while (m % 2 == 0) { if (k == s) return 2; m /= 2; k++; }
    for (int q = 3; m > 1; q += 2)
        while (m % q == 0) { if (k == s) return q; m /= q; k++; }
    return 1;
}
__host__ __device__ constexpr int nstages(int n)
{
    int s = 0;
    while (radix_at(n, s) > 1) s++;
    return s;
}
__host__ __device__ constexpr int ns_at(int n, int s)
{
    int p = 1;
    for (int i = 0; i < s; i++) p *= radix_at(n, i);
    return p;
}

template <typename V, int R, int DIR> __device__ __forceinline__ void dftR(V *v)
{
    if constexpr (R == 2) dft2<V, DIR>(v);
    else if constexpr (R == 3) dft3<V, DIR>(v);
    else if constexpr (R == 4) dft4<V, DIR>(v);
    else if constexpr (R == 5) dft5<V, DIR>(v);
    else if constexpr (R == 8) dft8<V, DIR>(v);
    else static_assert(R == 2, "unsupported radix in the fast path");
}

// one Stockham stage over a register array (Govindaraju et al. 2008 form)
template <typename V, int N, int DIR, int R, int NS>
__device__ __forceinline__ void rstage(const V (&a)[N], V (&b)[N], const V *__restrict__ tw)
{
    constexpr int M = N / R;
#pragma unroll
    for (int j = 0; j < M; j++) {
        const int k = j % NS;
        V v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = a[j + r * M];
        if (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; r++) {
                const int ti = k * r * (N / (NS * R));
                if (ti != 0) {
                    V w = tw[ti];
                    if (DIR > 0) w.y = -w.y;
                    v[r] = cmul(v[r], w);
                }
            }
        }
        dftR<V, R, DIR>(v);
        const int d0 = (j / NS) * NS * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) b[d0 + r * NS] = v[r];
    }
}

template <typename V, int N, int DIR, int S, bool DONE = (S >= nstages(N))>
struct Stages {
    static __device__ __forceinline__ void run(V (&a)[N], V (&b)[N], const V *tw)
    {
        rstage<V, N, DIR, radix_at(N, S), ns_at(N, S)>(a, b, tw);
        Stages<V, N, DIR, S + 1>::run(b, a, tw);
    }
};
template <typename V, int N, int DIR, int S>
struct Stages<V, N, DIR, S, true> {
    static __device__ __forceinline__ void run(V (&)[N], V (&)[N], const V *) {}
};

// In-register 1D FFT of x (result in x).  tw: N twiddles exp(-2 pi i j/N).
template <typename V, int N, int DIR>
__device__ __forceinline__ void line_fft(V (&x)[N], const V *__restrict__ tw)
{
    V y[N];
    Stages<V, N, DIR, 0>::run(x, y, tw);
    if constexpr (nstages(N) % 2 == 1) {
#pragma unroll
        for (int i = 0; i < N; i++) x[i] = y[i];
    }
}

// planes per CTA (XY passes); two plane sets must fit in 227 KB of smem
template <int N, int VB> struct Cfg {
    static constexpr int P0 = (N <= 16) ? 12 : (N <= 24 ? 8 : 4);
    static constexpr int PAD = N + ((N % 2 == 0) ? 1 : 0);           // row stride in smem
    static constexpr int P = (2 * P0 * N * PAD * VB > 200 * 1024) ? P0 / 2 : P0;
    static constexpr int THREADS = P * N;
};

// asynchronous global -> shared copy of one complex element (8 or 16 B)
template <typename V>
__device__ __forceinline__ void cp_async_elem(V *dst_smem, const V *src_gmem)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    if constexpr (sizeof(V) == 16)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src_gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src_gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

template <typename V>
__device__ __forceinline__ void stage_tw(const GridDesc &g, V *tws, int n)
{
    const V *src = twsrc<V>(g);
    for (int i = threadIdx.x; i < n; i += blockDim.x) tws[i] = src[i];   // cubic grid: axis 0 table
}

// ---------------------------------------------------------------- XYF ----
template <typename T, int N, class Op>
__global__ void __launch_bounds__(Cfg<N, sizeof(typename C2<T>::t)>::THREADS, 3) k_xyf_fast(Op op, int nplanes)
{
    using V = typename C2<T>::t;
    constexpr int P = Cfg<N, sizeof(typename C2<T>::t)>::P, PAD = Cfg<N, sizeof(typename C2<T>::t)>::PAD;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);
    V *A = tw + 128;
    stage_tw<V>(op.g, tw, N);
    const int pl = threadIdx.x / N, ln = threadIdx.x % N;
    const int pid0 = blockIdx.x * P;
    for (int f = 0; f < Op::NF; f++) {
        __syncthreads();
        // each thread fills column x = ln of its own plane (item and z fixed);
        // 12 elements (24 loads) in flight per thread
        if (pid0 + pl < nplanes) {
            const int item = (pid0 + pl) / N, z = (pid0 + pl) % N;
#pragma unroll 12
            for (int k = 0; k < N; k++)
                A[pl * N * PAD + k * PAD + ln] = op.xyf_load(item, f, ln, k, z, (size_t)z * N * N + (size_t)k * N + ln);
        }
        __syncthreads();
        V v[N];
        V *row = A + pl * N * PAD + ln * PAD;
#pragma unroll
        for (int i = 0; i < N; i++) v[i] = row[i];
        line_fft<V, N, -1>(v, tw);
#pragma unroll
        for (int i = 0; i < N; i++) row[i] = v[i];
        __syncthreads();
        const V *col = A + pl * N * PAD + ln;
#pragma unroll
        for (int i = 0; i < N; i++) v[i] = col[i * PAD];
        line_fft<V, N, -1>(v, tw);
        const int pid = pid0 + pl;
        if (pid < nplanes) {
            const int item = pid / N, z = pid % N;
            V *dst = op.tmp_grid(item, f) + (size_t)z * N * N + ln;
            if (((Op::BLI >> f) & 1) && op.m.prune) {
                // band-limited input: only the pencils its support meets are read by the Z pass
                const unsigned long long bits = op.pcol(item, ln);
#pragma unroll
                for (int i = 0; i < N; i++)
                    if ((bits >> i) & 1) dst[i * N] = v[i];
            } else {
#pragma unroll
                for (int i = 0; i < N; i++) dst[i * N] = v[i];
            }
        }
    }
}

// ------------------------------------------------------------------ Z ----
// Each z-line is split over a lane pair (s = lane & 1):
//   forward : one radix-2 DIF step across the pair via shuffles,
//             X[2k+s] = FFT_{N/2}( s ? (x[n] - x[n+N/2]) w^n : x[n] + x[n+N/2] )
//   inverse : FFT_{N/2} of the lane's half (frequencies 2k+s), then the
//             radix-2 DIT combine across the pair, y[n + s N/2] = E -+ w^-n O.
// Each thread holds N/2 values, so twice as many warps stay resident as
// with one thread per line.  Lanes keep the frequencies z = 2k+s for the
// G-space combination.  A CTA of 128 threads = 32 pencils x 2 halves x 2
// groups; group h handles inputs f = h, h+2, ... and outputs o = h, h+2, ...
template <typename V> __host__ __device__ constexpr int zcols() { return 32; }
constexpr int ZH = 2;

template <typename V>
__device__ __forceinline__ V shfl_xor1(V v)
{
    V r;
    r.x = __shfl_xor_sync(0xffffffffu, v.x, 1);
    r.y = __shfl_xor_sync(0xffffffffu, v.y, 1);
    return r;
}

// forward split transform: in natural order x[s*M + i] -> out X[2k+s]
template <typename V, int N>
__device__ __forceinline__ void fwd_split(V (&v)[N / 2], int s, const V *tw, const V *twM)
{
    constexpr int M = N / 2;
#pragma unroll
    for (int i = 0; i < M; i++) {
        const V o = shfl_xor1(v[i]);
        if (s == 0) v[i] = cadd(v[i], o);
        else {
            V d = csub(o, v[i]);              // x[i] - x[i+M]
            if (i != 0) d = cmul(d, tw[i]);
            v[i] = d;
        }
    }
    line_fft<V, M, -1>(v, twM);
}

// inverse split transform: in Y[2k+s] -> out natural y[s*M + n]
template <typename V, int N>
__device__ __forceinline__ void inv_split(V (&v)[N / 2], int s, const V *tw, const V *twM)
{
    constexpr int M = N / 2;
    line_fft<V, M, +1>(v, twM);               // s=0: E[n], s=1: O[n]
#pragma unroll
    for (int i = 0; i < M; i++) {
        const V o = shfl_xor1(v[i]);
        // s=0: y[n] = E + w^-n O ; s=1: y[n+M] = E - w^-n O
        V odd = s == 0 ? o : v[i];
        const V even = s == 0 ? v[i] : o;
        if (i != 0) { V w = tw[i]; w.y = -w.y; odd = cmul(odd, w); }
        v[i] = s == 0 ? cadd(even, odd) : csub(even, odd);
    }
}

template <typename T, int N, class Op>
__global__ void __launch_bounds__(128, Op::ZMINB) k_z_fast(Op op)
{
    using V = typename C2<T>::t;
    constexpr int TC = 32, M = N / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);   // [N]: exp(-2 pi i j/N)
    V *twM = tw + 64;                          // [M]: exp(-2 pi i j/M)
    V *S = tw + 128;                           // [NF][N][TC]
    stage_tw<V>(op.g, tw, N);
    __syncthreads();
    for (int i = threadIdx.x; i < M; i += blockDim.x) twM[i] = tw[2 * i];
    __syncthreads();
    const int item = blockIdx.y;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int s = lane & 1;
    const int cl = (w & 1) * 16 + (lane >> 1);   // pencil within the CTA
    const int h = w >> 1;                         // group
    const int c = blockIdx.x * TC + cl;
    const bool act = c < N * N;
    const int x = c % N, y = c / N;
    V v[M];
    for (int f = h; f < Op::NF; f += ZH) {
        if (act) {
            const V *src = op.zin_grid(item, f) + c + (size_t)s * M * N * N;
#pragma unroll
            for (int i = 0; i < M; i++) v[i] = src[(size_t)i * N * N];
        } else {
#pragma unroll
            for (int i = 0; i < M; i++) v[i] = czero<V>();
        }
        fwd_split<V, N>(v, s, tw, twM);
        V *st = S + f * N * TC + cl;
#pragma unroll
        for (int k = 0; k < M; k++) st[(2 * k + s) * TC] = v[k];
    }
    __syncthreads();
    for (int o = h; o < Op::NB; o += ZH) {
#pragma unroll
        for (int k = 0; k < M; k++) {
            const int z = 2 * k + s;
            V vin[Op::NF];
#pragma unroll
            for (int f = 0; f < Op::NF; f++) vin[f] = S[f * N * TC + z * TC + cl];
            v[k] = act ? op.zmix(item, o, x, y, z, vin) : czero<V>();
        }
        if (Op::ZINV) {
            inv_split<V, N>(v, s, tw, twM);
            if (act) {
                V *dst = op.out_grid(item, o) + c + (size_t)s * M * N * N;
#pragma unroll
                for (int i = 0; i < M; i++) dst[(size_t)i * N * N] = v[i];
            }
        } else if (act) {
            // G-space output: frequencies 2k+s
            V *dst = op.out_grid(item, o) + c;
#pragma unroll
            for (int k = 0; k < M; k++) dst[(size_t)(2 * k + s) * N * N] = v[k];
        }
    }
}

// Z pass variant with one thread per z-line (ZL groups of 32 pencils split
// the inputs / outputs); used by the terms whose G-space combination is
// light (tc2x, band part of tc3a2a4b2b5), where it measured faster.
constexpr int ZL = 4;
template <typename T, int N, class Op>
__global__ void __launch_bounds__(32 * ZL, Op::ZMINB) k_z_line(Op op)
{
    using V = typename C2<T>::t;
    constexpr int TC = 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);
    V *S = tw + 128;                      // [NF][N][TC]
    stage_tw<V>(op.g, tw, N);
    __syncthreads();
    const int item = blockIdx.y;
    const int lane = threadIdx.x % TC, h = threadIdx.x / TC;
    const int c = blockIdx.x * TC + lane;
    const bool act = c < N * N;
    const int x = c % N, y = c / N;
    V v[N];
    for (int f = h; f < Op::NF; f += ZL) {
        if (act) {
            const V *src = op.zin_grid(item, f) + c;
#pragma unroll
            for (int z = 0; z < N; z++) v[z] = src[(size_t)z * N * N];
        } else {
#pragma unroll
            for (int z = 0; z < N; z++) v[z] = czero<V>();
        }
        line_fft<V, N, -1>(v, tw);
        V *st = S + f * N * TC + lane;
#pragma unroll
        for (int z = 0; z < N; z++) st[z * TC] = v[z];
    }
    __syncthreads();
    for (int o = h; o < Op::NB; o += ZL) {
#pragma unroll
        for (int z = 0; z < N; z++) {
            V vin[Op::NF];
#pragma unroll
            for (int f = 0; f < Op::NF; f++) vin[f] = S[f * N * TC + z * TC + lane];
            v[z] = act ? op.zmix(item, o, x, y, z, vin) : czero<V>();
        }
        if (Op::ZINV) line_fft<V, N, +1>(v, tw);
        if (act) {
            V *dst = op.out_grid(item, o) + c;
#pragma unroll
            for (int z = 0; z < N; z++) dst[(size_t)z * N * N] = v[z];
        }
    }
}

// ---------------------------------------------------------------- XYI ----
// smem: twiddles + GS planes-of-P (results of a group) + 1 work set
template <typename T, int N, class Op>
__global__ void __launch_bounds__(Cfg<N, sizeof(typename C2<T>::t)>::THREADS, 2) k_xyi_fast(Op op, int nplanes)
{
    using V = typename C2<T>::t;
    constexpr int P = Cfg<N, sizeof(typename C2<T>::t)>::P, PAD = Cfg<N, sizeof(typename C2<T>::t)>::PAD;
    constexpr int PS = P * N * PAD;       // one set of P planes
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);
    V *W = tw + 128;                      // [GS + 1][P][N][PAD]
    stage_tw<V>(op.g, tw, N);
    const int pl = threadIdx.x / N, ln = threadIdx.x % N;
    const int pid0 = blockIdx.x * P;
    const int mypid = pid0 + pl;
    const bool mine = mypid < nplanes;
    const int tj = mine ? mypid / N : 0, z = mypid % N;
    // all planes of the CTA must belong to targets with the same source count
    const int ns = op.nsrc(pid0 / N);
    // register accumulation only in the FP32 path (an FP64 column would
    // double the register footprint of the line FFT)
    constexpr bool RACC = Op::REGACC && sizeof(V) == 8;
    // BOUT: one accumulator per output grid b (GS == 1); the b loop runs
    // outside the source loop and each b's column sum is flushed on its own
    constexpr bool BOUT = RACC && Op::BOUTER;
    static_assert(!BOUT || Op::GS == 1, "per-output accumulation needs GS == 1");
    V racc[RACC ? N : 1];
    for (int bo = 0; bo < (BOUT ? Op::NB : 1); bo++) {
#pragma unroll
    for (int i = 0; i < (RACC ? N : 1); i++) racc[i] = czero<V>();
    for (int si = 0; si < ns; si++) {
        for (int b0 = BOUT ? bo : 0; b0 < (BOUT ? bo + 1 : Op::NB); b0 += Op::GS) {
            V *keepc = W + PS + pl * N * PAD + ln;      // set 1, this thread's column
#pragma unroll
            for (int q = 0; q < Op::GS; q++) {
                V *A = W;
                __syncthreads();
                // plane copies global -> smem without passing through registers
                if (mine) {   // column x = ln of this thread's own plane
                    const V *src = op.xyi_grid(op.item_of(tj, si), b0 + q) + (size_t)z * N * N + ln;
#pragma unroll
                    for (int k = 0; k < N; k++) cp_async_elem(A + pl * N * PAD + k * PAD + ln, src + (size_t)k * N);
                }
                cp_async_wait_all();
                __syncthreads();
                V v[N];
                V *row = A + pl * N * PAD + ln * PAD;
#pragma unroll
                for (int i = 0; i < N; i++) v[i] = row[i];
                line_fft<V, N, +1>(v, tw);
#pragma unroll
                for (int i = 0; i < N; i++) row[i] = v[i];
                __syncthreads();
                const V *colp = A + pl * N * PAD + ln;
#pragma unroll
                for (int i = 0; i < N; i++) v[i] = colp[i * PAD];
                line_fft<V, N, +1>(v, tw);
                if (Op::GS > 1 && q < Op::GS - 1) {
                    // keep this grid's column (thread-private) for the group accumulation
#pragma unroll
                    for (int i = 0; i < N; i++) keepc[i * PAD] = v[i];
                } else if (mine) {
                    const int item = op.item_of(tj, si);
                    if (RACC && op.regacc_grid(b0)) {
#pragma unroll
                        for (int yy = 0; yy < N; yy++) {
                            V vals[1] = {v[yy]};
                            racc[yy] = cadd(racc[yy], op.xyi_term(tj, item, b0, (size_t)z * N * N + (size_t)yy * N + ln, vals));
                            if constexpr (Op::RACC_EXTRA) op.xyi_extra(tj, item, b0, (size_t)z * N * N + (size_t)yy * N + ln, vals);
                        }
                    } else {
#pragma unroll
                        for (int yy = 0; yy < N; yy++) {
                            V vals[Op::GS];
                            if constexpr (Op::GS > 1) { vals[0] = keepc[yy * PAD]; vals[Op::GS - 1] = v[yy]; }
                            else vals[0] = v[yy];
                            op.xyi_accum(tj, item, b0, (size_t)z * N * N + (size_t)yy * N + ln, vals);
                        }
                    }
                }
                if (Op::REFWD && Op::GS == 1) {
                    // derived plane: column values -> forward column FFT -> smem -> forward rows -> global
                    const bool want = op.refwd_want(b0);
                    if (want) {
                        // per-output sums wait in this thread's own column of the
                        // read set (no other thread touches it until the next
                        // load), which frees their registers for the two FFTs
                        V *stash = A + pl * N * PAD + ln;
                        if constexpr (BOUT) {
#pragma unroll
                            for (int i = 0; i < N; i++) stash[i * PAD] = racc[i];
                        }
                        const int item = op.item_of(tj, si);
#pragma unroll
                        for (int yy = 0; yy < N; yy++)
                            v[yy] = mine ? op.refwd_load(tj, item, b0, (size_t)z * N * N + (size_t)yy * N + ln, v[yy])
                                         : czero<V>();
                        line_fft<V, N, -1>(v, tw);
                        V *B = W + PS;          // work set
                        V *cb = B + pl * N * PAD + ln;
#pragma unroll
                        for (int i = 0; i < N; i++) cb[i * PAD] = v[i];
                        __syncthreads();
                        V *rb = B + pl * N * PAD + ln * PAD;
#pragma unroll
                        for (int i = 0; i < N; i++) v[i] = rb[i];
                        line_fft<V, N, -1>(v, tw);
#pragma unroll
                        for (int i = 0; i < N; i++) rb[i] = v[i];
                        __syncthreads();
                        if (mine) {
                            V *dstp = op.refwd_grid(op.item_of(tj, si), b0) + (size_t)z * N * N + ln;
#pragma unroll 4
                            for (int k = 0; k < N; k++) dstp[(size_t)k * N] = B[pl * N * PAD + k * PAD + ln];
                        }
                        if constexpr (BOUT) {
#pragma unroll
                            for (int i = 0; i < N; i++) racc[i] = stash[i * PAD];
                        }
                    }
                }
            }
        }
    }
    if constexpr (BOUT) {
        if (mine && op.regacc_grid(bo)) {
#pragma unroll
            for (int yy = 0; yy < N; yy++) op.xyi_flush_b(tj, bo, (size_t)z * N * N + (size_t)yy * N + ln, racc[yy]);
        }
    }
    }
    if (RACC && !BOUT && mine) {
#pragma unroll
        for (int yy = 0; yy < N; yy++) op.xyi_flush(tj, (size_t)z * N * N + (size_t)yy * N + ln, racc[yy]);
    }
}

// XYI with the next plane set prefetched: for terms without re-forwarded or
// grouped grids (GS == 1, no REFWD) the two plane sets alternate, and the
// asynchronous copies of step it + 1 (source, output grid) are in flight
// while step it is transformed and accumulated.
template <typename T, int N, class Op>
__global__ void __launch_bounds__(Cfg<N, sizeof(typename C2<T>::t)>::THREADS, 2) k_xyi_pf(Op op, int nplanes)
{
    using V = typename C2<T>::t;
    static_assert(Op::GS == 1, "prefetching XYI handles ungrouped outputs only");
    constexpr int P = Cfg<N, sizeof(V)>::P, PAD = Cfg<N, sizeof(V)>::PAD;
    constexpr int PS = P * N * PAD;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);
    V *W = tw + 128;                      // [2][P][N][PAD], alternating
    stage_tw<V>(op.g, tw, N);
    const int pl = threadIdx.x / N, ln = threadIdx.x % N;
    const int pid0 = blockIdx.x * P;
    const int mypid = pid0 + pl;
    const bool mine = mypid < nplanes;
    const int tj = mine ? mypid / N : 0, z = mypid % N;
    const int ns = op.nsrc(pid0 / N);
    constexpr bool RACC = Op::REGACC && sizeof(V) == 8;
    static_assert(!(RACC && Op::REFWD), "re-forwarded outputs accumulate through xyi_accum");
    V racc[RACC ? N : 1];
#pragma unroll
    for (int i = 0; i < (RACC ? N : 1); i++) racc[i] = czero<V>();
    const int total = ns * Op::NB;        // steps: it = si * NB + b
    auto issue = [&](int it) {
        if (mine) {
            const V *src = op.xyi_grid(op.item_of(tj, it / Op::NB), it % Op::NB) + (size_t)z * N * N + ln;
            V *dst = W + (it & 1) * PS + pl * N * PAD + ln;
#pragma unroll
            for (int k = 0; k < N; k++) cp_async_elem(dst + k * PAD, src + (size_t)k * N);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    issue(0);
    for (int it = 0; it < total; it++) {
        __syncthreads();                  // every thread is done with the set that step it + 1 overwrites
        if (it + 1 < total) {
            issue(it + 1);
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        __syncthreads();
        const int si = it / Op::NB, b0 = it % Op::NB;
        V *A = W + (it & 1) * PS;
        V v[N];
        V *row = A + pl * N * PAD + ln * PAD;
#pragma unroll
        for (int i = 0; i < N; i++) v[i] = row[i];
        line_fft<V, N, +1>(v, tw);
#pragma unroll
        for (int i = 0; i < N; i++) row[i] = v[i];
        __syncthreads();
        const V *colp = A + pl * N * PAD + ln;
#pragma unroll
        for (int i = 0; i < N; i++) v[i] = colp[i * PAD];
        line_fft<V, N, +1>(v, tw);
        if (mine) {
            const int item = op.item_of(tj, si);
            if (RACC && op.regacc_grid(b0)) {
#pragma unroll
                for (int yy = 0; yy < N; yy++) {
                    V vals[1] = {v[yy]};
                    racc[yy] = cadd(racc[yy], op.xyi_term(tj, item, b0, (size_t)z * N * N + (size_t)yy * N + ln, vals));
                    if constexpr (Op::RACC_EXTRA) op.xyi_extra(tj, item, b0, (size_t)z * N * N + (size_t)yy * N + ln, vals);
                }
            } else {
#pragma unroll
                for (int yy = 0; yy < N; yy++) {
                    V vals[1] = {v[yy]};
                    op.xyi_accum(tj, item, b0, (size_t)z * N * N + (size_t)yy * N + ln, vals);
                }
            }
        }
        if (Op::REFWD && op.refwd_want(b0)) {   // uniform over the CTA
            // derived plane, transformed forward in place in the current set:
            // columns (registers) -> own column -> rows -> global
            __syncthreads();                      // every column of the set has been read
            const int item = op.item_of(tj, si);
#pragma unroll
            for (int yy = 0; yy < N; yy++)
                v[yy] = mine ? op.refwd_load(tj, item, b0, (size_t)z * N * N + (size_t)yy * N + ln, v[yy]) : czero<V>();
            line_fft<V, N, -1>(v, tw);
            V *cb = A + pl * N * PAD + ln;
#pragma unroll
            for (int i = 0; i < N; i++) cb[i * PAD] = v[i];
            __syncthreads();
#pragma unroll
            for (int i = 0; i < N; i++) v[i] = row[i];
            line_fft<V, N, -1>(v, tw);
#pragma unroll
            for (int i = 0; i < N; i++) row[i] = v[i];
            __syncthreads();
            if (mine) {
                V *dstp = op.refwd_grid(item, b0) + (size_t)z * N * N + ln;
#pragma unroll 4
                for (int k = 0; k < N; k++) dstp[(size_t)k * N] = A[pl * N * PAD + k * PAD + ln];
            }
        }
    }
    if (RACC && mine) {
#pragma unroll
        for (int yy = 0; yy < N; yy++) op.xyi_flush(tj, (size_t)z * N * N + (size_t)yy * N + ln, racc[yy]);
    }
}

// ------------------------------- XY and Z passes, several threads per line --
// For N = TL * M with TL | M (36 = 6 x 6, 48 = 4 x 12) each line is
// transformed by TL threads in two stages (Cooley-Tukey, n = t + TL m,
// k = k1 + M k2), exchanged once through the plane in shared memory:
//   stage 1, thread t: u_t[k1] = w_N^{t k1} DFT_M over m of x[t + TL m];
//   stage 2, thread t for k1 = t + TL c (c < M / TL):
//            X[k1 + M k2] = DFT_TL over t' of u_t'[k1].
// Thread t holds the line at positions t + TL m (m < M) both before and after
// the transform: X[t + TL m'] in v[m'], m' = c + (M / TL) k2.  A thread
// holds M values instead of N, so a CTA of one plane (TL N threads) needs
// few registers and many CTAs stay resident.  Thread mapping r = t * N + l:
// consecutive lanes own consecutive lines l, so the row sweeps (odd stride
// PAD) and the column sweeps (stride 1 across lanes) are free of bank
// conflicts and the global copies are coalesced along x.
namespace t6 {
template <int N_, int TL_> struct Shape {
    static constexpr int N = N_, TL = TL_, M = N_ / TL_;
    static constexpr int PAD = N_ + ((N_ % 2 == 0) ? 1 : 0);
    static constexpr int THREADS = TL_ * N_;     // XY passes: one plane per CTA
    static constexpr int ZTHREADS = TL_ * 32;    // Z passes: 32 pencils per CTA
    // resident CTAs per SM the launch bounds ask for (register budget)
    static constexpr int MINB = M <= 6 ? 4 : 4;
    static constexpr int MINB_ZR = M <= 6 ? 3 : 2;
    static_assert(N_ % (TL_ * TL_) == 0, "two-stage lines need TL | N / TL");
    static_assert(N_ <= 64 && M <= 32 && TL_ <= 32, "pencil masks and twiddle slots");
};
// threads per line of each compiled grid size (0: one-thread-per-line forms only)
template <int N> struct ShapeOf { static constexpr int TL = 0; };
template <> struct ShapeOf<36> { static constexpr int TL = 6; };
template <> struct ShapeOf<48> { static constexpr int TL = 4; };

template <typename V>
struct Tw {
    const V *w;    // [N]  exp(-2 pi i j/N)
    const V *wm;   // [M]  exp(-2 pi i j/M)
    const V *wt;   // [TL] exp(-2 pi i j/TL)
};

// stage 1 of thread t on u[m] = x[t + TL m]: DFT_M, then the twiddles
template <typename V, class S, int DIR>
__device__ __forceinline__ void stage1(V (&u)[S::M], int t, const Tw<V> &tw)
{
    line_fft<V, S::M, DIR>(u, tw.wm);
#pragma unroll
    for (int k1 = 1; k1 < S::M; k1++) {
        V w = tw.w[t * k1];
        if (DIR > 0) w.y = -w.y;
        u[k1] = cmul(u[k1], w);
    }
}
// stage 2 of thread t from the exchanged values (u_j[k1] at
// base[(k1 TL + j) stride]): X[t + TL m'] into v[m']
template <typename V, class S, int DIR>
__device__ __forceinline__ void stage2(const V *base, int stride, int t, const Tw<V> &tw, V (&v)[S::M])
{
    constexpr int C = S::M / S::TL;
#pragma unroll
    for (int c = 0; c < C; c++) {
        const int k1 = t + S::TL * c;
        V w[S::TL];
#pragma unroll
        for (int j = 0; j < S::TL; j++) w[j] = base[(k1 * S::TL + j) * stride];
        line_fft<V, S::TL, DIR>(w, tw.wt);
#pragma unroll
        for (int k2 = 0; k2 < S::TL; k2++) v[c + C * k2] = w[k2];
    }
}

// line element i at base[i * stride]; all threads of the CTA call it.
// On return v[m] = X[t + TL m]; NAT: also written back in natural order.
template <typename V, class S, int DIR, bool NAT>
__device__ __forceinline__ void xform(V *base, int stride, int t, const Tw<V> &tw, V (&v)[S::M])
{
    V u[S::M];
#pragma unroll
    for (int m = 0; m < S::M; m++) u[m] = base[(t + S::TL * m) * stride];
    stage1<V, S, DIR>(u, t, tw);
    __syncthreads();
#pragma unroll
    for (int k1 = 0; k1 < S::M; k1++) base[(k1 * S::TL + t) * stride] = u[k1];
    __syncthreads();
    stage2<V, S, DIR>(base, stride, t, tw, v);
    if (NAT) {
        __syncthreads();
#pragma unroll
        for (int m = 0; m < S::M; m++) base[(t + S::TL * m) * stride] = v[m];
        __syncthreads();
    }
}

// twiddle tables in shared memory: N at 0, M at 64, TL at 96 (128 slots)
template <typename V, class S>
__device__ __forceinline__ Tw<V> stage(const GridDesc &g, V *tws)
{
    const V *src = twsrc<V>(g);
    for (int i = threadIdx.x; i < S::N; i += blockDim.x) tws[i] = src[i];
    __syncthreads();
    if (threadIdx.x < S::M) tws[64 + threadIdx.x] = tws[S::TL * threadIdx.x];
    if (threadIdx.x < S::TL) tws[96 + threadIdx.x] = tws[S::M * threadIdx.x];
    __syncthreads();
    return Tw<V>{tws, tws + 64, tws + 96};
}

// XYF: one (item, z) plane per CTA; pair products -> forward XY FFT -> tmp
template <typename T, class Op, class S>
__global__ void __launch_bounds__(S::THREADS, S::MINB) k_xyf_t6(Op op, int nplanes)
{
    using V = typename C2<T>::t;
    constexpr int N = S::N, TL = S::TL, M = S::M, PAD = S::PAD;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tws = reinterpret_cast<V *>(smem_raw);
    V *A = tws + 128;                     // [N][PAD]
    const Tw<V> tw = stage<V, S>(op.g, tws);
    const int t = threadIdx.x / N, l = threadIdx.x % N;
    const int pid = blockIdx.x;
    if (pid >= nplanes) return;           // uniform over the CTA
    const int item = pid / N, z = pid % N;
    const size_t pz = (size_t)z * N * N;
    for (int f = 0; f < Op::NF; f++) {
        __syncthreads();
#pragma unroll
        for (int m = 0; m < M; m++) {
            const int y = t + TL * m;
            A[y * PAD + l] = op.xyf_load(item, f, l, y, z, pz + (size_t)y * N + l);
        }
        __syncthreads();
        V v[M];
        xform<V, S, -1, true>(A + l * PAD, 1, t, tw, v);      // rows
        xform<V, S, -1, false>(A + l, PAD, t, tw, v);         // columns: v[m] at y = t + TL m
        V *dst = op.tmp_grid(item, f) + pz + l;
        if (((Op::BLI >> f) & 1) && op.m.prune) {
            const unsigned long long bits = op.pcol(item, l);
#pragma unroll
            for (int m = 0; m < M; m++)
                if ((bits >> (t + TL * m)) & 1) dst[(size_t)(t + TL * m) * N] = v[m];
        } else {
#pragma unroll
            for (int m = 0; m < M; m++) dst[(size_t)(t + TL * m) * N] = v[m];
        }
    }
}

// shared-memory accumulation of one output group (GS outputs in vals): the
// op's own xyi_sgroup, or its single slot xyi_slot(b0) (called on the derived
// op type, so that its overrides apply)
template <class Op, typename V, class F>
__device__ __forceinline__ void sacc_group(const Op &op, int tj, int item, int b0, size_t p, const V *vals, F &&add)
{
    if constexpr (Op::SACC_GROUP) {
        op.xyi_sgroup(tj, item, b0, p, vals, add);
    } else {
        const int slot = op.xyi_slot(b0);
        if (slot >= 0) add(slot, op.xyi_sterm(tj, item, b0, p, vals[Op::GS - 1]));
    }
}

// XYI: one (target, z) plane per CTA, looping over the chunk's (source,
// output) steps; the next step's plane is copied asynchronously into the
// second set.  GS > 1: the first GS - 1 outputs of a group wait in registers.
// (Op::XYI_MINB_EXTRA: more resident CTAs, FP32 at 36^3, for ops that fit the
// smaller register budget)
template <typename T, class Op, class S>
__global__ void __launch_bounds__(S::THREADS, S::MINB + ((S::M <= 6 && sizeof(T) == 4) ? Op::XYI_MINB_EXTRA : 0))
    k_xyi_t6(Op op, int nplanes)
{
    using V = typename C2<T>::t;
    constexpr int N = S::N, TL = S::TL, M = S::M, PAD = S::PAD;
    constexpr int PS = N * PAD;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tws = reinterpret_cast<V *>(smem_raw);
    V *W = tws + 128;                     // [2][N][PAD]
    const Tw<V> tw = stage<V, S>(op.g, tws);
    const int t = threadIdx.x / N, l = threadIdx.x % N;
    const int pid = blockIdx.x;
    if (pid >= nplanes) return;           // uniform over the CTA
    const int tj = pid / N, z = pid % N;
    const size_t pz = (size_t)z * N * N;
    const int ns = op.nsrc(tj);
    constexpr bool RACC = Op::REGACC && sizeof(V) == 8;
    constexpr int SA = sizeof(V) == 8 ? Op::SACC : 0;    // shared-memory accumulator planes (FP32)
    const bool sa_on = SA > 0 && op.sacc_on;
    const int nsa = sa_on ? op.sacc_n : 0;                // planes in use
    static_assert(!(Op::REFWD && Op::GS > 1), "re-forward needs GS == 1");
    static_assert(!(SA > 0 && RACC && !Op::RACC_EXTRA), "shared-memory accumulation replaces the register form");
    static_assert(!(SA > 0 && Op::GS > 1 && !Op::SACC_GROUP), "grouped outputs need the op's xyi_sgroup");
    V racc[M], keep[Op::GS][M];
#pragma unroll
    for (int i = 0; i < M; i++) racc[i] = czero<V>();
    V *SAcc = W + 2 * PS;                 // [SA][N][N]: this thread owns y = t + TL m, x = l
    // pruned chunks: the pencil-table entry of every source, looked up once
    // (the copies of each step then need one load of their column mask)
    int *sent = reinterpret_cast<int *>(SAcc + (size_t)nsa * N * N);
    if (op.m.prune) {
        for (int si = threadIdx.x; si < ns; si += blockDim.x) sent[si] = op.pent_of(op.item_of(tj, si));
        __syncthreads();
    }
    for (int a = 0; a < nsa; a++)
#pragma unroll
        for (int m = 0; m < M; m++) SAcc[(a * N + t + TL * m) * N + l] = czero<V>();
    const int total = ns * Op::NB;        // it = si * NB + b
    auto issue = [&](int it) {
        const int item = op.item_of(tj, it / Op::NB), b = it % Op::NB;
        const V *src = op.xyi_grid(item, b) + pz + l;
        V *dst = W + (it & 1) * PS + l;
        if (((Op::BLO >> b) & 1) && op.m.prune) {
            // band-limited output: the Z pass wrote only the pencils its support meets
            const unsigned long long bits = op.m.pbits[(size_t)sent[it / Op::NB] * op.g.n0 + l];
#pragma unroll
            for (int m = 0; m < M; m++) {
                if ((bits >> (t + TL * m)) & 1) cp_async_elem(dst + (t + TL * m) * PAD, src + (size_t)(t + TL * m) * N);
                else dst[(t + TL * m) * PAD] = czero<V>();
            }
        } else {
#pragma unroll
            for (int m = 0; m < M; m++) cp_async_elem(dst + (t + TL * m) * PAD, src + (size_t)(t + TL * m) * N);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    issue(0);
    for (int it = 0; it < total; it++) {
        __syncthreads();                  // the set that step it + 1 overwrites is no longer read
        if (it + 1 < total) {
            issue(it + 1);
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        __syncthreads();
        const int si = it / Op::NB, b = it % Op::NB, q = b % Op::GS, b0 = b - q;
        V *A = W + (it & 1) * PS;
        V v[M];
        xform<V, S, +1, true>(A + l * PAD, 1, t, tw, v);      // rows
        xform<V, S, +1, false>(A + l, PAD, t, tw, v);         // columns: v[m] at y = t + TL m
        if (Op::GS > 1 && q < Op::GS - 1) {
#pragma unroll
            for (int m = 0; m < M; m++) keep[q][m] = v[m];
            continue;
        }
        const int item = op.item_of(tj, si);
        const bool rg = RACC && op.regacc_grid(b0);
        if (rg) {
#pragma unroll
            for (int m = 0; m < M; m++) {
                V vals[1] = {v[m]};
                racc[m] = cadd(racc[m], op.xyi_term(tj, item, b0, pz + (size_t)(t + TL * m) * N + l, vals));
                if constexpr (Op::RACC_EXTRA)
                    if (!sa_on) op.xyi_extra(tj, item, b0, pz + (size_t)(t + TL * m) * N + l, vals);
            }
        }
        if (sa_on) {
            // this thread owns the accumulator points (x = l, y = t + TL m) of every slot;
            // with the register form the slots hold the op's other accumulators
#pragma unroll
            for (int m = 0; m < M; m++) {
                V vals[Op::GS];
#pragma unroll
                for (int g = 0; g < Op::GS - 1; g++) vals[g] = keep[g][m];
                vals[Op::GS - 1] = v[m];
                sacc_group(op, tj, item, b0, pz + (size_t)(t + TL * m) * N + l, vals, [&](int slot, V x) {
                    V *a = &SAcc[(slot * N + t + TL * m) * N + l];
                    *a = cadd(*a, x);
                });
            }
        } else if (rg) {
        } else {
#pragma unroll
            for (int m = 0; m < M; m++) {
                V vals[Op::GS];
#pragma unroll
                for (int g = 0; g < Op::GS - 1; g++) vals[g] = keep[g][m];
                vals[Op::GS - 1] = v[m];
                op.xyi_accum(tj, item, b0, pz + (size_t)(t + TL * m) * N + l, vals);
            }
        }
        if (Op::REFWD && op.refwd_want(b0)) {   // uniform over the CTA
            // derived plane (orbital x density) -> forward XY FFT in place -> global
            __syncthreads();                      // the column sweep has read the set
#pragma unroll
            for (int m = 0; m < M; m++) {
                const int y = t + TL * m;
                A[y * PAD + l] = op.refwd_load(tj, item, b0, pz + (size_t)y * N + l, v[m]);
            }
            __syncthreads();
            xform<V, S, -1, true>(A + l, PAD, t, tw, v);      // columns
            xform<V, S, -1, true>(A + l * PAD, 1, t, tw, v);  // rows
            V *dst = op.refwd_grid(item, b0) + pz + l;
#pragma unroll
            for (int m = 0; m < M; m++) dst[(size_t)(t + TL * m) * N] = A[(t + TL * m) * PAD + l];
        }
    }
    if (RACC) {
#pragma unroll
        for (int m = 0; m < M; m++) op.xyi_flush(tj, pz + (size_t)(t + TL * m) * N + l, racc[m]);
    }
    for (int a = 0; a < nsa; a++)
#pragma unroll
        for (int m = 0; m < M; m++)
            op.xyi_sflush(tj, a, pz + (size_t)(t + TL * m) * N + l, SAcc[(a * N + t + TL * m) * N + l]);
}
// shared memory of k_xyi_t6: twiddles, `sets` plane sets, `slots` FP32
// accumulator planes (0 unless the op's SACC path is on)
template <typename V, class Op, class S> __host__ inline size_t smem_xyi(int sets, int slots)
{
    return sizeof(V) * (128 + (size_t)sets * S::N * S::PAD + (sizeof(V) == 8 ? (size_t)slots * S::N * S::N : 0));
}

// Z pass: one item and 32 consecutive pencils (x, y) per CTA, TL threads
// per z-line (warp t owns z = t + TL m of all 32 pencils).  The NF inputs are
// transformed in place in S[f][z][32]; each output is combined into O[z][32]
// and transformed back from there.
// (Op::Z_MINB_EXTRA: more resident CTAs, FP32 at 36^3, for ops that fit the
// smaller register budget)
template <typename T, class Op, class S>
__global__ void __launch_bounds__(S::ZTHREADS, S::MINB + ((S::M <= 6 && sizeof(T) == 4) ? Op::Z_MINB_EXTRA : 0))
    k_z_t6(Op op)
{
    using V = typename C2<T>::t;
    constexpr int N = S::N, TL = S::TL, M = S::M, TC = 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tws = reinterpret_cast<V *>(smem_raw);
    V *Sb = tws + 128;                    // [NF][N][TC]
    // [N][TC] output plane: its own, or input plane Op::ZO_ALIAS (each thread
    // overwrites only the points it has just read for the first output, and
    // the later outputs read input 0 only)
    V *O = Sb + (Op::ZO_ALIAS >= 0 ? Op::ZO_ALIAS : Op::NF) * N * TC;
    const Tw<V> tw = stage<V, S>(op.g, tws);
    const int item = blockIdx.y;
    const int t = threadIdx.x / TC, cl = threadIdx.x % TC;
    // pruning: the CTA takes its 32 pencils from the pair's list (active
    // pencils first); a CTA past the active ones skips the band-limited
    // inputs (zero) and outputs (never read)
    const bool prune = op.m.prune != 0;
    const int slot = blockIdx.x * TC + cl;
    int c = slot;
    bool allin = false, pon = true;
    if (prune) {
        const int e = op.pent_of(item);
        allin = blockIdx.x * TC >= op.m.pnact[e];
        if (slot < N * N) {
            c = op.m.pperm[(size_t)e * op.m.np + slot];
            pon = slot < op.m.pnact[e];
        }
    }
    const bool act = slot < N * N;
    const int x = c % N, y = c / N;
#pragma unroll
    for (int f = 0; f < Op::NF; f++) {
        const bool bl = prune && ((Op::BLI >> f) & 1);
        const V *src = op.zin_grid(item, f) + c;
#pragma unroll
        for (int m = 0; m < M; m++) {
            const int z = t + TL * m;
            Sb[(f * N + z) * TC + cl] = (act && (!bl || pon)) ? src[(size_t)z * N * N] : czero<V>();
        }
    }
    __syncthreads();
    V v[M];
#pragma unroll
    for (int f = 0; f < Op::NF; f++)
        if (!(allin && ((Op::BLI >> f) & 1))) xform<V, S, -1, true>(Sb + f * N * TC + cl, TC, t, tw, v);
    for (int o = 0; o < Op::NB; o++) {
        const bool blo = prune && ((Op::BLO >> o) & 1);
        if (blo && allin) continue;       // uniform over the CTA
        if (Op::ZINV) __syncthreads();    // the previous output's sweep has read O
#pragma unroll
        for (int m = 0; m < M; m++) {
            const int z = t + TL * m;
            V vin[Op::NF];
#pragma unroll
            for (int f = 0; f < Op::NF; f++) vin[f] = Sb[(f * N + z) * TC + cl];
            const V r = act ? op.zmix(item, o, x, y, z, vin) : czero<V>();
            if (Op::ZINV) O[z * TC + cl] = r;
            else if (act) op.out_grid(item, o)[c + (size_t)z * N * N] = r;   // G-space output
        }
        if (Op::ZINV) {
            __syncthreads();
            xform<V, S, +1, false>(O + cl, TC, t, tw, v);   // v[m] at z = t + TL m
            if (act && (!blo || pon)) {
                V *dst = op.out_grid(item, o) + c;
#pragma unroll
                for (int m = 0; m < M; m++) dst[(size_t)(t + TL * m) * N * N] = v[m];
            }
        }
    }
}
template <typename V, class S, class Op> __host__ inline size_t smem_z()
{
    return sizeof(V) * (128 + (size_t)(Op::NF + (Op::ZO_ALIAS >= 0 ? 0 : 1)) * S::N * 32);
}
// Z pass with the transformed inputs kept in registers: thread (t, pencil)
// runs stage 1 of each input's z-line straight from global memory
// (z = t + TL m), exchanges once through shared memory, and after stage 2
// holds every input at z = t + TL m -- the points where it evaluates the
// G-space combination of every output.  Those values are already in the
// input order of the inverse transform's stage 1, so each output needs one
// exchange only.  Shared memory: one exchange buffer per input.
// (Op::ZR_MINB_EXTRA: more resident CTAs, FP32 at 36^3, for ops that fit the
// smaller register budget)
template <typename T, class Op, class S>
__global__ void __launch_bounds__(S::ZTHREADS, S::MINB_ZR + ((S::M <= 6 && sizeof(T) == 4) ? Op::ZR_MINB_EXTRA : 0))
    k_z_t6r(Op op)
{
    using V = typename C2<T>::t;
    constexpr int N = S::N, TL = S::TL, M = S::M, TC = 32, NF = Op::NF;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tws = reinterpret_cast<V *>(smem_raw);
    V *E = tws + 128;                     // [NF][N][TC] exchange buffers
    const Tw<V> tw = stage<V, S>(op.g, tws);
    const int item = blockIdx.y;
    const int t = threadIdx.x / TC, cl = threadIdx.x % TC;
    // pruning as in k_z_t6 (band-limited inputs read as zero off their support)
    const bool prune = op.m.prune != 0;
    const int slot = blockIdx.x * TC + cl;
    int c = slot;
    bool allin = false, pon = true;
    if (prune) {
        const int e = op.pent_of(item);
        allin = blockIdx.x * TC >= op.m.pnact[e];
        if (slot < N * N) {
            c = op.m.pperm[(size_t)e * op.m.np + slot];
            pon = slot < op.m.pnact[e];
        }
    }
    const bool act = slot < N * N;
    const int x = c % N, y = c / N;
    V X[NF][M];
#pragma unroll
    for (int f = 0; f < NF; f++) {
        const bool bl = prune && ((Op::BLI >> f) & 1);
        const V *src = op.zin_grid(item, f) + c;
#pragma unroll
        for (int m = 0; m < M; m++) X[f][m] = (act && (!bl || pon)) ? src[(size_t)(t + TL * m) * N * N] : czero<V>();
    }
#pragma unroll
    for (int f = 0; f < NF; f++) {
        stage1<V, S, -1>(X[f], t, tw);
#pragma unroll
        for (int k1 = 0; k1 < M; k1++) E[(f * N + k1 * TL + t) * TC + cl] = X[f][k1];
    }
    __syncthreads();
#pragma unroll
    for (int f = 0; f < NF; f++) stage2<V, S, -1>(E + f * N * TC + cl, TC, t, tw, X[f]);   // input f at z = t + TL m
    for (int o = 0; o < Op::NB; o++) {
        const bool blo = prune && ((Op::BLO >> o) & 1);
        if (blo && allin) continue;       // uniform over the CTA
        V v[M];
#pragma unroll
        for (int m = 0; m < M; m++) {
            V vin[NF];
#pragma unroll
            for (int f = 0; f < NF; f++) vin[f] = X[f][m];
            v[m] = act ? op.zmix(item, o, x, y, t + TL * m, vin) : czero<V>();
        }
        if (Op::ZINV) {
            // inverse: stage 1 over m in registers, one exchange, stage 2
            stage1<V, S, +1>(v, t, tw);
            __syncthreads();                  // the exchange buffer is free
#pragma unroll
            for (int k1 = 0; k1 < M; k1++) E[(k1 * TL + t) * TC + cl] = v[k1];
            __syncthreads();
            stage2<V, S, +1>(E + cl, TC, t, tw, v);   // v[m] at z = t + TL m
        }
        if (act && (!blo || pon)) {
            V *dst = op.out_grid(item, o) + c;
#pragma unroll
            for (int m = 0; m < M; m++) dst[(size_t)(t + TL * m) * N * N] = v[m];
        }
    }
}
template <typename V, class S> __host__ inline size_t smem_zr(int nf)
{
    return sizeof(V) * (128 + (size_t)nf * S::N * 32);
}

template <typename V, class S> __host__ inline size_t smem(int sets)
{
    return sizeof(V) * (128 + (size_t)sets * S::N * S::PAD);
}
} // namespace t6

// ------------------------------------------------- XY passes, line pairs --
// The same XY passes with each row / column split over a lane pair
// (s = lane & 1, as in the Z pass): half the registers per thread, so twice
// the warps stay resident.  Forward lines: natural halves x = s M + i in,
// frequencies 2k + s out (fwd_split); inverse lines: frequencies 2k + s in,
// natural halves out (inv_split).  Pairs are adjacent lanes, so a CTA holds
// whole warps: P N is a multiple of 16.
__host__ __device__ constexpr int gcd_c(int a, int b) { return b == 0 ? a : gcd_c(b, a % b); }
template <int N, int VB> struct CfgP {
    static constexpr int Q = 16 / gcd_c(N, 16);
    static constexpr int P = (96 + Q * N - 1) / (Q * N) * Q;         // >= 96 lines per CTA
    static constexpr int PAD = N + ((N % 2 == 0) ? 1 : 0);
    static constexpr int THREADS = 2 * P * N;
    // register cap: FP32 keeps >= 16 warps per SM, FP64 one CTA's worth
    static constexpr int CTAS = VB == 8 ? (512 + THREADS - 1) / THREADS : 1;
    static constexpr int REG0 = (65536 / (CTAS * THREADS)) & ~7;
    static constexpr int REG = REG0 < 168 ? REG0 : 168;
    static_assert(THREADS % 32 == 0, "line pairs need whole warps");
};

template <typename T, int N, class Op>
__global__ void __launch_bounds__(CfgP<N, sizeof(typename C2<T>::t)>::THREADS)
    __maxnreg__((CfgP<N, sizeof(typename C2<T>::t)>::REG)) k_xyf_pair(Op op, int nplanes)
{
    using V = typename C2<T>::t;
    using CF = CfgP<N, sizeof(V)>;
    constexpr int P = CF::P, PAD = CF::PAD, M = N / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);   // [N]
    V *twM = tw + 64;                          // [M]
    V *A = tw + 128;
    stage_tw<V>(op.g, tw, N);
    __syncthreads();
    for (int i = threadIdx.x; i < M; i += blockDim.x) twM[i] = tw[2 * i];
    const int s = threadIdx.x & 1, pi = threadIdx.x >> 1;
    const int pl = pi / N, ln = pi % N;
    const int pid0 = blockIdx.x * P;
    for (int f = 0; f < Op::NF; f++) {
        __syncthreads();
        // the 2N threads of a plane fill it: element r0 + 2 k N, r0 = 2 ln + s
        if (pid0 + pl < nplanes) {
            const int item = (pid0 + pl) / N, z = (pid0 + pl) % N;
            const int r0 = 2 * ln + s, x0 = r0 % N, y0 = r0 / N;
#pragma unroll 6
            for (int k = 0; k < M; k++) {
                const int y = y0 + 2 * k;
                A[pl * N * PAD + y * PAD + x0] = op.xyf_load(item, f, x0, y, z, (size_t)z * N * N + (size_t)y * N + x0);
            }
        }
        __syncthreads();
        V v[M];
        V *row = A + pl * N * PAD + ln * PAD;
#pragma unroll
        for (int i = 0; i < M; i++) v[i] = row[s * M + i];
        fwd_split<V, N>(v, s, tw, twM);
        __syncwarp();
#pragma unroll
        for (int k = 0; k < M; k++) row[2 * k + s] = v[k];
        __syncthreads();
        const V *col = A + pl * N * PAD + ln;
#pragma unroll
        for (int i = 0; i < M; i++) v[i] = col[(s * M + i) * PAD];
        fwd_split<V, N>(v, s, tw, twM);
        const int pid = pid0 + pl;
        if (pid < nplanes) {
            const int item = pid / N, z = pid % N;
            V *dst = op.tmp_grid(item, f) + (size_t)z * N * N + ln;
#pragma unroll
            for (int k = 0; k < M; k++) dst[(2 * k + s) * N] = v[k];
        }
    }
}

template <typename T, int N, class Op>
__global__ void __launch_bounds__(CfgP<N, sizeof(typename C2<T>::t)>::THREADS)
    __maxnreg__((CfgP<N, sizeof(typename C2<T>::t)>::REG)) k_xyi_pair(Op op, int nplanes)
{
    using V = typename C2<T>::t;
    using CF = CfgP<N, sizeof(V)>;
    constexpr int P = CF::P, PAD = CF::PAD, M = N / 2;
    constexpr int PS = P * N * PAD;       // one set of P planes
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tw = reinterpret_cast<V *>(smem_raw);
    V *twM = tw + 64;
    V *W = tw + 128;                      // [2][P][N][PAD]: read set, keep / work set
    stage_tw<V>(op.g, tw, N);
    __syncthreads();
    for (int i = threadIdx.x; i < M; i += blockDim.x) twM[i] = tw[2 * i];
    const int s = threadIdx.x & 1, pi = threadIdx.x >> 1;
    const int pl = pi / N, ln = pi % N;
    const int pid0 = blockIdx.x * P;
    const int mypid = pid0 + pl;
    const bool mine = mypid < nplanes;
    const int tj = mine ? mypid / N : 0, z = mypid % N;
    // all planes of the CTA must belong to targets with the same source count
    const int ns = op.nsrc(pid0 / N);
    constexpr bool RACC = Op::REGACC && sizeof(V) == 8;
    constexpr bool BOUT = RACC && Op::BOUTER;
    static_assert(!BOUT || Op::GS == 1, "per-output accumulation needs GS == 1");
    // this thread's rows y = s M + n of its column, as element offsets
    const size_t pz = (size_t)z * N * N + ln + (size_t)s * M * N;
    // plane copies: this thread moves elements r0 + 2 k N of its own plane
    const int r0 = 2 * ln + s, x0 = r0 % N, y0 = r0 / N;
    V racc[RACC ? M : 1];
    for (int bo = 0; bo < (BOUT ? Op::NB : 1); bo++) {
#pragma unroll
        for (int i = 0; i < (RACC ? M : 1); i++) racc[i] = czero<V>();
        for (int si = 0; si < ns; si++) {
            for (int b0 = BOUT ? bo : 0; b0 < (BOUT ? bo + 1 : Op::NB); b0 += Op::GS) {
                V *keepc = W + PS + pl * N * PAD + ln + s * M * PAD;   // set 1: this thread's half column
#pragma unroll
                for (int q = 0; q < Op::GS; q++) {
                    V *A = W;
                    __syncthreads();
                    if (mine) {   // element r0 + 2 k N of this thread's own plane
                        const V *src = op.xyi_grid(op.item_of(tj, si), b0 + q) + (size_t)z * N * N + (size_t)y0 * N + x0;
                        V *dsm = A + pl * N * PAD + y0 * PAD + x0;
#pragma unroll
                        for (int k = 0; k < M; k++) cp_async_elem(dsm + 2 * k * PAD, src + (size_t)2 * k * N);
                    }
                    cp_async_wait_all();
                    __syncthreads();
                    V v[M];
                    V *row = A + pl * N * PAD + ln * PAD;
#pragma unroll
                    for (int k = 0; k < M; k++) v[k] = row[2 * k + s];
                    inv_split<V, N>(v, s, tw, twM);
                    __syncwarp();
#pragma unroll
                    for (int i = 0; i < M; i++) row[s * M + i] = v[i];
                    __syncthreads();
                    V *colp = A + pl * N * PAD + ln;
#pragma unroll
                    for (int k = 0; k < M; k++) v[k] = colp[(2 * k + s) * PAD];
                    inv_split<V, N>(v, s, tw, twM);            // v[n]: row y = s M + n
                    if (Op::GS > 1 && q < Op::GS - 1) {
#pragma unroll
                        for (int i = 0; i < M; i++) keepc[i * PAD] = v[i];
                    } else if (mine) {
                        const int item = op.item_of(tj, si);
                        if (RACC && op.regacc_grid(b0)) {
#pragma unroll
                            for (int i = 0; i < M; i++) {
                                V vals[1] = {v[i]};
                                racc[i] = cadd(racc[i], op.xyi_term(tj, item, b0, pz + (size_t)i * N, vals));
                                if constexpr (Op::RACC_EXTRA) op.xyi_extra(tj, item, b0, pz + (size_t)i * N, vals);
                            }
                        } else {
#pragma unroll
                            for (int i = 0; i < M; i++) {
                                V vals[Op::GS];
                                if constexpr (Op::GS > 1) { vals[0] = keepc[i * PAD]; vals[Op::GS - 1] = v[i]; }
                                else vals[0] = v[i];
                                op.xyi_accum(tj, item, b0, pz + (size_t)i * N, vals);
                            }
                        }
                    }
                    if (Op::REFWD && Op::GS == 1) {
                        const bool want = op.refwd_want(b0);   // uniform over the CTA
                        if (want) {
                            // the column sums wait in the slots this thread read
                            V *stash = colp + s * PAD;
                            if constexpr (BOUT) {
#pragma unroll
                                for (int k = 0; k < M; k++) stash[2 * k * PAD] = racc[k];
                            }
                            const int item = op.item_of(tj, si);
#pragma unroll
                            for (int i = 0; i < M; i++)
                                v[i] = mine ? op.refwd_load(tj, item, b0, pz + (size_t)i * N, v[i]) : czero<V>();
                            fwd_split<V, N>(v, s, tw, twM);          // frequencies y = 2k + s
                            V *B = W + PS;
                            V *cb = B + pl * N * PAD + ln;
#pragma unroll
                            for (int k = 0; k < M; k++) cb[(2 * k + s) * PAD] = v[k];
                            __syncthreads();
                            V *rb = B + pl * N * PAD + ln * PAD;
#pragma unroll
                            for (int i = 0; i < M; i++) v[i] = rb[s * M + i];
                            fwd_split<V, N>(v, s, tw, twM);
                            __syncwarp();
#pragma unroll
                            for (int k = 0; k < M; k++) rb[2 * k + s] = v[k];
                            __syncthreads();
                            if (mine) {
                                V *dstp = op.refwd_grid(op.item_of(tj, si), b0) + (size_t)z * N * N + (size_t)y0 * N + x0;
                                const V *bs = B + pl * N * PAD + y0 * PAD + x0;
#pragma unroll 6
                                for (int k = 0; k < M; k++) dstp[(size_t)2 * k * N] = bs[2 * k * PAD];
                            }
                            if constexpr (BOUT) {
#pragma unroll
                                for (int k = 0; k < M; k++) racc[k] = stash[2 * k * PAD];
                            }
                        }
                    }
                }
            }
        }
        if constexpr (BOUT) {
            if (mine && op.regacc_grid(bo)) {
#pragma unroll
                for (int i = 0; i < M; i++) op.xyi_flush_b(tj, bo, pz + (size_t)i * N, racc[i]);
            }
        }
    }
    if (RACC && !BOUT && mine) {
#pragma unroll
        for (int i = 0; i < M; i++) op.xyi_flush(tj, pz + (size_t)i * N, racc[i]);
    }
}

template <typename V, int N> __host__ inline size_t smem_xy_pair(int sets)
{
    return sizeof(V) * (128 + (size_t)sets * CfgP<N, sizeof(V)>::P * N * CfgP<N, sizeof(V)>::PAD);
}

template <typename V, int N> __host__ inline size_t smem_xy_fast(int sets)
{
    return sizeof(V) * (128 + (size_t)sets * Cfg<N, sizeof(V)>::P * N * Cfg<N, sizeof(V)>::PAD);
}
template <typename V, int N> __host__ inline size_t smem_z_fast(int nf)
{
    return sizeof(V) * (128 + (size_t)nf * N * zcols<V>());
}

} // namespace fast
} // namespace tcg
