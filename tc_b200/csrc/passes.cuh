// passes.cuh -- the three fused pass kernels every operator term is built
// from, plus the generic 3D-FFT helpers (sphere scatter + backward FFT,
// forward FFT + sphere gather).
//
// A "pair pipeline" processes a chunk of items (target band t, occupied
// source u) as
//     XYF : NF grids per item  = XY-forward( op.xyf_load(...) )      -> tmp
//     Z   : NF tiles -> Z-forward -> op.zmix (G-space pointwise) -> NB tiles
//           -> Z-backward                                               -> tmp
//     XYI : per target, loop over the chunk's sources: XY-backward of each of
//           the NB grids, op.xyi_accum(...) folds it into R-space
//           accumulators owned by this CTA (no atomics, fixed order).
// so one exchange-type term costs two 3D FFTs of traffic per grid instead
// of two FFTs plus separate product / multiply / accumulate sweeps.
#pragma once
#include "fft.cuh"

namespace tcg {

constexpr int ZTC = 16;   // columns per Z-pass tile

template <typename V> __host__ __device__ inline size_t plane_bytes(int n0, int n1) { return sizeof(V) * (size_t)n0 * n1; }

// ------------------------------------------------------------ XYF pass ----
template <typename T, class Op>
__global__ void __launch_bounds__(256) k_xyf(Op op)
{
    using V = typename C2<T>::t;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tws = reinterpret_cast<V *>(smem_raw);
    const GridDesc &g = op.g;
    const int plane = g.n0 * g.n1;
    V *A = tws + 3 * MAXN, *B = A + plane;
    load_twiddles<V>(g, tws, 3);
    const int z = blockIdx.x, item = blockIdx.y;
    op.xyf_begin(item);
    for (int f = 0; f < Op::NF; f++) {
        for (int idx = threadIdx.x; idx < plane; idx += blockDim.x) {
            const int x = idx % g.n0, y = idx / g.n0;
            A[idx] = op.xyf_load(item, f, x, y, z, (size_t)z * plane + idx);
        }
        __syncthreads();
        V *r = fft_plane<V, -1>(A, B, tws, g);
        V *dst = op.tmp_grid(item, f) + (size_t)z * plane;
        for (int idx = threadIdx.x; idx < plane; idx += blockDim.x) dst[idx] = r[idx];
        __syncthreads();
    }
}

// -------------------------------------------------------------- Z pass ----
// smem: twiddles + NF input tiles + 2 work tiles
template <typename T, class Op>
__global__ void __launch_bounds__(256) k_z(Op op)
{
    using V = typename C2<T>::t;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tws = reinterpret_cast<V *>(smem_raw);
    const GridDesc &g = op.g;
    const int plane = g.n0 * g.n1, tile = ZTC * g.n2;
    V *in[Op::NF];
    V *base = tws + 3 * MAXN;
    for (int f = 0; f < Op::NF; f++) in[f] = base + f * tile;
    V *W0 = base + Op::NF * tile, *W1 = W0 + tile;
    load_twiddles<V>(g, tws, 4);
    const int c0 = blockIdx.x * ZTC, item = blockIdx.y;
    const int ncol = min(ZTC, plane - c0);
    op.z_begin(item);
    // load + forward along z (pointer swap keeps each result in its own slot)
    for (int f = 0; f < Op::NF; f++) {
        const V *src = op.zin_grid(item, f);
        for (int e = threadIdx.x; e < tile; e += blockDim.x) {
            const int zz = e / ZTC, cc = e % ZTC;
            in[f][e] = cc < ncol ? src[(size_t)zz * plane + c0 + cc] : czero<V>();
        }
        __syncthreads();
        V *r = fft_zcols<V, -1>(in[f], W0, tws, g, ZTC);
        if (r != in[f]) { V *t = in[f]; in[f] = r; W0 = t; }
    }
    // pointwise G-space combination, one output at a time
    for (int o = 0; o < Op::NB; o++) {
        for (int e = threadIdx.x; e < tile; e += blockDim.x) {
            const int zz = e / ZTC, cc = e % ZTC;
            V vin[Op::NF];
#pragma unroll
            for (int f = 0; f < Op::NF; f++) vin[f] = in[f][e];
            V out = czero<V>();
            if (cc < ncol) {
                const int c = c0 + cc;
                out = op.zmix(item, o, c % g.n0, c / g.n0, zz, vin);
            }
            W0[e] = out;
        }
        __syncthreads();
        V *r = Op::ZINV ? fft_zcols<V, +1>(W0, W1, tws, g, ZTC) : W0;
        V *dst = op.out_grid(item, o);
        for (int e = threadIdx.x; e < tile; e += blockDim.x) {
            const int zz = e / ZTC, cc = e % ZTC;
            if (cc < ncol) dst[(size_t)zz * plane + c0 + cc] = r[e];
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ XYI pass ----
// For each source of the target: XY-backward of the NB grids in groups of
// Op::GS (a group's planes are held together so accumulations may combine
// them, e.g. orbital * conj(orbital2)); optionally (Op::REFWD) a derived
// plane of each grid is XY-forwarded again and written to op.refwd_grid.
// smem: twiddles + (GS + 2) planes.
template <typename T, class Op>
__global__ void __launch_bounds__(256) k_xyi(Op op)
{
    using V = typename C2<T>::t;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tws = reinterpret_cast<V *>(smem_raw);
    const GridDesc &g = op.g;
    const int plane = g.n0 * g.n1;
    V *bufs = tws + 3 * MAXN;
    load_twiddles<V>(g, tws, 3);
    const int z = blockIdx.x, tj = blockIdx.y;
    const int ns = op.nsrc(tj);
    for (int si = 0; si < ns; si++) {
        const int item = op.item_of(tj, si);
        for (int b0 = 0; b0 < Op::NB; b0 += Op::GS) {
            // free list of the GS + 2 plane buffers (block-uniform)
            V *fl[Op::GS + 2];
#pragma unroll
            for (int w = 0; w < Op::GS + 2; w++) fl[w] = bufs + w * plane;
            int nfree = Op::GS + 2;
            V *res[Op::GS];
#pragma unroll
            for (int q = 0; q < Op::GS; q++) {
                V *A = fl[--nfree];
                V *S = fl[nfree - 1];
                const V *src = op.xyi_grid(item, b0 + q) + (size_t)z * plane;
                for (int idx = threadIdx.x; idx < plane; idx += blockDim.x) A[idx] = src[idx];
                __syncthreads();
                V *r = fft_plane<V, +1>(A, S, tws, g);
                res[q] = r;
                if (r != A) fl[nfree - 1] = A;   // result landed in S: A is free instead
            }
            for (int idx = threadIdx.x; idx < plane; idx += blockDim.x) {
                V vals[Op::GS];
#pragma unroll
                for (int q = 0; q < Op::GS; q++) vals[q] = res[q][idx];
                op.xyi_accum(tj, item, b0, (size_t)z * plane + idx, vals);
            }
            __syncthreads();
            if (Op::REFWD) {
                V *F0 = fl[0], *F1 = fl[1];
#pragma unroll
                for (int q = 0; q < Op::GS; q++) {
                    if (!op.refwd_want(b0 + q)) continue;
                    for (int idx = threadIdx.x; idx < plane; idx += blockDim.x)
                        F0[idx] = op.refwd_load(tj, item, b0 + q, (size_t)z * plane + idx, res[q][idx]);
                    __syncthreads();
                    V *r = fft_plane<V, -1>(F0, F1, tws, g);
                    V *dst = op.refwd_grid(item, b0 + q) + (size_t)z * plane;
                    for (int idx = threadIdx.x; idx < plane; idx += blockDim.x) dst[idx] = r[idx];
                    __syncthreads();
                }
            }
        }
    }
    op.xyi_end(tj, z);
}

// ------------------------------------------ generic 3D FFT helper passes --
// Items of a sphere -> R-space transform.
struct SphereItem {
    const double2 *coef;     // npw coefficients (G space, fp64)
    const int *inv;          // [N] grid point -> sphere index or -1
    const double2 *phase;    // [npw] phase factors
    void *out;               // [N] T2 R-space grid
    double kc[3];            // Cartesian k (gradient mode)
    int tr;                  // time reversal: conj(coef)
    int mode;                // 0 plain, 1..3: multiply by (k+G)_{mode-1}
};

// Z pass of a backward transform, loading straight from the sphere.
template <typename T>
__global__ void __launch_bounds__(256) k_sphere_z(GridDesc g, const SphereItem *items, const double *recip)
{
    using V = typename C2<T>::t;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tws = reinterpret_cast<V *>(smem_raw);
    const int plane = g.n0 * g.n1, tile = ZTC * g.n2;
    V *A = tws + 3 * MAXN, *B = A + tile;
    load_twiddles<V>(g, tws, 4);
    const SphereItem it = items[blockIdx.y];
    const int c0 = blockIdx.x * ZTC;
    const int ncol = min(ZTC, plane - c0);
    for (int e = threadIdx.x; e < tile; e += blockDim.x) {
        const int zz = e / ZTC, cc = e % ZTC;
        V v = czero<V>();
        if (cc < ncol) {
            const int c = c0 + cc;
            const size_t p = (size_t)zz * plane + c;
            const int ip = it.inv[p];
            if (ip >= 0) {
                double2 cf = it.coef[ip];
                if (it.tr) cf.y = -cf.y;
                cf = cmul(cf, it.phase[ip]);
                if (it.mode > 0) {
                    const int d = it.mode - 1;
                    const int m0 = miller(c % g.n0, g.n0), m1 = miller(c / g.n0, g.n1), m2 = miller(zz, g.n2);
                    const double Gd = recip[0 * 3 + d] * m0 + recip[1 * 3 + d] * m1 + recip[2 * 3 + d] * m2;
                    cf = cscale(cf, it.kc[d] + Gd);
                }
                v = from64<V>(cf);
            }
        }
        A[e] = v;
    }
    __syncthreads();
    V *r = fft_zcols<V, +1>(A, B, tws, g, ZTC);
    V *out = reinterpret_cast<V *>(it.out);
    for (int e = threadIdx.x; e < tile; e += blockDim.x) {
        const int zz = e / ZTC, cc = e % ZTC;
        if (cc < ncol) out[(size_t)zz * plane + c0 + cc] = r[e];
    }
}

// In-place XY pass over a list of grids (DIR = +1 backward, -1 forward).
// Grid pointers of an in-place transform list: a device array, or up to 8
// pointers passed by value (no upload, no synchronisation for short lists).
struct GridRefs {
    void *const *dev = nullptr;
    void *inl[8] = {};
    __device__ void *operator[](int i) const { return dev ? dev[i] : inl[i]; }
};

template <typename T, int DIR>
__global__ void __launch_bounds__(256) k_xy_inplace(GridDesc g, GridRefs grids)
{
    using V = typename C2<T>::t;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tws = reinterpret_cast<V *>(smem_raw);
    const int plane = g.n0 * g.n1;
    V *A = tws + 3 * MAXN, *B = A + plane;
    load_twiddles<V>(g, tws, 3);
    V *grid = reinterpret_cast<V *>(grids[blockIdx.y]) + (size_t)blockIdx.x * plane;
    for (int idx = threadIdx.x; idx < plane; idx += blockDim.x) A[idx] = grid[idx];
    __syncthreads();
    V *r = fft_plane<V, DIR>(A, B, tws, g);
    for (int idx = threadIdx.x; idx < plane; idx += blockDim.x) grid[idx] = r[idx];
}

// In-place Z pass over a list of grids, result scaled by `scale`.
template <typename T, int DIR>
__global__ void __launch_bounds__(256) k_z_inplace(GridDesc g, GridRefs grids, double scale)
{
    using V = typename C2<T>::t;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tws = reinterpret_cast<V *>(smem_raw);
    const int plane = g.n0 * g.n1, tile = ZTC * g.n2;
    V *A = tws + 3 * MAXN, *B = A + tile;
    load_twiddles<V>(g, tws, 4);
    V *grid = reinterpret_cast<V *>(grids[blockIdx.y]);
    const int c0 = blockIdx.x * ZTC;
    const int ncol = min(ZTC, plane - c0);
    for (int e = threadIdx.x; e < tile; e += blockDim.x) {
        const int zz = e / ZTC, cc = e % ZTC;
        A[e] = cc < ncol ? grid[(size_t)zz * plane + c0 + cc] : czero<V>();
    }
    __syncthreads();
    V *r = fft_zcols<V, DIR>(A, B, tws, g, ZTC);
    for (int e = threadIdx.x; e < tile; e += blockDim.x) {
        const int zz = e / ZTC, cc = e % ZTC;
        if (cc < ncol) grid[(size_t)zz * plane + c0 + cc] = cscale(r[e], (decltype(r[e].x))scale);
    }
}

// Forward Z pass + 1/N + gather onto a sphere: h[ip] += fac * grid(G).
struct GatherItem {
    const double2 *grid;     // fp64 accumulator after the forward XY pass
    const int *inv;          // [N]
    double2 *h;              // [npw] output (accumulate)
    double2 fac;             // complex factor (includes 1/N)
};

static __global__ void __launch_bounds__(256) k_gather_z(GridDesc g, const GatherItem *items)
{
    using V = double2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *tws = reinterpret_cast<V *>(smem_raw);
    const int plane = g.n0 * g.n1, tile = ZTC * g.n2;
    V *A = tws + 3 * MAXN, *B = A + tile;
    load_twiddles<V>(g, tws, 4);
    const GatherItem it = items[blockIdx.y];
    const int c0 = blockIdx.x * ZTC;
    const int ncol = min(ZTC, plane - c0);
    for (int e = threadIdx.x; e < tile; e += blockDim.x) {
        const int zz = e / ZTC, cc = e % ZTC;
        A[e] = cc < ncol ? it.grid[(size_t)zz * plane + c0 + cc] : czero<V>();
    }
    __syncthreads();
    V *r = fft_zcols<V, -1>(A, B, tws, g, ZTC);
    for (int e = threadIdx.x; e < tile; e += blockDim.x) {
        const int zz = e / ZTC, cc = e % ZTC;
        if (cc < ncol) {
            const size_t p = (size_t)zz * plane + c0 + cc;
            const int ip = it.inv[p];
            if (ip >= 0) {
                double2 v = cmul(r[e], it.fac);
                double2 h = it.h[ip];
                it.h[ip] = {h.x + v.x, h.y + v.y};
            }
        }
    }
}

} // namespace tcg
