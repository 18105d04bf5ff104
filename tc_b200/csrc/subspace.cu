// subspace.cu -- the dense band-by-band part of the block Davidson on the
// device, in FP64 (Diagonalization::block_davidson, diagonalization_davidson.cpp:
// 462-600; diagonalization_utils.cpp:7-119):
//   tcg_subspace_ritz   H_n,sub = Vref^H (H_n V) (ZGEMM), H_sub = sum_n H_n,sub,
//                       H_sub X = X D (general complex eigensolve, cuSOLVER
//                       Xgeev), eigenpairs sorted by the real part, X^-1 (LU),
//                       Ritz vectors V X and left vectors Vref (X^-1)^H (ZGEMM),
//                       energies diag(Xl^H H_n,sub X)
//   tcg_gram_schmidt    Gram_Schmidt / Gram_Schmidt_biortho of a block of vectors
//   tcg_davidson_expand the new trial vectors of one block: preconditioned
//                       residuals (make_a_new_trial_vector), each orthonormalised
//                       against the basis and appended unless it vanishes
// The band-by-band contractions are plain library GEMMs (cuBLAS ZGEMM runs
// them on the FP64 tensor pipe); the eigensolve and LU are cuSOLVER.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include "../../include/tcg.h"

namespace tcg {
void set_error(const char *fmt, ...);
}

namespace {

int fail(int code, const char *msg)
{
    tcg::set_error("%s", msg);
    return code;
}

#define SUB_CUDA(call)                                                                                        \
    do {                                                                                                      \
        cudaError_t e_ = (call);                                                                              \
        if (e_ != cudaSuccess) {                                                                              \
            tcg::set_error("CUDA error %s at %s:%d", cudaGetErrorString(e_), __FILE__, __LINE__);             \
            return TCG_ERR_CUDA;                                                                              \
        }                                                                                                     \
    } while (0)
#define SUB_BLAS(call)                                                                                        \
    do {                                                                                                      \
        cublasStatus_t e_ = (call);                                                                           \
        if (e_ != CUBLAS_STATUS_SUCCESS) {                                                                    \
            tcg::set_error("cuBLAS error %d at %s:%d", (int)e_, __FILE__, __LINE__);                          \
            return TCG_ERR_CUDA;                                                                              \
        }                                                                                                     \
    } while (0)
#define SUB_SOLV(call)                                                                                        \
    do {                                                                                                      \
        cusolverStatus_t e_ = (call);                                                                         \
        if (e_ != CUSOLVER_STATUS_SUCCESS) {                                                                  \
            tcg::set_error("cuSOLVER error %d at %s:%d", (int)e_, __FILE__, __LINE__);                        \
            return TCG_ERR_CUDA;                                                                              \
        }                                                                                                     \
    } while (0)

struct Handles {
    cublasHandle_t blas = nullptr;
    cusolverDnHandle_t solver = nullptr;
    cusolverDnParams_t params = nullptr;
};
std::mutex g_mu;
Handles g_h[64];

int handles(Handles **out)
{
    int dev = 0;
    SUB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(TCG_ERR_UNSUPPORTED, "device index >= 64");
    std::lock_guard<std::mutex> lk(g_mu);
    Handles &h = g_h[dev];
    if (!h.blas) {
        SUB_BLAS(cublasCreate(&h.blas));
        SUB_SOLV(cusolverDnCreate(&h.solver));
        SUB_SOLV(cusolverDnCreateParams(&h.params));
    }
    *out = &h;
    return TCG_OK;
}

// scratch of one call, freed on return
struct Scratch {
    std::vector<void *> p;
    ~Scratch()
    {
        for (void *q : p) cudaFree(q);
    }
    int get(void **out, size_t bytes)
    {
        *out = nullptr;
        if (cudaMalloc(out, std::max<size_t>(bytes, 16)) != cudaSuccess) {
            cudaGetLastError();
            return fail(TCG_ERR_NOMEM, "device allocation failed");
        }
        p.push_back(*out);
        return TCG_OK;
    }
};

__global__ void k_add3(int n, const double2 *a, const double2 *b, const double2 *c, double2 *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double2 s = {0, 0};
    if (a) s = {s.x + a[i].x, s.y + a[i].y};
    if (b) s = {s.x + b[i].x, s.y + b[i].y};
    if (c) s = {s.x + c[i].x, s.y + c[i].y};
    out[i] = s;
}

// column permutation (col-major n x n): out[:, j] = in[:, perm[j]]
__global__ void k_permute_cols(int n, const int *perm, const double2 *in, double2 *out)
{
    const int j = blockIdx.x;
    for (int r = threadIdx.x; r < n; r += blockDim.x) out[(size_t)j * n + r] = in[(size_t)perm[j] * n + r];
}

// identity (col-major n x n)
__global__ void k_identity(int n, double2 *a)
{
    const int j = blockIdx.x;
    for (int r = threadIdx.x; r < n; r += blockDim.x) a[(size_t)j * n + r] = make_double2(r == j ? 1.0 : 0.0, 0.0);
}

// conjugate transpose (col-major n x n)
__global__ void k_adjoint(int n, const double2 *in, double2 *out)
{
    const int j = blockIdx.x;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        const double2 v = in[(size_t)r * n + j];
        out[(size_t)j * n + r] = make_double2(v.x, -v.y);
    }
}

// e[i] = sum_{a,b} conj(L[a,i]) H[a,b] X[b,i]   (col-major, i < nout)
__global__ void k_diag_form(int n, int nout, const double2 *L, const double2 *H, const double2 *X, double2 *e)
{
    const int i = blockIdx.x;
    if (i >= nout) return;
    __shared__ double2 red[256];
    double2 s = {0, 0};
    for (int ab = threadIdx.x; ab < n * n; ab += blockDim.x) {
        const int a = ab % n, b = ab / n;
        const double2 l = L[(size_t)i * n + a], h = H[(size_t)b * n + a], x = X[(size_t)i * n + b];
        const double2 hx = {h.x * x.x - h.y * x.y, h.x * x.y + h.y * x.x};
        s.x += l.x * hx.x + l.y * hx.y;
        s.y += l.x * hx.y - l.y * hx.x;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] = {red[threadIdx.x].x + red[threadIdx.x + k].x,
                                                 red[threadIdx.x].y + red[threadIdx.x + k].y};
        __syncthreads();
    }
    if (threadIdx.x == 0) e[i] = red[0];
}

// one step of Gram-Schmidt on vector j: target -= <ref_i|target> basis_i for
// i < j, in order (modified Gram-Schmidt, as the reference's loop updates the
// target after each projection); one block
__global__ void k_gs_project(int npw, int j, const double2 *ref, const double2 *basis, double2 *target)
{
    __shared__ double2 red[256];
    for (int i = 0; i < j; i++) {
        const double2 *r = ref + (size_t)i * npw;
        double2 s = {0, 0};
        for (int p = threadIdx.x; p < npw; p += blockDim.x) {
            const double2 a = r[p], b = target[p];
            s.x += a.x * b.x + a.y * b.y;
            s.y += a.x * b.y - a.y * b.x;
        }
        red[threadIdx.x] = s;
        __syncthreads();
        for (int k = blockDim.x / 2; k > 0; k >>= 1) {
            if (threadIdx.x < k) red[threadIdx.x] = {red[threadIdx.x].x + red[threadIdx.x + k].x,
                                                     red[threadIdx.x].y + red[threadIdx.x + k].y};
            __syncthreads();
        }
        const double2 c = red[0];
        __syncthreads();
        const double2 *bs = basis + (size_t)i * npw;
        for (int p = threadIdx.x; p < npw; p += blockDim.x) {
            const double2 b = bs[p];
            target[p].x -= c.x * b.x - c.y * b.y;
            target[p].y -= c.x * b.y + c.y * b.x;
        }
        __syncthreads();
    }
}

// <a|b> into out (one block)
__global__ void k_dotc(int npw, const double2 *a, const double2 *b, double2 *out)
{
    __shared__ double2 red[256];
    double2 s = {0, 0};
    for (int p = threadIdx.x; p < npw; p += blockDim.x) {
        s.x += a[p].x * b[p].x + a[p].y * b[p].y;
        s.y += a[p].x * b[p].y - a[p].y * b[p].x;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] = {red[threadIdx.x].x + red[threadIdx.x + k].x,
                                                 red[threadIdx.x].y + red[threadIdx.x + k].y};
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// v /= c (complex), c read from the device
__global__ void k_scale_inv(int npw, const double2 *c, int conj_c, double2 *v)
{
    double2 d = *c;
    if (conj_c) d.y = -d.y;
    const double den = d.x * d.x + d.y * d.y;
    const double2 inv = {d.x / den, -d.y / den};
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npw; p += gridDim.x * blockDim.x) {
        const double2 a = v[p];
        v[p] = {a.x * inv.x - a.y * inv.y, a.x * inv.y + a.y * inv.x};
    }
}

// make_a_new_trial_vector (diagonalization_utils.cpp:165-211) for vector b
// of a block, one CTA each: with the kinetic expectation
// t = <phi| |k+G|^2 |phi> / <phi|phi> and x = |k+G|^2 / t, the Payne
// preconditioner K(x) = (27 + 18x + 12x^2 + 8x^3) / (27 + 18x + 12x^2 + 8x^3 + 16x^4)
// gives dst = -K (H phi - e phi), normalised, or zero when its norm is below 1e-8
__global__ void k_precondition(int npw, const double *kg2, const double2 *phi, const double2 *h1, const double2 *h2,
                               const double2 *h3, const double2 *eig, double2 *dst)
{
    __shared__ double ra[256], rb[256];
    const size_t off = (size_t)blockIdx.x * npw;
    double a = 0, n = 0;
    for (int p = threadIdx.x; p < npw; p += blockDim.x) {
        const double2 v = phi[off + p];
        const double q = v.x * v.x + v.y * v.y;
        a += kg2[p] * q;
        n += q;
    }
    ra[threadIdx.x] = a;
    rb[threadIdx.x] = n;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) {
            ra[threadIdx.x] += ra[threadIdx.x + k];
            rb[threadIdx.x] += rb[threadIdx.x + k];
        }
        __syncthreads();
    }
    const double kin = ra[0] / rb[0];
    const double2 e = eig[blockIdx.x];
    __syncthreads();
    double s = 0;
    for (int p = threadIdx.x; p < npw; p += blockDim.x) {
        const double x = kg2[p] / kin;
        const double c = (27 + x * (18 + x * (12 + x * 8))) / (27 + x * (18 + x * (12 + x * (8 + x * 16))));
        const double2 v = phi[off + p];
        double2 r = {-(e.x * v.x - e.y * v.y), -(e.x * v.y + e.y * v.x)};
        if (h1) r = {r.x + h1[off + p].x, r.y + h1[off + p].y};
        if (h2) r = {r.x + h2[off + p].x, r.y + h2[off + p].y};
        if (h3) r = {r.x + h3[off + p].x, r.y + h3[off + p].y};
        const double2 o = {-c * r.x, -c * r.y};
        dst[off + p] = o;
        s += o.x * o.x + o.y * o.y;
    }
    ra[threadIdx.x] = s;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) ra[threadIdx.x] += ra[threadIdx.x + k];
        __syncthreads();
    }
    const double nrm = sqrt(ra[0]);
    const double scale = nrm < 1e-8 ? 0.0 : 1.0 / nrm;
    for (int p = threadIdx.x; p < npw; p += blockDim.x) {
        const double2 o = dst[off + p];
        dst[off + p] = {o.x * scale, o.y * scale};
    }
}

} // namespace

extern "C" int tcg_davidson_expand(int32_t nbasis, int32_t nblock, int32_t npw, void *V, const void *phi,
                                   const void *H1phi, const void *H2phi, const void *H3phi, const double *kG2,
                                   const double *eig_ref, int32_t *nbasis_out, void *stream)
{
    if (nbasis < 0 || nblock < 0 || npw < 1 || !V || !nbasis_out || (nblock > 0 && (!phi || !kG2 || !eig_ref)) ||
        (nblock > 0 && !H1phi && !H2phi && !H3phi))
        return fail(TCG_ERR_ARG, "bad Davidson expansion arguments");
    *nbasis_out = nbasis;
    if (nblock == 0) return TCG_OK;
    cudaStream_t st = (cudaStream_t)stream;
    Scratch S;
    double2 *T, *de, *c;
    int rc;
    if ((rc = S.get((void **)&T, (size_t)nblock * npw * sizeof(double2))) ||
        (rc = S.get((void **)&de, nblock * sizeof(double2))) || (rc = S.get((void **)&c, sizeof(double2))))
        return rc;
    SUB_CUDA(cudaMemcpyAsync(de, eig_ref, nblock * sizeof(double2), cudaMemcpyHostToDevice, st));
    k_precondition<<<nblock, 256, 0, st>>>(npw, kG2, (const double2 *)phi, (const double2 *)H1phi,
                                           (const double2 *)H2phi, (const double2 *)H3phi, de, T);
    SUB_CUDA(cudaGetLastError());
    double2 *v = (double2 *)V;
    int r = nbasis;
    for (int b = 0; b < nblock; b++) {
        // Gram_Schmidt against the whole current basis, the new vectors of
        // this block included; a vector below norm 1e-8 is dropped
        // (diagonalization_davidson.cpp:297-318)
        double2 *tr = v + (size_t)r * npw;
        SUB_CUDA(cudaMemcpyAsync(tr, T + (size_t)b * npw, npw * sizeof(double2), cudaMemcpyDeviceToDevice, st));
        k_gs_project<<<1, 256, 0, st>>>(npw, r, v, v, tr);
        k_dotc<<<1, 256, 0, st>>>(npw, tr, tr, c);
        SUB_CUDA(cudaGetLastError());
        double2 nrm2;
        SUB_CUDA(cudaMemcpyAsync(&nrm2, c, sizeof(double2), cudaMemcpyDeviceToHost, st));
        SUB_CUDA(cudaStreamSynchronize(st));
        const double nrm = std::sqrt(nrm2.x);
        if (nrm < 1e-8) continue;
        const double2 hn = make_double2(nrm, 0.0);
        SUB_CUDA(cudaMemcpyAsync(c, &hn, sizeof(double2), cudaMemcpyHostToDevice, st));
        k_scale_inv<<<8, 256, 0, st>>>(npw, c, 0, tr);
        SUB_CUDA(cudaGetLastError());
        SUB_CUDA(cudaStreamSynchronize(st));
        r++;
    }
    *nbasis_out = r;
    return TCG_OK;
}

extern "C" int tcg_subspace_ritz(int32_t ndim, int32_t npw, int32_t nout, int32_t biortho, const void *V,
                                 const void *Vref, const void *H1V, const void *H2V, const void *H3V, double *eig_out,
                                 double *e_out, void *V_out, void *Vl_out, void *stream)
{
    if (ndim < 1 || npw < 1 || nout < 0 || nout > ndim) return fail(TCG_ERR_ARG, "bad subspace sizes");
    if (!V || !eig_out || (!H1V && !H2V && !H3V)) return fail(TCG_ERR_ARG, "null argument");
    if (nout > 0 && !V_out) return fail(TCG_ERR_ARG, "V_out is NULL");
    if (!Vref) Vref = V;
    Handles *hd;
    int rc = handles(&hd);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    SUB_BLAS(cublasSetStream(hd->blas, st));
    SUB_SOLV(cusolverDnSetStream(hd->solver, st));
    Scratch S;
    const size_t nn = (size_t)ndim * ndim;
    double2 *Hn[3] = {nullptr, nullptr, nullptr}, *H, *A, *W, *VR, *X, *Xinv, *XL, *E;
    const void *HV[3] = {H1V, H2V, H3V};
    for (int n = 0; n < 3; n++)
        if (HV[n] && (rc = S.get((void **)&Hn[n], nn * sizeof(double2)))) return rc;
    if ((rc = S.get((void **)&H, nn * sizeof(double2))) || (rc = S.get((void **)&A, nn * sizeof(double2))) ||
        (rc = S.get((void **)&W, ndim * sizeof(double2))) || (rc = S.get((void **)&VR, nn * sizeof(double2))) ||
        (rc = S.get((void **)&X, nn * sizeof(double2))) || (rc = S.get((void **)&Xinv, nn * sizeof(double2))) ||
        (rc = S.get((void **)&XL, nn * sizeof(double2))) || (rc = S.get((void **)&E, 3 * (size_t)ndim * sizeof(double2))))
        return rc;
    // H_n,sub(i, j) = <Vref_i | H_n V_j>   (diagonalization_davidson.cpp:462-475)
    const cuDoubleComplex one = make_cuDoubleComplex(1, 0), zero = make_cuDoubleComplex(0, 0);
    for (int n = 0; n < 3; n++)
        if (HV[n])
            SUB_BLAS(cublasZgemm(hd->blas, CUBLAS_OP_C, CUBLAS_OP_N, ndim, ndim, npw, &one, (const cuDoubleComplex *)Vref,
                                 npw, (const cuDoubleComplex *)HV[n], npw, &zero, (cuDoubleComplex *)Hn[n], ndim));
    k_add3<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>((int)nn, Hn[0], Hn[1], Hn[2], H);
    SUB_CUDA(cudaGetLastError());
    SUB_CUDA(cudaMemcpyAsync(A, H, nn * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    // H_sub X = X D (ComplexEigenSolver, :479-486)
    size_t dws = 0, hws = 0;
    SUB_SOLV(cusolverDnXgeev_bufferSize(hd->solver, hd->params, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_VECTOR,
                                        ndim, CUDA_C_64F, A, ndim, CUDA_C_64F, W, CUDA_C_64F, nullptr, ndim, CUDA_C_64F,
                                        VR, ndim, CUDA_C_64F, &dws, &hws));
    void *dwork;
    int *dinfo;
    if ((rc = S.get(&dwork, dws)) || (rc = S.get((void **)&dinfo, 64 * sizeof(int)))) return rc;
    std::vector<unsigned char> hwork(std::max<size_t>(hws, 16));
    SUB_SOLV(cusolverDnXgeev(hd->solver, hd->params, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_VECTOR, ndim,
                             CUDA_C_64F, A, ndim, CUDA_C_64F, W, CUDA_C_64F, nullptr, ndim, CUDA_C_64F, VR, ndim,
                             CUDA_C_64F, dwork, dws, hwork.data(), hws, dinfo));
    int info = 0;
    std::vector<double2> w(ndim);
    SUB_CUDA(cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st));
    SUB_CUDA(cudaMemcpyAsync(w.data(), W, ndim * sizeof(double2), cudaMemcpyDeviceToHost, st));
    SUB_CUDA(cudaStreamSynchronize(st));
    if (info != 0) return fail(TCG_ERR_NUMERIC, "diagonalization of H_subspace failed");
    // sort by the real part, ascending (sort_eigen, diagonalization_utils.cpp:82-119)
    std::vector<int> perm(ndim);
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return w[a].x < w[b].x; });
    for (int i = 0; i < ndim; i++) {
        eig_out[2 * i] = w[perm[i]].x;
        eig_out[2 * i + 1] = w[perm[i]].y;
    }
    int *dperm;
    if ((rc = S.get((void **)&dperm, ndim * sizeof(int)))) return rc;
    SUB_CUDA(cudaMemcpyAsync(dperm, perm.data(), ndim * sizeof(int), cudaMemcpyHostToDevice, st));
    k_permute_cols<<<ndim, 128, 0, st>>>(ndim, dperm, VR, X);
    // X^-1 by LU (eigenvectors.inverse(), :494); left eigenvectors (X^-1)^H
    int lwork = 0;
    SUB_SOLV(cusolverDnZgetrf_bufferSize(hd->solver, ndim, ndim, (cuDoubleComplex *)A, ndim, &lwork));
    void *lw;
    int *ipiv;
    if ((rc = S.get(&lw, (size_t)lwork * sizeof(double2))) || (rc = S.get((void **)&ipiv, ndim * sizeof(int)))) return rc;
    SUB_CUDA(cudaMemcpyAsync(A, X, nn * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    SUB_SOLV(cusolverDnZgetrf(hd->solver, ndim, ndim, (cuDoubleComplex *)A, ndim, (cuDoubleComplex *)lw, ipiv, dinfo));
    k_identity<<<ndim, 128, 0, st>>>(ndim, Xinv);
    SUB_SOLV(cusolverDnZgetrs(hd->solver, CUBLAS_OP_N, ndim, ndim, (const cuDoubleComplex *)A, ndim, ipiv,
                              (cuDoubleComplex *)Xinv, ndim, dinfo));
    SUB_CUDA(cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st));
    k_adjoint<<<ndim, 128, 0, st>>>(ndim, Xinv, XL);
    SUB_CUDA(cudaGetLastError());
    // Ritz vectors V X and left vectors Vref X_left (:497-530)
    if (nout > 0) {
        SUB_BLAS(cublasZgemm(hd->blas, CUBLAS_OP_N, CUBLAS_OP_N, npw, nout, ndim, &one, (const cuDoubleComplex *)V, npw,
                             (const cuDoubleComplex *)X, ndim, &zero, (cuDoubleComplex *)V_out, npw));
        if (Vl_out)
            SUB_BLAS(cublasZgemm(hd->blas, CUBLAS_OP_N, CUBLAS_OP_N, npw, nout, ndim, &one, (const cuDoubleComplex *)Vref,
                                 npw, (const cuDoubleComplex *)XL, ndim, &zero, (cuDoubleComplex *)Vl_out, npw));
    }
    // energies diag(L^H H_n,sub X), L = X_left for BITC, X otherwise (:583-596)
    if (e_out && nout > 0) {
        for (int n = 0; n < 3; n++)
            if (Hn[n]) k_diag_form<<<nout, 256, 0, st>>>(ndim, nout, biortho ? XL : X, Hn[n], X, E + (size_t)n * ndim);
        SUB_CUDA(cudaGetLastError());
        std::vector<double2> e(3 * (size_t)ndim, make_double2(0, 0));
        for (int n = 0; n < 3; n++)
            if (Hn[n]) SUB_CUDA(cudaMemcpyAsync(e.data() + (size_t)n * ndim, E + (size_t)n * ndim, nout * sizeof(double2),
                                                cudaMemcpyDeviceToHost, st));
        SUB_CUDA(cudaStreamSynchronize(st));
        for (int n = 0; n < 3; n++)
            for (int i = 0; i < nout; i++) {
                e_out[2 * ((size_t)n * nout + i)] = e[(size_t)n * ndim + i].x;
                e_out[2 * ((size_t)n * nout + i) + 1] = e[(size_t)n * ndim + i].y;
            }
    }
    SUB_CUDA(cudaStreamSynchronize(st));
    if (info != 0) return fail(TCG_ERR_NUMERIC, "eigenvector matrix of H_subspace is singular");
    return TCG_OK;
}

extern "C" int tcg_gram_schmidt(int32_t nvec, int32_t npw, void *V, void *Vl, void *stream)
{
    if (nvec < 0 || npw < 1 || !V) return fail(TCG_ERR_ARG, "bad Gram-Schmidt arguments");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch S;
    double2 *c;
    int rc;
    if ((rc = S.get((void **)&c, nvec * sizeof(double2)))) return rc;
    double2 *v = (double2 *)V, *l = (double2 *)Vl;
    for (int j = 0; j < nvec; j++) {
        double2 *tj = v + (size_t)j * npw;
        // |j> -= <ref_i|j> |i>, i < j  (Gram_Schmidt / Gram_Schmidt_biortho, utils:7-77)
        k_gs_project<<<1, 256, 0, st>>>(npw, j, l ? l : v, v, tj);
        k_dotc<<<1, 256, 0, st>>>(npw, tj, tj, c + j);            // |j|^2
        SUB_CUDA(cudaGetLastError());
        double2 nrm2;
        SUB_CUDA(cudaMemcpyAsync(&nrm2, c + j, sizeof(double2), cudaMemcpyDeviceToHost, st));
        SUB_CUDA(cudaStreamSynchronize(st));
        const double nrm = std::sqrt(nrm2.x);
        if (nrm < (l ? 1e-10 : 1e-8)) return fail(TCG_ERR_NUMERIC, "Linear independence breaks in block-Davidson algorithm.");
        double2 hn = make_double2(nrm, 0.0);
        SUB_CUDA(cudaMemcpyAsync(c + j, &hn, sizeof(double2), cudaMemcpyHostToDevice, st));
        k_scale_inv<<<8, 256, 0, st>>>(npw, c + j, 0, tj);
        if (l) {
            double2 *lj = l + (size_t)j * npw;
            // <j| -= <j|i> <i|, then <j|j> = 1 by dividing the left vector by conj(<l_j|v_j>)
            k_gs_project<<<1, 256, 0, st>>>(npw, j, v, l, lj);
            k_dotc<<<1, 256, 0, st>>>(npw, lj, tj, c + j);
            double2 cc;
            SUB_CUDA(cudaMemcpyAsync(&cc, c + j, sizeof(double2), cudaMemcpyDeviceToHost, st));
            SUB_CUDA(cudaStreamSynchronize(st));
            if (std::sqrt(cc.x * cc.x + cc.y * cc.y) < 1e-10)
                return fail(TCG_ERR_NUMERIC, "Linear independence breaks in block-Davidson algorithm.");
            k_scale_inv<<<8, 256, 0, st>>>(npw, c + j, 1, lj);
        }
        SUB_CUDA(cudaGetLastError());
    }
    SUB_CUDA(cudaStreamSynchronize(st));
    return TCG_OK;
}
