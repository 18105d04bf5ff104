// util.cuh -- error helpers, kernel launch wrapper, upload helper.
#pragma once
#include <mutex>
#include <string>
#include <vector>
#include <unordered_set>
#include "ctx.cuh"
#include "passes.cuh"

namespace tcg {

inline int fail(int code, const char *msg)
{
    set_error("%s", msg);
    return code;
}

// ---------------------------------------------------------------- plans --
inline int make_axis(int n, Axis &ax)
{
    if (n < 1 || n > MAXN) return fail(TCG_ERR_UNSUPPORTED, "FFT axis length outside 1..128");
    ax.n = n;
    ax.nst = 0;
    int m = n;
    while (m % 8 == 0 && ax.nst < MAXST) { ax.R[ax.nst++] = 8; m /= 8; }
    while (m % 4 == 0 && ax.nst < MAXST) { ax.R[ax.nst++] = 4; m /= 4; }
    while (m % 2 == 0 && ax.nst < MAXST) { ax.R[ax.nst++] = 2; m /= 2; }
    for (int q = 3; m > 1 && ax.nst < MAXST; q += 2)
        while (m % q == 0 && ax.nst < MAXST) {
            if (q > 16) return fail(TCG_ERR_UNSUPPORTED, "FFT axis length has a prime factor > 16");
            ax.R[ax.nst++] = q;
            m /= q;
        }
    if (m != 1) return fail(TCG_ERR_UNSUPPORTED, "FFT axis length not factorisable");
    return TCG_OK;
}

// smem sizes (bytes) of the pass kernels
template <typename V> inline size_t smem_xy(const GridDesc &g) { return sizeof(V) * (3 * MAXN + 2 * (size_t)g.n0 * g.n1); }
template <typename V> inline size_t smem_z(const GridDesc &g, int nf) { return sizeof(V) * (3 * MAXN + (size_t)(nf + 2) * ZTC * g.n2); }

// Launch with the dynamic-smem attribute set once per kernel.
inline std::mutex g_attr_mu;
inline std::unordered_set<const void *> g_attr_set;
// interned "op:pass" profiling tags
inline const char *tagname(const char *op, const char *pass)
{
    static std::mutex mu;
    static std::vector<std::string *> pool;
    std::lock_guard<std::mutex> lk(mu);
    std::string s = std::string(op) + ":" + pass;
    for (auto *p : pool)
        if (*p == s) return p->c_str();
    pool.push_back(new std::string(s));
    return pool.back()->c_str();
}

template <typename K, typename... Args>
inline int launch_tagged(tcg_ctx *c, const char *tag, double alg_bytes, K kernel, dim3 grid, dim3 block, size_t smem,
                         Args... args)
{
    if (grid.x == 0 || grid.y == 0 || grid.z == 0) return TCG_OK;
    if (smem > 48 * 1024) {
        std::lock_guard<std::mutex> lk(g_attr_mu);
        if (!g_attr_set.count((const void *)kernel)) {
            TCG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
            TCG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
            g_attr_set.insert((const void *)kernel);
        }
    }
    if (smem > 227 * 1024) return fail(TCG_ERR_UNSUPPORTED, "kernel shared memory exceeds 227 KB");
    tcg_ctx::ProfRec rec{(const void *)kernel, tag, nullptr, nullptr, alg_bytes};
    if (c->prof) {
        TCG_CUDA(cudaEventCreate(&rec.a));
        TCG_CUDA(cudaEventCreate(&rec.b));
        TCG_CUDA(cudaEventRecord(rec.a, c->stream));
    }
    kernel<<<grid, block, smem, c->stream>>>(args...);
    c->launches++;
    TCG_CUDA(cudaGetLastError());
    if (c->prof) {
        TCG_CUDA(cudaEventRecord(rec.b, c->stream));
        c->prof_recs.push_back(rec);
    }
    return TCG_OK;
}

template <typename K, typename... Args>
inline int launch(tcg_ctx *c, K kernel, dim3 grid, dim3 block, size_t smem, Args... args)
{
    return launch_tagged(c, c->stage, 0.0, kernel, grid, block, smem, args...);
}

// Names the stage whose untagged launches follow (profiling only).
struct PhaseScope {
    tcg_ctx *c;
    const char *old;
    PhaseScope(tcg_ctx *c_, const char *name) : c(c_), old(c_->stage) { c->stage = name; }
    ~PhaseScope() { c->stage = old; }
};

#define TRY(x)                     \
    do {                           \
        int rc_ = (x);             \
        if (rc_ != TCG_OK) return rc_; \
    } while (0)

inline int up(DBuf &b, const void *src, size_t bytes, cudaStream_t s)
{
    TRY(b.ensure(bytes));
    if (bytes) TCG_CUDA(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, s));
    return TCG_OK;
}


} // namespace tcg
