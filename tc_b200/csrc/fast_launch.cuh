// fast_launch.cuh -- launcher of the compile-time-size pass kernels (cubic
// grids).  Algorithmic bytes per launch as in run_chunk: N s per grid and pass.
#pragma once
#include "terms.cuh"
#include "fast.cuh"

namespace tcg {

template <typename T, int N, class Op>
int run_chunk_fast(tcg_ctx *c, const Op &op, int items, int nt, bool do_xyf, bool do_xyi)
{
    using V = typename C2<T>::t;
    using CF = fast::Cfg<N, sizeof(V)>;
    const double gb = (double)N * N * N * sizeof(V);
    // bytes a pass must move: N s per grid, the band-limited grids of a pruned
    // chunk only on the pencils their support meets (fraction op.m.pfrac)
    const double fr = op.m.prune ? op.m.pfrac : 1.0;
    const int bli = __builtin_popcount(Op::BLI), blo = __builtin_popcount(Op::BLO);
    const double nf_eff = (Op::NF - bli) + fr * bli, nb_eff = (Op::NB - blo) + fr * blo;
    const int np_f = items * N, np_i = nt * N;
    using CP = fast::CfgP<N, sizeof(V)>;
    const bool fpair = c->xy_kernels ? c->xy_kernels == 2 : Op::XYF_PAIR;
    const bool ipair = c->xy_kernels ? c->xy_kernels == 2 : Op::XYI_PAIR;
    // grids with a several-threads-per-line shape (36: 6 x 6, 48: 4 x 12):
    // the inverse XY pass runs in that form unless another is forced; the
    // forward pass measured faster with one thread per line in FP32 and with
    // the split form in FP64 (where a whole line per thread spills)
    constexpr int TLN = fast::t6::ShapeOf<N>::TL;
    using SH = fast::t6::Shape<TLN ? N : 36, TLN ? TLN : 6>;   // (36 x 6 unused where TLN = 0)
    const bool t6i = TLN > 0 && (c->xy_kernels == 0 || c->xy_kernels == 3);
    const bool t6f = TLN > 0 && (c->xy_kernels == 3 ||
                                 (c->xy_kernels == 0 && (sizeof(V) == 16 || (N == 48 && Op::XYF_SPLIT48))));
    if constexpr (TLN > 0) {
        if (t6f && do_xyf)
            TRY(launch_tagged(c, tagname(Op::NAME, "xyf"), (double)items * nf_eff * gb, fast::t6::k_xyf_t6<T, Op, SH>,
                              dim3(np_f), dim3(SH::THREADS), fast::t6::smem<V, SH>(1), op, np_f));
    }
    if (do_xyf && !t6f) {
        if (!fpair)
            TRY(launch_tagged(c, tagname(Op::NAME, "xyf"), (double)items * nf_eff * gb, fast::k_xyf_fast<T, N, Op>,
                              dim3((np_f + CF::P - 1) / CF::P), dim3(CF::THREADS), fast::smem_xy_fast<V, N>(1), op, np_f));
        else
            TRY(launch_tagged(c, tagname(Op::NAME, "xyf"), (double)items * Op::NF * gb, fast::k_xyf_pair<T, N, Op>,
                              dim3((np_f + CP::P - 1) / CP::P), dim3(CP::THREADS), fast::smem_xy_pair<V, N>(1), op, np_f));
    }
    constexpr int TC = fast::zcols<V>();
    const bool zsplit = c->z_kernels ? c->z_kernels == 2 : Op::ZSPLIT;
    // several threads per z-line unless a form is forced
    bool zt6 = false;
    if constexpr (TLN > 0) {
        zt6 = c->z_kernels == 0 || c->z_kernels == 3 || c->z_kernels == 4;
        // default: inputs transformed in place in shared memory (k_z_t6); the
        // terms with Op::ZREG keep them in registers in FP32 (k_z_t6r)
        if (c->z_kernels == 3 || (c->z_kernels == 0 && !(Op::ZREG && sizeof(V) == 8)))
            TRY(launch_tagged(c, tagname(Op::NAME, "z"), (double)items * (nf_eff + (Op::ZINV ? nb_eff : 0)) * gb,
                              fast::t6::k_z_t6<T, Op, SH>, dim3((N * N + TC - 1) / TC, items), dim3(SH::ZTHREADS),
                              fast::t6::smem_z<V, SH, Op>(), op));
        else if (zt6)
            TRY(launch_tagged(c, tagname(Op::NAME, "z"), (double)items * (nf_eff + (Op::ZINV ? nb_eff : 0)) * gb,
                              fast::t6::k_z_t6r<T, Op, SH>, dim3((N * N + TC - 1) / TC, items), dim3(SH::ZTHREADS),
                              fast::t6::smem_zr<V, SH>(Op::NF), op));
    }
    if (zt6) {
    } else if (zsplit)
        TRY(launch_tagged(c, tagname(Op::NAME, "z"), (double)items * (Op::NF + (Op::ZINV ? Op::NB : 0)) * gb,
                          fast::k_z_fast<T, N, Op>, dim3((N * N + TC - 1) / TC, items), dim3(128),
                          fast::smem_z_fast<V, N>(Op::NF), op));
    else
        TRY(launch_tagged(c, tagname(Op::NAME, "z"), (double)items * (Op::NF + (Op::ZINV ? Op::NB : 0)) * gb,
                          fast::k_z_line<T, N, Op>, dim3((N * N + TC - 1) / TC, items), dim3(32 * fast::ZL),
                          fast::smem_z_fast<V, N>(Op::NF), op));
    if constexpr (TLN > 0) {
        if (t6i && do_xyi) {
            const int nref = Op::REFWD ? Op::NB - 1 : 0;
            return launch_tagged(c, tagname(Op::NAME, "xyi"), (double)items * (nb_eff + nref) * gb,
                                 fast::t6::k_xyi_t6<T, Op, SH>, dim3(np_i), dim3(SH::THREADS),
                                 fast::t6::smem_xyi<V, Op, SH>(2, op.sacc_on ? op.sacc_n : 0) +
                                     (op.m.prune ? (size_t)op.ns * sizeof(int) : 0),
                                 op, np_i);
        }
    }
    if (do_xyi) {
        const int nref = Op::REFWD ? Op::NB - 1 : 0;
        if constexpr (Op::GS == 1 && !(Op::REGACC && Op::REFWD)) {
            if (!ipair && !c->no_prefetch)
                return launch_tagged(c, tagname(Op::NAME, "xyi"), (double)items * (Op::NB + nref) * gb,
                                     fast::k_xyi_pf<T, N, Op>, dim3((np_i + CF::P - 1) / CF::P), dim3(CF::THREADS),
                                     fast::smem_xy_fast<V, N>(2), op, np_i);
        }
        if (!ipair)
            TRY(launch_tagged(c, tagname(Op::NAME, "xyi"), (double)items * (Op::NB + nref) * gb, fast::k_xyi_fast<T, N, Op>,
                              dim3((np_i + CF::P - 1) / CF::P), dim3(CF::THREADS), fast::smem_xy_fast<V, N>(2), op, np_i));
        else
            TRY(launch_tagged(c, tagname(Op::NAME, "xyi"), (double)items * (Op::NB + nref) * gb, fast::k_xyi_pair<T, N, Op>,
                              dim3((np_i + CP::P - 1) / CP::P), dim3(CP::THREADS), fast::smem_xy_pair<V, N>(2), op, np_i));
    }
    return TCG_OK;
}

} // namespace tcg
