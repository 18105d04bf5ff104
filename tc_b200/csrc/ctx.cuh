// ctx.cuh -- the library context: device copies of the system / state,
// FFT plans, scratch arenas, launch helpers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include <unordered_set>
#include "../../include/tcg.h"
#include "fft.cuh"

namespace tcg {

void set_error(const char *fmt, ...);

struct Status {
    int code = TCG_OK;
};

#define TCG_CUDA(call)                                                                    \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            tcg::set_error("CUDA error %s at %s:%d (%s)", cudaGetErrorString(e_), __FILE__, \
                           __LINE__, #call);                                              \
            return TCG_ERR_CUDA;                                                          \
        }                                                                                 \
    } while (0)

// Device buffer (owned).
struct DBuf {
    void *p = nullptr;
    size_t bytes = 0;
    int ensure(size_t b)
    {
        if (b <= bytes) return TCG_OK;
        // kernels queued earlier may still read the old buffer
        if (p) { cudaDeviceSynchronize(); cudaFree(p); }
        p = nullptr;
        bytes = 0;
        if (b == 0) return TCG_OK;
        if (cudaMalloc(&p, b) != cudaSuccess) {
            cudaGetLastError();
            set_error("cudaMalloc of %zu bytes failed", b);
            return TCG_ERR_NOMEM;
        }
        bytes = b;
        return TCG_OK;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <typename X> X *as() const { return reinterpret_cast<X *>(p); }
};

struct Host {
    // system
    int n[3] = {0, 0, 0}, N = 0;
    double recip[9], lattice[9], omega = 0;
    int method = 0, nspin = 1, nk = 0, nk_all = 0, num_kpoints = 0;
    std::vector<int> nsym_k, kall_off, ik_of_all, npw;
    std::vector<double> kvec;               // [nk_all][3]
    std::vector<uint8_t> time_rev;
    std::vector<int> rot_index;
    int nsymop = 0;
    std::vector<int> rotation;              // [nsymop][9]
    std::vector<double> translation;        // [nsymop][3]
    std::vector<size_t> gidx_off;           // [nspin*nk_all] offset in gindex / phase
    std::vector<int> gidx_host;             // host copy of gindex (pseudopotential set-up)
    double A[4], F[4];
    bool A_zero = true;
    bool div = false;
    double alpha = 0;
    std::vector<double> sum_vaux;
    // state
    bool have_state = false;
    std::vector<int> nbands, nocc;          // [nspin], [nspin][nk]
    std::vector<double> filling;            // [nspin][nk][nbands]
    std::vector<size_t> orb_off;            // [nspin*nk] complex offset of band 0
    std::vector<size_t> occ_off;            // [nspin*nk_all] grid offset into Rocc
    size_t nocc_grids = 0;
    bool qp_ready = false;                  // tc3a2a4b2b5 occupied-pair stage done for this state
    bool qp_pending = false;                // a partial stage awaits the caller's sum and tcg_qp_finish
    // one-body data
    bool have_pseudo = false, have_vloc = false;
    int nl_ncomp = 0;                       // projector components (atom, projector, m)
    std::vector<size_t> nl_koff;            // [nk] offset of k in nlB
    size_t nl_dval_off = 0;                 // byte offset of the D values in nlD
    std::vector<size_t> g0_off;             // [nspin*nk] offset of (s, k) in gidx0
};

// cubic grid sizes whose pass kernels split each line over several threads
// (fast::t6::ShapeOf: 36 = 6 x 6, 48 = 4 x 12); only those forms honour
// pruned transforms
inline bool split_line_grid(int n) { return n == 36 || n == 48; }

struct tcg_ctx_impl;
} // namespace tcg

struct tcg_ctx {
    int device = 0;
    int prec = TCG_PREC_FP64;
    cudaStream_t stream = nullptr;
    tcg::Host h;
    tcg::GridDesc gd;
    // static device data
    tcg::DBuf tw64, tw32, recip;            // twiddles, reciprocal vectors (9 doubles)
    tcg::DBuf inv;                          // [nspin][nk_all][N] int32
    tcg::DBuf phase;                        // [sum npw] double2
    // state
    tcg::DBuf phik, chik;                   // G-space fp64 (chik only for BITC)
    tcg::DBuf fill;                         // [nspin][nk][nbands] doubles
    tcg::DBuf Rocc, Rchi, Rgrad;            // R-space occupied grids (compute precision)
    tcg::DBuf dens;                         // [2][N] double2
    tcg::DBuf densT;                        // [3][N] compute precision: n_0, n_1, n_0 + n_1
    tcg::DBuf occfill;                      // [nocc_grids] doubles: filling of each occupied grid
    // local three-body potentials built per state
    tcg::DBuf Vloc;                         // [nspin][N] double2 (tc3a1 + tc3b1 + ...)
    tcg::DBuf dnu, dnuT;                    // [nspin][3][N] fp64 / compute precision
    tcg::DBuf V3a1, V3b1, V3a2, V3b2;       // [nspin][N] fp64 local three-body potentials
    tcg::DBuf VH;                           // [N] fp64 Hartree potential (hf2h)
    tcg::DBuf V2h;                          // [nspin][N] fp64 TC Hartree potential (tc2h [2a_h] + [2b_h2])
    tcg::DBuf pgw;                          // [3][N] fp64 work: sum_q f conj(chi_q) grad phi_q (tc2h [2b_h2])
    // one-body data (tcg_set_pseudo) and per-apply scratch
    tcg::DBuf gidx0;                        // [nspin][sum npw] grid index of each plane wave at isym 0
    tcg::DBuf vloc;                         // [N] fp64 local pseudopotential (real), or empty
    tcg::DBuf nlB;                          // [sum_k ncomp npw_k] complex exp(iG.R) x projector
    tcg::DBuf nlD;                          // CSR of D between projector components
    tcg::DBuf acc1, h1buf;                  // one-body accumulators / device copies
    tcg::DBuf gpsi, adjw, adjt;             // energy gradients: occupied block + outputs, pair grids, tables
    // pruned transforms (36^3 path): per (irreducible k, all-k q) pair, the
    // (x, y) pencils of the grid that the support of a pair density touches
    tcg::DBuf prune_tab;                    // masks [nk][nk_all][NP] u8, perms [..][NP] u16, counts [..] i32
    bool prune_ok = false;                  // table built and usable
    std::vector<int> prune_nact;            // host copy of the table's active-pencil counts
    bool no_prune = false;                  // TCG_NO_PRUNE: full transforms everywhere
    bool use_sacc = false;                  // TCG_SACC: shared-memory accumulation in the 3a3b6A and fused (2x3A) inverse XY passes
    bool no_fuse = false;                   // TCG_NO_FUSE: tc2x and tc3a3b3b4b6 run as separate passes
    bool qp_sacc = true;                    // TCG_NO_QP_SACC clears: shared-memory accumulation in the
                                            // occupied-pair inverse XY pass (36^3, FP32)
    tcg::DBuf Qt, Bt;                       // tc3a2a4b2b5 rotated intermediates [nocc_grids][3][N]
    tcg::DBuf accP, qtg;                    // occupied-pair accumulators / gathered q2 grids
    tcg::DBuf div3b6;                       // [nspin][N] fp64 temp_div_3b6 in R space
    std::vector<double2> t1_3b6;            // [nspin][nk] temp_div_3b6_1
    // per-apply scratch
    tcg::DBuf psi, h2, h3;                  // packed fp64
    tcg::DBuf Rpsi, Rgpsi, acc2, acc3, qsum, tmp, tmp2, aux, items, meta;
    tcg::DBuf rotw, q3b2w, nGw, Ww;           // per-state scratch kept across states (no per-step cudaMalloc / cudaFree)
    tcg::DBuf ftab;                         // mixed path: FP32 G-space coefficient records of a chunk
    tcg::DBuf w3x;                          // [targets][3][N] compute precision: b3 dnu_d psi + b4 qsum_d (3bX input)
    int ftab_nrec = 1;
    int fast_n = 0;                         // cubic grid size with compiled fast kernels (0: generic path)
    bool force_generic = false;             // use the generic pass kernels even if fast_n is set
    int xy_kernels = 0;                     // fast XY passes: 0 default, 1 all line, 2 all lane-pair, 3 split lines (36^3, 48^3)
    bool no_prefetch = false;               // fast XYI: no prefetch of the next plane set
    const char *stage = "misc";            // profiling tag of untagged launches (the current stage)
    int z_kernels = 0;                      // fast Z pass: 0 per-term choice, 1 one thread per line, 2 lane pairs,
                                            // 3 / 4 split lines in shared memory / registers (36^3, 48^3)
    size_t tmp_budget = 0;                  // bytes per chunk of pass temporaries (0: default 8 GiB)
    int min_targets = 0;                    // targets per chunk (0: default, about 12 waves of XYI CTAs)
    int64_t launches = 0;
    // optional per-kernel timing with CUDA events on the context stream
    bool prof = false;
    struct ProfRec { const void *fn; const char *tag; cudaEvent_t a, b; double bytes; };
    std::vector<ProfRec> prof_recs;
};
