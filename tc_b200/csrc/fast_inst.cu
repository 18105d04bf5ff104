// fast_inst.cu -- explicit instantiation of the fast pass kernels for one
// cubic grid size N = TCG_FAST_N (the build compiles this file once per N).
#include "fast_launch.cuh"

#ifndef TCG_FAST_N
#error "TCG_FAST_N must be defined"
#endif

namespace tcg {
template <typename T> using OpQPBitc = OpQP<T, true>;
template <typename T> using OpQPTc = OpQP<T, false>;
template <typename T> using OpQPBitcEq = OpQP<T, true, true>;
template <typename T> using OpQPTcEq = OpQP<T, false, true>;
template <typename T> using OpTC3AEq = OpTC3A<T, true>;
template <typename T> using OpTC3BEq = OpTC3B<T, true>;
#define TCG_INST(T, OP) \
    template int run_chunk_fast<T, TCG_FAST_N, OP>(tcg_ctx *, const OP &, int, int, bool, bool);
#define TCG_INST_ALL(T)                \
    TCG_INST(T, OpHF2X<T>)             \
    TCG_INST(T, OpTC2X<T>)             \
    TCG_INST(T, OpTC3A<T>)             \
    TCG_INST(T, OpTC3B<T>)             \
    TCG_INST(T, OpTC3C<T>)             \
    TCG_INST(T, OpPairFwd<T>)          \
    TCG_INST(T, OpBand<T>)             \
    TCG_INST(T, OpQPBitc<T>)           \
    TCG_INST(T, OpQPTc<T>)             \
    TCG_INST(T, OpQPBitcEq<T>)         \
    TCG_INST(T, OpQPTcEq<T>)           \
    TCG_INST(T, OpTC3AEq<T>)           \
    TCG_INST(T, OpTC3BEq<T>)           \
    TCG_INST(T, OpTC2X3<T>)            \
    TCG_INST(T, OpTC3X<T>)
TCG_INST_ALL(float)
TCG_INST_ALL(double)
} // namespace tcg
