// jastrow.cuh -- RPA Jastrow factor on the device (jastrow_functions.cpp:6-97,
// derived parameters jastrow_initialize.cpp:86-110).
//   u(G)       = 4 pi A / (G^2 (1 + F^2 G^2)),          u(0) = -4 pi A F^2
//   V_2body(G) = 4pi/G^2 - 4pi A/(1+F^2G^2)
//                + (pi A^2/F^2/G) [pi F^2G^2 + (4+2F^2G^2) atan(FG/2) - (4+4F^2G^2) atan(FG)],
//   V_2body(0) = -2 pi A^2 / F
// With all A zero the reference falls back to plain Coulomb 4pi/G^2 (0 at G=0).
#pragma once
#include <cmath>
#include "ctx.cuh"

namespace tcg {

struct Jastrow {
    double fourpiA[4], F2[4], F[4], piAAF2inv[4];
    int A_zero;
    __device__ __forceinline__ double uk(const double *G, int s1, int s2) const
    {
        if (A_zero) return 0.0;
        const int i = s1 * 2 + s2;
        const double G2 = G[0] * G[0] + G[1] * G[1] + G[2] * G[2];
        if (G2 < 1e-12) return -fourpiA[i] * F2[i];
        return fourpiA[i] / (G2 * (G2 * F2[i] + 1));
    }
    __device__ __forceinline__ double tc2body(const double *G, int s1, int s2) const
    {
        const double PI = 3.14159265358979323846;
        const double G2 = G[0] * G[0] + G[1] * G[1] + G[2] * G[2];
        if (A_zero) return G2 > 1e-12 ? 4.0 * PI / G2 : 0.0;
        const int i = s1 * 2 + s2;
        if (G2 < 1e-12) return -2 * piAAF2inv[i] * F[i];
        const double G1 = sqrt(G2), FG1 = F[i] * G1, F2G2 = F2[i] * G2;
        return 4.0 * PI / G2 - fourpiA[i] / (1 + F2G2) +
               (piAAF2inv[i] / G1) * (PI * F2G2 + (4 + 2 * F2G2) * atan(FG1 / 2) - (4 + 4 * F2G2) * atan(FG1));
    }
};

inline Jastrow make_jastrow(const Host &h)
{
    const double PI = 3.14159265358979323846;
    Jastrow J;
    J.A_zero = h.A_zero ? 1 : 0;
    for (int i = 0; i < 4; i++) {
        const double A = h.A[i], F = h.F[i];
        J.fourpiA[i] = 4.0 * PI * A;
        J.F[i] = F;
        J.F2[i] = F * F;
        J.piAAF2inv[i] = PI * A * A * (1.0 / (F * F));
    }
    return J;
}

} // namespace tcg
