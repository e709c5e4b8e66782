// Material laws on the device, written in terms of the displacement gradient
// H = F - I so that no O(1) terms cancel (this keeps the FP32 element path
// accurate at small strain).  Algebraically identical to the reference's
// first Piola-Kirchhoff stress:
//   Neo-Hookean    src/material/NeoHookean.cpp:4-20
//   Mooney-Rivlin  src/material/MooneyRivlin.cpp:4-24
//   Yeoh           src/material/Yeoh.cpp:4-19
// Identities used (F = I + H, J = det F, cof F = J F^{-T}):
//   J - 1       = tr H + tr cof(H) + det H
//   cof F       = I + B,   B = (tr H) I - H^T + cof(H)
//   I1 - 3      = 2 tr H + |H|^2
//   P_I1bar     = J^{-2/3} (2F - 2/3 I1 F^{-T}) = 2 J^{-2/3} [H - (c-1) I - c B],
//                 c = I1 / (3J)
//   P_I2bar     = J^{-4/3} (2F(I1 I - C) - 4/3 I2 F^{-T})
//               = J^{-4/3} (2[t I - E + (2+t) H - H E] - 4 (c2-1) I - 4 c2 B),
//                 E = C - I, t = tr E, c2 = I2 / (3J)
//   volumetric  = 2/D1 (J-1) J F^{-T} = 2/D1 (J-1) (I + B)
#pragma once
#include <cuda_runtime.h>

#include "efem_internal.h"

namespace efem {

// log|1 + x|.  The laws take J^{-2/3} as (J^2)^{-1/3} = |J|^{-2/3}, as the
// reference does (std::pow(I3, 1/3) with I3 = J^2): an inverted element
// (J < 0) gets a finite stress, not NaN, so a line-search trial that inverts
// elements is judged on its residual exactly as in the reference.
template <typename T>
__device__ __forceinline__ T dlogabs1p(T x);
template <>
__device__ __forceinline__ double dlogabs1p<double>(double x) { return x > -1.0 ? log1p(x) : log(-(1.0 + x)); }
template <>
__device__ __forceinline__ float dlogabs1p<float>(float x) { return x > -1.0f ? log1pf(x) : logf(-(1.0f + x)); }
// J^{-1/3} (negative for J < 0)
template <typename T>
__device__ __forceinline__ T drcbrt(T x);
template <>
__device__ __forceinline__ double drcbrt<double>(double x) { return rcbrt(x); }
template <>
__device__ __forceinline__ float drcbrt<float>(float x) { return rcbrtf(x); }

// cofactor matrix (row-major): cof(A)_ij = A_{i+1,j+1} A_{i+2,j+2} - A_{i+1,j+2} A_{i+2,j+1}
template <typename T>
__device__ __forceinline__ void cof3(const T* A, T* C)
{
    C[0] = A[4] * A[8] - A[5] * A[7];
    C[1] = A[5] * A[6] - A[3] * A[8];
    C[2] = A[3] * A[7] - A[4] * A[6];
    C[3] = A[7] * A[2] - A[8] * A[1];
    C[4] = A[8] * A[0] - A[6] * A[2];
    C[5] = A[6] * A[1] - A[7] * A[0];
    C[6] = A[1] * A[5] - A[2] * A[4];
    C[7] = A[2] * A[3] - A[0] * A[5];
    C[8] = A[0] * A[4] - A[1] * A[3];
}

// Kinematic quantities shared by the laws.
template <typename T>
struct Kin {
    T B[9];      // cof F - I
    T delta;     // J - 1
    T a;         // I1 - 3
};

template <typename T>
__device__ __forceinline__ void kinematics(const T* H, Kin<T>& k)
{
    T cH[9];
    cof3(H, cH);
    const T trH = H[0] + H[4] + H[8];
    const T trc = cH[0] + cH[4] + cH[8];
    const T detH = H[0] * cH[0] + H[1] * cH[1] + H[2] * cH[2];
    k.delta = trH + trc + detH;
    T hh = 0;
#pragma unroll
    for (int i = 0; i < 9; i++) hh += H[i] * H[i];
    k.a = T(2) * trH + hh;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) k.B[3 * i + j] = (i == j ? trH : T(0)) - H[3 * j + i] + cH[3 * i + j];
}

// P(F) for F = I + H, row-major 3x3.  MT: the law when every element of a
// block has the same one (EFEM_NEO_HOOKEAN, EFEM_MOONEY_RIVLIN, EFEM_YEOH),
// so that only its code is compiled in; -1: any law, chosen per element.
template <typename T, int MT = -1>
__device__ __forceinline__ void piola(const MatParams<T>& mp, const T* H, T* P)
{
    const bool yeoh = MT == EFEM_YEOH || (MT < 0 && mp.type == EFEM_YEOH);
    const bool mr = MT == EFEM_MOONEY_RIVLIN || (MT < 0 && mp.type == EFEM_MOONEY_RIVLIN);
    Kin<T> k;
    kinematics(H, k);
    // J^{-2/3} = rc^2 with rc = J^{-1/3}: the reference's (J^2)^{-1/3}, finite
    // for an inverted element (rc < 0), with one transcendental call
    const T J = T(1) + k.delta;
    const T rc = drcbrt(J);
    const T Jm23 = rc * rc;
    const T inv1pd = T(1) / J;
    const T cm1 = (k.a * T(1.0 / 3.0) - k.delta) * inv1pd;  // c - 1
    const T c = T(1) + cm1;
    T coef = mp.C10;
    if (yeoh) {
        // I1bar - 3 = 3 (J^{-2/3} - 1) + (I1 - 3) J^{-2/3}, where with
        // y = J^{1/3} = J rc^2 (so y - 1 = delta / (y^2 + y + 1)),
        // J^{-2/3} - 1 = -delta (y + 1) rc^2 / (y^2 + y + 1): no cancellation
        const T y = J * Jm23;
        const T jm1 = -k.delta * (y + T(1)) * Jm23 / (y * y + y + T(1));
        const T t = T(3) * jm1 + k.a * Jm23;
        coef = mp.C10 + T(2) * mp.C20 * t + T(3) * mp.C30 * t * t;
    }
    const T s1 = T(2) * coef * Jm23;
    const T vol = T(2) / mp.D1 * k.delta;
#pragma unroll
    for (int i = 0; i < 9; i++) {
        const T id = (i % 4 == 0) ? T(1) : T(0);
        P[i] = s1 * (H[i] - cm1 * id - c * k.B[i]) + vol * (id + k.B[i]);
    }
    if (mr) {
        T E[9];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
                E[3 * i + j] = H[3 * i + j] + H[3 * j + i] + H[i] * H[j] + H[3 + i] * H[3 + j] + H[6 + i] * H[6 + j];
        const T t = E[0] + E[4] + E[8];  // = a
        T ee = 0;
#pragma unroll
        for (int i = 0; i < 9; i++) ee += E[i] * E[i];
        const T i2 = T(2) * t + T(0.5) * (t * t - ee);  // I2 - 3
        const T c2m1 = (i2 * T(1.0 / 3.0) - k.delta) * inv1pd;
        const T c2 = T(1) + c2m1;
        const T s2 = mp.C01 * Jm23 * Jm23;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const T HE = H[3 * i] * E[j] + H[3 * i + 1] * E[3 + j] + H[3 * i + 2] * E[6 + j];
                const T id = (i == j) ? T(1) : T(0);
                const T q = T(2) * (t * id - E[3 * i + j] + (T(2) + t) * H[3 * i + j] - HE) - T(4) * c2m1 * id
                    - T(4) * c2 * k.B[3 * i + j];
                P[3 * i + j] += s2 * q;
            }
    }
}

}  // namespace efem
