// True tangent, adjoint solve and parameter sensitivities.  The reference has
// none of these (it only ever forms the approximate Jacobian, see
// src/fe/ElementConstraint.cpp:164-205); they are built on its residual
// (ElementConstraint.cpp:139-162, ExternalConstraint.cpp:829-959):
//
//   K(u) v      the directional derivative of R at u along v, computed by the
//               residual kernels instantiated on forward-mode dual numbers
//               (value + derivative), so the tangent is exact to rounding;
//   K(u)^T w    the element part of K is the Hessian of the stored energy and
//               is symmetric, so K_el^T w = K_el w; the pressure part is not
//               (follower and directed loads are not conservative) and is
//               transposed face by face: one dual seed per face unknown gives
//               the column d f_face / d u_j, dotted with w on the face; an
//               adjoint solve stores these face blocks once at its u and
//               applies them in every Krylov iteration, and likewise the
//               Gauss-point tangents dP/dH of the elements, so that K_el v
//               in its iterations is C : grad v without dual numbers;
//   dR/dtheta   the same kernels with the seed on a material constant
//               (C10, C01, C20, C30, D1 of one material) or on the scale of one
//               pressure load;
//   adjoint     K(u)^T lambda = dJ/du by restarted GMRES, right-preconditioned
//               with the approximate-Jacobian Cholesky factor H0 of the
//               solve; then dJ/dtheta_k = -lambda . dR/dtheta_k.
//
// Parameter order: for every material slot of the model (its material
// table), C10, C01, C20, C30, D1; then one scale per pressure load in input
// order (a follower load's pressure value, a directed load's vector scale).
#include <cuda_runtime.h>

#include <cstdlib>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "dual.cuh"
#include "efem_internal.h"
#include "mechanics.cuh"

namespace efem {

template <>
__device__ __forceinline__ Dual drcbrt<Dual>(Dual x)
{
    const double r = rcbrt(x.v);
    return Dual(r, -(1.0 / 3.0) * (r * r) * (r * r) * x.d);  // d J^{-1/3} / dJ = -J^{-4/3} / 3
}

namespace {

constexpr int kBlock = 128;
constexpr int kVec = 256;        // threads of the vector kernels
constexpr int kDotBlocks = 128;  // CTAs per dot product
constexpr size_t kStoredBytes = size_t(8) << 30;  // most device memory the stored tangents may take

struct TanElemArgs {
    int n, n_free;
    const int* __restrict__ conn;   // [NEN][n]
    const int* __restrict__ mat;    // [n]
    const double* __restrict__ vol;
    const double* __restrict__ J0inv;
    const double* __restrict__ dN;
    const double* __restrict__ gw;
    const MatParams<Dual>* __restrict__ mats;
    const double* __restrict__ u;
    const double* __restrict__ v;   // direction (nullptr: none)
    double* __restrict__ out;       // += derivative of r
};

// elements per CTA of the tangent kernel (dual numbers double the shared memory)
__host__ __device__ constexpr int tan_epb(int ngp) { return (kBlock / ngp) < 1 ? 1 : ((kBlock / ngp) > 32 ? 32 : kBlock / ngp); }

// The element residual of residual.cu on dual numbers: out += d r_el.
template <int NEN, int NGP>
__global__ void __launch_bounds__(kBlock) k_elem_tangent(TanElemArgs a)
{
    constexpr int EPB = tan_epb(NGP);
    __shared__ Dual s_u[EPB][NEN][3];
    __shared__ Dual s_S[EPB][NGP][9];
    __shared__ double s_dN[NGP][NEN][3];
    __shared__ int s_node[EPB][NEN];
    const int tid = threadIdx.x;
    for (int i = tid; i < NGP * NEN * 3; i += kBlock) (&s_dN[0][0][0])[i] = a.dN[i];
    const int e0 = blockIdx.x * EPB;
    for (int i = tid; i < EPB * NEN; i += kBlock) {
        const int el = i % EPB, nd = i / EPB, e = e0 + el;
        int node = a.n_free;
        Dual x[3];
        if (e < a.n) {
            node = a.conn[static_cast<size_t>(nd) * a.n + e];
            if (node < a.n_free)
#pragma unroll
                for (int c = 0; c < 3; c++) x[c] = Dual(a.u[3 * node + c], a.v ? a.v[3 * node + c] : 0.0);
        }
        s_node[el][nd] = node;
#pragma unroll
        for (int c = 0; c < 3; c++) s_u[el][nd][c] = x[c];
    }
    __syncthreads();
    if (tid < EPB * NGP) {
        const int el = tid / NGP, g = tid % NGP, e = e0 + el;
        if (e < a.n) {
            Dual A[9];
            for (int q = 0; q < NEN; q++)
#pragma unroll
                for (int i = 0; i < 3; i++)
#pragma unroll
                    for (int k = 0; k < 3; k++) A[3 * i + k] += s_u[el][q][i] * Dual(s_dN[g][q][k]);
            const double* Ji = a.J0inv + (static_cast<size_t>(e) * NGP + g) * 9;
            Dual H[9];
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++)
                    H[3 * i + j] = A[3 * i] * Dual(Ji[j]) + A[3 * i + 1] * Dual(Ji[3 + j]) + A[3 * i + 2] * Dual(Ji[6 + j]);
            const MatParams<Dual> mp = a.mats[a.mat[e]];
            Dual P[9];
            piola(mp, H, P);
            const Dual wv = Dual(a.vol[e] * a.gw[g]);
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++)
                    s_S[el][g][3 * i + j] =
                        wv * (P[3 * i] * Dual(Ji[3 * j]) + P[3 * i + 1] * Dual(Ji[3 * j + 1]) + P[3 * i + 2] * Dual(Ji[3 * j + 2]));
        }
    }
    __syncthreads();
    for (int i = tid; i < EPB * NEN; i += kBlock) {
        const int el = i % EPB, nd = i / EPB, e = e0 + el;
        if (e >= a.n) continue;
        const int node = s_node[el][nd];
        if (node >= a.n_free) continue;
        double r[3] = { 0, 0, 0 };
        for (int g = 0; g < NGP; g++) {
            const double* d = s_dN[g][nd];
            const Dual* S = s_S[el][g];
#pragma unroll
            for (int c = 0; c < 3; c++) r[c] += S[3 * c].d * d[0] + S[3 * c + 1].d * d[1] + S[3 * c + 2].d * d[2];
        }
#pragma unroll
        for (int c = 0; c < 3; c++) atomicAdd(a.out + 3 * node + c, r[c]);
    }
}

// The Gauss-point tangents at a fixed u: C[9 m + p][e NGP + g] = dP_p / dH_m
// (H = du/dX), one thread per (element, Gauss point, m) with the dual seed
// on H_m; stored once per adjoint solve so that every Krylov iteration's
// K_el v is a linear map of grad v instead of a dual-number P(F).
template <int NEN, int NGP>
__global__ void __launch_bounds__(kBlock) k_gp_tangent(TanElemArgs a, double* __restrict__ C)
{
    const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long long ng = static_cast<long long>(a.n) * NGP;
    if (idx >= ng * 9) return;
    const int m = static_cast<int>(idx % 9);
    const long long eg = idx / 9;
    const int e = static_cast<int>(eg / NGP), g = static_cast<int>(eg % NGP);
    double A[9] = { 0, 0, 0, 0, 0, 0, 0, 0, 0 };
    for (int q = 0; q < NEN; q++) {
        const int node = a.conn[static_cast<size_t>(q) * a.n + e];
        if (node >= a.n_free) continue;
        const double* dN = a.dN + (g * NEN + q) * 3;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const double ui = a.u[3 * node + i];
#pragma unroll
            for (int k = 0; k < 3; k++) A[3 * i + k] += ui * dN[k];
        }
    }
    const double* Ji = a.J0inv + (static_cast<size_t>(e) * NGP + g) * 9;
    Dual H[9];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++)
            H[3 * i + j] = Dual(A[3 * i] * Ji[j] + A[3 * i + 1] * Ji[3 + j] + A[3 * i + 2] * Ji[6 + j], 3 * i + j == m ? 1.0 : 0.0);
    const MatParams<Dual> mp = a.mats[a.mat[e]];
    Dual P[9];
    piola(mp, H, P);
#pragma unroll
    for (int p = 0; p < 9; p++) C[static_cast<size_t>(9 * m + p) * ng + eg] = P[p].d;
}

// out += K_el v from the stored Gauss-point tangents: the phases of
// k_elem_tangent with dP = C : dH, dH = grad v, in place of the dual P(F).
template <int NEN, int NGP>
__global__ void __launch_bounds__(kBlock) k_elem_tangent_stored(TanElemArgs a, const double* __restrict__ C)
{
    constexpr int EPB = tan_epb(NGP);
    constexpr int SV = (NEN * 3) | 1, SS = 9 | 1;
    __shared__ double s_v[EPB][SV];
    __shared__ double s_S[EPB][NGP][SS];
    __shared__ double s_dN[NGP][NEN][3];
    __shared__ int s_node[EPB][NEN];
    const int tid = threadIdx.x;
    for (int i = tid; i < NGP * NEN * 3; i += kBlock) (&s_dN[0][0][0])[i] = a.dN[i];
    const int e0 = blockIdx.x * EPB;
    for (int i = tid; i < EPB * NEN; i += kBlock) {
        const int el = i % EPB, nd = i / EPB, e = e0 + el;
        int node = a.n_free;
        double x[3] = { 0, 0, 0 };
        if (e < a.n) {
            node = a.conn[static_cast<size_t>(nd) * a.n + e];
            if (node < a.n_free)
#pragma unroll
                for (int c = 0; c < 3; c++) x[c] = a.v[3 * node + c];
        }
        s_node[el][nd] = node;
#pragma unroll
        for (int c = 0; c < 3; c++) s_v[el][3 * nd + c] = x[c];
    }
    __syncthreads();
    if (tid < EPB * NGP) {
        const int el = tid / NGP, g = tid % NGP, e = e0 + el;
        if (e < a.n) {
            double A[9] = { 0, 0, 0, 0, 0, 0, 0, 0, 0 };
            for (int q = 0; q < NEN; q++)
#pragma unroll
                for (int i = 0; i < 3; i++)
#pragma unroll
                    for (int k = 0; k < 3; k++) A[3 * i + k] += s_v[el][3 * q + i] * s_dN[g][q][k];
            const double* Ji = a.J0inv + (static_cast<size_t>(e) * NGP + g) * 9;
            double dH[9];
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) dH[3 * i + j] = A[3 * i] * Ji[j] + A[3 * i + 1] * Ji[3 + j] + A[3 * i + 2] * Ji[6 + j];
            const size_t ng = static_cast<size_t>(a.n) * NGP, eg = static_cast<size_t>(e) * NGP + g;
            double dP[9] = { 0, 0, 0, 0, 0, 0, 0, 0, 0 };
#pragma unroll
            for (int mm = 0; mm < 9; mm++)
#pragma unroll
                for (int p = 0; p < 9; p++) dP[p] += C[(9 * mm + p) * ng + eg] * dH[mm];
            const double wv = a.vol[e] * a.gw[g];
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++)
                    s_S[el][g][3 * i + j] = wv * (dP[3 * i] * Ji[3 * j] + dP[3 * i + 1] * Ji[3 * j + 1] + dP[3 * i + 2] * Ji[3 * j + 2]);
        }
    }
    __syncthreads();
    for (int i = tid; i < EPB * NEN; i += kBlock) {
        const int el = i % EPB, nd = i / EPB, e = e0 + el;
        if (e >= a.n) continue;
        const int node = s_node[el][nd];
        if (node >= a.n_free) continue;
        double r[3] = { 0, 0, 0 };
        for (int g = 0; g < NGP; g++) {
            const double* d = s_dN[g][nd];
            const double* S = s_S[el][g];
#pragma unroll
            for (int c = 0; c < 3; c++) r[c] += S[3 * c] * d[0] + S[3 * c + 1] * d[1] + S[3 * c + 2] * d[2];
        }
#pragma unroll
        for (int c = 0; c < 3; c++) atomicAdd(a.out + 3 * node + c, r[c]);
    }
}

struct TanFaceArgs {
    int n, n_free;
    const int* __restrict__ conn;
    const int* __restrict__ table;
    const int* __restrict__ load_idx;
    const double* __restrict__ A0;
    const double* __restrict__ J0inv;
    const double* __restrict__ load;
    const int* __restrict__ t_ngp;
    const double* __restrict__ t_w;
    const double* __restrict__ t_N;
    const double* __restrict__ t_dN;
    const double* __restrict__ u;
    const double* __restrict__ v;       // direction (nullptr: none)
    const double* __restrict__ dscale;  // per pressure load: derivative of its scale (nullptr: none)
    const double* __restrict__ w;       // transpose products: the vector K^T is applied to
    double* __restrict__ out;
};

// Nodal forces f_q (all NEN nodes, dual) of face f with node displacements uu,
// as in the face residual of residual.cu; the load value's derivative is
// dscale times the load (pressure value, or directed vector).
template <int NEN>
__device__ void face_forces(const TanFaceArgs& a, int f, const Dual (*uu)[3], Dual (*fq)[3])
{
    const int t = a.table[f];
    const int ngp = a.t_ngp[t];
    const double* L = a.load + 4 * f;
    const bool directed = L[0] != 0.0;
    const double ds = a.dscale ? a.dscale[a.load_idx[f]] : 0.0;
    Dual cA[MAX_FGP][3];
    for (int g = 0; g < ngp; g++) {
        const double* dN = a.t_dN + (static_cast<size_t>(t) * MAX_FGP + g) * NEN * 3;
        Dual A[9];
        for (int q = 0; q < NEN; q++)
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int k = 0; k < 3; k++) A[3 * i + k] += uu[q][i] * Dual(dN[3 * q + k]);
        const double* Ji = a.J0inv + (static_cast<size_t>(f) * MAX_FGP + g) * 9;
        Dual H[9];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
                H[3 * i + j] = A[3 * i] * Dual(Ji[j]) + A[3 * i + 1] * Dual(Ji[3 + j]) + A[3 * i + 2] * Dual(Ji[6 + j]);
        Kin<Dual> k;
        kinematics(H, k);
        const Dual A0[3] = { Dual(a.A0[3 * f]), Dual(a.A0[3 * f + 1]), Dual(a.A0[3 * f + 2]) };
#pragma unroll
        for (int i = 0; i < 3; i++) cA[g][i] = A0[i] + k.B[3 * i] * A0[0] + k.B[3 * i + 1] * A0[1] + k.B[3 * i + 2] * A0[2];
        if (directed) cA[g][0] = sqrt(cA[g][0] * cA[g][0] + cA[g][1] * cA[g][1] + cA[g][2] * cA[g][2]);
    }
    for (int q = 0; q < NEN; q++) {
        Dual s[3];
        for (int g = 0; g < ngp; g++) {
            const Dual wn = Dual(a.t_w[t * MAX_FGP + g] * a.t_N[(static_cast<size_t>(t) * MAX_FGP + g) * NEN + q]);
            if (directed) {
                s[0] += wn * cA[g][0];
            } else {
#pragma unroll
                for (int i = 0; i < 3; i++) s[i] += wn * cA[g][i];
            }
        }
        if (directed) {
#pragma unroll
            for (int i = 0; i < 3; i++) fq[q][i] = Dual(L[1 + i]) * s[0] + Dual(0.0, ds * L[1 + i] * s[0].v);
        } else {
#pragma unroll
            for (int i = 0; i < 3; i++) fq[q][i] = Dual(L[1]) * s[i] + Dual(0.0, ds * s[i].v);
        }
    }
}

// out -= d f (the face part of R is -f): K_face v, or dR/dscale
template <int NEN>
__global__ void __launch_bounds__(kBlock) k_face_tangent(TanFaceArgs a)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= a.n) return;
    int node[NEN];
    Dual uu[NEN][3];
    for (int q = 0; q < NEN; q++) {
        node[q] = a.conn[static_cast<size_t>(q) * a.n + f];
        const bool fr = node[q] < a.n_free;
#pragma unroll
        for (int c = 0; c < 3; c++)
            uu[q][c] = fr ? Dual(a.u[3 * node[q] + c], a.v ? a.v[3 * node[q] + c] : 0.0) : Dual(0.0);
    }
    Dual fq[NEN][3];
    face_forces<NEN>(a, f, uu, fq);
    for (int q = 0; q < NEN; q++) {
        if (node[q] >= a.n_free) continue;
#pragma unroll
        for (int c = 0; c < 3; c++) atomicAdd(a.out + 3 * node[q] + c, -fq[q][c].d);
    }
}

// out_j -= sum_i w_i d f_i / d u_j for every free unknown j of every face:
// one thread per (face, local unknown), the seed on that unknown
template <int NEN>
__global__ void __launch_bounds__(kBlock) k_face_transpose(TanFaceArgs a)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = idx / (3 * NEN), j = idx % (3 * NEN);
    if (f >= a.n) return;
    const int qj = j / 3, cj = j % 3;
    int node[NEN];
    Dual uu[NEN][3];
    for (int q = 0; q < NEN; q++) {
        node[q] = a.conn[static_cast<size_t>(q) * a.n + f];
        const bool fr = node[q] < a.n_free;
#pragma unroll
        for (int c = 0; c < 3; c++) uu[q][c] = fr ? Dual(a.u[3 * node[q] + c], (q == qj && c == cj) ? 1.0 : 0.0) : Dual(0.0);
    }
    if (node[qj] >= a.n_free) return;
    Dual fq[NEN][3];
    face_forces<NEN>(a, f, uu, fq);
    double s = 0.0;
    for (int q = 0; q < NEN; q++) {
        if (node[q] >= a.n_free) continue;
#pragma unroll
        for (int c = 0; c < 3; c++) s += a.w[3 * node[q] + c] * fq[q][c].d;
    }
    atomicAdd(a.out + 3 * node[qj] + cj, -s);
}

// The face tangent blocks at a fixed u: blk[f][i][j] = d f_i / d u_j over the
// 3 NEN local unknowns (rows i of fixed nodes are 0; columns j of fixed nodes
// are not written).  One thread per (face, local unknown j), seeded as in
// k_face_transpose, so each block costs one set of dual passes per adjoint
// solve instead of one per Krylov iteration.
template <int NEN>
__global__ void __launch_bounds__(kBlock) k_face_block(TanFaceArgs a, double* __restrict__ blk)
{
    constexpr int ND = 3 * NEN;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = idx / ND, j = idx % ND;
    if (f >= a.n) return;
    const int qj = j / 3, cj = j % 3;
    int node[NEN];
    Dual uu[NEN][3];
    for (int q = 0; q < NEN; q++) {
        node[q] = a.conn[static_cast<size_t>(q) * a.n + f];
        const bool fr = node[q] < a.n_free;
#pragma unroll
        for (int c = 0; c < 3; c++) uu[q][c] = fr ? Dual(a.u[3 * node[q] + c], (q == qj && c == cj) ? 1.0 : 0.0) : Dual(0.0);
    }
    if (node[qj] >= a.n_free) return;
    Dual fq[NEN][3];
    face_forces<NEN>(a, f, uu, fq);
    double* b = blk + static_cast<size_t>(f) * ND * ND + j;
    for (int q = 0; q < NEN; q++) {
        const bool fr = node[q] < a.n_free;
#pragma unroll
        for (int c = 0; c < 3; c++) b[(3 * q + c) * ND] = fr ? fq[q][c].d : 0.0;
    }
}

// out_j -= sum_i w_i blk[f][i][j]: the transpose product of k_face_transpose
// from the stored blocks, one thread per (face, local unknown j); a warp's
// reads of row i are consecutive in j.
template <int NEN>
__global__ void __launch_bounds__(kBlock) k_face_block_apply(TanFaceArgs a, const double* __restrict__ blk)
{
    constexpr int ND = 3 * NEN;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = idx / ND, j = idx % ND;
    if (f >= a.n) return;
    const int nj = a.conn[static_cast<size_t>(j / 3) * a.n + f];
    if (nj >= a.n_free) return;
    const double* b = blk + static_cast<size_t>(f) * ND * ND + j;
    double s0 = 0.0, s1 = 0.0;
    for (int q = 0; q < NEN; q++) {
        const int nq = a.conn[static_cast<size_t>(q) * a.n + f];
        if (nq >= a.n_free) continue;
        const double* wq = a.w + 3 * nq;
        s0 += wq[0] * b[(3 * q) * ND] + wq[2] * b[(3 * q + 2) * ND];
        s1 += wq[1] * b[(3 * q + 1) * ND];
    }
    atomicAdd(a.out + 3 * nj + j % 3, -(s0 + s1));
}

// ---------------------------------------------------------------- vectors
// per-CTA partial sums of the dot products x_k . y (k < nk) into part[k][blockIdx.x]
__global__ void __launch_bounds__(kVec) k_dots(const double* __restrict__ X, size_t ldx, int nk,
    const double* __restrict__ y, size_t n, double* __restrict__ part)
{
    __shared__ double sh[kVec / 32];
    const int k = blockIdx.y;
    const double* x = X + k * ldx;
    double s = 0.0;
    for (size_t i = blockIdx.x * (size_t)kVec + threadIdx.x; i < n; i += (size_t)gridDim.x * kVec) s += x[i] * y[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < kVec / 32; q++) t += sh[q];
        part[static_cast<size_t>(k) * gridDim.x + blockIdx.x] = t;
    }
}

// y += sum_k c_k x_k, two entries per thread (16-byte loads; ldx and n even,
// y and X 16-byte aligned)
__global__ void __launch_bounds__(kVec) k_axpys2(double* __restrict__ y, const double* __restrict__ X, size_t ldx, int nk,
    const double* __restrict__ c, size_t n)
{
    const size_t n2 = n / 2, ld2 = ldx / 2;
    const double2* X2 = reinterpret_cast<const double2*>(X);
    double2* y2 = reinterpret_cast<double2*>(y);
    for (size_t i = blockIdx.x * (size_t)kVec + threadIdx.x; i < n2; i += (size_t)gridDim.x * kVec) {
        double2 s0 = y2[i], s1 = make_double2(0.0, 0.0), s2 = s1, s3 = s1;
        int k = 0;
        for (; k + 4 <= nk; k += 4) {
            const double2 a = X2[k * ld2 + i], b = X2[(k + 1) * ld2 + i];
            const double2 d = X2[(k + 2) * ld2 + i], e = X2[(k + 3) * ld2 + i];
            s0.x += c[k] * a.x;
            s0.y += c[k] * a.y;
            s1.x += c[k + 1] * b.x;
            s1.y += c[k + 1] * b.y;
            s2.x += c[k + 2] * d.x;
            s2.y += c[k + 2] * d.y;
            s3.x += c[k + 3] * e.x;
            s3.y += c[k + 3] * e.y;
        }
        for (; k < nk; k++) {
            const double2 a = X2[k * ld2 + i];
            s0.x += c[k] * a.x;
            s0.y += c[k] * a.y;
        }
        y2[i] = make_double2((s0.x + s1.x) + (s2.x + s3.x), (s0.y + s1.y) + (s2.y + s3.y));
    }
}

// y += sum_k c_k x_k (coefficients in device memory)
__global__ void __launch_bounds__(kVec) k_axpys(double* __restrict__ y, const double* __restrict__ X, size_t ldx, int nk,
    const double* __restrict__ c, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)kVec + threadIdx.x; i < n; i += (size_t)gridDim.x * kVec) {
        // four independent sums keep four loads of X in flight per thread
        double s0 = y[i], s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int k = 0;
        for (; k + 4 <= nk; k += 4) {
            s0 += c[k] * X[k * ldx + i];
            s1 += c[k + 1] * X[(k + 1) * ldx + i];
            s2 += c[k + 2] * X[(k + 2) * ldx + i];
            s3 += c[k + 3] * X[(k + 3) * ldx + i];
        }
        for (; k < nk; k++) s0 += c[k] * X[k * ldx + i];
        y[i] = (s0 + s1) + (s2 + s3);
    }
}

// one warp per row k < nk: s_k = sum of part[k][0..nb) in order; hacc[k] = s_k
// (accumulate: hacc[k] += s_k) and coef[k] = -s_k
__global__ void k_rows_reduce(const double* __restrict__ part, int nk, int nb, double* __restrict__ hacc,
    double* __restrict__ coef, int accumulate)
{
    const int k = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (k >= nk) return;
    double s = 0.0;
    for (int b = lane; b < nb; b += 32) s += part[static_cast<size_t>(k) * nb + b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        hacc[k] = accumulate ? hacc[k] + s : s;
        coef[k] = -s;
    }
}

// *out = sqrt(sum of part[0..nb))
__global__ void k_norm_reduce(const double* __restrict__ part, int nb, double* __restrict__ out)
{
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += 32) s += part[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) *out = ::sqrt(s);
}

// y = x / *s (0 when *s is 0)
__global__ void __launch_bounds__(kVec) k_scale_inv(double* __restrict__ y, const double* __restrict__ x,
    const double* __restrict__ s, size_t n)
{
    const double d = *s;
    const double f = d > 0.0 ? 1.0 / d : 0.0;
    for (size_t i = blockIdx.x * (size_t)kVec + threadIdx.x; i < n; i += (size_t)gridDim.x * kVec) y[i] = f * x[i];
}

__global__ void __launch_bounds__(kVec) k_scale_copy(double* __restrict__ y, const double* __restrict__ x, double s, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)kVec + threadIdx.x; i < n; i += (size_t)gridDim.x * kVec) y[i] = s * x[i];
}

int vec_grid(size_t n) { return static_cast<int>(std::min<size_t>(592, std::max<size_t>(1, (n + kVec - 1) / kVec))); }

// y += sum_k c_k X_k (rows of stride ldx): the 16-byte form when the layout allows
void launch_axpys(cudaStream_t st, double* y, const double* X, size_t ldx, int nk, const double* c, size_t n)
{
    const bool v2 = n % 2 == 0 && ldx % 2 == 0 && reinterpret_cast<uintptr_t>(y) % 16 == 0 &&
        reinterpret_cast<uintptr_t>(X) % 16 == 0;
    if (v2) k_axpys2<<<vec_grid(n / 2), kVec, 0, st>>>(y, X, ldx, nk, c, n);
    else k_axpys<<<vec_grid(n), kVec, 0, st>>>(y, X, ldx, nk, c, n);
}

}  // namespace

struct AdjointWS {
    size_t n = 0;
    int restart = 0;
    double *V = nullptr, *Z = nullptr;  // Krylov basis and preconditioned basis, (restart + 1) x n
    double *w = nullptr, *x = nullptr, *b = nullptr, *t = nullptr, *u = nullptr, *io = nullptr;
    double *part = nullptr, *coef = nullptr;
    double* hcol = nullptr;    // device: the Hessenberg column being formed
    double* h_hcol = nullptr;  // pinned host copy
    MatParams<Dual>* mats = nullptr;
    double* dscale = nullptr;
    std::vector<double> h_part;
    // stored tangents at u, used while blocks_ready is set (inside one adjoint
    // solve): per face set the face blocks (k_face_block), per element block
    // the Gauss-point tangents (k_gp_tangent)
    std::vector<double*> fblk, gpt;
    bool blocks_ready = false;
};

void free_adjoint(Model& m)
{
    if (!m.aws) return;
    AdjointWS& w = *m.aws;
    for (double** p : { &w.V, &w.Z, &w.w, &w.x, &w.b, &w.t, &w.u, &w.io, &w.part, &w.coef, &w.dscale, &w.hcol })
        dev_free(*p);
    if (w.mats) cudaFree(w.mats);
    if (w.h_hcol) cudaFreeHost(w.h_hcol);
    for (double*& p : w.fblk) dev_free(p);
    for (double*& p : w.gpt) dev_free(p);
    delete m.aws;
    m.aws = nullptr;
}

namespace {

constexpr int kRestart = 100;

efem_status alloc_aws(Model& m)
{
    const size_t n = 3 * static_cast<size_t>(m.n_free);
    if (m.aws && m.aws->n == n) return EFEM_OK;
    free_adjoint(m);
    m.aws = new AdjointWS();
    AdjointWS& w = *m.aws;
    w.n = n;
    w.restart = kRestart;
    efem_status s;
    const size_t nb = static_cast<size_t>(kRestart + 1) * std::max<size_t>(n, 1);
    if ((s = dev_alloc(&w.V, nb)) != EFEM_OK) return s;
    if ((s = dev_alloc(&w.Z, nb)) != EFEM_OK) return s;
    for (double** p : { &w.w, &w.x, &w.b, &w.t, &w.u, &w.io })
        if ((s = dev_alloc(p, std::max<size_t>(n, 1))) != EFEM_OK) return s;
    if ((s = dev_alloc(&w.part, static_cast<size_t>(kRestart + 1) * kDotBlocks)) != EFEM_OK) return s;
    if ((s = dev_alloc(&w.coef, static_cast<size_t>(kRestart + 1))) != EFEM_OK) return s;
    if ((s = dev_alloc(&w.hcol, static_cast<size_t>(kRestart + 2))) != EFEM_OK) return s;
    EFEM_CUDA(cudaMallocHost(&w.h_hcol, sizeof(double) * (kRestart + 2)));
    if ((s = dev_alloc(&w.dscale, static_cast<size_t>(std::max(m.n_pressure_loads, 1)))) != EFEM_OK) return s;
    EFEM_CUDA(cudaMalloc(&w.mats, sizeof(MatParams<Dual>) * MAX_MATS));
    w.h_part.resize(static_cast<size_t>(kRestart + 1) * kDotBlocks);
    return EFEM_OK;
}

// material table on dual numbers; seed (slot, k) puts derivative 1 on constant
// k (0 C10, 1 C01, 2 C20, 3 C30, 4 D1) of material slot `slot` (-1: none)
efem_status upload_dual_mats(Model& m, int slot, int k)
{
    std::vector<MatParams<Dual>> h(std::max<size_t>(m.materials_used.size(), 1));
    for (size_t i = 0; i < m.materials_used.size(); i++) {
        const HostMaterial& hm = m.materials_used[i];
        const bool s = static_cast<int>(i) == slot;
        h[i].type = hm.type;
        h[i].C10 = Dual(hm.C10, s && k == 0 ? 1.0 : 0.0);
        h[i].C01 = Dual(hm.C01, s && k == 1 ? 1.0 : 0.0);
        h[i].C20 = Dual(hm.C20, s && k == 2 ? 1.0 : 0.0);
        h[i].C30 = Dual(hm.C30, s && k == 3 ? 1.0 : 0.0);
        h[i].D1 = Dual(hm.D1, s && k == 4 ? 1.0 : 0.0);
    }
    EFEM_CUDA(cudaMemcpyAsync(m.aws->mats, h.data(), sizeof(MatParams<Dual>) * h.size(), cudaMemcpyHostToDevice, m.stream));
    return EFEM_OK;
}

// out += K_el v (dual kernels; from the stored Gauss-point tangents when
// stored is set, which needs v and blocks_ready), or dR/dtheta with v = nullptr
void launch_elem_tangent(Model& m, const double* u, const double* v, double* out, bool stored = false)
{
    for (size_t bi = 0; bi < m.blocks.size(); bi++) {
        auto& b = m.blocks[bi];
        if (b.n == 0) continue;
        TanElemArgs a { b.n, m.n_free, b.conn, b.mat, b.vol, b.J0inv, b.dN, b.gw, m.aws->mats, u, v, out };
        const double* C = stored ? m.aws->gpt[bi] : nullptr;
        auto go = [&](auto kern, auto kern_stored, int ngp) {
            const int epb = tan_epb(ngp);
            if (C) kern_stored<<<(b.n + epb - 1) / epb, kBlock, 0, m.stream>>>(a, C);
            else kern<<<(b.n + epb - 1) / epb, kBlock, 0, m.stream>>>(a);
            m.launches++;
        };
#define EFEM_TAN(NEN, NGP) go(k_elem_tangent<NEN, NGP>, k_elem_tangent_stored<NEN, NGP>, NGP)
        if (b.nen == 4 && b.ngp == 1) EFEM_TAN(4, 1);
        else if (b.nen == 10 && b.ngp == 4) EFEM_TAN(10, 4);
        else if (b.nen == 10 && b.ngp == 1) EFEM_TAN(10, 1);
        else if (b.nen == 8 && b.ngp == 8) EFEM_TAN(8, 8);
        else if (b.nen == 8 && b.ngp == 1) EFEM_TAN(8, 1);
        else if (b.nen == 20 && b.ngp == 27) EFEM_TAN(20, 27);
        else if (b.nen == 20 && b.ngp == 8) EFEM_TAN(20, 8);
#undef EFEM_TAN
    }
}

// mode 0: out -= K_face v;  1: out -= dF/dscale;  2: out -= K_face^T w
void launch_face_tangent(Model& m, const double* u, const double* v, const double* dscale, const double* w,
    double* out, bool transpose)
{
    const AdjointWS* ws = m.aws;
    for (size_t fs = 0; fs < m.faces.size(); fs++) {
        auto& f = m.faces[fs];
        if (f.n == 0) continue;
        TanFaceArgs a { f.n, m.n_free, f.conn, f.table, f.load_idx, f.A0, f.J0inv, f.load, f.t_ngp, f.t_w, f.t_N,
            f.t_dN, u, v, dscale, w, out };
        const int nthreads = transpose ? f.n * 3 * f.nen : f.n;
        const int grid = (nthreads + kBlock - 1) / kBlock;
        const double* blk = transpose && ws && ws->blocks_ready ? ws->fblk[fs] : nullptr;
        m.launches++;
        switch (f.nen) {
        case 4:
            if (blk) k_face_block_apply<4><<<grid, kBlock, 0, m.stream>>>(a, blk);
            else if (transpose) k_face_transpose<4><<<grid, kBlock, 0, m.stream>>>(a);
            else k_face_tangent<4><<<grid, kBlock, 0, m.stream>>>(a);
            break;
        case 8:
            if (blk) k_face_block_apply<8><<<grid, kBlock, 0, m.stream>>>(a, blk);
            else if (transpose) k_face_transpose<8><<<grid, kBlock, 0, m.stream>>>(a);
            else k_face_tangent<8><<<grid, kBlock, 0, m.stream>>>(a);
            break;
        case 10:
            if (blk) k_face_block_apply<10><<<grid, kBlock, 0, m.stream>>>(a, blk);
            else if (transpose) k_face_transpose<10><<<grid, kBlock, 0, m.stream>>>(a);
            else k_face_tangent<10><<<grid, kBlock, 0, m.stream>>>(a);
            break;
        case 20:
            if (blk) k_face_block_apply<20><<<grid, kBlock, 0, m.stream>>>(a, blk);
            else if (transpose) k_face_transpose<20><<<grid, kBlock, 0, m.stream>>>(a);
            else k_face_tangent<20><<<grid, kBlock, 0, m.stream>>>(a);
            break;
        }
    }
}

// Out of device memory for the stored tangents: free them and go on with the
// dual-number products (blocks_ready stays unset).
efem_status drop_stored(AdjointWS& w)
{
    for (double*& p : w.fblk) dev_free(p);
    for (double*& p : w.gpt) dev_free(p);
    w.blocks_ready = false;
    return EFEM_OK;
}

// Device memory for stored tangents.  Running out of memory is not an error
// (*oom is set and the caller falls back to the dual-number products); any
// other failure is.  The environment variable EFEM_TEST_STORED_OOM=1 makes
// every such allocation report out of memory, so that tests reach the
// fallback without filling the GPU.
efem_status stored_alloc(double** p, size_t n, bool* oom)
{
    *p = nullptr;
    *oom = false;
    if (n == 0) return EFEM_OK;
    const char* force = std::getenv("EFEM_TEST_STORED_OOM");
    if (force && force[0] == '1') {
        *oom = true;
        return EFEM_OK;
    }
    const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(double));
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();  // not sticky: clear it so that later checks do not see it
        *p = nullptr;
        *oom = true;
        return EFEM_OK;
    }
    if (e != cudaSuccess) {
        *p = nullptr;
        set_error(std::string("cudaMalloc of the stored tangents: ") + cudaGetErrorString(e));
        return EFEM_ERR_CUDA;
    }
    return EFEM_OK;
}

// The stored tangents at u for the Krylov iterations of one adjoint solve:
// the face blocks of every face set and the Gauss-point tangents of every
// element block.  Sets blocks_ready only when all of them fit in
// kStoredBytes and in device memory; otherwise every product recomputes them
// on dual numbers.
efem_status build_stored_tangents(Model& m, const double* u)
{
    AdjointWS& w = *m.aws;
    w.blocks_ready = false;
    size_t total = 0;
    for (auto& f : m.faces) total += sizeof(double) * f.n * static_cast<size_t>(9 * f.nen * f.nen);
    for (auto& b : m.blocks) total += sizeof(double) * b.n * static_cast<size_t>(81 * b.ngp);
    if (total == 0 || total > kStoredBytes) return EFEM_OK;
    w.gpt.resize(m.blocks.size(), nullptr);
    for (size_t bi = 0; bi < m.blocks.size(); bi++) {
        auto& b = m.blocks[bi];
        if (b.n == 0) continue;
        const long long nthreads = 9LL * b.n * b.ngp;
        if (!w.gpt[bi]) {
            bool oom = false;
            const efem_status as = stored_alloc(&w.gpt[bi], static_cast<size_t>(9 * nthreads), &oom);
            if (as != EFEM_OK) return as;
            if (oom) return drop_stored(w);
        }
        TanElemArgs a { b.n, m.n_free, b.conn, b.mat, b.vol, b.J0inv, b.dN, b.gw, w.mats, u, nullptr, nullptr };
        const unsigned grid = static_cast<unsigned>((nthreads + kBlock - 1) / kBlock);
        double* C = w.gpt[bi];
        m.launches++;
        if (b.nen == 4 && b.ngp == 1) k_gp_tangent<4, 1><<<grid, kBlock, 0, m.stream>>>(a, C);
        else if (b.nen == 10 && b.ngp == 4) k_gp_tangent<10, 4><<<grid, kBlock, 0, m.stream>>>(a, C);
        else if (b.nen == 10 && b.ngp == 1) k_gp_tangent<10, 1><<<grid, kBlock, 0, m.stream>>>(a, C);
        else if (b.nen == 8 && b.ngp == 8) k_gp_tangent<8, 8><<<grid, kBlock, 0, m.stream>>>(a, C);
        else if (b.nen == 8 && b.ngp == 1) k_gp_tangent<8, 1><<<grid, kBlock, 0, m.stream>>>(a, C);
        else if (b.nen == 20 && b.ngp == 27) k_gp_tangent<20, 27><<<grid, kBlock, 0, m.stream>>>(a, C);
        else if (b.nen == 20 && b.ngp == 8) k_gp_tangent<20, 8><<<grid, kBlock, 0, m.stream>>>(a, C);
    }
    w.fblk.resize(m.faces.size(), nullptr);
    for (size_t fs = 0; fs < m.faces.size(); fs++) {
        auto& f = m.faces[fs];
        if (f.n == 0) continue;
        if (!w.fblk[fs]) {
            bool oom = false;
            const efem_status as = stored_alloc(&w.fblk[fs], f.n * static_cast<size_t>(9 * f.nen * f.nen), &oom);
            if (as != EFEM_OK) return as;
            if (oom) return drop_stored(w);
        }
        TanFaceArgs a { f.n, m.n_free, f.conn, f.table, f.load_idx, f.A0, f.J0inv, f.load, f.t_ngp, f.t_w, f.t_N,
            f.t_dN, u, nullptr, nullptr, nullptr, nullptr };
        const int grid = (f.n * 3 * f.nen + kBlock - 1) / kBlock;
        m.launches++;
        switch (f.nen) {
        case 4: k_face_block<4><<<grid, kBlock, 0, m.stream>>>(a, w.fblk[fs]); break;
        case 8: k_face_block<8><<<grid, kBlock, 0, m.stream>>>(a, w.fblk[fs]); break;
        case 10: k_face_block<10><<<grid, kBlock, 0, m.stream>>>(a, w.fblk[fs]); break;
        case 20: k_face_block<20><<<grid, kBlock, 0, m.stream>>>(a, w.fblk[fs]); break;
        }
    }
    EFEM_CUDA(cudaGetLastError());
    w.blocks_ready = true;
    return EFEM_OK;
}

// out = K(u) v  (transpose: K(u)^T v); device pointers; dual materials without seeds uploaded
efem_status tangent(Model& m, const double* u, const double* v, double* out, bool transpose)
{
    EFEM_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * 3 * m.n_free, m.stream));
    launch_elem_tangent(m, u, v, out, m.aws->blocks_ready);
    if (transpose)
        launch_face_tangent(m, u, nullptr, nullptr, v, out, true);
    else
        launch_face_tangent(m, u, v, nullptr, nullptr, out, false);
    EFEM_CUDA(cudaGetLastError());
    return EFEM_OK;
}

// out = dR/dtheta_k at u (parameter order in the file comment)
efem_status param_derivative(Model& m, const double* u, int k, double* out)
{
    const int nm = static_cast<int>(m.materials_used.size());
    EFEM_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * 3 * m.n_free, m.stream));
    if (k < 5 * nm) {
        efem_status s = upload_dual_mats(m, k / 5, k % 5);
        if (s != EFEM_OK) return s;
        launch_elem_tangent(m, u, nullptr, out);
        s = upload_dual_mats(m, -1, 0);
        if (s != EFEM_OK) return s;
    } else {
        std::vector<double> ds(std::max(m.n_pressure_loads, 1), 0.0);
        ds[k - 5 * nm] = 1.0;
        EFEM_CUDA(cudaMemcpyAsync(m.aws->dscale, ds.data(), sizeof(double) * ds.size(), cudaMemcpyHostToDevice, m.stream));
        launch_face_tangent(m, u, nullptr, m.aws->dscale, nullptr, out, false);
        // synchronise before ds goes out of scope
        EFEM_CUDA(cudaStreamSynchronize(m.stream));
    }
    EFEM_CUDA(cudaGetLastError());
    return EFEM_OK;
}

// dot products X_k . y for k < nk (X rows of stride n), summed on the host in CTA order
efem_status dots(Model& m, const double* X, int nk, const double* y, double* res)
{
    AdjointWS& w = *m.aws;
    const size_t n = w.n;
    k_dots<<<dim3(kDotBlocks, nk), kVec, 0, m.stream>>>(X, n, nk, y, n, w.part);
    m.launches++;
    EFEM_CUDA(cudaMemcpyAsync(w.h_part.data(), w.part, sizeof(double) * nk * kDotBlocks, cudaMemcpyDeviceToHost, m.stream));
    EFEM_CUDA(cudaStreamSynchronize(m.stream));
    for (int k = 0; k < nk; k++) {
        double s = 0.0;
        for (int b = 0; b < kDotBlocks; b++) s += w.h_part[static_cast<size_t>(k) * kDotBlocks + b];
        res[k] = s;
    }
    return EFEM_OK;
}

efem_status axpys(Model& m, double* y, const double* X, int nk, const double* c)
{
    AdjointWS& w = *m.aws;
    EFEM_CUDA(cudaMemcpyAsync(w.coef, c, sizeof(double) * nk, cudaMemcpyHostToDevice, m.stream));
    launch_axpys(m.stream, y, X, w.n, nk, w.coef, w.n);
    m.launches++;
    EFEM_CUDA(cudaStreamSynchronize(m.stream));  // c is host memory owned by the caller
    return EFEM_OK;
}

// Restarted GMRES(kRestart) for K(u)^T x = b, right-preconditioned with H0
// (x = H0 z); classical Gram-Schmidt applied twice.  x starts at 0.
efem_status adjoint_gmres(Model& m, const double* u, double tol, int max_it, int* iters, double* relres,
    double* bytes)
{
    AdjointWS& w = *m.aws;
    const size_t n = w.n;
    const int R = w.restart;
    // algorithmic bytes of one Krylov iteration: the basis copy, H0, the
    // transpose tangent (element part as an FP64 residual plus v and the zeroed
    // output, plus the stored Gauss-point tangents; the stored face blocks or,
    // without them, the faces' residual bytes), the norm and the scaling; plus
    // two Gram-Schmidt passes over the j + 1 basis vectors (dots: the basis and
    // w; updates: the basis, w read and written)
    const double nd = 8.0 * static_cast<double>(n);
    efem_model_info mi {};
    precond_info(m, &mi);
    long long rb = 0;
    double rf = 0.0;
    residual_work(m, 8, &rb, &rf, !w.blocks_ready);
    double fb = 0.0;
    if (w.blocks_ready) {
        for (auto& f : m.faces) fb += static_cast<double>(f.n) * (72.0 * f.nen * f.nen + 4.0 * f.nen);
        for (auto& b : m.blocks) fb += static_cast<double>(b.n) * b.ngp * 81.0 * 8.0;
    }
    const double it_bytes = 2.0 * nd + 16.0 * static_cast<double>(mi.factor_nnz) + 5.0 * nd + static_cast<double>(rb) +
        2.0 * nd + fb + 3.0 * nd;
    *bytes = 0.0;
    double bnorm = 0.0;
    efem_status s = dots(m, w.b, 1, w.b, &bnorm);
    if (s != EFEM_OK) return s;
    bnorm = std::sqrt(bnorm);
    EFEM_CUDA(cudaMemsetAsync(w.x, 0, sizeof(double) * n, m.stream));
    *iters = 0;
    *relres = 0.0;
    if (bnorm == 0.0) return EFEM_OK;
    std::vector<double> H(static_cast<size_t>(R + 1) * R), cs(R), sn(R), g(R + 1), y(R);
    double beta = bnorm;  // residual of x = 0
    EFEM_CUDA(cudaMemcpyAsync(w.t, w.b, sizeof(double) * n, cudaMemcpyDeviceToDevice, m.stream));
    int total = 0;
    while (total < max_it) {
        // V_0 = r / beta, r = t
        k_scale_copy<<<vec_grid(n), kVec, 0, m.stream>>>(w.V, w.t, 1.0 / beta, n);
        m.launches++;
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int j = 0;
        bool done = false;
        for (; j < R && total < max_it; j++, total++) {
            double* Zj = w.Z + j * n;
            EFEM_CUDA(cudaMemcpyAsync(Zj, w.V + j * n, sizeof(double) * n, cudaMemcpyDeviceToDevice, m.stream));
            if ((s = precond_enqueue(m, Zj, m.stream)) != EFEM_OK) return s;
            m.launches++;
            if ((s = tangent(m, u, Zj, w.w, true)) != EFEM_OK) return s;
            *bytes += it_bytes + 2.0 * (2.0 * (j + 1) * nd + 3.0 * nd);
            // two passes of classical Gram-Schmidt, coefficients kept on the device
            // (with H0 a good preconditioner, K^T H0 v is close to the basis: the
            // first pass removes most of w in nearly every iteration, so a
            // conditional second pass would almost always run)
            for (int pass = 0; pass < 2; pass++) {
                k_dots<<<dim3(kDotBlocks, j + 1), kVec, 0, m.stream>>>(w.V, n, j + 1, w.w, n, w.part);
                k_rows_reduce<<<(j + 1 + 7) / 8, 256, 0, m.stream>>>(w.part, j + 1, kDotBlocks, w.hcol, w.coef, pass);
                launch_axpys(m.stream, w.w, w.V, n, j + 1, w.coef, n);
                m.launches += 3;
            }
            k_dots<<<dim3(kDotBlocks, 1), kVec, 0, m.stream>>>(w.w, n, 1, w.w, n, w.part);
            k_norm_reduce<<<1, 32, 0, m.stream>>>(w.part, kDotBlocks, w.hcol + j + 1);
            k_scale_inv<<<vec_grid(n), kVec, 0, m.stream>>>(w.V + (j + 1) * n, w.w, w.hcol + j + 1, n);
            m.launches += 3;
            EFEM_CUDA(cudaMemcpyAsync(w.h_hcol, w.hcol, sizeof(double) * (j + 2), cudaMemcpyDeviceToHost, m.stream));
            EFEM_CUDA(cudaStreamSynchronize(m.stream));
            for (int i = 0; i <= j + 1; i++) H[static_cast<size_t>(i) * R + j] = w.h_hcol[i];
            const double hn = w.h_hcol[j + 1];
            // Givens rotations on column j
            for (int i = 0; i < j; i++) {
                const double a = H[static_cast<size_t>(i) * R + j], c = H[static_cast<size_t>(i + 1) * R + j];
                H[static_cast<size_t>(i) * R + j] = cs[i] * a + sn[i] * c;
                H[static_cast<size_t>(i + 1) * R + j] = -sn[i] * a + cs[i] * c;
            }
            const double a = H[static_cast<size_t>(j) * R + j], c = H[static_cast<size_t>(j + 1) * R + j];
            const double rr = std::hypot(a, c);
            cs[j] = rr > 0.0 ? a / rr : 1.0;
            sn[j] = rr > 0.0 ? c / rr : 0.0;
            H[static_cast<size_t>(j) * R + j] = rr;
            H[static_cast<size_t>(j + 1) * R + j] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            *relres = std::fabs(g[j + 1]) / bnorm;
            if (*relres <= tol || hn == 0.0) {
                j++;
                total++;
                done = true;
                break;
            }
        }
        // x += Z y, H y = g (upper triangular j x j)
        for (int i = j - 1; i >= 0; i--) {
            double t = g[i];
            for (int k = i + 1; k < j; k++) t -= H[static_cast<size_t>(i) * R + k] * y[k];
            y[i] = t / H[static_cast<size_t>(i) * R + i];
        }
        if ((s = axpys(m, w.x, w.Z, j, y.data())) != EFEM_OK) return s;
        if ((s = precond_check(m)) != EFEM_OK) return s;
        if (done) break;
        // true residual t = b - K^T x for the restart
        if ((s = tangent(m, u, w.x, w.w, true)) != EFEM_OK) return s;
        k_scale_copy<<<vec_grid(n), kVec, 0, m.stream>>>(w.t, w.b, 1.0, n);
        m.launches++;
        const double minus1 = -1.0;
        if ((s = axpys(m, w.t, w.w, 1, &minus1)) != EFEM_OK) return s;
        if ((s = dots(m, w.t, 1, w.t, &beta)) != EFEM_OK) return s;
        beta = std::sqrt(beta);
        *relres = beta / bnorm;
        if (*relres <= tol) break;
    }
    *iters = total;
    return EFEM_OK;
}

double ms_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

// ------------------------------------------------------------------ host entry points (C ABI helpers)
efem_status adjoint_io(Model& m, double** io)
{
    efem_status s = alloc_aws(m);
    if (s != EFEM_OK) return s;
    *io = m.aws->io;
    return EFEM_OK;
}

int n_params(const Model& m) { return 5 * static_cast<int>(m.materials_used.size()) + m.n_pressure_loads; }

efem_status hvp(Model& m, const double* d_u, const double* d_v, double* d_out, bool transpose)
{
    efem_status s = alloc_aws(m);
    if (s != EFEM_OK) return s;
    if ((s = upload_dual_mats(m, -1, 0)) != EFEM_OK) return s;
    return tangent(m, d_u, d_v, d_out, transpose);
}

efem_status residual_param_derivative(Model& m, const double* d_u, int k, double* d_out)
{
    if (k < 0 || k >= n_params(m)) {
        set_error("parameter index out of range");
        return EFEM_ERR_ARG;
    }
    efem_status s = alloc_aws(m);
    if (s != EFEM_OK) return s;
    return param_derivative(m, d_u, k, d_out);
}

efem_status adjoint(Model& m, const double* d_u, const double* d_dJdu, double* dJdtheta, double* d_lambda,
    efem_adjoint_info* info)
{
    const auto t0 = std::chrono::steady_clock::now();
    std::memset(info, 0, sizeof(*info));
    const long long launches0 = m.launches;
    efem_status s = alloc_aws(m);
    if (s != EFEM_OK) return s;
    AdjointWS& w = *m.aws;
    const size_t n = w.n;
    int ok = 0;
    double msf = 0.0;
    if ((s = precond_setup(m, false, &ok, &msf)) != EFEM_OK) return s;
    if (!ok) {
        set_error("approximate Jacobian is not positive definite (no preconditioner for the adjoint solve)");
        return EFEM_ERR_NAN;
    }
    if ((s = upload_dual_mats(m, -1, 0)) != EFEM_OK) return s;
    EFEM_CUDA(cudaMemcpyAsync(w.u, d_u, sizeof(double) * n, cudaMemcpyDeviceToDevice, m.stream));
    EFEM_CUDA(cudaMemcpyAsync(w.b, d_dJdu, sizeof(double) * n, cudaMemcpyDeviceToDevice, m.stream));
    const double tol = m.opts.adjoint_tolerance > 0 ? m.opts.adjoint_tolerance : 1e-8;
    const int max_it = m.opts.adjoint_max_iterations > 0 ? m.opts.adjoint_max_iterations : 2000;
    int iters = 0;
    double rel = 0.0;
    if ((s = build_stored_tangents(m, w.u)) != EFEM_OK) return s;
    s = adjoint_gmres(m, w.u, tol, max_it, &iters, &rel, &info->solve_bytes);
    w.blocks_ready = false;  // the blocks hold K at this u only
    if (s != EFEM_OK) return s;
    info->iterations = iters;
    info->rel_residual = rel;
    if (rel <= tol) info->flags |= EFEM_SOLVE_CONVERGED;
    EFEM_CUDA(cudaStreamSynchronize(m.stream));
    info->ms_solve = ms_since(t0);
    // dJ/dtheta_k = -lambda . dR/dtheta_k
    const auto t1 = std::chrono::steady_clock::now();
    const int np = n_params(m);
    for (int k = 0; k < np; k++) {
        if ((s = param_derivative(m, w.u, k, w.t)) != EFEM_OK) return s;
        double d = 0.0;
        if ((s = dots(m, w.t, 1, w.x, &d)) != EFEM_OK) return s;
        dJdtheta[k] = -d;
    }
    if (d_lambda) EFEM_CUDA(cudaMemcpyAsync(d_lambda, w.x, sizeof(double) * n, cudaMemcpyDeviceToDevice, m.stream));
    EFEM_CUDA(cudaStreamSynchronize(m.stream));
    info->ms_params = ms_since(t1);
    info->ms_total = ms_since(t0);
    info->n_kernel_launches = m.launches - launches0;
    return EFEM_OK;
}

}  // namespace efem
