// Stored strain energy of the body, summed in FP64:
//   E(u) = sum_e V_e sum_g w_g W(F_g)
// with the strain-energy functions whose derivative dW/dF is the reference's
// first Piola-Kirchhoff stress (so dE/du is the element part of R):
//   Neo-Hookean    W = C10 (I1bar - 3) + (J - 1)^2 / D1       (src/material/NeoHookean.cpp:4-20)
//   Mooney-Rivlin  W = C10 (I1bar - 3) + C01 (I2bar - 3) + (J - 1)^2 / D1   (MooneyRivlin.cpp:4-24)
//   Yeoh           W = sum_k C_k0 (I1bar - 3)^k + (J - 1)^2 / D1           (Yeoh.cpp:4-19)
// written, like the stress, in terms of H = F - I so that nothing cancels:
//   I1bar - 3 = 3 expm1(-2/3 ln J) + (I1 - 3) J^{-2/3}
//   I2bar - 3 = 3 expm1(-4/3 ln J) + (I2 - 3) J^{-4/3}
// The reference itself never evaluates an energy; this is for objectives and
// energy-based checks.  The sum is deterministic: one FP64 partial per CTA,
// added in CTA order.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "efem_internal.h"
#include "mechanics.cuh"

namespace efem {

namespace {

constexpr int kBlock = 128;

__device__ double strain_energy(const MatParams<double>& mp, const double* H)
{
    Kin<double> k;
    kinematics(H, k);
    const double lJ = dlogabs1p(k.delta);  // log|J|: |J|^{-2/3} as in the reference
    const double Jm23 = exp(-2.0 / 3.0 * lJ);
    const double i1 = 3.0 * expm1(-2.0 / 3.0 * lJ) + k.a * Jm23;  // I1bar - 3
    double W = k.delta * k.delta / mp.D1;
    if (mp.type == EFEM_YEOH)
        W += mp.C10 * i1 + mp.C20 * i1 * i1 + mp.C30 * i1 * i1 * i1;
    else
        W += mp.C10 * i1;
    if (mp.type == EFEM_MOONEY_RIVLIN) {
        double E[9];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                E[3 * i + j] = H[3 * i + j] + H[3 * j + i] + H[i] * H[j] + H[3 + i] * H[3 + j] + H[6 + i] * H[6 + j];
        const double t = E[0] + E[4] + E[8];
        double ee = 0.0;
        for (int i = 0; i < 9; i++) ee += E[i] * E[i];
        const double i2 = 2.0 * t + 0.5 * (t * t - ee);  // I2 - 3
        W += mp.C01 * (3.0 * expm1(-4.0 / 3.0 * lJ) + i2 * Jm23 * Jm23);
    }
    return W;
}

// one thread per (element, Gauss point); per-CTA partial sums
__global__ void __launch_bounds__(kBlock) k_energy(int n, int nen, int ngp, int n_free, const int* __restrict__ conn,
    const int* __restrict__ mat, const double* __restrict__ vol, const double* __restrict__ J0inv,
    const double* __restrict__ dN, const double* __restrict__ gw, const MatParams<double>* __restrict__ mats,
    const double* __restrict__ u, double* __restrict__ part)
{
    __shared__ double sh[kBlock / 32];
    const long long idx = static_cast<long long>(blockIdx.x) * kBlock + threadIdx.x;
    double W = 0.0;
    if (idx < static_cast<long long>(n) * ngp) {
        const int e = static_cast<int>(idx / ngp), g = static_cast<int>(idx % ngp);
        double A[9] = { 0, 0, 0, 0, 0, 0, 0, 0, 0 };
        for (int q = 0; q < nen; q++) {
            const int node = conn[static_cast<size_t>(q) * n + e];
            if (node >= n_free) continue;
            const double* d = dN + (static_cast<size_t>(g) * nen + q) * 3;
            for (int i = 0; i < 3; i++)
                for (int k = 0; k < 3; k++) A[3 * i + k] += u[3 * node + i] * d[k];
        }
        const double* Ji = J0inv + (static_cast<size_t>(e) * ngp + g) * 9;
        double H[9];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) H[3 * i + j] = A[3 * i] * Ji[j] + A[3 * i + 1] * Ji[3 + j] + A[3 * i + 2] * Ji[6 + j];
        W = vol[e] * gw[g] * strain_energy(mats[mat[e]], H);
    }
    for (int o = 16; o > 0; o >>= 1) W += __shfl_xor_sync(0xffffffffu, W, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = W;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < kBlock / 32; q++) s += sh[q];
        part[blockIdx.x] = s;
    }
}

// per-CTA partial sums of f . u
__global__ void __launch_bounds__(kBlock) k_dot_part(const double* __restrict__ f, const double* __restrict__ u,
    size_t n, double* __restrict__ part)
{
    __shared__ double sh[kBlock / 32];
    double s = 0.0;
    for (size_t i = blockIdx.x * static_cast<size_t>(kBlock) + threadIdx.x; i < n; i += static_cast<size_t>(gridDim.x) * kBlock)
        s += f[i] * u[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < kBlock / 32; q++) t += sh[q];
        part[blockIdx.x] = t;
    }
}

}  // namespace

// Total potential of conservative loads, Pi(u) = E(u) - f_ext . u: its
// gradient is the residual R(u), so the Armijo line search can test it.
efem_status total_potential(Model& m, const double* d_u, double* pi)
{
    double e = 0.0;
    efem_status s = strain_energy_sum(m, d_u, &e);
    if (s != EFEM_OK) return s;
    const size_t n = 3 * static_cast<size_t>(m.n_free);
    double w = 0.0;
    if (n > 0) {
        const int grid = static_cast<int>(std::min<size_t>(296, (n + kBlock - 1) / kBlock));
        double* part = nullptr;
        EFEM_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&part), sizeof(double) * grid, m.stream));
        k_dot_part<<<grid, kBlock, 0, m.stream>>>(m.d_fext, d_u, n, part);
        m.launches++;
        std::vector<double> h(grid);
        EFEM_CUDA(cudaMemcpyAsync(h.data(), part, sizeof(double) * grid, cudaMemcpyDeviceToHost, m.stream));
        EFEM_CUDA(cudaFreeAsync(part, m.stream));
        EFEM_CUDA(cudaStreamSynchronize(m.stream));
        for (double x : h) w += x;
    }
    *pi = e - w;
    return EFEM_OK;
}

efem_status strain_energy_sum(Model& m, const double* d_u, double* energy)
{
    double total = 0.0;
    for (auto& b : m.blocks) {
        if (b.n == 0) continue;
        const long long threads = static_cast<long long>(b.n) * b.ngp;
        const int grid = static_cast<int>((threads + kBlock - 1) / kBlock);
        double* part = nullptr;
        EFEM_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&part), sizeof(double) * grid, m.stream));
        k_energy<<<grid, kBlock, 0, m.stream>>>(b.n, b.nen, b.ngp, m.n_free, b.conn, b.mat, b.vol, b.J0inv, b.dN, b.gw,
            m.d_mats, d_u, part);
        m.launches++;
        std::vector<double> h(grid);
        EFEM_CUDA(cudaMemcpyAsync(h.data(), part, sizeof(double) * grid, cudaMemcpyDeviceToHost, m.stream));
        EFEM_CUDA(cudaFreeAsync(part, m.stream));
        EFEM_CUDA(cudaStreamSynchronize(m.stream));
        for (double x : h) total += x;
    }
    *energy = total;
    return EFEM_OK;
}

}  // namespace efem
