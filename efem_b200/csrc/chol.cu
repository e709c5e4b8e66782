// Approximate-Jacobian Cholesky preconditioner on the GPU.
//
// Replaces the reference's Eigen SimplicialLLT factor of K~ = L (x) I3
// (src/simulation/nlsolver/LBFGS.h:65-81) and its solve inside the two-loop
// recursion (src/simulation/nlsolver/LBFGSMat.h:119-120).  The scalar node
// matrix L is factored (the same H0 = K~^{-1} up to rounding) and applied to
// the three displacement components at once.
//
// Numeric factorisation, multifrontal, one level of the supernodal
// elimination tree per launch (leaves first), one CTA per front:
//   1. extend-add: the children's update blocks are added into the front
//      through the precomputed relative indices (children in a fixed order, so
//      the factor is bitwise repeatable);
//   2. partial dense Cholesky of the r x r front: 32-column blocks, diagonal
//      block in shared memory, panel TRSM row-parallel, trailing SYRK in 64x64
//      register-blocked tiles.
// Then each diagonal block L_JJ is inverted explicitly, so the triangular
// solves are matrix-vector products.
//
// Solves (3 right-hand sides interleaved per node), one launch per level:
//   forward  (leaves -> root): f = [b_J; 0] + sum over children of their update
//            vectors; y_J = L_JJ^{-1} f_J; update g = f_R - L_RJ y_J;
//   backward (root -> leaves): x_J = L_JJ^{-T} (y_J - L_RJ^T x_R), x_R gathered
//            from the ancestors' results.
// No atomics anywhere: results are deterministic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "chol_symbolic.h"
#include "efem_internal.h"

namespace efem {

struct Precond {
    Symbolic S;
    bool ready = false;     // symbolic analysis done and uploaded
    bool factored = false;  // numeric factor present
    bool ok = false;        // factor is positive definite
    double ms_factor = 0;
    int max_r = 0, max_c = 0;
    std::vector<int> lev_max_r, lev_max_c;
    int *d_first = nullptr, *d_ncol = nullptr, *d_nrow = nullptr, *d_rows = nullptr, *d_child_ptr = nullptr,
        *d_child_list = nullptr, *d_relind = nullptr, *d_level_list = nullptr, *d_perm = nullptr, *d_fail = nullptr;
    long long *d_front_off = nullptr, *d_rows_off = nullptr, *d_relind_off = nullptr, *d_dinv_off = nullptr,
              *d_upd_off = nullptr, *d_a_pos = nullptr, *d_a_src = nullptr;
    double *d_front = nullptr, *d_dinv = nullptr, *d_upd = nullptr, *d_w = nullptr, *d_vals = nullptr;
};

namespace {

constexpr int kFT = 256;  // factor threads
constexpr int kNB = 32;   // factor column block
constexpr int kST = 128;  // solve threads

struct FrontArgs {
    const int *first, *ncol, *nrow, *rows, *child_ptr, *child_list, *relind, *level_list;
    const long long *front_off, *rows_off, *relind_off, *dinv_off, *upd_off;
    double* front;
    double* dinv;
    double* upd;
    double* w;
    int* fail;
};

__global__ void k_scatter_a(double* __restrict__ front, const long long* __restrict__ pos,
    const long long* __restrict__ src, const double* __restrict__ vals, long long n)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        front[pos[k]] = vals[src[k]];
}

// extend-add of the children, then partial Cholesky of the front
__global__ void __launch_bounds__(kFT) k_factor(FrontArgs a, int level_base)
{
    const int s = a.level_list[level_base + blockIdx.x];
    const int r = a.nrow[s], c = a.ncol[s];
    double* F = a.front + a.front_off[s];
    const int tid = threadIdx.x;

    for (int q = a.child_ptr[s]; q < a.child_ptr[s + 1]; q++) {
        const int ch = a.child_list[q];
        const int rc = a.nrow[ch], cc = a.ncol[ch], m = rc - cc;
        const int* ri = a.relind + a.relind_off[ch];
        const double* U = a.front + a.front_off[ch];
        for (int idx = tid; idx < m * m; idx += kFT) {
            const int i = idx % m, j = idx / m;
            if (i < j) continue;
            F[ri[i] + static_cast<long long>(ri[j]) * r] += U[(cc + i) + static_cast<long long>(cc + j) * rc];
        }
        __syncthreads();
    }

    __shared__ double D[kNB][kNB + 1];
    __shared__ double Pi[64][kNB + 1];
    __shared__ double Pj[64][kNB + 1];
    for (int k0 = 0; k0 < c; k0 += kNB) {
        const int kb = min(kNB, c - k0);
        // (a) diagonal block
        for (int idx = tid; idx < kb * kb; idx += kFT) {
            const int i = idx % kb, j = idx / kb;
            D[i][j] = (i >= j) ? F[(k0 + i) + static_cast<long long>(k0 + j) * r] : 0.0;
        }
        __syncthreads();
        for (int j = 0; j < kb; j++) {
            if (tid == 0) {
                double d = D[j][j];
                if (!(d > 0.0)) {
                    *a.fail = 1;
                    d = 1.0;
                }
                D[j][j] = sqrt(d);
            }
            __syncthreads();
            const double dj = D[j][j];
            for (int i = j + 1 + tid; i < kb; i += kFT) D[i][j] /= dj;
            __syncthreads();
            const int t = kb - j - 1;
            for (int idx = tid; idx < t * t; idx += kFT) {
                const int ii = j + 1 + idx % t, kk = j + 1 + idx / t;
                if (ii >= kk) D[ii][kk] -= D[ii][j] * D[kk][j];
            }
            __syncthreads();
        }
        for (int idx = tid; idx < kb * kb; idx += kFT) {
            const int i = idx % kb, j = idx / kb;
            if (i >= j) F[(k0 + i) + static_cast<long long>(k0 + j) * r] = D[i][j];
        }
        // (b) panel: rows below the block, x L^T = f
        for (int i = k0 + kb + tid; i < r; i += kFT) {
            double x[kNB];
#pragma unroll
            for (int j = 0; j < kNB; j++) x[j] = j < kb ? F[i + static_cast<long long>(k0 + j) * r] : 0.0;
#pragma unroll
            for (int j = 0; j < kNB; j++) {
                if (j < kb) {
                    double sum = x[j];
#pragma unroll
                    for (int k = 0; k < kNB; k++)
                        if (k < j) sum -= x[k] * D[j][k];
                    x[j] = sum / D[j][j];
                }
            }
#pragma unroll
            for (int j = 0; j < kNB; j++)
                if (j < kb) F[i + static_cast<long long>(k0 + j) * r] = x[j];
        }
        __syncthreads();
        // (c) trailing lower triangle -= P P^T, P = F[base:r, k0:k0+kb]
        const int base = k0 + kb, m2 = r - base;
        const int nt = (m2 + 63) / 64;
        for (int tj = 0; tj < nt; tj++)
            for (int ti = tj; ti < nt; ti++) {
                for (int idx = tid; idx < 64 * kNB; idx += kFT) {
                    const int p = idx % 64, k = idx / 64;
                    const int gi = base + ti * 64 + p, gj = base + tj * 64 + p;
                    Pi[p][k] = (k < kb && gi < r) ? F[gi + static_cast<long long>(k0 + k) * r] : 0.0;
                    Pj[p][k] = (k < kb && gj < r) ? F[gj + static_cast<long long>(k0 + k) * r] : 0.0;
                }
                __syncthreads();
                const int a0 = (tid % 16) * 4, b0 = (tid / 16) * 4;
                double acc[4][4];
#pragma unroll
                for (int x = 0; x < 4; x++)
#pragma unroll
                    for (int y = 0; y < 4; y++) acc[x][y] = 0.0;
                for (int k = 0; k < kb; k++) {
                    double pa[4], pb[4];
#pragma unroll
                    for (int x = 0; x < 4; x++) {
                        pa[x] = Pi[a0 + x][k];
                        pb[x] = Pj[b0 + x][k];
                    }
#pragma unroll
                    for (int x = 0; x < 4; x++)
#pragma unroll
                        for (int y = 0; y < 4; y++) acc[x][y] += pa[x] * pb[y];
                }
#pragma unroll
                for (int x = 0; x < 4; x++)
#pragma unroll
                    for (int y = 0; y < 4; y++) {
                        const int gi = base + ti * 64 + a0 + x, gj = base + tj * 64 + b0 + y;
                        if (gi < r && gj < r && gi >= gj) F[gi + static_cast<long long>(gj) * r] -= acc[x][y];
                    }
                __syncthreads();
            }
    }
}

// Dinv = L_JJ^{-1}, one thread per column of the inverse
__global__ void k_inverse(FrontArgs a, int ns)
{
    const int s = blockIdx.x;
    if (s >= ns) return;
    const int r = a.nrow[s], c = a.ncol[s];
    const double* F = a.front + a.front_off[s];
    double* X = a.dinv + a.dinv_off[s];
    for (int j = threadIdx.x; j < c; j += blockDim.x) {
        for (int i = 0; i < j; i++) X[i + static_cast<long long>(j) * c] = 0.0;
        X[j + static_cast<long long>(j) * c] = 1.0 / F[j + static_cast<long long>(j) * r];
        for (int i = j + 1; i < c; i++) {
            double sum = 0.0;
            for (int k = j; k < i; k++) sum += F[i + static_cast<long long>(k) * r] * X[k + static_cast<long long>(j) * c];
            X[i + static_cast<long long>(j) * c] = -sum / F[i + static_cast<long long>(i) * r];
        }
    }
}

__global__ void k_gather_rhs(double* __restrict__ w, const double* __restrict__ v, const int* __restrict__ perm, int n)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int o = perm[k];
        w[3 * k] = v[3 * o];
        w[3 * k + 1] = v[3 * o + 1];
        w[3 * k + 2] = v[3 * o + 2];
    }
}

__global__ void k_scatter_sol(double* __restrict__ v, const double* __restrict__ w, const int* __restrict__ perm, int n)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int o = perm[k];
        v[3 * o] = w[3 * k];
        v[3 * o + 1] = w[3 * k + 1];
        v[3 * o + 2] = w[3 * k + 2];
    }
}

__global__ void __launch_bounds__(kST) k_forward(FrontArgs a, int level_base)
{
    extern __shared__ double sm[];
    const int s = a.level_list[level_base + blockIdx.x];
    const int r = a.nrow[s], c = a.ncol[s], m = r - c, f0 = a.first[s];
    double* f = sm;          // [r][3]
    double* y = sm + 3 * r;  // [c][3]
    const int tid = threadIdx.x;
    for (int k = tid; k < r; k += kST) {
        const bool own = k < c;
        f[3 * k] = own ? a.w[3 * (f0 + k)] : 0.0;
        f[3 * k + 1] = own ? a.w[3 * (f0 + k) + 1] : 0.0;
        f[3 * k + 2] = own ? a.w[3 * (f0 + k) + 2] : 0.0;
    }
    __syncthreads();
    for (int q = a.child_ptr[s]; q < a.child_ptr[s + 1]; q++) {
        const int ch = a.child_list[q];
        const int mc = a.nrow[ch] - a.ncol[ch];
        const int* ri = a.relind + a.relind_off[ch];
        const double* g = a.upd + a.upd_off[ch];
        for (int k = tid; k < mc; k += kST) {
            const int t = ri[k];
            f[3 * t] += g[3 * k];
            f[3 * t + 1] += g[3 * k + 1];
            f[3 * t + 2] += g[3 * k + 2];
        }
        __syncthreads();
    }
    const double* Di = a.dinv + a.dinv_off[s];
    for (int i = tid; i < c; i += kST) {
        double y0 = 0, y1 = 0, y2 = 0;
        for (int k = 0; k <= i; k++) {
            const double d = Di[i + static_cast<long long>(k) * c];
            y0 += d * f[3 * k];
            y1 += d * f[3 * k + 1];
            y2 += d * f[3 * k + 2];
        }
        y[3 * i] = y0;
        y[3 * i + 1] = y1;
        y[3 * i + 2] = y2;
        a.w[3 * (f0 + i)] = y0;
        a.w[3 * (f0 + i) + 1] = y1;
        a.w[3 * (f0 + i) + 2] = y2;
    }
    __syncthreads();
    const double* F = a.front + a.front_off[s];
    double* g = a.upd + a.upd_off[s];
    for (int k = tid; k < m; k += kST) {
        double g0 = f[3 * (c + k)], g1 = f[3 * (c + k) + 1], g2 = f[3 * (c + k) + 2];
        for (int j = 0; j < c; j++) {
            const double l = F[(c + k) + static_cast<long long>(j) * r];
            g0 -= l * y[3 * j];
            g1 -= l * y[3 * j + 1];
            g2 -= l * y[3 * j + 2];
        }
        g[3 * k] = g0;
        g[3 * k + 1] = g1;
        g[3 * k + 2] = g2;
    }
}

__device__ __forceinline__ double wsum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(kST) k_backward(FrontArgs a, int level_base)
{
    extern __shared__ double sm[];
    const int s = a.level_list[level_base + blockIdx.x];
    const int r = a.nrow[s], c = a.ncol[s], m = r - c, f0 = a.first[s];
    double* xr = sm;          // [m][3]
    double* t = sm + 3 * m;   // [c][3]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = kST / 32;
    const int* rows = a.rows + a.rows_off[s];
    for (int k = tid; k < m; k += kST) {
        const int g = rows[c + k];
        xr[3 * k] = a.w[3 * g];
        xr[3 * k + 1] = a.w[3 * g + 1];
        xr[3 * k + 2] = a.w[3 * g + 2];
    }
    __syncthreads();
    const double* F = a.front + a.front_off[s];
    for (int j = warp; j < c; j += nw) {
        double s0 = 0, s1 = 0, s2 = 0;
        const double* col = F + static_cast<long long>(j) * r + c;
        for (int k = lane; k < m; k += 32) {
            const double l = col[k];
            s0 += l * xr[3 * k];
            s1 += l * xr[3 * k + 1];
            s2 += l * xr[3 * k + 2];
        }
        s0 = wsum(s0);
        s1 = wsum(s1);
        s2 = wsum(s2);
        if (lane == 0) {
            t[3 * j] = a.w[3 * (f0 + j)] - s0;
            t[3 * j + 1] = a.w[3 * (f0 + j) + 1] - s1;
            t[3 * j + 2] = a.w[3 * (f0 + j) + 2] - s2;
        }
    }
    __syncthreads();
    const double* Di = a.dinv + a.dinv_off[s];
    for (int i = warp; i < c; i += nw) {
        double s0 = 0, s1 = 0, s2 = 0;
        const double* col = Di + static_cast<long long>(i) * c;  // column i of L_JJ^{-1} = row i of its transpose
        for (int k = i + lane; k < c; k += 32) {
            const double d = col[k];
            s0 += d * t[3 * k];
            s1 += d * t[3 * k + 1];
            s2 += d * t[3 * k + 2];
        }
        s0 = wsum(s0);
        s1 = wsum(s1);
        s2 = wsum(s2);
        if (lane == 0) {
            a.w[3 * (f0 + i)] = s0;
            a.w[3 * (f0 + i) + 1] = s1;
            a.w[3 * (f0 + i) + 2] = s2;
        }
    }
}

FrontArgs args_of(Precond& P)
{
    return FrontArgs { P.d_first, P.d_ncol, P.d_nrow, P.d_rows, P.d_child_ptr, P.d_child_list, P.d_relind,
        P.d_level_list, P.d_front_off, P.d_rows_off, P.d_relind_off, P.d_dinv_off, P.d_upd_off, P.d_front, P.d_dinv,
        P.d_upd, P.d_w, P.d_fail };
}

}  // namespace

void free_precond(Model& m)
{
    if (!m.precond) return;
    Precond& P = *m.precond;
    for (int** p : { &P.d_first, &P.d_ncol, &P.d_nrow, &P.d_rows, &P.d_child_ptr, &P.d_child_list, &P.d_relind,
             &P.d_level_list, &P.d_perm, &P.d_fail })
        dev_free(*p);
    for (long long** p : { &P.d_front_off, &P.d_rows_off, &P.d_relind_off, &P.d_dinv_off, &P.d_upd_off, &P.d_a_pos, &P.d_a_src })
        dev_free(*p);
    for (double** p : { &P.d_front, &P.d_dinv, &P.d_upd, &P.d_w, &P.d_vals }) dev_free(*p);
    delete m.precond;
    m.precond = nullptr;
}

void precond_info(const Model& m, efem_model_info* info)
{
    if (!m.precond) return;
    const Symbolic& S = m.precond->S;
    info->factor_nnz = S.nnz_L;
    info->n_supernodes = S.ns;
    info->n_levels = static_cast<int>(S.level_ptr.size()) - 1;
    info->factor_gflop = S.flops * 1e-9;
    long long dn = 0;
    for (int s = 0; s < S.ns; s++) dn += static_cast<long long>(S.ncol[s]) * (S.ncol[s] + 1) / 2;
    info->factor_dinv_nnz = dn;
}

static efem_status precond_factor(Model& m, int* ok, double* ms_factor);

efem_status precond_setup(Model& m, bool refactor, int* ok, double* ms_factor)
{
    if (m.precond && m.precond->ready && !refactor) {
        *ok = m.precond->ok;
        *ms_factor = 0.0;
        return EFEM_OK;
    }
    if (m.precond && m.precond->ready) return precond_factor(m, ok, ms_factor);
    free_precond(m);
    m.precond = new Precond();
    Precond& P = *m.precond;
    Symbolic& S = P.S;
    // host: assemble L, order, analyse
    std::vector<int> rp, ci;
    std::vector<double> vals;
    assemble_L_csr(m, rp, ci, vals);
    std::vector<double> coords(3 * static_cast<size_t>(m.n_free));
    for (int i = 0; i < m.n_free; i++)
        for (int k = 0; k < 3; k++) coords[3 * i + k] = m.X[3 * static_cast<size_t>(m.node_of_dnode[i]) + k];
    symbolic_analysis(m.n_free, rp, ci, coords.data(), S);
    const int nlev = static_cast<int>(S.level_ptr.size()) - 1;
    P.lev_max_r.assign(nlev, 0);
    P.lev_max_c.assign(nlev, 0);
    for (int l = 0; l < nlev; l++)
        for (int q = S.level_ptr[l]; q < S.level_ptr[l + 1]; q++) {
            const int s = S.level_list[q];
            P.lev_max_r[l] = std::max(P.lev_max_r[l], S.nrow[s]);
            P.lev_max_c[l] = std::max(P.lev_max_c[l], S.ncol[s]);
            P.max_r = std::max(P.max_r, S.nrow[s]);
        }
    if (static_cast<size_t>(P.max_r) * 6 * sizeof(double) > 200 * 1024) {
        set_error("a front of the approximate-Jacobian factor is too large for the solve kernels ("
            + std::to_string(P.max_r) + " rows)");
        return EFEM_ERR_UNSUPPORTED;
    }
    // device arrays
    efem_status st;
#define UP(p, v)                                       \
    if ((st = dev_upload(&(p), (v))) != EFEM_OK) return st;
    UP(P.d_first, S.first);
    UP(P.d_ncol, S.ncol);
    UP(P.d_nrow, S.nrow);
    UP(P.d_rows, S.rows);
    UP(P.d_child_ptr, S.child_ptr);
    UP(P.d_child_list, S.child_list);
    UP(P.d_relind, S.relind);
    UP(P.d_level_list, S.level_list);
    UP(P.d_perm, S.perm);
    UP(P.d_front_off, S.front_off);
    UP(P.d_rows_off, S.rows_off);
    UP(P.d_relind_off, S.relind_off);
    UP(P.d_dinv_off, S.dinv_off);
    UP(P.d_upd_off, S.upd_off);
    UP(P.d_a_pos, S.a_pos);
    UP(P.d_a_src, S.a_src);
    UP(P.d_vals, vals);
#undef UP
    if ((st = dev_alloc(&P.d_front, static_cast<size_t>(S.front_size))) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_dinv, static_cast<size_t>(std::max<long long>(S.dinv_size, 1)))) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_upd, static_cast<size_t>(std::max<long long>(S.upd_size, 1)))) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_w, 3 * static_cast<size_t>(std::max(S.n, 1)))) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_fail, 1)) != EFEM_OK) return st;
    EFEM_CUDA(cudaFuncSetAttribute(k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    EFEM_CUDA(cudaFuncSetAttribute(k_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    P.ready = true;  // analysed; the numeric factor follows
    return precond_factor(m, ok, ms_factor);
}

// Numeric factorisation (every solve, like LBFGSSolver::updateApproxJacobi):
// scatter L into the fronts, factor level by level, invert the diagonal blocks.
static efem_status precond_factor(Model& m, int* ok, double* ms_factor)
{
    Precond& P = *m.precond;
    const Symbolic& S = P.S;
    const int nlev = static_cast<int>(S.level_ptr.size()) - 1;
    cudaEvent_t e0, e1;
    EFEM_CUDA(cudaEventCreate(&e0));
    EFEM_CUDA(cudaEventCreate(&e1));
    EFEM_CUDA(cudaEventRecord(e0, m.stream));
    EFEM_CUDA(cudaMemsetAsync(P.d_front, 0, sizeof(double) * S.front_size, m.stream));
    EFEM_CUDA(cudaMemsetAsync(P.d_fail, 0, sizeof(int), m.stream));
    const long long na = static_cast<long long>(S.a_pos.size());
    k_scatter_a<<<static_cast<int>(std::min<long long>(1184, (na + 255) / 256 + 1)), 256, 0, m.stream>>>(
        P.d_front, P.d_a_pos, P.d_a_src, P.d_vals, na);
    FrontArgs a = args_of(P);
    for (int l = 0; l < nlev; l++) {
        const int cnt = S.level_ptr[l + 1] - S.level_ptr[l];
        k_factor<<<cnt, kFT, 0, m.stream>>>(a, S.level_ptr[l]);
    }
    k_inverse<<<S.ns, 128, 0, m.stream>>>(a, S.ns);
    m.launches += 2 + nlev;
    EFEM_CUDA(cudaGetLastError());
    EFEM_CUDA(cudaEventRecord(e1, m.stream));
    int fail = 0;
    EFEM_CUDA(cudaMemcpyAsync(&fail, P.d_fail, sizeof(int), cudaMemcpyDeviceToHost, m.stream));
    EFEM_CUDA(cudaStreamSynchronize(m.stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    P.ms_factor = ms;
    P.ok = fail == 0;
    P.factored = true;
    *ok = P.ok;
    *ms_factor = ms;
    return EFEM_OK;
}

efem_status precond_apply(Model& m, double* d_v)
{
    if (!m.precond || !m.precond->factored || !m.precond->ok) {
        set_error("preconditioner not factored");
        return EFEM_ERR_ARG;
    }
    Precond& P = *m.precond;
    const Symbolic& S = P.S;
    const int n = S.n;
    if (n == 0) return EFEM_OK;
    const int g = std::min(1184, (n + 255) / 256);
    k_gather_rhs<<<g, 256, 0, m.stream>>>(P.d_w, d_v, P.d_perm, n);
    FrontArgs a = args_of(P);
    const int nlev = static_cast<int>(S.level_ptr.size()) - 1;
    for (int l = 0; l < nlev; l++) {
        const int cnt = S.level_ptr[l + 1] - S.level_ptr[l];
        const size_t sm = sizeof(double) * 3 * (P.lev_max_r[l] + P.lev_max_c[l]);
        k_forward<<<cnt, kST, sm, m.stream>>>(a, S.level_ptr[l]);
    }
    for (int l = nlev - 1; l >= 0; l--) {
        const int cnt = S.level_ptr[l + 1] - S.level_ptr[l];
        const size_t sm = sizeof(double) * 3 * (P.lev_max_r[l] + P.lev_max_c[l]);
        k_backward<<<cnt, kST, sm, m.stream>>>(a, S.level_ptr[l]);
    }
    k_scatter_sol<<<g, 256, 0, m.stream>>>(d_v, P.d_w, P.d_perm, n);
    m.launches += 2 + 2 * nlev;
    EFEM_CUDA(cudaGetLastError());
    return EFEM_OK;
}

// ============================================================================
// Allocation-free H0 application.
//
// Some callers cannot call cudaMalloc at the moment they need H0 v: code that
// runs while a CUDA stream capture is open (cudaMalloc is not allowed there),
// code inside another framework's allocator (a caching allocator that owns the
// device's free memory and must not see foreign allocations), or real-time
// control loops that forbid the implicit device synchronisation an allocation
// can cause.  For them efem_precond_apply_noalloc runs the same forward and
// backward sweeps as efem_precond_apply, but its working vectors (the permuted
// right-hand side, 3 per free node, and the fronts' update vectors) live in
// the fixed array below instead of buffers owned by the model.
//
// Limits and sharing:
//   * the array holds kNoAllocDoubles doubles (16 MiB); a model that needs
//     more (3 * free nodes + its update-vector length) is rejected;
//   * every GPU that loads this library keeps the array until the process
//     exits;
//   * all calls share the array and it keeps the last call's contents; every
//     entry is written before it is read, so nothing has to be cleared, but
//     calls that overlap on the GPU (other streams, other threads, other
//     models) race on it and must be serialised by the caller.
// ============================================================================
namespace {
constexpr size_t kNoAllocDoubles = size_t(2) << 20;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// device address of g_noalloc_scratch, looked up once per device; in host
// code the array's name is only a host-side stand-in, never a device address
std::mutex g_noalloc_mutex;
double* g_noalloc_addr[256] = {};

efem_status noalloc_scratch(int device, double** out)
{
    if (device < 0 || device >= 256) {
        set_error("device ordinal out of range for the static workspace");
        return EFEM_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[device]) {
        EFEM_CUDA(cudaSetDevice(device));
        void* p = nullptr;
        EFEM_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_addr[device] = static_cast<double*>(p);
    }
    *out = g_noalloc_addr[device];
    return EFEM_OK;
}
}  // namespace

}  // namespace efem

extern "C" efem_status efem_precond_apply_noalloc(void* model, double* d_v)
{
    using namespace efem;
    if (!model || !d_v) {
        set_error("null model or vector");
        return EFEM_ERR_ARG;
    }
    Model& m = *static_cast<Model*>(model);
    if (!m.on_device || !m.precond || !m.precond->factored || !m.precond->ok) {
        set_error("efem_precond_apply_noalloc needs an existing positive-definite factor: call efem_solve or "
                  "efem_precond_apply once first");
        return EFEM_ERR_ARG;
    }
    Precond& P = *m.precond;
    const Symbolic& S = P.S;
    const int n = S.n;
    const size_t need = 3 * static_cast<size_t>(n) + static_cast<size_t>(S.upd_size);
    if (need > kNoAllocDoubles) {
        set_error("model needs " + std::to_string(need) + " doubles of workspace; the static workspace of "
            "efem_precond_apply_noalloc holds " + std::to_string(kNoAllocDoubles));
        return EFEM_ERR_ARG;
    }
    double* scratch = nullptr;
    efem_status st = noalloc_scratch(m.device, &scratch);
    if (st != EFEM_OK) return st;
    EFEM_CUDA(cudaSetDevice(m.device));
    if (n == 0) return EFEM_OK;
    FrontArgs a = args_of(P);
    a.w = scratch;
    a.upd = scratch + 3 * static_cast<size_t>(n);
    const int g = std::min(1184, (n + 255) / 256);
    k_gather_rhs<<<g, 256, 0, m.stream>>>(a.w, d_v, P.d_perm, n);
    const int nlev = static_cast<int>(S.level_ptr.size()) - 1;
    for (int l = 0; l < nlev; l++) {
        const int cnt = S.level_ptr[l + 1] - S.level_ptr[l];
        const size_t sm = sizeof(double) * 3 * (P.lev_max_r[l] + P.lev_max_c[l]);
        k_forward<<<cnt, kST, sm, m.stream>>>(a, S.level_ptr[l]);
    }
    for (int l = nlev - 1; l >= 0; l--) {
        const int cnt = S.level_ptr[l + 1] - S.level_ptr[l];
        const size_t sm = sizeof(double) * 3 * (P.lev_max_r[l] + P.lev_max_c[l]);
        k_backward<<<cnt, kST, sm, m.stream>>>(a, S.level_ptr[l]);
    }
    k_scatter_sol<<<g, 256, 0, m.stream>>>(d_v, a.w, P.d_perm, n);
    EFEM_CUDA(cudaGetLastError());
    EFEM_CUDA(cudaStreamSynchronize(m.stream));
    return EFEM_OK;
}

