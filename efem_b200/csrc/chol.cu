// Approximate-Jacobian Cholesky preconditioner on the GPU.
//
// Replaces the reference's Eigen SimplicialLLT factor of K~ = L (x) I3
// (src/simulation/nlsolver/LBFGS.h:65-81) and its solve inside the two-loop
// recursion (src/simulation/nlsolver/LBFGSMat.h:119-120).  The scalar node
// matrix L is factored (the same H0 = K~^{-1} up to rounding) and applied to
// the three displacement components at once.
//
// Numeric factorisation (multifrontal, one level of the supernodal
// elimination tree at a time, leaves first):
//   k_extend_add  one CTA per front: add the children's update blocks through
//                 the precomputed relative indices, children in a fixed order
//                 (the factor is bitwise repeatable);
//   per 32-column panel step of the level's fronts:
//   k_panel       one CTA per front: Cholesky of the 32x32 diagonal block in
//                 shared memory, then the panel TRSM, row-parallel;
//   k_syrk        one CTA per 64x64 tile of every front's trailing lower
//                 triangle: register-blocked rank-32 update.
//   k_inverse     one warp per 32 columns of each diagonal block: L_JJ^{-1},
//                 stored row-major, so the solves are matrix-vector products.
//
// Solve H0 v (3 right-hand sides interleaved per node), per level and in
// tiles of 32 rows (or columns) of a front, so that large fronts spread over
// many CTAs:
//   forward   k_fwd_y: y_J = L_JJ^{-1} f_J, f = b_J + children's updates
//             k_fwd_g: g = f_R - L_RJ y_J (the update passed to the parent)
//   backward  k_bwd_t: t_J = y_J - L_RJ^T x_R (x_R from the ancestors)
//             k_bwd_x: x_J = L_JJ^{-T} t_J
// Every sum is formed in a fixed order (no atomics): results are deterministic.
// The whole solve (gather, 4 launches per level, scatter) is replayed as one
// CUDA graph per input vector.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "chol_symbolic.h"
#include "efem_internal.h"

namespace efem {

namespace {
constexpr int kFT = 256;  // factor threads
constexpr int kNB = 32;   // factor panel width
constexpr int kTS = 64;   // SYRK tile
constexpr int kST = 256;  // solve threads: one warp per output row / column
constexpr int kSW = kST / 32;  // outputs per solve CTA
constexpr int kRT = 32;   // columns per CTA of the inverse / transpose kernels

struct Tile {
    int s;    // front
    int off;  // first row / column of the tile (multiple of kRT)
};
}  // namespace

struct Precond {
    Symbolic S;
    bool ready = false;     // symbolic analysis done and uploaded
    bool factored = false;  // numeric factor present
    bool ok = false;        // factor is positive definite
    double ms_factor = 0;
    int max_r = 0, max_c = 0, max_m = 0, nlev = 0;
    // solve schedule: tiles per level for the four solve kernels
    std::vector<int> fy_off, fg_off, bt_off, bx_off;  // nlev + 1 offsets each
    std::vector<int> lev_max_c, lev_max_m;
    // factor schedule: per (level, step) the fronts with a panel at that step and the SYRK tiles
    struct Step {
        int level, k0, panel_off, panel_cnt, syrk_off, syrk_cnt;
    };
    std::vector<Step> steps;
    std::vector<int> lev_first_step;  // index into steps, nlev + 1
    int n_inv_tiles = 0;
    int *d_first = nullptr, *d_ncol = nullptr, *d_nrow = nullptr, *d_rows = nullptr, *d_child_ptr = nullptr,
        *d_child_list = nullptr, *d_relind = nullptr, *d_level_list = nullptr, *d_perm = nullptr, *d_fail = nullptr,
        *d_panel_list = nullptr;
    long long *d_front_off = nullptr, *d_rows_off = nullptr, *d_relind_off = nullptr, *d_dinv_off = nullptr,
              *d_upd_off = nullptr, *d_a_pos = nullptr, *d_a_src = nullptr;
    Tile *d_fy = nullptr, *d_fg = nullptr, *d_bt = nullptr, *d_bx = nullptr, *d_inv = nullptr;
    int *d_contrib_ptr = nullptr, *d_contrib_idx = nullptr, *d_below_front = nullptr;
    Tile *d_ea = nullptr, *d_oinv = nullptr;  // extend-add column tiles, off-diagonal inverse column groups
    std::vector<int> ea_off;                  // nlev + 1
    int n_oinv = 0;
    long long* d_lt_off = nullptr;
    double *d_dinvT = nullptr, *d_lt = nullptr;
    int4* d_syrk = nullptr;
    double *d_front = nullptr, *d_dinv = nullptr, *d_upd = nullptr, *d_w = nullptr, *d_y = nullptr, *d_t = nullptr,
           *d_vals = nullptr;
    // graph replay of the solve, per (input vector, work buffers)
    cudaStream_t capture = nullptr;
    std::map<std::pair<double*, double*>, cudaGraphExec_t> graphs;
};

namespace {

struct FrontArgs {
    const int *first, *ncol, *nrow, *rows, *child_ptr, *child_list, *relind, *level_list, *contrib_ptr, *contrib_idx,
        *below_front;
    const long long *front_off, *rows_off, *relind_off, *dinv_off, *upd_off, *lt_off;
    double* front;
    double* dinv;   // L_JJ^{-1}, row-major
    double* dinvT;  // its transpose, row-major
    double* lt;     // L_RJ, row-major
    int* fail;
};

struct SolveBufs {
    double* w;    // b, then x (permuted order, 3 per node)
    double* y;    // forward result
    double* t;    // backward intermediate
    double* upd;  // fronts' update vectors
};

__device__ __forceinline__ double wsum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ------------------------------------------------------------------ factorisation
__global__ void k_scatter_a(double* __restrict__ front, const long long* __restrict__ pos,
    const long long* __restrict__ src, const double* __restrict__ vals, long long n)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        front[pos[k]] = vals[src[k]];
}

// Children's update blocks into the fronts of one level, one warp per front
// column p (8 per CTA): the contributions landing on column p are added in
// child order, each one a column j of a child's update block whose rows
// i >= j go to the parent rows relind[i].  No two warps touch the same entry,
// so the sums need no atomics and are bitwise repeatable.
__global__ void __launch_bounds__(kFT) k_extend_add(FrontArgs a, const Tile* __restrict__ tiles)
{
    const Tile tl = tiles[blockIdx.x];
    const int s = tl.s;
    const int p = tl.off + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    const int r = a.nrow[s];
    if (p >= r) return;
    double* Fp = a.front + a.front_off[s] + static_cast<long long>(p) * r;
    const long long row = a.rows_off[s] + p;
    for (int q = a.contrib_ptr[row]; q < a.contrib_ptr[row + 1]; q++) {
        const int idx = a.contrib_idx[q];
        const int ch = a.below_front[idx];
        const int j = idx - static_cast<int>(a.upd_off[ch] / 3);
        const int rc = a.nrow[ch], cc = a.ncol[ch], m = rc - cc;
        const int* ri = a.relind + a.relind_off[ch];
        const double* U = a.front + a.front_off[ch] + static_cast<long long>(cc + j) * rc + cc;
        for (int i = j + lane; i < m; i += 32) Fp[ri[i]] += U[i];
        __syncwarp();
    }
}

// diagonal block and panel of step k0, one CTA per front in the step's list
__global__ void __launch_bounds__(kFT) k_panel(FrontArgs a, const int* __restrict__ list, int k0)
{
    const int s = list[blockIdx.x];
    const int r = a.nrow[s], c = a.ncol[s];
    const int kb = min(kNB, c - k0);
    double* F = a.front + a.front_off[s];
    const int tid = threadIdx.x;
    __shared__ double D[kNB][kNB + 1];
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
    // rows below the block: x L^T = f
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
}

// trailing lower triangle -= P P^T for one 64x64 tile; tile = (front, ti, tj)
__global__ void __launch_bounds__(kFT) k_syrk(FrontArgs a, const int4* __restrict__ tiles, int k0)
{
    const int4 tl = tiles[blockIdx.x];
    const int s = tl.x, ti = tl.y, tj = tl.z;
    const int r = a.nrow[s], c = a.ncol[s];
    const int kb = min(kNB, c - k0);
    const int base = k0 + kb;
    double* F = a.front + a.front_off[s];
    const int tid = threadIdx.x;
    __shared__ double Pi[kTS][kNB + 1];
    __shared__ double Pj[kTS][kNB + 1];
    for (int idx = tid; idx < kTS * kNB; idx += kFT) {
        const int p = idx % kTS, k = idx / kTS;
        const int gi = base + ti * kTS + p, gj = base + tj * kTS + p;
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
            const int gi = base + ti * kTS + a0 + x, gj = base + tj * kTS + b0 + y;
            if (gi < r && gj < r && gi >= gj) F[gi + static_cast<long long>(gj) * r] -= acc[x][y];
        }
}

// Inverse of the diagonal block, row-major: X = L_JJ^{-1}.  One warp per 32
// columns; lane j owns column j and reads only its own earlier entries.
// L_JJ^{-1} in two passes.  Pass 1: the inverse of every 32x32 diagonal tile,
// one warp per tile, column j of the inverse by forward substitution in
// shared memory; the tile's upper triangle is written as zeros because pass 2
// reads whole tiles.
__global__ void __launch_bounds__(32) k_diag_inv(FrontArgs a, const Tile* __restrict__ tiles)
{
    const Tile tl = tiles[blockIdx.x];
    const int s = tl.s, j0 = tl.off;
    const int r = a.nrow[s], c = a.ncol[s];
    const int kb = min(kRT, c - j0);
    const double* F = a.front + a.front_off[s];
    __shared__ double D[kRT][kRT + 1];
    __shared__ double X[kRT][kRT + 1];
    const int j = threadIdx.x;
    for (int k = 0; k < kb; k++) D[j][k] = j < kb ? F[static_cast<long long>(j0 + k) * r + j0 + j] : 0.0;
    __syncwarp();
    for (int i = 0; i < kb; i++) {  // thread j owns column j of X
        double v = 0.0;
        if (i == j) {
            v = 1.0 / D[i][i];
        } else if (i > j) {
            double acc = 0.0;
            for (int k = j; k < i; k++) acc += D[i][k] * X[k][j];
            v = -acc / D[i][i];
        }
        X[i][j] = v;
    }
    __syncwarp();
    if (j >= kb) return;
    double* Xg = a.dinv + a.dinv_off[s];
    double* XTg = a.dinvT + a.dinv_off[s];
    for (int i = 0; i < kb; i++) {
        Xg[static_cast<long long>(j0 + i) * c + j0 + j] = X[i][j];
        XTg[static_cast<long long>(j0 + i) * c + j0 + j] = X[j][i];
    }
}

// Pass 2: the tiles below the diagonal, for 8 columns [j0, j0+8) per CTA.
// With J the diagonal tile holding the columns, block row I > J of the
// inverse is X_IJ = -X_II sum_{K=J}^{I-1} L_IK X_KJ (left-looking, the
// columns are independent).  The next L_IK / X_KJ tiles are fetched into
// registers while the current ones are multiplied.
constexpr int kIC = 8;     // columns per CTA
constexpr int kIT = 128;   // threads per CTA
__global__ void __launch_bounds__(kIT) k_offdiag_inv(FrontArgs a, const Tile* __restrict__ tiles)
{
    const Tile tl = tiles[blockIdx.x];
    const int s = tl.s, j0 = tl.off;
    const int r = a.nrow[s], c = a.ncol[s];
    const int jb0 = (j0 / kRT) * kRT;
    if (jb0 + kRT >= c) return;  // no tile below the diagonal one
    const double* F = a.front + a.front_off[s];
    double* X = a.dinv + a.dinv_off[s];
    double* XT = a.dinvT + a.dinv_off[s];
    __shared__ double As[kRT][kRT + 1];
    __shared__ double Bs[kRT][kIC + 1];
    const int tid = threadIdx.x, jj = tid & (kIC - 1), ii = tid >> 3;  // rows ii and ii + 16
    const int ncols = min(kIC, c - j0);
    double pa[kRT * kRT / kIT], pb[kRT * kIC / kIT];
    auto fetch = [&](int i0, int ib, int k0) {
#pragma unroll
        for (int q = 0; q < kRT * kRT / kIT; q++) {
            const int idx = tid + q * kIT, kk = idx >> 5, rr = idx & 31;
            pa[q] = rr < ib ? F[static_cast<long long>(k0 + kk) * r + i0 + rr] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < kRT * kIC / kIT; q++) {
            const int idx = tid + q * kIT, kk = idx >> 3, cc = idx & 7;
            pb[q] = cc < ncols ? X[static_cast<long long>(k0 + kk) * c + j0 + cc] : 0.0;
        }
    };
    for (int i0 = jb0 + kRT; i0 < c; i0 += kRT) {
        const int ib = min(kRT, c - i0);
        double acc0 = 0.0, acc1 = 0.0;
        fetch(i0, ib, jb0);
        for (int k0 = jb0; k0 < i0; k0 += kRT) {
#pragma unroll
            for (int q = 0; q < kRT * kRT / kIT; q++) {
                const int idx = tid + q * kIT;
                As[idx & 31][idx >> 5] = pa[q];
            }
#pragma unroll
            for (int q = 0; q < kRT * kIC / kIT; q++) {
                const int idx = tid + q * kIT;
                Bs[idx >> 3][idx & 7] = pb[q];
            }
            __syncthreads();
            if (k0 + kRT < i0) fetch(i0, ib, k0 + kRT);
#pragma unroll 8
            for (int kk = 0; kk < kRT; kk++) {
                const double b = Bs[kk][jj];
                acc0 += As[ii][kk] * b;
                acc1 += As[ii + 16][kk] * b;
            }
            __syncthreads();
        }
        // X_IJ = -X_II T, X_II lower triangular with its zeros stored
        Bs[ii][jj] = acc0;
        Bs[ii + 16][jj] = acc1;
        for (int idx = tid; idx < kRT * kRT; idx += kIT) {
            const int rr = idx >> 5, kk = idx & 31;
            As[rr][kk] = (rr < ib && kk < ib) ? X[static_cast<long long>(i0 + rr) * c + i0 + kk] : 0.0;
        }
        __syncthreads();
        double x0 = 0.0, x1 = 0.0;
#pragma unroll 8
        for (int kk = 0; kk < kRT; kk++) {
            const double t = Bs[kk][jj];
            x0 += As[ii][kk] * t;
            x1 += As[ii + 16][kk] * t;
        }
        if (jj < ncols) {
            if (ii < ib) {
                X[static_cast<long long>(i0 + ii) * c + j0 + jj] = -x0;
                XT[static_cast<long long>(j0 + jj) * c + i0 + ii] = -x0;
            }
            if (ii + 16 < ib) {
                X[static_cast<long long>(i0 + ii + 16) * c + j0 + jj] = -x1;
                XT[static_cast<long long>(j0 + jj) * c + i0 + ii + 16] = -x1;
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ solves
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

// Dot product of a contiguous row with a 3-component vector held in shared
// memory, over k in [k0, k1); the 32 lanes stride the row with four loads in
// flight each, then the warp reduces.
__device__ __forceinline__ void warp_dot3(const double* __restrict__ row, const double* __restrict__ v, int k0, int k1,
    int vbase, int lane, double& s0, double& s1, double& s2)
{
    double a0 = 0, a1 = 0, a2 = 0;
    int k = k0 + lane;
    for (; k + 96 < k1; k += 128) {
        const double d0 = row[k], d1 = row[k + 32], d2 = row[k + 64], d3 = row[k + 96];
        const double* v0 = v + 3 * (k - vbase);
        a0 += d0 * v0[0] + d1 * v0[96] + d2 * v0[192] + d3 * v0[288];
        a1 += d0 * v0[1] + d1 * v0[97] + d2 * v0[193] + d3 * v0[289];
        a2 += d0 * v0[2] + d1 * v0[98] + d2 * v0[194] + d3 * v0[290];
    }
    for (; k < k1; k += 32) {
        const double d = row[k];
        const double* v0 = v + 3 * (k - vbase);
        a0 += d * v0[0];
        a1 += d * v0[1];
        a2 += d * v0[2];
    }
    s0 = wsum(a0);
    s1 = wsum(a1);
    s2 = wsum(a2);
}

// f_t = (b_t for own columns) + the children's update entries landing on row t
__device__ __forceinline__ void assemble_row(const FrontArgs& a, const SolveBufs& b, int s, int t, bool own, int f0,
    double& f0v, double& f1v, double& f2v)
{
    double x0 = 0, x1 = 0, x2 = 0;
    if (own) {
        x0 = b.w[3 * (f0 + t)];
        x1 = b.w[3 * (f0 + t) + 1];
        x2 = b.w[3 * (f0 + t) + 2];
    }
    const long long row = a.rows_off[s] + t;
    for (int q = a.contrib_ptr[row]; q < a.contrib_ptr[row + 1]; q++) {
        const double* g = b.upd + 3LL * a.contrib_idx[q];
        x0 += g[0];
        x1 += g[1];
        x2 += g[2];
    }
    f0v = x0;
    f1v = x1;
    f2v = x2;
}

// y rows [i0, i0+8) of front s: y_i = sum_{k<=i} (L_JJ^{-1})_ik f_k, one warp per row
__global__ void __launch_bounds__(kST) k_fwd_y(FrontArgs a, SolveBufs b, const Tile* __restrict__ tiles)
{
    extern __shared__ double sm[];
    const Tile tl = tiles[blockIdx.x];
    const int s = tl.s, i0 = tl.off;
    const int c = a.ncol[s], f0 = a.first[s];
    const int kmax = min(c, i0 + kSW);
    double* f = sm;  // [kmax][3]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int k = tid; k < kmax; k += kST) assemble_row(a, b, s, k, true, f0, f[3 * k], f[3 * k + 1], f[3 * k + 2]);
    __syncthreads();
    const int i = i0 + warp;
    if (i >= kmax) return;
    double y0, y1, y2;
    warp_dot3(a.dinv + a.dinv_off[s] + static_cast<long long>(i) * c, f, 0, i + 1, 0, lane, y0, y1, y2);
    if (lane == 0) {
        b.y[3 * (f0 + i)] = y0;
        b.y[3 * (f0 + i) + 1] = y1;
        b.y[3 * (f0 + i) + 2] = y2;
    }
}

// update rows [k0, k0+8) of front s: g_k = f_{c+k} - (L_RJ)_k . y_J, one warp per row
__global__ void __launch_bounds__(kST) k_fwd_g(FrontArgs a, SolveBufs b, const Tile* __restrict__ tiles)
{
    extern __shared__ double sm[];
    const Tile tl = tiles[blockIdx.x];
    const int s = tl.s, k0 = tl.off;
    const int r = a.nrow[s], c = a.ncol[s], m = r - c, f0 = a.first[s];
    double* y = sm;  // [c][3]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int k = tid; k < 3 * c; k += kST) y[k] = b.y[3 * f0 + k];
    __syncthreads();
    const int k = k0 + warp;
    if (k >= m) return;
    double d0, d1, d2;
    warp_dot3(a.lt + a.lt_off[s] + static_cast<long long>(k) * c, y, 0, c, 0, lane, d0, d1, d2);
    if (lane == 0) {
        double f0v, f1v, f2v;
        assemble_row(a, b, s, c + k, false, f0, f0v, f1v, f2v);
        double* g = b.upd + a.upd_off[s] + 3 * k;
        g[0] = f0v - d0;
        g[1] = f1v - d1;
        g[2] = f2v - d2;
    }
}

// columns [j0, j0+8) of front s: t_j = y_j - (L_RJ)^T_j . x_R, one warp per column
__global__ void __launch_bounds__(kST) k_bwd_t(FrontArgs a, SolveBufs b, const Tile* __restrict__ tiles)
{
    extern __shared__ double sm[];
    const Tile tl = tiles[blockIdx.x];
    const int s = tl.s, j0 = tl.off;
    const int r = a.nrow[s], c = a.ncol[s], m = r - c, f0 = a.first[s];
    double* xr = sm;  // [m][3]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int* rows = a.rows + a.rows_off[s] + c;
    for (int k = tid; k < m; k += kST) {
        const int g = rows[k];
        xr[3 * k] = b.w[3 * g];
        xr[3 * k + 1] = b.w[3 * g + 1];
        xr[3 * k + 2] = b.w[3 * g + 2];
    }
    __syncthreads();
    const int j = j0 + warp;
    if (j >= c) return;
    double s0, s1, s2;
    warp_dot3(a.front + a.front_off[s] + static_cast<long long>(j) * r + c, xr, 0, m, 0, lane, s0, s1, s2);
    if (lane == 0) {
        b.t[3 * (f0 + j)] = b.y[3 * (f0 + j)] - s0;
        b.t[3 * (f0 + j) + 1] = b.y[3 * (f0 + j) + 1] - s1;
        b.t[3 * (f0 + j) + 2] = b.y[3 * (f0 + j) + 2] - s2;
    }
}

// rows [i0, i0+8) of front s: x_i = sum_{k>=i} (L_JJ^{-1})_ki t_k, one warp per row
__global__ void __launch_bounds__(kST) k_bwd_x(FrontArgs a, SolveBufs b, const Tile* __restrict__ tiles)
{
    extern __shared__ double sm[];
    const Tile tl = tiles[blockIdx.x];
    const int s = tl.s, i0 = tl.off;
    const int c = a.ncol[s], f0 = a.first[s];
    double* t = sm;  // [c - i0][3]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int k = tid; k < 3 * (c - i0); k += kST) t[k] = b.t[3 * (f0 + i0) + k];
    __syncthreads();
    const int i = i0 + warp;
    if (i >= c) return;
    double x0, x1, x2;
    warp_dot3(a.dinvT + a.dinv_off[s] + static_cast<long long>(i) * c, t, i, c, i0, lane, x0, x1, x2);
    if (lane == 0) {
        b.w[3 * (f0 + i)] = x0;
        b.w[3 * (f0 + i) + 1] = x1;
        b.w[3 * (f0 + i) + 2] = x2;
    }
}

// row-major copy of every front's L_RJ, columns [j0, j0+32) per CTA
__global__ void __launch_bounds__(256) k_transpose_lt(FrontArgs a, const Tile* __restrict__ tiles)
{
    const Tile tl = tiles[blockIdx.x];
    const int s = tl.s, j0 = tl.off;
    const int r = a.nrow[s], c = a.ncol[s], m = r - c;
    const int j = j0 + (threadIdx.x & 31);
    if (j >= c) return;
    const double* F = a.front + a.front_off[s] + static_cast<long long>(j) * r + c;
    double* LT = a.lt + a.lt_off[s] + j;
    for (int k = threadIdx.x >> 5; k < m; k += 8) LT[static_cast<long long>(k) * c] = F[k];
}

FrontArgs args_of(Precond& P)
{
    return FrontArgs { P.d_first, P.d_ncol, P.d_nrow, P.d_rows, P.d_child_ptr, P.d_child_list, P.d_relind,
        P.d_level_list, P.d_contrib_ptr, P.d_contrib_idx, P.d_below_front, P.d_front_off, P.d_rows_off, P.d_relind_off, P.d_dinv_off,
        P.d_upd_off, P.d_lt_off, P.d_front, P.d_dinv, P.d_dinvT, P.d_lt, P.d_fail };
}

// enqueue one H0 application (gather, levels, scatter) on stream st
void enqueue_solve(const Precond& P, const FrontArgs& a, const SolveBufs& b, double* d_v, cudaStream_t st)
{
    const Symbolic& S = P.S;
    const int n = S.n;
    const int g = std::min(1184, (n + 255) / 256);
    k_gather_rhs<<<g, 256, 0, st>>>(b.w, d_v, P.d_perm, n);
    for (int l = 0; l < P.nlev; l++) {
        const size_t smc = sizeof(double) * 3 * std::max(P.lev_max_c[l], 1);
        const int ny = P.fy_off[l + 1] - P.fy_off[l];
        k_fwd_y<<<ny, kST, smc, st>>>(a, b, P.d_fy + P.fy_off[l]);
        const int ng = P.fg_off[l + 1] - P.fg_off[l];
        if (ng > 0) k_fwd_g<<<ng, kST, smc, st>>>(a, b, P.d_fg + P.fg_off[l]);
    }
    for (int l = P.nlev - 1; l >= 0; l--) {
        const int nt = P.bt_off[l + 1] - P.bt_off[l];
        k_bwd_t<<<nt, kST, sizeof(double) * 3 * std::max(P.lev_max_m[l], 1), st>>>(a, b, P.d_bt + P.bt_off[l]);
        const int nx = P.bx_off[l + 1] - P.bx_off[l];
        k_bwd_x<<<nx, kST, sizeof(double) * 3 * std::max(P.lev_max_c[l], 1), st>>>(a, b, P.d_bx + P.bx_off[l]);
    }
    k_scatter_sol<<<g, 256, 0, st>>>(d_v, b.w, P.d_perm, n);
}

}  // namespace

void free_precond(Model& m)
{
    if (!m.precond) return;
    Precond& P = *m.precond;
    for (auto& kv : P.graphs) cudaGraphExecDestroy(kv.second);
    P.graphs.clear();
    if (P.capture) cudaStreamDestroy(P.capture);
    for (int** p : { &P.d_first, &P.d_ncol, &P.d_nrow, &P.d_rows, &P.d_child_ptr, &P.d_child_list, &P.d_relind,
             &P.d_level_list, &P.d_perm, &P.d_fail, &P.d_panel_list, &P.d_contrib_ptr, &P.d_contrib_idx, &P.d_below_front })
        dev_free(*p);
    for (long long** p : { &P.d_front_off, &P.d_rows_off, &P.d_relind_off, &P.d_dinv_off, &P.d_upd_off, &P.d_a_pos,
             &P.d_a_src, &P.d_lt_off })
        dev_free(*p);
    for (Tile** p : { &P.d_fy, &P.d_fg, &P.d_bt, &P.d_bx, &P.d_inv, &P.d_ea, &P.d_oinv }) dev_free(*p);
    dev_free(P.d_syrk);
    for (double** p : { &P.d_front, &P.d_dinv, &P.d_dinvT, &P.d_lt, &P.d_upd, &P.d_w, &P.d_y, &P.d_t, &P.d_vals })
        dev_free(*p);
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
    if (m.precond && m.precond->factored && !refactor) {
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
    P.nlev = static_cast<int>(S.level_ptr.size()) - 1;
    const int nlev = P.nlev;
    // solve and factor schedules
    std::vector<Tile> fy, fg, bt, bx, inv, ea, oinv;
    P.ea_off.assign(1, 0);
    std::vector<int> panel_list;
    std::vector<int4> syrk;
    P.fy_off.assign(1, 0);
    P.fg_off.assign(1, 0);
    P.bt_off.assign(1, 0);
    P.bx_off.assign(1, 0);
    P.lev_max_c.assign(nlev, 0);
    P.lev_max_m.assign(nlev, 0);
    P.lev_first_step.assign(1, 0);
    for (int l = 0; l < nlev; l++) {
        int maxc = 0;
        for (int q = S.level_ptr[l]; q < S.level_ptr[l + 1]; q++) {
            const int s = S.level_list[q];
            const int c = S.ncol[s], mm = S.nrow[s] - c;
            P.lev_max_c[l] = std::max(P.lev_max_c[l], c);
            P.lev_max_m[l] = std::max(P.lev_max_m[l], mm);
            P.max_r = std::max(P.max_r, S.nrow[s]);
            P.max_c = std::max(P.max_c, c);
            P.max_m = std::max(P.max_m, mm);
            maxc = std::max(maxc, c);
            for (int o = 0; o < c; o += kSW) {
                fy.push_back({ s, o });
                bt.push_back({ s, o });
                bx.push_back({ s, o });
            }
            for (int o = 0; o < c; o += kRT) inv.push_back({ s, o });
            for (int jb = 0; jb + kRT < c; jb += kRT)  // diagonal tiles with rows below them
                for (int o = jb; o < jb + kRT; o += kIC) oinv.push_back({ s, o });
            if (S.child_ptr[s + 1] > S.child_ptr[s])
                for (int o = 0; o < S.nrow[s]; o += kFT / 32) ea.push_back({ s, o });
            for (int o = 0; o < mm; o += kSW) fg.push_back({ s, o });
        }
        P.fy_off.push_back(static_cast<int>(fy.size()));
        P.fg_off.push_back(static_cast<int>(fg.size()));
        P.bt_off.push_back(static_cast<int>(bt.size()));
        P.bx_off.push_back(static_cast<int>(bx.size()));
        P.ea_off.push_back(static_cast<int>(ea.size()));
        for (int k0 = 0; k0 < maxc; k0 += kNB) {
            Precond::Step st { l, k0, static_cast<int>(panel_list.size()), 0, static_cast<int>(syrk.size()), 0 };
            for (int q = S.level_ptr[l]; q < S.level_ptr[l + 1]; q++) {
                const int s = S.level_list[q];
                const int c = S.ncol[s], r = S.nrow[s];
                if (c <= k0) continue;
                panel_list.push_back(s);
                const int kb = std::min(kNB, c - k0);
                const int m2 = r - k0 - kb;
                const int nt = (m2 + kTS - 1) / kTS;
                for (int tj = 0; tj < nt; tj++)
                    for (int ti = tj; ti < nt; ti++) syrk.push_back(make_int4(s, ti, tj, 0));
            }
            st.panel_cnt = static_cast<int>(panel_list.size()) - st.panel_off;
            st.syrk_cnt = static_cast<int>(syrk.size()) - st.syrk_off;
            P.steps.push_back(st);
        }
        P.lev_first_step.push_back(static_cast<int>(P.steps.size()));
    }
    P.n_inv_tiles = static_cast<int>(inv.size());
    P.n_oinv = static_cast<int>(oinv.size());
    const size_t smem_need = sizeof(double) * 3 * static_cast<size_t>(std::max(P.max_c, P.max_m));
    if (smem_need > 200 * 1024) {
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
    UP(P.d_lt_off, S.lt_off);
    UP(P.d_contrib_ptr, S.contrib_ptr);
    UP(P.d_contrib_idx, S.contrib_idx);
    UP(P.d_a_pos, S.a_pos);
    UP(P.d_a_src, S.a_src);
    UP(P.d_vals, vals);
    UP(P.d_fy, fy);
    UP(P.d_fg, fg);
    UP(P.d_bt, bt);
    UP(P.d_bx, bx);
    UP(P.d_inv, inv);
    UP(P.d_oinv, oinv);
    UP(P.d_ea, ea);
    UP(P.d_below_front, S.below_front);
    UP(P.d_panel_list, panel_list);
    UP(P.d_syrk, syrk);
#undef UP
    const size_t n3 = 3 * static_cast<size_t>(std::max(S.n, 1));
    if ((st = dev_alloc(&P.d_front, static_cast<size_t>(S.front_size))) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_dinv, static_cast<size_t>(std::max<long long>(S.dinv_size, 1)))) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_dinvT, static_cast<size_t>(std::max<long long>(S.dinv_size, 1)))) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_lt, static_cast<size_t>(std::max<long long>(S.lt_size, 1)))) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_upd, static_cast<size_t>(std::max<long long>(S.upd_size, 1)))) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_w, n3)) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_y, n3)) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_t, n3)) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_fail, 1)) != EFEM_OK) return st;
    for (const void* k : { (const void*)k_fwd_y, (const void*)k_fwd_g, (const void*)k_bwd_t, (const void*)k_bwd_x })
        EFEM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    EFEM_CUDA(cudaStreamCreateWithFlags(&P.capture, cudaStreamNonBlocking));
    P.ready = true;  // analysed; the numeric factor follows
    return precond_factor(m, ok, ms_factor);
}

// Numeric factorisation (every solve, like LBFGSSolver::updateApproxJacobi):
// scatter L into the fronts, factor level by level, invert the diagonal blocks.
static efem_status precond_factor(Model& m, int* ok, double* ms_factor)
{
    Precond& P = *m.precond;
    const Symbolic& S = P.S;
    cudaEvent_t e0, e1;
    EFEM_CUDA(cudaEventCreate(&e0));
    EFEM_CUDA(cudaEventCreate(&e1));
    EFEM_CUDA(cudaEventRecord(e0, m.stream));
    EFEM_CUDA(cudaMemsetAsync(P.d_front, 0, sizeof(double) * S.front_size, m.stream));
    EFEM_CUDA(cudaMemsetAsync(P.d_fail, 0, sizeof(int), m.stream));
    const long long na = static_cast<long long>(S.a_pos.size());
    k_scatter_a<<<static_cast<int>(std::min<long long>(1184, (na + 255) / 256 + 1)), 256, 0, m.stream>>>(
        P.d_front, P.d_a_pos, P.d_a_src, P.d_vals, na);
    m.launches++;
    FrontArgs a = args_of(P);
    for (int l = 0; l < P.nlev; l++) {
        const int cnt = P.ea_off[l + 1] - P.ea_off[l];
        if (cnt > 0) {
            k_extend_add<<<cnt, kFT, 0, m.stream>>>(a, P.d_ea + P.ea_off[l]);
            m.launches++;
        }
        for (int q = P.lev_first_step[l]; q < P.lev_first_step[l + 1]; q++) {
            const Precond::Step& stp = P.steps[q];
            k_panel<<<stp.panel_cnt, kFT, 0, m.stream>>>(a, P.d_panel_list + stp.panel_off, stp.k0);
            m.launches++;
            if (stp.syrk_cnt > 0) {
                k_syrk<<<stp.syrk_cnt, kFT, 0, m.stream>>>(a, P.d_syrk + stp.syrk_off, stp.k0);
                m.launches++;
            }
        }
    }
    if (P.n_inv_tiles > 0) {
        k_diag_inv<<<P.n_inv_tiles, 32, 0, m.stream>>>(a, P.d_inv);
        m.launches += 2;
        if (P.n_oinv > 0) {
            k_offdiag_inv<<<P.n_oinv, kIT, 0, m.stream>>>(a, P.d_oinv);
            m.launches++;
        }
        k_transpose_lt<<<P.n_inv_tiles, 256, 0, m.stream>>>(a, P.d_inv);
    }
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

// One H0 application, replayed from a CUDA graph captured (once per input
// vector and work buffers) on the preconditioner's private stream.
static efem_status apply_with(Model& m, double* d_v, const SolveBufs& b)
{
    Precond& P = *m.precond;
    if (P.S.n == 0) return EFEM_OK;
    const auto key = std::make_pair(d_v, b.w);
    auto it = P.graphs.find(key);
    if (it == P.graphs.end()) {
        if (P.graphs.size() >= 8) {  // callers passing many distinct vectors: start over
            EFEM_CUDA(cudaStreamSynchronize(m.stream));
            for (auto& kv : P.graphs) cudaGraphExecDestroy(kv.second);
            P.graphs.clear();
        }
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        EFEM_CUDA(cudaStreamBeginCapture(P.capture, cudaStreamCaptureModeThreadLocal));
        enqueue_solve(P, args_of(P), b, d_v, P.capture);
        EFEM_CUDA(cudaStreamEndCapture(P.capture, &g));
        EFEM_CUDA(cudaGraphInstantiate(&ge, g, 0));
        cudaGraphDestroy(g);
        it = P.graphs.emplace(key, ge).first;
    }
    EFEM_CUDA(cudaGraphLaunch(it->second, m.stream));
    m.launches += 2 + 4LL * P.nlev;
    return EFEM_OK;
}

efem_status precond_apply(Model& m, double* d_v)
{
    if (!m.precond || !m.precond->factored || !m.precond->ok) {
        set_error("preconditioner not factored");
        return EFEM_ERR_ARG;
    }
    Precond& P = *m.precond;
    return apply_with(m, d_v, SolveBufs { P.d_w, P.d_y, P.d_t, P.d_upd });
}

efem_status precond_enqueue(Model& m, double* d_v, cudaStream_t stream)
{
    if (!m.precond || !m.precond->factored || !m.precond->ok) {
        set_error("preconditioner not factored");
        return EFEM_ERR_ARG;
    }
    Precond& P = *m.precond;
    if (P.S.n == 0) return EFEM_OK;
    enqueue_solve(P, args_of(P), SolveBufs { P.d_w, P.d_y, P.d_t, P.d_upd }, d_v, stream);
    return EFEM_OK;
}

long long precond_launch_count(const Model& m)
{
    return m.precond ? 2 + 4LL * m.precond->nlev : 0;
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
// right-hand side and solution, the forward and backward intermediates, 3 per
// free node each, and the fronts' update vectors) live in the fixed array
// below instead of buffers owned by the model.
//
// Limits and sharing:
//   * the array holds kNoAllocDoubles doubles (16 MiB); a model that needs
//     more (9 * free nodes + its update-vector length) is rejected;
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
    const size_t n3 = 3 * static_cast<size_t>(S.n);
    const size_t need = 3 * n3 + static_cast<size_t>(S.upd_size);
    if (need > kNoAllocDoubles) {
        set_error("model needs " + std::to_string(need) + " doubles of workspace; the static workspace of "
            "efem_precond_apply_noalloc holds " + std::to_string(kNoAllocDoubles));
        return EFEM_ERR_ARG;
    }
    double* scratch = nullptr;
    efem_status st = noalloc_scratch(m.device, &scratch);
    if (st != EFEM_OK) return st;
    EFEM_CUDA(cudaSetDevice(m.device));
    if (S.n == 0) return EFEM_OK;
    const SolveBufs b { scratch, scratch + n3, scratch + 2 * n3, scratch + 3 * n3 };
    enqueue_solve(P, args_of(P), b, d_v, m.stream);
    EFEM_CUDA(cudaGetLastError());
    EFEM_CUDA(cudaStreamSynchronize(m.stream));
    return EFEM_OK;
}
