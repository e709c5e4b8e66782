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
//   k_panel       per front and chunk of rows: Cholesky of the 32x32
//                 diagonal block in shared memory (one warp), then the
//                 panel TRSM on the chunk's rows; k_panel_store then writes
//                 the factored diagonal blocks into the fronts;
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
constexpr int kRT = 32;   // columns per CTA of the inverse / transpose kernels
constexpr int kStageBudget = 4096;        // staged doubles per solve tile (rows of a tile x row length)
constexpr long long kWholeBudget = 4096;  // staged doubles up to which one CTA solves a whole front

// one work item of the persistent triangular solve
struct SolveItem {
    int kind, s, r0, r1;  // kind, front, rows [r0, r1) of the tile
    int cbeg, cend;       // contributions assembled for the front's own rows (or the tile's)
    int cbeg2, cend2;     // update tiles: contributions of the tile's below-diagonal rows
};

struct Tile {
    int s;    // front
    int off;  // first row / column of the tile (multiple of kRT)
};

// a subtree solved by one CTA (see k_sub_fwd) and its chunks of factor rows
struct SubTree {
    int lo, hi;             // fronts [lo, hi] in postorder; hi is the root
    int j0, ncols;          // the subtree's columns [j0, j0 + ncols) (new numbering)
    int chunk0, nchunk_f;   // forward chunks
    int bchunk0, nchunk_b;  // backward chunks
};

struct SubChunk {
    int s;      // front
    int kind;   // 0: rows of L_JJ^{-1}; 1: rows of W; 2: rows of L_JJ^{-T} and of W^T
    int a, b;   // rows [a, b)
    int first;  // the front's first chunk of the sweep
};

constexpr int kSubStage = 4096;  // doubles per stage buffer (two buffers)
}  // namespace

struct Precond {
    Symbolic S;
    bool ready = false;     // symbolic analysis done and uploaded
    bool factored = false;  // numeric factor present
    bool ok = false;        // factor is positive definite
    double ms_factor = 0;
    int max_r = 0, max_c = 0, max_m = 0, nlev = 0;
    // solve schedule: the persistent kernel's items, launch shape
    int n_items = 0, solve_grid = 1, solve_grid_full = 1, slots = 1;
    size_t solve_smem = 0;
    SolveItem* d_items = nullptr;
    std::vector<int> h_item_front;  // the front of every item (host)
    int* d_item_group = nullptr;    // batch unions: member of every item
    const int* d_frozen = nullptr;  // batch unions: per-member flag, 1 = skip its items
    int *d_tgt = nullptr, *d_parent = nullptr, *d_cnt = nullptr, *d_prow = nullptr;
    // subtree solves below the cut level (sub_levels levels of the tree)
    int sub_levels = 0, n_subs = 0;
    int sub_max_r = 0, sub_max_cols = 0, sub_max_depth = 0, sub_max_m = 0, sub_max_c = 0, sub_max_mroot = 0;
    size_t sub_smem_f = 0, sub_smem_b = 0;
    SubTree* d_subs = nullptr;
    SubChunk* d_chunks = nullptr;
    int *d_depth = nullptr, *d_xidx = nullptr;
    int stage_d = 0, work_d = 0;
    // factor schedule: per (level, step) the fronts with a panel at that step and the SYRK tiles
    struct Step {
        int level, k0, panel_off, panel_cnt, syrk_off, syrk_cnt, panel_chunks;
    };
    std::vector<Step> steps;
    std::vector<int> lev_first_step;  // index into steps, nlev + 1
    int n_inv_tiles = 0;
    int *d_first = nullptr, *d_ncol = nullptr, *d_nrow = nullptr, *d_rows = nullptr, *d_child_ptr = nullptr,
        *d_child_list = nullptr, *d_relind = nullptr, *d_level_list = nullptr, *d_perm = nullptr, *d_fail = nullptr,
        *d_panel_list = nullptr;
    long long *d_front_off = nullptr, *d_rows_off = nullptr, *d_relind_off = nullptr, *d_dinv_off = nullptr,
              *d_upd_off = nullptr, *d_a_pos = nullptr, *d_a_src = nullptr;
    Tile* d_inv = nullptr;
    int *d_contrib_ptr = nullptr, *d_contrib_idx = nullptr, *d_below_front = nullptr;
    Tile *d_ea = nullptr, *d_oinv = nullptr;  // extend-add column tiles, off-diagonal inverse column groups
    std::vector<int> ea_off;                  // nlev + 1
    int n_oinv = 0;
    long long* d_lt_off = nullptr;
    double *d_dinvT = nullptr, *d_w = nullptr, *d_wt = nullptr;
    int4* d_wtiles = nullptr;  // (front, 64-row tile, 64-column tile) of every W
    int n_wtiles = 0;
    int4* d_syrk = nullptr;
    double* d_diag_tmp = nullptr;  // factored diagonal blocks of one panel step, [fronts in step][kNB][kNB]
    int max_panel_cnt = 0;
    double *d_front = nullptr, *d_dinv = nullptr, *d_upd = nullptr, *d_y = nullptr, *d_t = nullptr,
           *d_vals = nullptr;
    // graph replay of the numeric factorisation (the same launches every solve)
    cudaGraphExec_t factor_exec = nullptr;
    long long factor_launches = 0;
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
    double* w;      // W = L_RJ L_JJ^{-1}, row-major (r - c) x c
    double* wt;     // W^T, row-major c x (r - c)
    int* fail;
};


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

// Diagonal block and panel of step k0 for the fronts in the step's list.
// Grid (fronts, row chunks): every CTA factors the panel's kb x kb diagonal
// block (one warp, left-looking, with the reciprocals of the pivots so that
// no division sits on a dependent chain; every CTA computes the same block,
// so the factor does not depend on the grid) and solves up to kFT of the rows
// below it, one per thread.  Chunk 0 leaves the factored block in tmp, and
// k_panel_store copies it into the front afterwards: written in place, it
// could reach a chunk CTA of a later wave before that CTA has read the
// unfactored block.
__global__ void __launch_bounds__(kFT) k_panel(FrontArgs a, const int* __restrict__ list, int k0,
    double* __restrict__ tmp)
{
    const int s = list[blockIdx.x];
    const int r = a.nrow[s], c = a.ncol[s];
    const int kb = min(kNB, c - k0);
    const int row0 = k0 + kb + static_cast<int>(blockIdx.y) * kFT;
    if (blockIdx.y > 0 && row0 >= r) return;  // uniform over the CTA
    double* F = a.front + a.front_off[s];
    const int tid = threadIdx.x;
    __shared__ double D[kNB][kNB + 1];
    __shared__ double Dinv[kNB];  // 1 / L_jj: the divisions leave the dependent chains
    for (int idx = tid; idx < kb * kb; idx += kFT) {
        const int i = idx % kb, j = idx / kb;
        D[i][j] = (i >= j) ? F[(k0 + i) + static_cast<long long>(k0 + j) * r] : 0.0;
    }
    __syncthreads();
    if (tid < 32) {
        const int i = tid;
        for (int j = 0; j < kb; j++) {
            if (i == j) {
                double d = D[j][j];
                for (int k = 0; k < j; k++) d -= D[j][k] * D[j][k];
                if (!(d > 0.0)) {
                    if (blockIdx.y == 0) *a.fail = 1;
                    d = 1.0;
                }
                const double sd = sqrt(d);
                D[j][j] = sd;
                Dinv[j] = 1.0 / sd;
            }
            __syncwarp();
            if (i > j && i < kb) {
                double t = D[i][j];
                for (int k = 0; k < j; k++) t -= D[i][k] * D[j][k];
                D[i][j] = t * Dinv[j];
            }
            __syncwarp();
        }
    }
    __syncthreads();
    if (blockIdx.y == 0)
        for (int idx = tid; idx < kb * kb; idx += kFT) {
            const int i = idx % kb, j = idx / kb;
            if (i >= j) tmp[static_cast<size_t>(blockIdx.x) * kNB * kNB + idx] = D[i][j];
        }
    // rows below the block: x L^T = f
    for (int i = row0 + tid; i < min(r, row0 + kFT); i += kFT) {
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
                x[j] = sum * Dinv[j];
            }
        }
#pragma unroll
        for (int j = 0; j < kNB; j++)
            if (j < kb) F[i + static_cast<long long>(k0 + j) * r] = x[j];
    }
}

// the factored diagonal blocks of a panel step, from k_panel's tmp into the fronts
__global__ void __launch_bounds__(kFT) k_panel_store(FrontArgs a, const int* __restrict__ list, int k0,
    const double* __restrict__ tmp)
{
    const int s = list[blockIdx.x];
    const int r = a.nrow[s], c = a.ncol[s];
    const int kb = min(kNB, c - k0);
    double* F = a.front + a.front_off[s];
    for (int idx = threadIdx.x; idx < kb * kb; idx += kFT) {
        const int i = idx % kb, j = idx / kb;
        if (i >= j) F[(k0 + i) + static_cast<long long>(k0 + j) * r] = tmp[static_cast<size_t>(blockIdx.x) * kNB * kNB + idx];
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
//
// One persistent launch runs the whole solve H0 v (in place on v, 3 values per
// node).  Its work is a list of items in dependency order -- the forward
// sweep leaves first, then the backward sweep root first -- and every CTA
// takes the next item from a ticket counter.  An item waits until the items
// it depends on have finished (per-front completion counters), so a front
// starts as soon as its children (forward) or its parent (backward) are done,
// with no barrier between levels.  An item only waits on items with smaller
// tickets, which were taken by CTAs already running (a CTA takes its next
// ticket while it works on the current one, which keeps this true), so the
// wait always ends whatever the number of resident CTAs; each wait is still
// bounded, and a wait that runs out sets the error flag and makes every later
// wait give up.
//
// Before it waits, a CTA stages everything of its item that does not depend
// on other items -- the factor rows it multiplies with (odd row stride in
// shared memory, so lanes on different rows hit different banks) and the
// index lists of the assembly -- with cp.async, so only the dependent vectors
// are fetched after the wait.
//
// Item kinds.  A small front is one item per sweep; a large one is split into
// tiles of rows sized so that a tile's factor rows fill about kStageBudget
// doubles.  Every output row is a dot product computed by a group of g lanes
// (g = 32 for a handful of long rows, down to one thread per row for many
// short ones).  With W = L_RJ L_JJ^{-1} from the factorisation, each sweep has
// one dependent step per tree level:
//   kFwdFront  y_J = L_JJ^{-1} f_J and g = f_R - W f_J for a whole front
//   kFwdY      y rows of one tile         (waits: children's g)
//   kFwdG      update rows of one tile    (waits: children's g)
//   kBwdFront  x_J = L_JJ^{-T} y_J - W^T x_R for a whole front
//   kBwdX      x rows of one tile         (waits: own y, parent's x)
enum ItemKind { kFwdFront = 0, kFwdY = 1, kFwdG = 2, kBwdFront = 3, kBwdX = 5 };

// device counters, one int array: [cY ns][cGin ns][exits, ns - 1 unused][cX ns][ticket][error]
struct SolveArgs {
    FrontArgs a;
    const int* parent;
    const int* prow;          // per front row (rows_off[s] + t): the node's index in v
    const SolveItem* items;
    const int* tgt;           // targets of the four counter groups
    int n_items, ns;
    int stage_d, work_d;      // shared-memory layout: staged doubles, work doubles, then ints
    double* v;
    double* y;
    double* t;
    double* upd;
    int* cnt;
    unsigned long long* stamp;  // when set: global timer at the start of the solve
    int spin_limit;             // polls of one wait before the solve gives up
    int test_wait;              // 1: the last item's wait target is raised by one (it can only run out)
    int n3;                     // entries of v (3 per free node)
    const int* item_group;      // batch unions: the member each item belongs to
    const int* frozen;          // batch unions: 1 for a member that no longer iterates (its items are skipped)
};

constexpr int kSpinLimit = 1 << 22;  // default polls of one wait (about half a second)

__device__ __forceinline__ int ld_acquire(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// thread 0 only: wait until *c >= target; false after `limit` polls (the
// error flag is then set) or when another wait has already given up
__device__ bool wait_ge(const int* c, int target, int* err, int limit)
{
    for (int it = 0;; it++) {
        if (ld_acquire(c) >= target) return true;
        if (*reinterpret_cast<volatile int*>(err)) return false;
        if (it >= limit) {
            atomicExch(err, 1);
            return false;
        }
        __nanosleep(64);
    }
}

__device__ __forceinline__ void ld3(const double* p, double& a, double& b, double& c)
{
    a = __ldcg(p);
    b = __ldcg(p + 1);
    c = __ldcg(p + 2);
}

__device__ __forceinline__ void cp8(double* dst, const double* src)
{
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void stage_i(int* dst, const int* src, int n)
{
    for (int i = threadIdx.x; i < n; i += kST) {
        const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst + i));
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src + i) : "memory");
    }
}
// rows [0, R) of a matrix with leading dimension ld, entries k in [lo(row), hi(row)),
// into dst with row stride lp; lo / hi: 0 = 0 / L, 1 = 0 / row0 + row + 1 (lower
// triangle), 2 = row0 + row / L (upper triangle); one warp per row
__device__ __forceinline__ void stage_rows(double* dst, int lp, const double* src, long long ld, int R, int L, int tri,
    int row0)
{
    const int lane = threadIdx.x & 31;
    for (int rr = threadIdx.x >> 5; rr < R; rr += kST / 32) {
        const int lo = tri == 2 ? row0 + rr : 0;
        const int hi = tri == 1 ? row0 + rr + 1 : L;
        const double* sr = src + rr * ld;
        double* dr = dst + rr * lp;
        for (int k = lo + lane; k < hi; k += 32) cp8(dr + k, sr + k);
    }
}
__device__ __forceinline__ void stage_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void stage_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void stage_wait_but_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

__device__ __forceinline__ int odd(int L) { return L | 1; }
__device__ __forceinline__ int lanes_per_row(int R)
{
    int g = kST;
    while (g > 1 && (kST / g) < R) g >>= 1;
    return g;
}

// Dot products of staged rows [0, R) (row stride lp) with a 3-component vector
// v in shared memory (entry k at v[3 (k - vbase)]), over k in [lo, hi) with
// lo / hi as in stage_rows.  Each row gets a group of g threads (g = kST / R
// rounded to a power of two: a whole CTA for one row, one thread per row for
// kST rows); a group wider than a warp adds its warps' partial sums through
// shared memory.  Every sum has a fixed order.  out is called with
// (row, s0, s1, s2) by the first thread of each group.
template <typename Out>
__device__ __forceinline__ void rows_dot(const double* M, int lp, const double* v, int vbase, int R, int L, int tri,
    int row0, Out out)
{
    __shared__ double part[kST / 32][3];
    const int g = lanes_per_row(R);
    const int lig = threadIdx.x & (g - 1), grp = threadIdx.x / g, ngrp = kST / g;
    for (int base = 0; base < R; base += ngrp) {  // uniform trip count across the CTA
        const int rr = base + grp;
        const bool valid = rr < R;
        const int lo = !valid ? 0 : (tri == 2 ? row0 + rr : 0);
        const int hi = !valid ? 0 : (tri == 1 ? row0 + rr + 1 : L);
        const double* row = M + rr * lp;
        double a0 = 0, a1 = 0, a2 = 0, b0 = 0, b1 = 0, b2 = 0;
        int k = lo + lig;
        for (; k + g < hi; k += 2 * g) {
            const double d = row[k], e = row[k + g];
            const double* vv = v + 3 * (k - vbase);
            const double* vw = vv + 3 * g;
            a0 += d * vv[0];
            a1 += d * vv[1];
            a2 += d * vv[2];
            b0 += e * vw[0];
            b1 += e * vw[1];
            b2 += e * vw[2];
        }
        if (k < hi) {
            const double d = row[k];
            const double* vv = v + 3 * (k - vbase);
            a0 += d * vv[0];
            a1 += d * vv[1];
            a2 += d * vv[2];
        }
        a0 += b0;
        a1 += b1;
        a2 += b2;
        const int w = g < 32 ? g : 32;
        for (int o = w >> 1; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        }
        if (g > 32) {  // several warps per row
            const int wid = threadIdx.x >> 5;
            if ((threadIdx.x & 31) == 0) {
                part[wid][0] = a0;
                part[wid][1] = a1;
                part[wid][2] = a2;
            }
            __syncthreads();
            if (valid && lig == 0) {
                a0 = a1 = a2 = 0.0;
                for (int q = wid; q < wid + g / 32; q++) {
                    a0 += part[q][0];
                    a1 += part[q][1];
                    a2 += part[q][2];
                }
                out(rr, a0, a1, a2);
            }
            __syncthreads();
        } else if (valid && lig == 0) {
            out(rr, a0, a1, a2);
        }
    }
}

// f_t for front rows [t0, t1) into f (3 per row): the right-hand side for own
// columns (t < c) plus the children's update entries landing on the row, from
// the staged contribution pointers cp (row t0 first) and indices ci (starting
// at contribution cbeg) and the staged node indices pr (row t0 first).  Each
// thread first issues the loads of up to kBatch rows (right-hand side and the
// first two contributions of each) and only then adds them, so the rows cost
// one memory latency instead of one each; further contributions (rows with
// more than two children behind them) follow in order.
constexpr int kBatch = 2;
__device__ __forceinline__ void assemble(const SolveArgs& A, int t0, int t1, int c, const int* cp, const int* ci,
    int cbeg, const int* pr, double* f)
{
    for (int base = t0; base < t1; base += kST * kBatch) {
        double b[kBatch][3], g[kBatch][2][3];
#pragma unroll
        for (int u = 0; u < kBatch; u++) {
            const int t = base + static_cast<int>(threadIdx.x) + u * kST;
            const bool valid = t < t1;
            const int q0 = valid ? cp[t - t0] : 0, q1 = valid ? cp[t - t0 + 1] : 0;
            b[u][0] = b[u][1] = b[u][2] = 0.0;
            if (valid && t < c) ld3(A.v + 3LL * pr[t - t0], b[u][0], b[u][1], b[u][2]);
#pragma unroll
            for (int e = 0; e < 2; e++) {
                g[u][e][0] = g[u][e][1] = g[u][e][2] = 0.0;
                if (q0 + e < q1) ld3(A.upd + 3LL * ci[q0 + e - cbeg], g[u][e][0], g[u][e][1], g[u][e][2]);
            }
        }
#pragma unroll
        for (int u = 0; u < kBatch; u++) {
            const int t = base + static_cast<int>(threadIdx.x) + u * kST;
            if (t >= t1) continue;
            double x0 = b[u][0] + g[u][0][0] + g[u][1][0];
            double x1 = b[u][1] + g[u][0][1] + g[u][1][1];
            double x2 = b[u][2] + g[u][0][2] + g[u][1][2];
            for (int q = cp[t - t0] + 2; q < cp[t - t0 + 1]; q++) {
                double h0, h1, h2;
                ld3(A.upd + 3LL * ci[q - cbeg], h0, h1, h2);
                x0 += h0;
                x1 += h1;
                x2 += h2;
            }
            double* o = f + 3 * (t - t0);
            o[0] = x0;
            o[1] = x1;
            o[2] = x2;
        }
    }
}

// n doubles from global memory written by other CTAs of this launch into
// shared memory, loads batched ahead of the stores
__device__ __forceinline__ void copy_cg(double* dst, const double* src, int n)
{
    for (int base = 0; base < n; base += kST * 8) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int i = base + static_cast<int>(threadIdx.x) + u * kST;
            v[u] = i < n ? __ldcg(src + i) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int i = base + static_cast<int>(threadIdx.x) + u * kST;
            if (i < n) dst[i] = v[u];
        }
    }
}

// x_R: the solution on n front rows whose node indices are pr[0..n), gathered
// from v (3 per node) into shared memory, loads batched ahead of the stores
__device__ __forceinline__ void gather3(double* dst, const double* v, const int* pr, int n)
{
    for (int base = 0; base < n; base += kST * kBatch) {
        double x[kBatch][3];
#pragma unroll
        for (int u = 0; u < kBatch; u++) {
            const int k = base + static_cast<int>(threadIdx.x) + u * kST;
            x[u][0] = x[u][1] = x[u][2] = 0.0;
            if (k < n) ld3(v + 3LL * pr[k], x[u][0], x[u][1], x[u][2]);
        }
#pragma unroll
        for (int u = 0; u < kBatch; u++) {
            const int k = base + static_cast<int>(threadIdx.x) + u * kST;
            if (k < n) {
                dst[3 * k] = x[u][0];
                dst[3 * k + 1] = x[u][1];
                dst[3 * k + 2] = x[u][2];
            }
        }
    }
}

__global__ void __launch_bounds__(kST) k_solve(SolveArgs A)
{
    griddep_wait();
    extern __shared__ double sm[];
    double* st = sm;                                  // staged factor rows
    double* wk = sm + A.stage_d;                      // work vectors
    int* si = reinterpret_cast<int*>(wk + A.work_d);  // staged index lists
    __shared__ int item_sh, ok_sh, ok2_sh;
    const int ns = A.ns;
    int* cY = A.cnt;
    int* cGin = A.cnt + ns;
    int* cX = A.cnt + 3 * ns;
    int* ticket = A.cnt + 4 * ns;
    int* err = ticket + 1;
    const int* tY = A.tgt;
    const int* tGin = A.tgt + ns;
    const int* tX = A.tgt + 3 * ns;
    int* exits = A.cnt + 2 * ns;
    const int tid = threadIdx.x;
    const FrontArgs& a = A.a;
    int next = 0;  // thread 0: the ticket taken ahead
    if (tid == 0) {
        next = atomicAdd(ticket, 1);
        if (next == 0 && A.stamp) {
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            *A.stamp = t;
        }
    }
    for (;;) {
        if (tid == 0) item_sh = next;
        __syncthreads();
        const int it = item_sh;
        if (it >= A.n_items) {
            griddep_launch();  // no more items for this CTA
            break;
        }
        if (A.frozen && A.frozen[A.item_group[it]]) {
            // a batch member that stopped iterating: its tree of fronts (no
            // other member's items depend on it) is skipped whole
            if (tid == 0) next = atomicAdd(ticket, 1);
            __syncthreads();
            continue;
        }
        const int bump = A.test_wait && it == A.n_items - 1 ? 1 : 0;
        const SolveItem d = A.items[it];
        const int kind = d.kind, s = d.s, r0 = d.r0, r1 = d.r1, R = r1 - r0, cbeg = d.cbeg, cend = d.cend;
        const int p = A.parent[s];
        const int r = a.nrow[s], c = a.ncol[s], m = r - c, f0 = a.first[s];
        const long long ro = a.rows_off[s];
        const double* X = a.dinv + a.dinv_off[s];
        const double* XT = a.dinvT + a.dinv_off[s];
        const double* W = a.w + a.lt_off[s];
        const double* WT = a.wt + a.lt_off[s];
        const int lc = odd(c), lm = odd(m);
        const int nci = cend - cbeg, nci2 = d.cend2 - d.cbeg2;
        // stage what does not depend on other items
        switch (kind) {
        case kFwdFront:
            stage_rows(st, lc, X, c, c, c, 1, 0);           // L_JJ^{-1} rows (lower)
            stage_rows(st + c * lc, lc, W, c, m, c, 0, 0);  // W rows
            stage_i(si, a.contrib_ptr + ro, r + 1);
            stage_i(si + r + 1, a.contrib_idx + cbeg, nci);
            stage_i(si + r + 1 + nci, A.prow + ro, c);
            break;
        case kFwdY:
            stage_rows(st, lc, X + static_cast<long long>(r0) * c, c, R, c, 1, r0);
            stage_i(si, a.contrib_ptr + ro, r1 + 1);
            stage_i(si + r1 + 1, a.contrib_idx + cbeg, nci);
            stage_i(si + r1 + 1 + nci, A.prow + ro, r1);
            break;
        case kFwdG: {
            stage_rows(st, lc, W + static_cast<long long>(r0) * c, c, R, c, 0, 0);
            int* q = si;
            stage_i(q, a.contrib_ptr + ro, c + 1);
            stage_i(q + c + 1, a.contrib_idx + cbeg, nci);
            stage_i(q + c + 1 + nci, A.prow + ro, c);
            q += 2 * c + 1 + nci;
            stage_i(q, a.contrib_ptr + ro + c + r0, R + 1);
            stage_i(q + R + 1, a.contrib_idx + d.cbeg2, nci2);
            break;
        }
        case kBwdFront:
            stage_rows(st, lc, XT, c, c, c, 2, 0);             // L_JJ^{-T} rows (upper)
            stage_rows(st + c * lc, lm, WT, m, c, m, 0, 0);  // W^T rows
            stage_i(si, A.prow + ro, r);
            break;
        default:  // kBwdX
            stage_rows(st, lc, XT + static_cast<long long>(r0) * c, c, R, c, 2, r0);
            stage_rows(st + R * lc, lm, WT + static_cast<long long>(r0) * m, m, R, m, 0, 0);
            stage_i(si, A.prow + ro, r);
            break;
        }
        stage_commit();
        // The next ticket is drawn once this item's dependencies are in (a
        // few microseconds before the CTA is free), not when the item starts:
        // a CTA whose item waits on a long chain would otherwise hold up the
        // item of the ticket it drew.  Backward items wait in two steps: their
        // own front's forward result first, the parent's solution last.
        const bool bwd = kind == kBwdFront || kind == kBwdX;
        if (tid == 0) {
            const bool ok = bwd ? wait_ge(cY + s, tY[s] + bump, err, A.spin_limit)
                                : wait_ge(cGin + s, tGin[s] + bump, err, A.spin_limit);
            ok_sh = ok;
            if (!bwd || !ok) next = atomicAdd(ticket, 1);
        }
        // backward items: thread 0 waits for the parent's x, then draws the next ticket
        auto parent_wait = [&]() {
            if (tid == 0) {
                ok2_sh = p < 0 || wait_ge(cX + p, tX[p], err, A.spin_limit);
                next = atomicAdd(ticket, 1);
            }
            __syncthreads();
        };
        stage_wait();
        __syncthreads();
        if (ok_sh) {
            switch (kind) {
            case kFwdFront: {
                double* f = wk;  // [r][3]
                const int* ci = si + r + 1;
                assemble(A, 0, r, c, si, ci, cbeg, ci + nci, f);
                __syncthreads();
                rows_dot(st, lc, f, 0, c, c, 1, 0, [&](int i, double y0, double y1, double y2) {
                    double* yg = A.y + 3LL * (f0 + i);
                    yg[0] = y0;
                    yg[1] = y1;
                    yg[2] = y2;
                });
                double* g = A.upd + a.upd_off[s];
                rows_dot(st + c * lc, lc, f, 0, m, c, 0, 0, [&](int k, double d0, double d1, double d2) {
                    const double* fk = f + 3 * (c + k);
                    g[3 * k] = fk[0] - d0;
                    g[3 * k + 1] = fk[1] - d1;
                    g[3 * k + 2] = fk[2] - d2;
                });
                break;
            }
            case kFwdY: {
                double* f = wk;  // [r1][3]
                const int* ci = si + r1 + 1;
                assemble(A, 0, r1, c, si, ci, cbeg, ci + nci, f);
                __syncthreads();
                rows_dot(st, lc, f, 0, R, c, 1, r0, [&](int i, double y0, double y1, double y2) {
                    double* yg = A.y + 3LL * (f0 + r0 + i);
                    yg[0] = y0;
                    yg[1] = y1;
                    yg[2] = y2;
                });
                break;
            }
            case kFwdG: {
                double* fj = wk;          // [c][3]
                double* fr = wk + 3 * c;  // [R][3]
                const int* q = si;
                const int* ci = q + c + 1;
                assemble(A, 0, c, c, q, ci, cbeg, ci + nci, fj);
                q += 2 * c + 1 + nci;
                assemble(A, c + r0, c + r1, c, q, q + R + 1, d.cbeg2, nullptr, fr);
                __syncthreads();
                double* g = A.upd + a.upd_off[s] + 3LL * r0;
                rows_dot(st, lc, fj, 0, R, c, 0, 0, [&](int k, double d0, double d1, double d2) {
                    g[3 * k] = fr[3 * k] - d0;
                    g[3 * k + 1] = fr[3 * k + 1] - d1;
                    g[3 * k + 2] = fr[3 * k + 2] - d2;
                });
                break;
            }
            case kBwdFront: {
                double* yj = wk;               // [c][3]
                double* xr = wk + 3 * c;       // [m][3]
                double* xs = wk + 3 * r;       // [c][3]
                copy_cg(yj, A.y + 3LL * f0, 3 * c);
                __syncthreads();
                // L_JJ^{-T} y_J needs only this front's forward result
                rows_dot(st, lc, yj, 0, c, c, 2, 0, [&](int i, double x0, double x1, double x2) {
                    xs[3 * i] = x0;
                    xs[3 * i + 1] = x1;
                    xs[3 * i + 2] = x2;
                });
                parent_wait();
                if (!ok2_sh) break;
                gather3(xr, A.v, si + c, m);
                __syncthreads();
                rows_dot(st + c * lc, lm, xr, 0, c, m, 0, 0, [&](int i, double s0, double s1, double s2) {
                    double* o = A.v + 3LL * si[i];
                    o[0] = xs[3 * i] - s0;
                    o[1] = xs[3 * i + 1] - s1;
                    o[2] = xs[3 * i + 2] - s2;
                });
                break;
            }
            default: {  // kBwdX
                double* yj = wk;                      // [c - r0][3]
                double* xr = wk + 3 * (c - r0);       // [m][3]
                double* xs = xr + 3 * m;              // [R][3]
                copy_cg(yj, A.y + 3LL * (f0 + r0), 3 * (c - r0));
                __syncthreads();
                rows_dot(st, lc, yj, r0, R, c, 2, r0, [&](int i, double x0, double x1, double x2) {
                    xs[3 * i] = x0;
                    xs[3 * i + 1] = x1;
                    xs[3 * i + 2] = x2;
                });
                parent_wait();
                if (!ok2_sh) break;
                gather3(xr, A.v, si + c, m);
                __syncthreads();
                rows_dot(st + R * lc, lm, xr, 0, R, m, 0, 0, [&](int i, double s0, double s1, double s2) {
                    double* o = A.v + 3LL * si[r0 + i];
                    o[0] = xs[3 * i] - s0;
                    o[1] = xs[3 * i + 1] - s1;
                    o[2] = xs[3 * i + 2] - s2;
                });
                break;
            }
            }
        }
        __syncthreads();  // the item's results are written
        if (tid == 0) {
            __threadfence();
            switch (kind) {
            case kFwdFront:
                atomicAdd(cY + s, 1);
                if (p >= 0) atomicAdd(cGin + p, 1);
                break;
            case kFwdY: atomicAdd(cY + s, 1); break;
            case kFwdG:
                if (p >= 0) atomicAdd(cGin + p, 1);
                break;
            default: atomicAdd(cX + s, 1); break;  // kBwdFront, kBwdX
            }
        }
    }
    // A solve that gave up leaves v partly overwritten: the last CTA to
    // leave fills it with NaN, so that a caller who cannot read the error
    // flag (a replayed graph) still sees that the result is not valid.
    if (tid == 0) {
        __threadfence();
        ok_sh = atomicAdd(exits, 1) == static_cast<int>(gridDim.x) - 1 && *reinterpret_cast<volatile int*>(err);
    }
    __syncthreads();
    if (ok_sh) {
        __threadfence();
        for (int i = tid; i < A.n3; i += kST) A.v[i] = __longlong_as_double(0x7ff8000000000000LL);
    }
}

// ---------------------------------------------------------------- subtree solves
// Below a cut level the elimination tree has many small fronts, and in the
// dataflow solve above every one of its levels costs an inter-CTA
// notification step (a few microseconds) per sweep.  There, each subtree is
// solved by one CTA from start to end instead: its fronts in postorder
// (forward) or reverse postorder (backward), the factor rows streamed through
// a double-buffered cp.async stage in chunks listed at set-up, and what passes
// between the subtree's fronts kept in shared memory -- the children's
// updates are added straight into the parent's assembly buffer (one buffer per
// depth below the subtree root), the solution on ancestor rows is read from
// the CTA's own copy.  Only the subtree root's update leaves the CTA (for its
// parent's assembly in k_solve), and the backward sweep reads the solution on
// the root's below rows once.  The subtree forward sweep runs before k_solve
// and the backward sweep after it, so the three launches need no counters.
// Sums keep the dataflow solve's order: b, then the children in list order.


struct SubArgs {
    FrontArgs a;
    const int* parent;
    const int* prow;
    const int* perm;
    const SubTree* subs;
    const SubChunk* chunks;
    const int* depth;  // per front: depth below its subtree root
    const int* xidx;   // per front row t >= c: >= 0 local column of the row; < 0: -(q + 1), the root's q-th below row
    int max_r, max_cols, max_depth, max_m, max_c, max_mroot;
    double* v;
    double* y;
    double* upd;
    unsigned long long* stamp;
};

__device__ __forceinline__ void sub_stage(const SubArgs& A, const SubChunk& ch, double* dst)
{
    const FrontArgs& a = A.a;
    const int s = ch.s, c = a.ncol[s], m = a.nrow[s] - c, R = ch.b - ch.a;
    const int lc = odd(c), lm = odd(m);
    if (ch.kind == 0) {
        stage_rows(dst, lc, a.dinv + a.dinv_off[s] + static_cast<long long>(ch.a) * c, c, R, c, 1, ch.a);
    } else if (ch.kind == 1) {
        stage_rows(dst, lc, a.w + a.lt_off[s] + static_cast<long long>(ch.a) * c, c, R, c, 0, 0);
    } else {
        stage_rows(dst, lc, a.dinvT + a.dinv_off[s] + static_cast<long long>(ch.a) * c, c, R, c, 2, ch.a);
        stage_rows(dst + R * lc, lm, a.wt + a.lt_off[s] + static_cast<long long>(ch.a) * m, m, R, m, 0, 0);
    }
    stage_commit();
}

// Forward sweep of one subtree per CTA: y_J = L_JJ^{-1} f_J for every front
// and the updates g = f_R - W f_J, added into the parent's buffer or, for the
// subtree root, written to the update array.
__global__ void __launch_bounds__(kST) k_sub_fwd(SubArgs A)
{
    extern __shared__ double sm[];
    double* buf[2] = { sm, sm + kSubStage };
    double* bsub = sm + 2 * kSubStage;          // [ncols][3] right-hand side on the subtree's columns
    double* acc = bsub + 3 * A.max_cols;        // [max_depth][max_r][3] assembly buffers
    const SubTree T = A.subs[blockIdx.x];
    const FrontArgs& a = A.a;
    if (A.stamp && blockIdx.x == 0 && threadIdx.x == 0) {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        *A.stamp = t;
    }
    const int nch = T.nchunk_f;
    if (nch > 0) sub_stage(A, A.chunks[T.chunk0], buf[0]);
    for (int i = threadIdx.x; i < T.ncols; i += kST) {
        const double* src = A.v + 3LL * A.perm[T.j0 + i];
        bsub[3 * i] = src[0];
        bsub[3 * i + 1] = src[1];
        bsub[3 * i + 2] = src[2];
    }
    __syncthreads();
    for (int i = 0; i < nch; i++) {
        const SubChunk ch = A.chunks[T.chunk0 + i];
        if (i + 1 < nch) sub_stage(A, A.chunks[T.chunk0 + i + 1], buf[(i + 1) & 1]);
        const int s = ch.s, c = a.ncol[s], r = a.nrow[s], lc = odd(c);
        double* f = acc + static_cast<size_t>(A.depth[s]) * 3 * A.max_r;
        const bool inner = s != T.hi;  // the parent belongs to the subtree
        const int p = A.parent[s];
        if (ch.first) {
            if (a.child_ptr[s] == a.child_ptr[s + 1]) {  // no children: f = (b_J, 0)
                const int jc = a.first[s] - T.j0;
                for (int t = threadIdx.x; t < r; t += kST) {
                    const bool own = t < c;
                    f[3 * t] = own ? bsub[3 * (jc + t)] : 0.0;
                    f[3 * t + 1] = own ? bsub[3 * (jc + t) + 1] : 0.0;
                    f[3 * t + 2] = own ? bsub[3 * (jc + t) + 2] : 0.0;
                }
            }
            if (inner && a.child_list[a.child_ptr[p]] == s) {  // first child: open the parent's buffer
                double* fp = acc + static_cast<size_t>(A.depth[p]) * 3 * A.max_r;
                const int cp = a.ncol[p], rp = a.nrow[p], jp = a.first[p] - T.j0;
                for (int t = threadIdx.x; t < rp; t += kST) {
                    const bool own = t < cp;
                    fp[3 * t] = own ? bsub[3 * (jp + t)] : 0.0;
                    fp[3 * t + 1] = own ? bsub[3 * (jp + t) + 1] : 0.0;
                    fp[3 * t + 2] = own ? bsub[3 * (jp + t) + 2] : 0.0;
                }
            }
        }
        if (i + 1 < nch)
            stage_wait_but_one();
        else
            stage_wait();
        __syncthreads();
        const double* cur = buf[i & 1];
        const int R = ch.b - ch.a;
        if (ch.kind == 0) {
            double* yg = A.y + 3LL * (a.first[s] + ch.a);
            rows_dot(cur, lc, f, 0, R, c, 1, ch.a, [&](int rr, double y0, double y1, double y2) {
                yg[3 * rr] = y0;
                yg[3 * rr + 1] = y1;
                yg[3 * rr + 2] = y2;
            });
        } else {
            double* fp = inner ? acc + static_cast<size_t>(A.depth[p]) * 3 * A.max_r : nullptr;
            const int* rel = a.relind + a.relind_off[s];
            double* g = A.upd + a.upd_off[s];
            rows_dot(cur, lc, f, 0, R, c, 0, 0, [&](int rr, double d0, double d1, double d2) {
                const int q = ch.a + rr;
                const double* fq = f + 3 * (c + q);
                const double g0 = fq[0] - d0, g1 = fq[1] - d1, g2 = fq[2] - d2;
                if (inner) {
                    double* o = fp + 3 * rel[q];
                    o[0] += g0;
                    o[1] += g1;
                    o[2] += g2;
                } else {
                    g[3 * q] = g0;
                    g[3 * q + 1] = g1;
                    g[3 * q + 2] = g2;
                }
            });
        }
        __syncthreads();  // the buffer is free for the chunk after next; updates are visible
    }
}

// Backward sweep of one subtree per CTA, fronts root first:
// x_J = L_JJ^{-T} y_J - W^T x_R, x_R from the CTA's own copy of the solution.
__global__ void __launch_bounds__(kST) k_sub_bwd(SubArgs A)
{
    extern __shared__ double sm[];
    double* buf[2] = { sm, sm + kSubStage };
    double* ysub = sm + 2 * kSubStage;        // [ncols][3]
    double* xs = ysub + 3 * A.max_cols;       // [ncols][3] solution on the subtree's columns
    double* xr = xs + 3 * A.max_cols;         // [max_mroot][3] solution on the root's below rows
    double* xR = xr + 3 * A.max_mroot;        // [max_m][3] x_R of the current front
    double* tmp = xR + 3 * A.max_m;           // [max_c][3]
    const SubTree T = A.subs[blockIdx.x];
    const FrontArgs& a = A.a;
    const int nch = T.nchunk_b;
    if (nch > 0) sub_stage(A, A.chunks[T.bchunk0], buf[0]);
    for (int i = threadIdx.x; i < 3 * T.ncols; i += kST) ysub[i] = __ldcg(A.y + 3LL * T.j0 + i);
    {
        const int root = T.hi, cr = a.ncol[root], mr = a.nrow[root] - cr;
        const int* pr = A.prow + a.rows_off[root] + cr;
        for (int q = threadIdx.x; q < mr; q += kST) {
            const double* src = A.v + 3LL * pr[q];
            xr[3 * q] = __ldcg(src);
            xr[3 * q + 1] = __ldcg(src + 1);
            xr[3 * q + 2] = __ldcg(src + 2);
        }
    }
    __syncthreads();
    for (int i = 0; i < nch; i++) {
        const SubChunk ch = A.chunks[T.bchunk0 + i];
        if (i + 1 < nch) sub_stage(A, A.chunks[T.bchunk0 + i + 1], buf[(i + 1) & 1]);
        const int s = ch.s, c = a.ncol[s], m = a.nrow[s] - c, lc = odd(c), lm = odd(m);
        const long long ro = a.rows_off[s];
        const int jc = a.first[s] - T.j0;
        if (ch.first) {  // x on the front's below rows, from the subtree's columns or the root's below rows
            const int* xi = A.xidx + ro + c;
            for (int q = threadIdx.x; q < m; q += kST) {
                const int li = xi[q];
                const double* src = li >= 0 ? xs + 3 * li : xr + 3 * (-li - 1);
                xR[3 * q] = src[0];
                xR[3 * q + 1] = src[1];
                xR[3 * q + 2] = src[2];
            }
        }
        if (i + 1 < nch)
            stage_wait_but_one();
        else
            stage_wait();
        __syncthreads();
        const double* cur = buf[i & 1];
        const int R = ch.b - ch.a;
        rows_dot(cur, lc, ysub + 3 * jc, 0, R, c, 2, ch.a, [&](int rr, double x0, double x1, double x2) {
            tmp[3 * rr] = x0;
            tmp[3 * rr + 1] = x1;
            tmp[3 * rr + 2] = x2;
        });
        __syncthreads();
        const int* pr = A.prow + ro + ch.a;
        double* xo = xs + 3 * (jc + ch.a);
        rows_dot(cur + R * lc, lm, xR, 0, R, m, 0, 0, [&](int rr, double s0, double s1, double s2) {
            const double x0 = tmp[3 * rr] - s0, x1 = tmp[3 * rr + 1] - s1, x2 = tmp[3 * rr + 2] - s2;
            xo[3 * rr] = x0;
            xo[3 * rr + 1] = x1;
            xo[3 * rr + 2] = x2;
            double* o = A.v + 3LL * pr[rr];
            o[0] = x0;
            o[1] = x1;
            o[2] = x2;
        });
        __syncthreads();
    }
}

// W = L_RJ L_JJ^{-1} for every front, one 64 x 64 tile of W per CTA (4 x 4
// per thread), L_RJ from the front's panel and L_JJ^{-1} (lower triangular,
// entries above the diagonal masked) in blocks of 32; written row-major as W
// and as its transpose.  With W the forward sweep forms a front's update
// g = f_R - W f_J without waiting for y_J, and the backward sweep forms
// x_J = L_JJ^{-T} y_J - W^T x_R in one step.
__global__ void __launch_bounds__(256) k_w(FrontArgs a, const int4* __restrict__ tiles)
{
    const int4 tl = tiles[blockIdx.x];
    const int s = tl.x, k0 = tl.y * 64, j0 = tl.z * 64;
    const int r = a.nrow[s], c = a.ncol[s], m = r - c;
    const double* F = a.front + a.front_off[s];
    const double* X = a.dinv + a.dinv_off[s];
    __shared__ double As[32][64 + 1];  // As[i][k] = L_RJ[k0 + k][i0 + i]
    __shared__ double Bs[32][64 + 1];  // Bs[i][j] = X[i0 + i][j0 + j]
    const int tid = threadIdx.x, tk = (tid & 15) * 4, tj = (tid >> 4) * 4;
    double acc[4][4] = {};
    for (int i0 = (j0 / 32) * 32; i0 < c; i0 += 32) {
        for (int idx = tid; idx < 32 * 64; idx += 256) {
            const int i = idx >> 6, kk = idx & 63;
            const int gi = i0 + i, gk = k0 + kk, gj = j0 + kk;
            As[i][kk] = (gi < c && gk < m) ? F[static_cast<long long>(gi) * r + c + gk] : 0.0;
            Bs[i][kk] = (gi < c && gj < c && gi >= gj) ? X[static_cast<long long>(gi) * c + gj] : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int i = 0; i < 32; i++) {
            double av[4], bv[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                av[q] = As[i][tk + q];
                bv[q] = Bs[i][tj + q];
            }
#pragma unroll
            for (int x = 0; x < 4; x++)
#pragma unroll
                for (int y = 0; y < 4; y++) acc[x][y] += av[x] * bv[y];
        }
        __syncthreads();
    }
    double* W = a.w + a.lt_off[s];
    double* WT = a.wt + a.lt_off[s];
#pragma unroll
    for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) {
            const int gk = k0 + tk + x, gj = j0 + tj + y;
            if (gk < m && gj < c) {
                W[static_cast<long long>(gk) * c + gj] = acc[x][y];
                WT[static_cast<long long>(gj) * m + gk] = acc[x][y];
            }
        }
}

FrontArgs args_of(Precond& P)
{
    return FrontArgs { P.d_first, P.d_ncol, P.d_nrow, P.d_rows, P.d_child_ptr, P.d_child_list, P.d_relind,
        P.d_level_list, P.d_contrib_ptr, P.d_contrib_idx, P.d_below_front, P.d_front_off, P.d_rows_off,
        P.d_relind_off, P.d_dinv_off, P.d_upd_off, P.d_lt_off, P.d_front, P.d_dinv, P.d_dinvT, P.d_w, P.d_wt, P.d_fail };
}

// the work buffers of one solve
struct SolveBufs {
    double* y;    // forward result, 3 per node
    double* t;    // backward intermediate, 3 per node
    double* upd;  // fronts' update vectors
    int* cnt;     // completion counters, ticket, error flag (4 ns + 2)
};

// limits of the persistent solve's device-side waits (efem_options.wait_limit, wait_test)
struct WaitCfg {
    int limit, test;
};
WaitCfg wait_cfg(const Model& m)
{
    return WaitCfg { m.opts.wait_limit > 0 ? m.opts.wait_limit : kSpinLimit, m.opts.wait_test ? 1 : 0 };
}

// enqueue one H0 application (counter reset unless the caller cleared them,
// then the persistent solve) on stream st
efem_status enqueue_solve(const Precond& P, const FrontArgs& a, const SolveBufs& b, double* d_v, cudaStream_t st,
    WaitCfg wc, bool clear = true, unsigned long long* stamp = nullptr)
{
    const int ns = P.S.ns;
    if (clear) EFEM_CUDA(cudaMemsetAsync(b.cnt, 0, sizeof(int) * (4 * static_cast<size_t>(ns) + 2), st));
    const SubArgs B { a, P.d_parent, P.d_prow, P.d_perm, P.d_subs, P.d_chunks, P.d_depth, P.d_xidx, P.sub_max_r,
        P.sub_max_cols, P.sub_max_depth, P.sub_max_m, P.sub_max_c, P.sub_max_mroot, d_v, b.y, b.upd, stamp };
    if (P.n_subs > 0) k_sub_fwd<<<P.n_subs, kST, P.sub_smem_f, st>>>(B);
    SolveArgs A { a, P.d_parent, P.d_prow, P.d_items, P.d_tgt, P.n_items, ns, P.stage_d, P.work_d, d_v, b.y, b.t,
        b.upd, b.cnt, P.n_subs > 0 ? nullptr : stamp, wc.limit, wc.test, 3 * P.S.n, P.d_item_group,
        P.d_item_group ? P.d_frozen : nullptr };
    if (P.n_items > 0) launch_k(k_solve, P.solve_grid, kST, P.solve_smem, st, A);
    if (P.n_subs > 0) k_sub_bwd<<<P.n_subs, kST, P.sub_smem_b, st>>>(B);
    return EFEM_OK;
}

}  // namespace

void free_precond(Model& m)
{
    if (!m.precond) return;
    m.epoch++;
    Precond& P = *m.precond;
    for (auto& kv : P.graphs) cudaGraphExecDestroy(kv.second);
    P.graphs.clear();
    if (P.factor_exec) cudaGraphExecDestroy(P.factor_exec);
    if (P.capture) cudaStreamDestroy(P.capture);
    for (int** p : { &P.d_first, &P.d_ncol, &P.d_nrow, &P.d_rows, &P.d_child_ptr, &P.d_child_list, &P.d_relind,
             &P.d_level_list, &P.d_perm, &P.d_fail, &P.d_panel_list, &P.d_contrib_ptr, &P.d_contrib_idx, &P.d_below_front, &P.d_tgt, &P.d_parent, &P.d_cnt, &P.d_prow, &P.d_depth, &P.d_xidx })
        dev_free(*p);
    for (long long** p : { &P.d_front_off, &P.d_rows_off, &P.d_relind_off, &P.d_dinv_off, &P.d_upd_off, &P.d_a_pos,
             &P.d_a_src, &P.d_lt_off })
        dev_free(*p);
    for (Tile** p : { &P.d_inv, &P.d_ea, &P.d_oinv }) dev_free(*p);
    dev_free(P.d_items);
    dev_free(P.d_item_group);
    dev_free(P.d_subs);
    dev_free(P.d_chunks);
    dev_free(P.d_syrk);
    dev_free(P.d_wtiles);
    for (double** p : { &P.d_front, &P.d_dinv, &P.d_dinvT, &P.d_w, &P.d_wt, &P.d_upd, &P.d_y, &P.d_t, &P.d_vals,
             &P.d_diag_tmp })
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
    info->solve_subtree_levels = m.precond->sub_levels;
    info->n_solve_subtrees = m.precond->n_subs;
    info->solve_ctas = m.precond->solve_grid;
    info->solve_smem_bytes = static_cast<int>(m.precond->solve_smem);
}

thread_local int t_batch = 0;

// the persistent solve's grid for the calling thread (see precond_sync_grid)
static int solve_grid_for(const Precond& P)
{
    if (t_batch <= 0) return P.solve_grid_full;
    return std::max(1, std::min(P.n_items, P.slots / t_batch));
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
    std::vector<Tile> inv, ea, oinv;
    P.ea_off.assign(1, 0);
    std::vector<int> panel_list;
    std::vector<int4> syrk;
    P.lev_first_step.assign(1, 0);
    for (int l = 0; l < nlev; l++) {
        int maxc = 0;
        for (int q = S.level_ptr[l]; q < S.level_ptr[l + 1]; q++) {
            const int s = S.level_list[q];
            const int c = S.ncol[s], mm = S.nrow[s] - c;
            P.max_r = std::max(P.max_r, S.nrow[s]);
            P.max_c = std::max(P.max_c, c);
            P.max_m = std::max(P.max_m, mm);
            maxc = std::max(maxc, c);
            for (int o = 0; o < c; o += kRT) inv.push_back({ s, o });
            for (int jb = 0; jb + kRT < c; jb += kRT)  // diagonal tiles with rows below them
                for (int o = jb; o < jb + kRT; o += kIC) oinv.push_back({ s, o });
            if (S.child_ptr[s + 1] > S.child_ptr[s])
                for (int o = 0; o < S.nrow[s]; o += kFT / 32) ea.push_back({ s, o });
        }
        P.ea_off.push_back(static_cast<int>(ea.size()));
        for (int k0 = 0; k0 < maxc; k0 += kNB) {
            Precond::Step st { l, k0, static_cast<int>(panel_list.size()), 0, static_cast<int>(syrk.size()), 0, 1 };
            for (int q = S.level_ptr[l]; q < S.level_ptr[l + 1]; q++) {
                const int s = S.level_list[q];
                const int c = S.ncol[s], r = S.nrow[s];
                if (c <= k0) continue;
                panel_list.push_back(s);
                const int kb = std::min(kNB, c - k0);
                const int m2 = r - k0 - kb;
                st.panel_chunks = std::max(st.panel_chunks, (m2 + kFT - 1) / kFT);
                const int nt = (m2 + kTS - 1) / kTS;
                for (int tj = 0; tj < nt; tj++)
                    for (int ti = tj; ti < nt; ti++) syrk.push_back(make_int4(s, ti, tj, 0));
            }
            st.panel_cnt = static_cast<int>(panel_list.size()) - st.panel_off;
            st.syrk_cnt = static_cast<int>(syrk.size()) - st.syrk_off;
            P.max_panel_cnt = std::max(P.max_panel_cnt, st.panel_cnt);
            P.steps.push_back(st);
        }
        P.lev_first_step.push_back(static_cast<int>(P.steps.size()));
    }
    P.n_inv_tiles = static_cast<int>(inv.size());
    std::vector<int4> wtiles;
    for (int s = 0; s < S.ns; s++) {
        const int c = S.ncol[s], mm = S.nrow[s] - c;
        for (int tk = 0; tk * 64 < mm; tk++)
            for (int tj = 0; tj * 64 < c; tj++) wtiles.push_back(make_int4(s, tk, tj, 0));
    }
    P.n_wtiles = static_cast<int>(wtiles.size());
    P.n_oinv = static_cast<int>(oinv.size());
    auto odd_h = [](int L) { return L | 1; };
    // Subtree solves: fronts on the lowest K levels are solved per subtree by
    // one CTA (k_sub_fwd / k_sub_bwd), the levels above by the dataflow
    // k_solve.  opts.solve_subtree_levels = K asks for them (K is lowered
    // until the subtrees fit in shared memory); the default (-1) is K = 0.
    // Measured on the 20 480-element C3D8 beam (11 levels), one H0
    // application inside the solve costs 274 us per iteration with K = 0 and
    // 290, 322, 361, 450 us with K = 1, 2, 3, 4: a subtree CTA streams its
    // factor rows one 32 KB chunk ahead, about 20 GB/s, and works through its
    // fronts one after another, which is slower than the notification steps
    // of the levels it replaces.
    std::vector<int> lev(S.ns, 0), nsub(S.ns, 1), sdepth(S.ns, 0);
    for (int l = 0; l < nlev; l++)
        for (int q = S.level_ptr[l]; q < S.level_ptr[l + 1]; q++) lev[S.level_list[q]] = l;
    for (int s = 0; s < S.ns; s++)
        if (S.parent[s] >= 0) nsub[S.parent[s]] += nsub[s];
    bool postorder = true;  // every subtree is the index range [s - nsub[s] + 1, s]
    for (int s = 0; s < S.ns && postorder; s++)
        for (int k = s - nsub[s] + 1; k < s && postorder; k++) {
            int u = k;
            while (u >= 0 && u < s) u = S.parent[u];
            postorder = u == s;
        }
    struct SubPlan {
        bool ok = true;
        int max_r = 1, max_cols = 1, max_depth = 1, max_m = 1, max_c = 1, max_mroot = 1;
        size_t smem_f = 0, smem_b = 0;
        std::vector<int> roots;
    };
    auto plan = [&](int K) {
        SubPlan p;
        if (K <= 0) return p;
        for (int s = 0; s < S.ns; s++)
            if (lev[s] < K && (S.parent[s] < 0 || lev[S.parent[s]] >= K)) p.roots.push_back(s);
        for (int root : p.roots) {
            int cols = 0;
            for (int k = root; k > root - nsub[root]; k--) {  // parents before children
                sdepth[k] = k == root ? 0 : sdepth[S.parent[k]] + 1;
                const int c = S.ncol[k], r = S.nrow[k], mm = r - c;
                cols += c;
                p.max_r = std::max(p.max_r, r);
                p.max_m = std::max(p.max_m, mm);
                p.max_c = std::max(p.max_c, c);
                p.max_depth = std::max(p.max_depth, sdepth[k] + 1);
                if (odd_h(c) + odd_h(mm) > kSubStage) p.ok = false;
            }
            p.max_cols = std::max(p.max_cols, cols);
            p.max_mroot = std::max(p.max_mroot, S.nrow[root] - S.ncol[root]);
        }
        p.smem_f = sizeof(double) * (2 * static_cast<size_t>(kSubStage) + 3 * static_cast<size_t>(p.max_cols)
            + 3 * static_cast<size_t>(p.max_depth) * p.max_r);
        p.smem_b = sizeof(double) * (2 * static_cast<size_t>(kSubStage) + 6 * static_cast<size_t>(p.max_cols)
            + 3 * static_cast<size_t>(p.max_mroot + p.max_m + p.max_c));
        if (std::max(p.smem_f, p.smem_b) > 200 * 1024) p.ok = false;
        return p;
    };
    int K = 0;
    if (postorder && m.opts.solve_subtree_levels > 0)
        for (K = std::min(m.opts.solve_subtree_levels, nlev); K > 0 && !plan(K).ok; K--) {
        }
    const SubPlan sp = plan(K);  // also leaves sdepth for the chosen subtrees
    std::vector<char> in_sub(S.ns, 0);
    for (int s = 0; s < S.ns; s++) in_sub[s] = lev[s] < K;
    std::vector<SubTree> subs;
    std::vector<SubChunk> chunks;
    std::vector<int> xidx(S.rows.size(), 0);
    for (int root : sp.roots) {
        SubTree T {};
        T.lo = root - nsub[root] + 1;
        T.hi = root;
        T.j0 = S.first[T.lo];
        T.ncols = S.first[root] + S.ncol[root] - T.j0;
        T.chunk0 = static_cast<int>(chunks.size());
        for (int k = T.lo; k <= T.hi; k++) {
            const int c = S.ncol[k], mm = S.nrow[k] - c, rx = std::max(1, kSubStage / odd_h(c));
            for (int a0 = 0; a0 < c; a0 += rx) chunks.push_back(SubChunk { k, 0, a0, std::min(c, a0 + rx), a0 == 0 });
            for (int a0 = 0; a0 < mm; a0 += rx) chunks.push_back(SubChunk { k, 1, a0, std::min(mm, a0 + rx), 0 });
        }
        T.nchunk_f = static_cast<int>(chunks.size()) - T.chunk0;
        T.bchunk0 = static_cast<int>(chunks.size());
        for (int k = T.hi; k >= T.lo; k--) {
            const int c = S.ncol[k], mm = S.nrow[k] - c, rb = std::max(1, kSubStage / (odd_h(c) + odd_h(mm)));
            for (int a0 = 0; a0 < c; a0 += rb) chunks.push_back(SubChunk { k, 2, a0, std::min(c, a0 + rb), a0 == 0 });
            // below rows: a column of the subtree, or one of the root's below rows
            const long long ro = S.rows_off[k];
            const int* rb0 = S.rows.data() + S.rows_off[root] + S.ncol[root];
            const int nrb = S.nrow[root] - S.ncol[root];
            for (int t = c; t < S.nrow[k]; t++) {
                const int row = S.rows[ro + t];
                if (row >= T.j0 && row < T.j0 + T.ncols) {
                    xidx[ro + t] = row - T.j0;
                } else {
                    const int q = static_cast<int>(std::lower_bound(rb0, rb0 + nrb, row) - rb0);
                    if (q >= nrb || rb0[q] != row) {
                        set_error("internal: a subtree row is neither a subtree column nor a root row");
                        return EFEM_ERR_CUDA;
                    }
                    xidx[ro + t] = -(q + 1);
                }
            }
        }
        T.nchunk_b = static_cast<int>(chunks.size()) - T.bchunk0;
        subs.push_back(T);
    }
    P.sub_levels = K;
    P.n_subs = static_cast<int>(subs.size());
    P.sub_max_r = sp.max_r;
    P.sub_max_cols = sp.max_cols;
    P.sub_max_depth = sp.max_depth;
    P.sub_max_m = sp.max_m;
    P.sub_max_c = sp.max_c;
    P.sub_max_mroot = sp.max_mroot;
    P.sub_smem_f = sp.smem_f;
    P.sub_smem_b = sp.smem_b;
    // solve items above the cut: forward sweep by level (leaves first),
    // backward sweep by level (root first).  Each item records the ranges of
    // contributions its rows assemble, and the shared memory it stages is
    // sized here.
    // Tiles take a multiple of 4 rows, at least 4.  A front with rows longer
    // than kStageBudget / 4 then stages more than the budget, and on a mesh
    // like the C3D20 cap that halves the CTAs per SM for every item of the
    // solve; so the schedule is also built with tiles of 1-3 rows for such
    // fronts (more items, more repeated assembly), and the one with more CTAs
    // per SM is kept (the 4-row one on a tie).
    struct Schedule {
        std::vector<SolveItem> items;
        std::vector<int> tgt;
        size_t stage_d = 1, work_d = 1, ints = 1;
        size_t smem() const { return sizeof(double) * (stage_d + work_d) + sizeof(int) * ints; }
    };
    std::vector<char> whole(S.ns, 0);
    auto schedule = [&](int min_rows, Schedule& sch) {
        std::vector<SolveItem>& items = sch.items;
        std::vector<int>& tgt = sch.tgt;
        tgt.assign(4 * static_cast<size_t>(S.ns), 0);
        size_t& stage_d = sch.stage_d;
        size_t& work_d = sch.work_d;
        size_t& ints = sch.ints;
        auto need = [&](size_t sd, size_t wd, size_t ni) {
            stage_d = std::max(stage_d, sd);
            work_d = std::max(work_d, wd);
            ints = std::max(ints, ni);
        };
        auto tile = [&](int per_row) {  // rows per tile when a row stages per_row doubles
            const int t = kStageBudget / per_row;
            return t >= 4 ? std::min(256, t / 4 * 4) : std::max(min_rows, t);
        };
        auto ntiles = [&](int n, int per_row) { const int t = tile(per_row); return (n + t - 1) / t; };
        auto crange = [&](int s, int t0, int t1) {  // contributions of front rows [t0, t1)
            const long long ro = S.rows_off[s];
            return t1 > t0 ? std::make_pair(S.contrib_ptr[ro + t0], S.contrib_ptr[ro + t1]) : std::make_pair(0, 0);
        };
        for (int s = 0; s < S.ns; s++) {
            const int c = S.ncol[s], mm = S.nrow[s] - c, r = S.nrow[s];
            const int lc = odd_h(c), lm = odd_h(mm);
            whole[s] = static_cast<long long>(r) * lc <= kWholeBudget && static_cast<long long>(c) * (lc + lm) <= kWholeBudget;
            tgt[s] = whole[s] ? 1 : ntiles(c, lc);  // y of s complete
            if (S.parent[s] >= 0 && !in_sub[s])     // children's g complete (subtree roots finish before k_solve)
                tgt[S.ns + S.parent[s]] += whole[s] ? 1 : ntiles(mm, lc);
            tgt[3 * S.ns + s] = whole[s] ? 1 : ntiles(c, lc + lm);                              // x of s complete
        }
        for (int l = K; l < nlev; l++) {
            for (int q = S.level_ptr[l]; q < S.level_ptr[l + 1]; q++) {
                const int s = S.level_list[q];
                const int c = S.ncol[s], r = S.nrow[s], mm = r - c, lc = odd_h(c);
                if (whole[s]) {
                    const auto cr = crange(s, 0, r);
                    items.push_back(SolveItem { kFwdFront, s, 0, c, cr.first, cr.second, 0, 0 });
                    need(static_cast<size_t>(r) * lc, 3 * static_cast<size_t>(r), r + 1 + (cr.second - cr.first) + c);
                    continue;
                }
                const int ty = tile(lc);
                for (int o = 0; o < c; o += ty) {
                    const int i1 = std::min(c, o + ty);
                    const auto cr = crange(s, 0, i1);
                    items.push_back(SolveItem { kFwdY, s, o, i1, cr.first, cr.second, 0, 0 });
                    need(static_cast<size_t>(i1 - o) * lc, 3 * static_cast<size_t>(i1), i1 + 1 + (cr.second - cr.first) + i1);
                }
                const auto cj = crange(s, 0, c);
                for (int o = 0; o < mm; o += ty) {
                    const int k1 = std::min(mm, o + ty);
                    const auto cr = crange(s, c + o, c + k1);
                    items.push_back(SolveItem { kFwdG, s, o, k1, cj.first, cj.second, cr.first, cr.second });
                    need(static_cast<size_t>(k1 - o) * lc, 3 * static_cast<size_t>(c + k1 - o),
                        2 * static_cast<size_t>(c) + 1 + (cj.second - cj.first) + (k1 - o + 1) + (cr.second - cr.first));
                }
            }
        }
        for (int l = nlev - 1; l >= K; l--) {
            for (int q = S.level_ptr[l]; q < S.level_ptr[l + 1]; q++) {
                const int s = S.level_list[q];
                const int c = S.ncol[s], r = S.nrow[s], mm = r - c, lc = odd_h(c), lm = odd_h(mm);
                if (whole[s]) {
                    items.push_back(SolveItem { kBwdFront, s, 0, c, 0, 0, 0, 0 });
                    need(static_cast<size_t>(c) * (lc + lm), 3 * static_cast<size_t>(r + c), r);
                    continue;
                }
                const int tx = tile(lc + lm);
                for (int o = 0; o < c; o += tx) {
                    const int i1 = std::min(c, o + tx);
                    items.push_back(SolveItem { kBwdX, s, o, i1, 0, 0, 0, 0 });
                    need(static_cast<size_t>(i1 - o) * (lc + lm), 3 * static_cast<size_t>(c - o + mm + i1 - o), r);
                }
            }
        }
    };
    Schedule sch4, sch1;
    schedule(4, sch4);
    schedule(1, sch1);
    EFEM_CUDA(cudaFuncSetAttribute(k_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    int per4 = 0, per1 = 0;
    if (sch4.smem() <= 200 * 1024)
        EFEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per4, k_solve, kST, sch4.smem()));
    if (sch1.smem() <= 200 * 1024)
        EFEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per1, k_solve, kST, sch1.smem()));
    Schedule& sch = per1 > per4 ? sch1 : sch4;
    std::vector<SolveItem>& items = sch.items;
    std::vector<int>& tgt = sch.tgt;
    const size_t stage_d = sch.stage_d, work_d = sch.work_d, ints = sch.ints;
    P.n_items = static_cast<int>(items.size());
    P.h_item_front.resize(items.size());
    for (size_t i = 0; i < items.size(); i++) P.h_item_front[i] = items[i].s;
    P.stage_d = static_cast<int>(stage_d);
    P.work_d = static_cast<int>(work_d);
    P.solve_smem = sizeof(double) * (stage_d + work_d) + sizeof(int) * ints;
    if (P.solve_smem > 200 * 1024) {
        set_error("a front of the approximate-Jacobian factor is too large for the solve kernel ("
            + std::to_string(P.max_r) + " rows)");
        return EFEM_ERR_UNSUPPORTED;
    }
    // node index in v of every front row
    std::vector<int> prow(S.rows.size());
    for (size_t q = 0; q < S.rows.size(); q++) prow[q] = S.perm[S.rows[q]];
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
    UP(P.d_parent, S.parent);
    UP(P.d_prow, prow);
    UP(P.d_items, items);
    UP(P.d_tgt, tgt);
    if (P.n_subs > 0) {
        UP(P.d_subs, subs);
        UP(P.d_chunks, chunks);
        UP(P.d_depth, sdepth);
        UP(P.d_xidx, xidx);
    }
    UP(P.d_inv, inv);
    UP(P.d_oinv, oinv);
    UP(P.d_wtiles, wtiles);
    UP(P.d_ea, ea);
    UP(P.d_below_front, S.below_front);
    UP(P.d_panel_list, panel_list);
    UP(P.d_syrk, syrk);
#undef UP
    const size_t n3 = 3 * static_cast<size_t>(std::max(S.n, 1));
    if ((st = dev_alloc(&P.d_front, static_cast<size_t>(S.front_size))) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_dinv, static_cast<size_t>(std::max<long long>(S.dinv_size, 1)))) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_dinvT, static_cast<size_t>(std::max<long long>(S.dinv_size, 1)))) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_w, static_cast<size_t>(std::max<long long>(S.lt_size, 1)))) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_wt, static_cast<size_t>(std::max<long long>(S.lt_size, 1)))) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_upd, static_cast<size_t>(std::max<long long>(S.upd_size, 1)))) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_y, n3)) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_t, n3)) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_cnt, 4 * static_cast<size_t>(S.ns) + 2)) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_fail, 1)) != EFEM_OK) return st;
    if ((st = dev_alloc(&P.d_diag_tmp, static_cast<size_t>(std::max(P.max_panel_cnt, 1)) * kNB * kNB)) != EFEM_OK)
        return st;
    // persistent solve: as many CTAs as fit on the device at once
    EFEM_CUDA(cudaFuncSetAttribute(k_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    int per_sm = 0, sms = 0;
    EFEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve, kST, P.solve_smem));
    EFEM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m.device));
    P.slots = std::max(1, per_sm) * std::max(1, sms);
    P.solve_grid_full = std::max(1, std::min(P.n_items, P.slots));
    P.solve_grid = solve_grid_for(P);
    if (P.n_subs > 0) {
        EFEM_CUDA(cudaFuncSetAttribute(k_sub_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        EFEM_CUDA(cudaFuncSetAttribute(k_sub_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    }
    EFEM_CUDA(cudaStreamCreateWithFlags(&P.capture, cudaStreamNonBlocking));
    P.ready = true;  // analysed; the numeric factor follows
    return precond_factor(m, ok, ms_factor);
}

// Numeric factorisation (every solve, like LBFGSSolver::updateApproxJacobi):
// scatter L into the fronts, factor level by level, invert the diagonal blocks.
// the launches of one numeric factorisation, in order, on stream st; returns
// the number of kernels
static long long enqueue_factor(Precond& P, cudaStream_t st)
{
    const Symbolic& S = P.S;
    long long n = 0;
    cudaMemsetAsync(P.d_front, 0, sizeof(double) * S.front_size, st);
    cudaMemsetAsync(P.d_fail, 0, sizeof(int), st);
    const long long na = static_cast<long long>(S.a_pos.size());
    k_scatter_a<<<static_cast<int>(std::min<long long>(1184, (na + 255) / 256 + 1)), 256, 0, st>>>(
        P.d_front, P.d_a_pos, P.d_a_src, P.d_vals, na);
    n++;
    FrontArgs a = args_of(P);
    for (int l = 0; l < P.nlev; l++) {
        const int cnt = P.ea_off[l + 1] - P.ea_off[l];
        if (cnt > 0) {
            k_extend_add<<<cnt, kFT, 0, st>>>(a, P.d_ea + P.ea_off[l]);
            n++;
        }
        for (int q = P.lev_first_step[l]; q < P.lev_first_step[l + 1]; q++) {
            const Precond::Step& stp = P.steps[q];
            k_panel<<<dim3(stp.panel_cnt, stp.panel_chunks), kFT, 0, st>>>(a, P.d_panel_list + stp.panel_off, stp.k0,
                P.d_diag_tmp);
            k_panel_store<<<stp.panel_cnt, kFT, 0, st>>>(a, P.d_panel_list + stp.panel_off, stp.k0, P.d_diag_tmp);
            n += 2;
            if (stp.syrk_cnt > 0) {
                k_syrk<<<stp.syrk_cnt, kFT, 0, st>>>(a, P.d_syrk + stp.syrk_off, stp.k0);
                n++;
            }
        }
    }
    if (P.n_inv_tiles > 0) {
        k_diag_inv<<<P.n_inv_tiles, 32, 0, st>>>(a, P.d_inv);
        n++;
        if (P.n_oinv > 0) {
            k_offdiag_inv<<<P.n_oinv, kIT, 0, st>>>(a, P.d_oinv);
            n++;
        }
        if (P.n_wtiles > 0) {
            k_w<<<P.n_wtiles, 256, 0, st>>>(a, P.d_wtiles);
            n++;
        }
    }
    return n;
}

// The factorisation's few hundred dependent launches are captured once into a
// CUDA graph and replayed every solve (shorter gaps between the launches).
static efem_status precond_factor(Model& m, int* ok, double* ms_factor)
{
    Precond& P = *m.precond;
    if (!P.factor_exec) {
        std::lock_guard<std::mutex> lock(capture_mutex());
        cudaGraph_t g = nullptr;
        EFEM_CUDA(cudaStreamBeginCapture(P.capture, cudaStreamCaptureModeThreadLocal));
        P.factor_launches = enqueue_factor(P, P.capture);
        const cudaError_t e = cudaStreamEndCapture(P.capture, &g);
        if (e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            set_error(std::string("capture of the factorisation: ") + cudaGetErrorString(e));
            return EFEM_ERR_CUDA;
        }
        const cudaError_t ei = cudaGraphInstantiate(&P.factor_exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            P.factor_exec = nullptr;
            set_error(std::string("factorisation graph: ") + cudaGetErrorString(ei));
            return EFEM_ERR_CUDA;
        }
    }
    cudaEvent_t e0, e1;
    EFEM_CUDA(cudaEventCreate(&e0));
    EFEM_CUDA(cudaEventCreate(&e1));
    EFEM_CUDA(cudaEventRecord(e0, m.stream));
    EFEM_CUDA(cudaGraphLaunch(P.factor_exec, m.stream));
    m.launches += P.factor_launches;
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
    const auto key = std::make_pair(d_v, b.y);
    auto it = P.graphs.find(key);
    if (it == P.graphs.end()) {
        if (P.graphs.size() >= 8) {  // callers passing many distinct vectors: start over
            EFEM_CUDA(cudaStreamSynchronize(m.stream));
            for (auto& kv : P.graphs) cudaGraphExecDestroy(kv.second);
            P.graphs.clear();
        }
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        std::lock_guard<std::mutex> lock(capture_mutex());
        EFEM_CUDA(cudaStreamBeginCapture(P.capture, cudaStreamCaptureModeThreadLocal));
        const efem_status es = enqueue_solve(P, args_of(P), b, d_v, P.capture, wait_cfg(m));
        EFEM_CUDA(cudaStreamEndCapture(P.capture, &g));
        if (es != EFEM_OK) {
            cudaGraphDestroy(g);
            return es;
        }
        EFEM_CUDA(cudaGraphInstantiate(&ge, g, 0));
        cudaGraphDestroy(g);
        it = P.graphs.emplace(key, ge).first;
    }
    EFEM_CUDA(cudaGraphLaunch(it->second, m.stream));
    m.launches += 1;
    return EFEM_OK;
}

void precond_drop_graphs(Model& m)
{
    if (!m.precond) return;
    if (m.on_device) cudaStreamSynchronize(m.stream);
    for (auto& kv : m.precond->graphs) cudaGraphExecDestroy(kv.second);
    m.precond->graphs.clear();
    m.epoch++;  // the solver's iteration graphs hold the persistent solve's arguments too
}

efem_status precond_sync_grid(Model& m)
{
    if (!m.precond || !m.precond->ready) return EFEM_OK;
    Precond& P = *m.precond;
    const int want = solve_grid_for(P);
    if (want == P.solve_grid) return EFEM_OK;
    EFEM_CUDA(cudaStreamSynchronize(m.stream));
    for (auto& kv : P.graphs) cudaGraphExecDestroy(kv.second);
    P.graphs.clear();
    P.solve_grid = want;
    m.epoch++;  // the solver's iteration graphs hold the old grid
    return EFEM_OK;
}

efem_status precond_apply(Model& m, double* d_v)
{
    if (!m.precond || !m.precond->factored || !m.precond->ok) {
        set_error("preconditioner not factored");
        return EFEM_ERR_ARG;
    }
    Precond& P = *m.precond;
    return apply_with(m, d_v, SolveBufs { P.d_y, P.d_t, P.d_upd, P.d_cnt });
}

efem_status precond_enqueue(Model& m, double* d_v, cudaStream_t stream, bool clear, unsigned long long* stamp)
{
    if (!m.precond || !m.precond->factored || !m.precond->ok) {
        set_error("preconditioner not factored");
        return EFEM_ERR_ARG;
    }
    Precond& P = *m.precond;
    if (P.S.n == 0) return EFEM_OK;
    return enqueue_solve(P, args_of(P), SolveBufs { P.d_y, P.d_t, P.d_upd, P.d_cnt }, d_v, stream, wait_cfg(m), clear,
        stamp);
}

efem_status precond_set_groups(Model& m, const std::vector<int>& group_of_free_node, const int* d_frozen)
{
    if (!m.precond || !m.precond->ready) {
        set_error("precond_set_groups: no solve schedule");
        return EFEM_ERR_ARG;
    }
    Precond& P = *m.precond;
    if (P.n_subs > 0) return EFEM_OK;  // subtree solves do not skip; leave the schedule as it is
    std::vector<int> g(std::max(1, P.n_items), 0);
    for (int i = 0; i < P.n_items; i++) {
        const int s = P.h_item_front[i];
        g[i] = group_of_free_node[P.S.perm[P.S.first[s]]];
    }
    dev_free(P.d_item_group);
    efem_status st = dev_upload(&P.d_item_group, g);
    if (st != EFEM_OK) return st;
    P.d_frozen = d_frozen;
    for (auto& kv : P.graphs) cudaGraphExecDestroy(kv.second);  // captured solves hold the old arguments
    P.graphs.clear();
    m.epoch++;
    return EFEM_OK;
}

bool precond_has_groups(const Model& m) { return m.precond && m.precond->d_item_group; }

void precond_counters(const Model& m, int** cnt, int* n)
{
    *cnt = m.precond ? m.precond->d_cnt : nullptr;
    *n = m.precond ? 4 * m.precond->S.ns + 2 : 0;
}

long long precond_launch_count(const Model& m)
{
    if (!m.precond) return 0;
    return (m.precond->n_items > 0 ? 1 : 0) + (m.precond->n_subs > 0 ? 2 : 0);
}

const int* precond_error_flag(const Model& m)
{
    return m.precond && m.precond->d_cnt ? m.precond->d_cnt + 4LL * m.precond->S.ns + 1 : nullptr;
}

static efem_status check_solve_flag(const int* d_flag, cudaStream_t st)
{
    int flag = 0;
    EFEM_CUDA(cudaMemcpyAsync(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    EFEM_CUDA(cudaStreamSynchronize(st));
    if (flag) {
        set_error("the triangular solve of the preconditioner gave up waiting for a front");
        return EFEM_ERR_TIMEOUT;
    }
    return EFEM_OK;
}

efem_status precond_check(Model& m)
{
    const int* f = precond_error_flag(m);
    return f ? check_solve_flag(f, m.stream) : EFEM_OK;
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
// backward sweeps as efem_precond_apply, but its working memory (the forward
// and backward intermediates, 3 per free node each, the fronts' update
// vectors, and the solve's completion counters) lives in the fixed array
// below instead of buffers owned by the model.
//
// Limits and sharing:
//   * the array holds kNoAllocDoubles doubles (16 MiB); a model that needs
//     more (6 * free nodes + its update-vector length + 2 * fronts + 1) is
//     rejected;
//   * every GPU that loads this library keeps the array until the process
//     exits;
//   * all calls share the array and it keeps the last call's contents; the
//     counters are cleared by each call and every other entry is written
//     before it is read, but calls that overlap on the GPU (other streams, other threads, other
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
    // two vectors of 3 per free node are the least any model needs: refuse
    // models that cannot fit before asking for anything else
    if (6 * static_cast<size_t>(m.n_free) > kNoAllocDoubles) {
        set_error("model needs at least " + std::to_string(6 * static_cast<size_t>(m.n_free))
            + " doubles of workspace; the static workspace of efem_precond_apply_noalloc holds "
            + std::to_string(kNoAllocDoubles));
        return EFEM_ERR_ARG;
    }
    if (!m.on_device || !m.precond || !m.precond->factored || !m.precond->ok) {
        set_error("efem_precond_apply_noalloc needs an existing positive-definite factor: call efem_solve or "
                  "efem_precond_apply once first");
        return EFEM_ERR_ARG;
    }
    Precond& P = *m.precond;
    const Symbolic& S = P.S;
    const size_t n3 = 3 * static_cast<size_t>(S.n);
    const size_t n_cnt = 4 * static_cast<size_t>(S.ns) + 2;
    const size_t need = 2 * n3 + static_cast<size_t>(S.upd_size) + (n_cnt + 1) / 2;
    if (need > kNoAllocDoubles) {
        set_error("model needs " + std::to_string(need) + " doubles of workspace; the static workspace of "
            "efem_precond_apply_noalloc holds " + std::to_string(kNoAllocDoubles));
        return EFEM_ERR_ARG;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    EFEM_CUDA(cudaStreamIsCapturing(m.stream, &cs));
    const bool capturing = cs != cudaStreamCaptureStatusNone;
    double* scratch = nullptr;
    if (capturing) {  // only a cached address: no CUDA runtime call that a capture forbids
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        scratch = m.device >= 0 && m.device < 256 ? g_noalloc_addr[m.device] : nullptr;
        if (!scratch) {
            set_error("efem_precond_apply_noalloc: the first call on a device must come before any stream "
                      "capture (it looks up the static workspace's device address)");
            return EFEM_ERR_ARG;
        }
    } else {
        efem_status st = noalloc_scratch(m.device, &scratch);
        if (st != EFEM_OK) return st;
        EFEM_CUDA(cudaSetDevice(m.device));
    }
    if (S.n == 0) return EFEM_OK;
    // This thread's host-side calls below (pointer check, flag read) must not
    // invalidate a capture that the caller has open on some other stream.
    cudaStreamCaptureMode mode = cudaStreamCaptureModeRelaxed;
    EFEM_CUDA(cudaThreadExchangeStreamCaptureMode(&mode));
    struct Restore {
        cudaStreamCaptureMode mode;
        ~Restore() { cudaThreadExchangeStreamCaptureMode(&mode); }
    } restore { mode };
    if (!capturing) {  // d_v must be memory this GPU addresses (not checked while capturing)
        cudaPointerAttributes a {};
        const bool ok = cudaPointerGetAttributes(&a, d_v) == cudaSuccess
            && (a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == m.device)
                || (a.type == cudaMemoryTypeHost && a.devicePointer != nullptr));
        if (!ok) {
            cudaGetLastError();
            set_error("d_v is not device memory of the model's GPU");
            return EFEM_ERR_ARG;
        }
    }
    int* counters = reinterpret_cast<int*>(scratch + 2 * n3 + S.upd_size);
    const SolveBufs b { scratch, scratch + n3, scratch + 2 * n3, counters };
    efem_status st = enqueue_solve(P, args_of(P), b, d_v, m.stream, wait_cfg(m));
    if (st != EFEM_OK) return st;
    EFEM_CUDA(cudaGetLastError());
    if (capturing) return EFEM_OK;  // recorded into the caller's graph; a give-up shows as NaN in d_v
    return check_solve_flag(counters + 4LL * S.ns + 1, m.stream);
}
