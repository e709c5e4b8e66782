// L-BFGS solve on the GPU: the reference's solver semantics
// (src/simulation/nlsolver/LBFGS.h:96-174, LBFGSMat.h:59-131,
// LineSearchFEA.h:37-68) with every vector operation on the device.
//
// Vector work is done by grid-stride kernels; dot products and max-norms use a
// deterministic two-level reduction (per-CTA partials, the last CTA to finish
// combines them in a fixed order), so results are bitwise repeatable.  The
// L-BFGS state -- history pointer and count, alpha_j, ys_j, theta -- lives in
// device memory and is produced and consumed by kernels only.
//
// The two-loop recursion of LBFGSMat::apply_Hv runs as four passes over the
// history instead of 2m dependent ones.  With the m x m matrix
// G[a][b] = s_a . y_b kept up to date (the new pair's row and column are
// formed in the same pass as s and y themselves), the first loop's
// alpha_i = rho_i s_i . (q0 - sum_{k newer} alpha_k y_k) needs only the dot
// products s_i . q0, and the second loop's beta_i only y_i . z0 (z0 = H0 q):
//   pass 1  s, y of the new pair; G's new row and column; s_i . q0 for all i;
//           the last CTA runs the alpha recursion (m^2 scalar operations)
//   pass 2  q = q0 - sum alpha_i y_i                  (then H0 on q -> z0)
//   pass 3  y_i . z0 for all i; the last CTA runs the beta recursion
//   pass 4  d = z0 + sum (alpha_i - beta_i) s_i, fused with the start of the
//           line search (r.d, xp = x, rp = r) and its first trial x = xp + d.
// This is the same recursion evaluated with the same vectors; only the order
// of the floating-point sums differs.
//
// Iterations run on the device.  After the first one (driven from the host),
// a CUDA graph holds the loop: a while node over iterations whose body is the
// four passes with H0, the residual at the first trial and the line-search
// reductions, then a nested while node over the further trials of the line
// search, then a one-thread kernel that applies the reference's convergence
// and iteration-limit tests and sets the loop condition.  The accept / scale
// rule of the line search is applied by a one-thread kernel as well.  Both
// loops are bounded: the line search by max_linesearch, the iterations by a
// per-launch cap, after which the host reads the state and launches the graph
// again.  Scalars the host reads are written into mapped host memory, and the
// time spent in the residual and in H0 is summed on the device from the GPU's
// global timer.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>

#include "efem_internal.h"

namespace efem {

thread_local bool t_pdl = false;

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 592;  // 4 x 148 SMs
constexpr int kMaxHist = 64;
constexpr int kRowBlocks = 128;  // CTAs per history slot in the dot-product passes (m > kMaxFast)
constexpr int kMaxFast = 8;      // history lengths with the 1D-grid passes k_pass1_m / k_pass3_m

// device-resident solver state
struct Scalars {
    double dg, rinf, xinf, x2;  // line-search reads (r.d, ||r||_inf, ||x||_inf, ||x||_2^2)
    double dg0;                 // r.d at the start of the line search
    double perr;                // the preconditioner's solve gave up waiting (nonzero)
    double theta;
    double ys[kMaxHist];
    double alpha[kMaxHist];
    double coef[kMaxHist];      // alpha - beta, per slot
    double G[kMaxHist][kMaxHist];  // G[a][b] = s_a . y_b
    int ptr, ncorr;             // LBFGSMat::m_ptr, m_ncorr
    unsigned int counter[8];
    // device-driven iterations
    double eps, step;           // residual criterion; current line-search step
    int max_iter, max_ls, cap;  // iteration limit (0: none), trials per line search, iterations per launch
    int k, launch_iters, ls_t, status;
    unsigned long long n_res, n_extra, n_body;  // residual evaluations, extra trials, device-driven iterations
    unsigned long long t0_res, t_res, t0_pc, t_pc;  // global-timer stamps and sums (ns)
    // convergence trace: record i = the state after iteration i's line search
    // (record 0: the initial residual); kTraceCols doubles per record
    double* trace;
    int trace_cap, tr_i, tr_evals;
    unsigned long long t_start;
    // mixed precision's FP32 phase: it ends when the best ||r||_inf has not
    // halved for stall_iters iterations (0: no such test)
    double best_rinf;
    int best_k, stall_iters;
};

// trace record: seconds since the solve started (GPU global timer), ||r||_2,
// ||r||_inf, the step of the trial, residual evaluations in the iteration
constexpr int kTraceCols = 5;

// host-mapped read-back slots
enum { kRdDg = 0, kRdRinf, kRdXinf, kRdX2, kRdDg0, kRdPerr, kRdStatus, kRdK, kRdNRes, kRdNExtra, kRdNBody, kRdTRes,
    kRdTPc, kRdTrN, kRdCount };
// device loop status
enum { kRunning = 0, kConverged = 1, kMaxIters = 2, kNonFinite = 3, kPrecondFail = 4, kCapReached = 5, kStalled = 6 };

__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// max that keeps a NaN (fmax drops it): a non-finite residual or solution
// must show in its infinity norm (Integrator.cpp:28-34 tests for it)
__device__ __forceinline__ double nan_max(double a, double b) { return (b > a || b != b) ? b : a; }

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nan_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block reduction of NV values, ops[k] = 0 sum / 1 max.  Result valid in thread 0.
template <int NV>
__device__ void block_reduce(double* v, const int* ops)
{
    __shared__ double sh[NV][kThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        v[k] = ops[k] ? warp_max(v[k]) : warp_sum(v[k]);
        if (lane == 0) sh[k][w] = v[k];
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            const double x = lane < kThreads / 32 ? sh[k][lane] : 0.0;
            v[k] = ops[k] ? warp_max(x) : warp_sum(x);
        }
    }
    __syncthreads();
}

// Finish a grid reduction: every CTA stores its partials; the last CTA
// combines them in CTA order.  Returns true in thread 0 of the last CTA with
// the totals in v.
template <int NV>
__device__ bool grid_finish(double* v, const int* ops, double* partials, unsigned int* counter)
{
    __shared__ bool last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) partials[blockIdx.x * NV + k] = v[k];
        __threadfence();
        const unsigned int t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) acc[k] = 0.0;
    for (int b = threadIdx.x; b < gridDim.x; b += kThreads)
#pragma unroll
        for (int k = 0; k < NV; k++) {
            const double p = *(volatile double*)&partials[b * NV + k];
            acc[k] = ops[k] ? nan_max(acc[k], p) : acc[k] + p;
        }
    block_reduce<NV>(acc, ops);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) v[k] = acc[k];
        *counter = 0u;
    }
    return threadIdx.x == 0;
}

// Rows of dot products over a 2D grid: blockIdx.y selects a row (a history
// slot), blockIdx.x strides the vector.  Each CTA stores NV partials of its
// row; the last CTA of the whole grid sums every row's partials in CTA order
// into out[row * NV + k] and returns true (all threads of that CTA).
template <int NV>
__device__ bool rows_finish(const double* v, double* partials, unsigned int* counter, double* out)
{
    __shared__ double sh[NV][kThreads / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        const double x = warp_sum(v[k]);
        if (lane == 0) sh[k][w] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const size_t base = (static_cast<size_t>(blockIdx.y) * gridDim.x + blockIdx.x) * NV;
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double x = 0.0;
            for (int q = 0; q < kThreads / 32; q++) x += sh[k][q];
            partials[base + k] = x;
        }
        __threadfence();
        const unsigned int t = atomicAdd(counter, 1u);
        last = (t == gridDim.x * gridDim.y - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    // one warp per (row, value): lanes over the CTAs of the row, then a fixed-order shuffle
    const int nsum = gridDim.y * NV;
    for (int q = w; q < nsum; q += kThreads / 32) {
        const int row = q / NV, k = q - row * NV;
        double x = 0.0;
        for (int b = lane; b < static_cast<int>(gridDim.x); b += 32)
            x += *(volatile double*)&partials[(static_cast<size_t>(row) * gridDim.x + b) * NV + k];
        x = warp_sum(x);
        if (lane == 0) out[q] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

#define GRID_STRIDE(i, n) for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

__global__ void k_state_init(Scalars* S, int m)
{
    S->ptr = m;  // makes ptr % m == 0 on the first correction (LBFGSMat.h:68)
    S->ncorr = 0;
    S->theta = 1.0;
}

// x = xp + step d (a host-driven trial; the step is kept for the trace)
__global__ void k_trial(double* __restrict__ x, const double* __restrict__ xp, const double* __restrict__ d, double step,
    size_t n, Scalars* S)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) S->step = step;
    GRID_STRIDE(i, n) x[i] = __fma_rn(step, d[i], xp[i]);
}

// line-search scalars: dg = r.d, rinf = ||r||_inf, xinf = ||x||_inf, x2 = ||x||^2,
// stored in S and in the host-mapped read-back array; with a trace buffer the
// trial also (over)writes the current iteration's record, so the record left
// is the accepted trial's
// With `decide` (inside the device-driven line search) the last CTA also
// applies the accept / scale rule of LineSearchFEA.h:43-67: accept when
// |r.d| <= |r0.d|; otherwise scale the step by 1.5 (same sign) or 0.5 and try
// again, at most max_ls trials in all; it sets the line-search loop condition.
__global__ void __launch_bounds__(kThreads) k_ls_reduce(const double* __restrict__ r, const double* __restrict__ d,
    const double* __restrict__ x, size_t n, Scalars* S, double* partials, const int* perr, double* hread,
    cudaGraphConditionalHandle h, int decide)
{
    griddep_wait();
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        S->t_res += gtimer() - S->t0_res;  // the residual just ended
        // the loop stops unless the last CTA below decides on another trial
        if (decide) cudaGraphSetConditional(h, 0u);
    }
    double v[5] = { 0, 0, 0, 0, 0 };
    const int ops[5] = { 0, 1, 1, 0, 0 };
    GRID_STRIDE(i, n)
    {
        const double ri = r[i], xi = x[i];
        v[0] += ri * d[i];
        v[1] = nan_max(v[1], fabs(ri));
        v[2] = nan_max(v[2], fabs(xi));
        v[3] += xi * xi;
        v[4] += ri * ri;
    }
    griddep_launch();
    block_reduce<5>(v, ops);
    if (grid_finish<5>(v, ops, partials, &S->counter[0])) {
        S->dg = v[0];
        S->rinf = v[1];
        S->xinf = v[2];
        S->x2 = v[3];
        S->perr = perr ? static_cast<double>(*perr) : 0.0;
        S->n_res++;
        S->tr_evals++;
        if (S->trace && S->tr_i < S->trace_cap) {
            double* rec = S->trace + static_cast<size_t>(S->tr_i) * kTraceCols;
            rec[0] = static_cast<double>(gtimer() - S->t_start) * 1e-9;
            rec[1] = sqrt(v[4]);
            rec[2] = v[1];
            rec[3] = S->step;
            rec[4] = static_cast<double>(S->tr_evals);
        }
        hread[kRdTrN] = static_cast<double>(S->tr_i + 1);
        hread[kRdDg] = S->dg;
        hread[kRdRinf] = S->rinf;
        hread[kRdXinf] = S->xinf;
        hread[kRdX2] = S->x2;
        hread[kRdDg0] = S->dg0;
        hread[kRdPerr] = S->perr;
        hread[kRdNRes] = static_cast<double>(S->n_res);
        hread[kRdTRes] = static_cast<double>(S->t_res);
        hread[kRdTPc] = static_cast<double>(S->t_pc);
        if (decide) {
            const int t = ++S->ls_t;
            const double dg = S->dg, dg0 = S->dg0;
            const bool again = !(fabs(dg) <= fabs(dg0)) && t < S->max_ls;
            if (again) {
                S->step *= dg * dg0 > 0 ? 1.5 : 0.5;
                S->n_extra++;
            }
            cudaGraphSetConditional(h, again ? 1u : 0u);
        }
    }
}

// start of the line search fused with its first trial (step 1):
// dg0 = r.d, xp = x, rp = r, x = x + d
__global__ void __launch_bounds__(kThreads) k_ls_begin_trial(const double* __restrict__ r, const double* __restrict__ d,
    double* __restrict__ x, double* __restrict__ xp, double* __restrict__ rp, size_t n, Scalars* S, double* partials)
{
    double v[1] = { 0 };
    const int ops[1] = { 0 };
    GRID_STRIDE(i, n)
    {
        const double ri = r[i], di = d[i], xi = x[i];
        v[0] += ri * di;
        xp[i] = xi;
        rp[i] = ri;
        x[i] = xi + 1.0 * di;
    }
    block_reduce<1>(v, ops);
    if (grid_finish<1>(v, ops, partials, &S->counter[1])) {
        S->dg0 = v[0];
        S->step = 1.0;
        S->tr_i++;  // iteration 1's trace record
        S->tr_evals = 0;
    }
}

// Pass 1 (LBFGSMat::add_correction, LBFGSMat.h:81-98, and the dot products of
// the first loop).  Grid (kRowBlocks, m + 1): row j < m forms s.Y_j, S_j.y and
// S_j.q0 (q0 = -r) for history slot j, with the new pair standing in for the
// slot it replaces; row m writes the new pair and forms s.y and y.y.  The
// last CTA updates G, ys, theta, the pointer and count, and runs the first
// loop's recursion (newest pair first).
__global__ void __launch_bounds__(kThreads) k_pass1(const double* __restrict__ x, const double* __restrict__ xp,
    const double* __restrict__ r, const double* __restrict__ rp, double* __restrict__ Sh, double* __restrict__ Yh,
    size_t n, int m, Scalars* S, double* partials, double* sums)
{
    griddep_wait();
    const int loc = S->ptr % m;
    const int ncorr = S->ncorr < m ? S->ncorr + 1 : m;  // count after the insertion; slots 0..ncorr-1 hold pairs
    const int row = blockIdx.y;
    double v[3] = { 0, 0, 0 };
    if (row == m) {
        double* s = Sh + loc * n;
        double* y = Yh + loc * n;
        for (size_t i = blockIdx.x * (size_t)kThreads + threadIdx.x; i < n; i += (size_t)gridDim.x * kThreads) {
            const double si = x[i] - xp[i], yi = r[i] - rp[i];
            s[i] = si;
            y[i] = yi;
            v[0] += si * yi;
            v[1] += yi * yi;
        }
    } else if (row < ncorr) {
        const double* sj = Sh + row * n;
        const double* yj = Yh + row * n;
        const bool self = row == loc;
        for (size_t i = blockIdx.x * (size_t)kThreads + threadIdx.x; i < n; i += (size_t)gridDim.x * kThreads) {
            const double si = x[i] - xp[i], yi = r[i] - rp[i];
            const double sji = self ? si : sj[i], yji = self ? yi : yj[i];
            v[0] += si * yji;      // s_new . y_j
            v[1] += sji * yi;      // s_j . y_new
            v[2] -= sji * r[i];    // s_j . q0
        }
    }
    if (!rows_finish<3>(v, partials, &S->counter[2], sums)) return;
    // last CTA: the small recursion runs on copies in shared memory (m x m G, ys, alpha)
    extern __shared__ double dyn[];
    double* sG = dyn;
    double* sys = dyn + m * m;
    double* sal = sys + m;
    const int tid = threadIdx.x;
    for (int q = tid; q < m * m; q += kThreads) sG[q] = S->G[q / m][q % m];
    for (int j = tid; j < m; j += kThreads) sys[j] = S->ys[j];
    __syncthreads();
    const double ys = sums[3 * m], yy = sums[3 * m + 1];
    for (int j = tid; j < ncorr; j += kThreads) {
        sG[loc * m + j] = sums[3 * j];
        sG[j * m + loc] = sums[3 * j + 1];
    }
    __syncthreads();
    if (tid == 0) {
        sG[loc * m + loc] = ys;
        sys[loc] = ys;
        // first loop (LBFGSMat.h:106-113): newest slot first
        for (int i = 0; i < ncorr; i++) {
            const int j = ((loc - i) % m + m) % m;
            double t = sums[3 * j + 2];
            for (int k = 0; k < i; k++) {
                const int jk = ((loc - k) % m + m) % m;
                t -= sal[jk] * sG[j * m + jk];
            }
            sal[j] = t / sys[j];
        }
        S->theta = yy / ys;
        S->ptr = loc + 1;
        S->ncorr = ncorr;
        S->ys[loc] = ys;
    }
    __syncthreads();
    for (int j = tid; j < ncorr; j += kThreads) {
        S->G[loc][j] = sG[loc * m + j];
        S->G[j][loc] = sG[j * m + loc];
        S->alpha[j] = sal[j];
    }
}

// Sums of NV values over a 1D grid in a fixed order: every CTA stores its
// block sums; the last CTA to finish adds them up -- each thread the CTAs
// b = t, t + kThreads, ... for all NV values at once (independent loads, a
// couple of round trips), then a block reduction -- into out[0, NV).
// Returns true in every thread of the last CTA.
template <int NV>
__device__ bool grid_sums(double* v, double* partials, unsigned int* counter, double* out)
{
    __shared__ bool last;
    int ops[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) ops[k] = 0;
    block_reduce<NV>(v, ops);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) partials[blockIdx.x * NV + k] = v[k];
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) acc[k] = 0.0;
    for (int b = threadIdx.x; b < static_cast<int>(gridDim.x); b += kThreads) {
        const volatile double* pb = partials + static_cast<size_t>(b) * NV;
        double p[NV];
#pragma unroll
        for (int k = 0; k < NV; k++) p[k] = pb[k];
#pragma unroll
        for (int k = 0; k < NV; k++) acc[k] += p[k];
    }
    block_reduce<NV>(acc, ops);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) out[k] = acc[k];
        *counter = 0u;
    }
    __syncthreads();
    return true;
}

// Pass 1 for a history of M <= 8 pairs on a 1D grid: each thread reads x, xp,
// r, rp once for all slots (the 2D k_pass1 re-reads them per slot) and keeps
// the 3M + 2 dot products in registers; the last CTA runs the same recursion.
template <int M>
__global__ void __launch_bounds__(kThreads) k_pass1_m(const double* __restrict__ x, const double* __restrict__ xp,
    const double* __restrict__ r, const double* __restrict__ rp, double* __restrict__ Sh, double* __restrict__ Yh,
    size_t n, Scalars* S, double* partials)
{
    griddep_wait();
    constexpr int NV = 3 * M + 2;
    const int m = M;
    const int loc = S->ptr % m;
    const int ncorr = S->ncorr < m ? S->ncorr + 1 : m;
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = 0.0;
    double* snew = Sh + loc * n;
    double* ynew = Yh + loc * n;
    GRID_STRIDE(i, n)
    {
        const double si = x[i] - xp[i], ri = r[i], yi = ri - rp[i];
        snew[i] = si;
        ynew[i] = yi;
        v[3 * M] += si * yi;
        v[3 * M + 1] += yi * yi;
#pragma unroll
        for (int j = 0; j < M; j++) {
            if (j < ncorr) {
                const bool self = j == loc;
                const double sj = self ? si : Sh[j * n + i], yj = self ? yi : Yh[j * n + i];
                v[3 * j] += si * yj;      // s_new . y_j
                v[3 * j + 1] += sj * yi;  // s_j . y_new
                v[3 * j + 2] -= sj * ri;  // s_j . q0
            }
        }
    }
    griddep_launch();
    __shared__ double tot[NV];
    if (!grid_sums<NV>(v, partials, &S->counter[2], tot)) return;
    extern __shared__ double dyn[];
    double* sG = dyn;
    double* sys = dyn + m * m;
    double* sal = sys + m;
    const int tid = threadIdx.x;
    for (int q = tid; q < m * m; q += kThreads) sG[q] = S->G[q / m][q % m];
    for (int j = tid; j < m; j += kThreads) sys[j] = S->ys[j];
    __syncthreads();
    const double ys = tot[3 * M], yy = tot[3 * M + 1];
    for (int j = tid; j < ncorr; j += kThreads) {
        sG[loc * m + j] = tot[3 * j];
        sG[j * m + loc] = tot[3 * j + 1];
    }
    __syncthreads();
    if (tid == 0) {
        sG[loc * m + loc] = ys;
        sys[loc] = ys;
        for (int i = 0; i < ncorr; i++) {  // first loop (LBFGSMat.h:106-113): newest slot first
            const int j = ((loc - i) % m + m) % m;
            double t = tot[3 * j + 2];
            for (int k = 0; k < i; k++) {
                const int jk = ((loc - k) % m + m) % m;
                t -= sal[jk] * sG[j * m + jk];
            }
            sal[j] = t / sys[j];
        }
        S->theta = yy / ys;
        S->ptr = loc + 1;
        S->ncorr = ncorr;
        S->ys[loc] = ys;
    }
    __syncthreads();
    for (int j = tid; j < ncorr; j += kThreads) {
        S->G[loc][j] = sG[loc * m + j];
        S->G[j][loc] = sG[j * m + loc];
        S->alpha[j] = sal[j];
    }
}

// Pass 3 for M <= 8 on a 1D grid: z read once for all slots
template <int M>
__global__ void __launch_bounds__(kThreads) k_pass3_m(const double* __restrict__ z, const double* __restrict__ Yh,
    size_t n, Scalars* S, double* partials, int time_pc)
{
    griddep_wait();
    const int m = M, ncorr = S->ncorr;
    if (blockIdx.x == 0 && threadIdx.x == 0 && time_pc) S->t_pc += gtimer() - S->t0_pc;  // H0 just ended
    double v[M];
#pragma unroll
    for (int k = 0; k < M; k++) v[k] = 0.0;
    GRID_STRIDE(i, n)
    {
        const double zi = z[i];
#pragma unroll
        for (int j = 0; j < M; j++)
            if (j < ncorr) v[j] += Yh[j * n + i] * zi;
    }
    griddep_launch();
    __shared__ double tot[M];
    if (!grid_sums<M>(v, partials, &S->counter[3], tot)) return;
    extern __shared__ double dyn[];
    double* sG = dyn;
    double* sys = dyn + m * m;
    double* sal = sys + m;
    double* scf = sal + m;
    const int tid = threadIdx.x;
    for (int q = tid; q < m * m; q += kThreads) sG[q] = S->G[q / m][q % m];
    for (int j = tid; j < m; j += kThreads) {
        sys[j] = S->ys[j];
        sal[j] = S->alpha[j];
    }
    __syncthreads();
    if (tid == 0) {  // second loop (LBFGSMat.h:121-128), oldest pair first
        const int ptr = S->ptr;
        for (int o = 0; o < ncorr; o++) {
            const int j = ((ptr - ncorr + o) % m + m) % m;
            double t = tot[j];
            for (int p = 0; p < o; p++) {
                const int jp = ((ptr - ncorr + p) % m + m) % m;
                t += scf[jp] * sG[jp * m + j];
            }
            scf[j] = sal[j] - t / sys[j];
        }
    }
    __syncthreads();
    for (int j = tid; j < ncorr; j += kThreads) S->coef[j] = scf[j];
}

// Pass 2: q = (q0 - sum_j alpha_j y_j) [/ theta when H0 = I / theta]; also
// clears the preconditioner solve's counters for the H0 application that follows
__global__ void __launch_bounds__(kThreads) k_pass2(double* __restrict__ q, const double* __restrict__ r,
    const double* __restrict__ Yh, size_t n, int m, int divide_theta, const Scalars* S, int* clear, int n_clear)
{
    griddep_wait();
    __shared__ double al[kMaxHist];
    const int ncorr = S->ncorr;
    for (int j = threadIdx.x; j < ncorr; j += kThreads) al[j] = S->alpha[j];
    __syncthreads();
    const double th = S->theta;
    GRID_STRIDE(i, n)
    {
        double qi = -r[i];
        for (int j = 0; j < ncorr; j++) qi -= al[j] * Yh[j * n + i];
        q[i] = divide_theta ? qi / th : qi;
    }
    griddep_launch();
    if (clear)
        for (int k = blockIdx.x * kThreads + threadIdx.x; k < n_clear; k += gridDim.x * kThreads) clear[k] = 0;
}

// Pass 3: y_j . z0 for every slot (grid (kRowBlocks, m)); the last CTA runs
// the second loop's recursion (LBFGSMat.h:121-128), oldest pair first
__global__ void __launch_bounds__(kThreads) k_pass3(const double* __restrict__ z, const double* __restrict__ Yh, size_t n,
    int m, Scalars* S, double* partials, double* sums, int time_pc)
{
    griddep_wait();
    const int ncorr = S->ncorr, row = blockIdx.y;
    if (blockIdx.x == 0 && row == 0 && threadIdx.x == 0 && time_pc) S->t_pc += gtimer() - S->t0_pc;  // H0 just ended
    double v[1] = { 0 };
    if (row < ncorr) {
        const double* yj = Yh + row * n;
        for (size_t i = blockIdx.x * (size_t)kThreads + threadIdx.x; i < n; i += (size_t)gridDim.x * kThreads)
            v[0] += yj[i] * z[i];
    }
    if (!rows_finish<1>(v, partials, &S->counter[3], sums)) return;
    // last CTA: the recursion on shared-memory copies of G, ys, alpha
    extern __shared__ double dyn[];
    double* sG = dyn;
    double* sys = dyn + m * m;
    double* sal = sys + m;
    double* scf = sal + m;
    const int tid = threadIdx.x;
    for (int q = tid; q < m * m; q += kThreads) sG[q] = S->G[q / m][q % m];
    for (int j = tid; j < m; j += kThreads) {
        sys[j] = S->ys[j];
        sal[j] = S->alpha[j];
    }
    __syncthreads();
    if (tid == 0) {
        const int ptr = S->ptr;
        for (int o = 0; o < ncorr; o++) {
            const int j = ((ptr - ncorr + o) % m + m) % m;
            double t = sums[j];
            for (int p = 0; p < o; p++) {
                const int jp = ((ptr - ncorr + p) % m + m) % m;
                t += scf[jp] * sG[jp * m + j];
            }
            scf[j] = sal[j] - t / sys[j];
        }
    }
    __syncthreads();
    for (int j = tid; j < ncorr; j += kThreads) S->coef[j] = scf[j];
}

// Pass 4: d = z0 + sum_j coef_j s_j, the start of the line search (r.d,
// xp = x, rp = r, step 1) and its first trial: x = xp + 1 d, r = -f_ext for
// the residual that follows (whose start time is stamped by the last CTA)
__global__ void __launch_bounds__(kThreads) k_pass4(double* __restrict__ d, const double* __restrict__ z,
    const double* __restrict__ Sh, double* __restrict__ r, double* __restrict__ x, double* __restrict__ xp,
    double* __restrict__ rp, const double* __restrict__ fext, size_t n, Scalars* S, double* partials)
{
    griddep_wait();
    __shared__ double cf[kMaxHist];
    const int ncorr = S->ncorr;
    for (int j = threadIdx.x; j < ncorr; j += kThreads) cf[j] = S->coef[j];
    __syncthreads();
    double v[1] = { 0 };
    const int ops[1] = { 0 };
    GRID_STRIDE(i, n)
    {
        double di = z[i];
        for (int j = 0; j < ncorr; j++) di += cf[j] * Sh[j * n + i];
        d[i] = di;
        const double ri = r[i], xi = x[i];
        v[0] += ri * di;
        xp[i] = xi;
        rp[i] = ri;
        x[i] = xi + 1.0 * di;
        r[i] = -fext[i];
    }
    griddep_launch();
    block_reduce<1>(v, ops);
    if (grid_finish<1>(v, ops, partials, &S->counter[1])) {
        S->dg0 = v[0];
        S->step = 1.0;
        S->ls_t = 0;
        S->tr_i++;  // the next iteration's trace record
        S->tr_evals = 0;
        S->t0_res = gtimer();
    }
}

__global__ void k_neg_copy(double* __restrict__ q, const double* __restrict__ r, size_t n)
{
    GRID_STRIDE(i, n) q[i] = -r[i];
}

// a trial of the device-driven line search: x = xp + step d with the step
// held on the device, and r = -f_ext to start the residual at x (its start
// time is stamped for the residual's timing)
__global__ void k_trial_dev(double* __restrict__ x, const double* __restrict__ xp, const double* __restrict__ d,
    double* __restrict__ r, const double* __restrict__ fext, size_t n, Scalars* S)
{
    griddep_wait();
    if (blockIdx.x == 0 && threadIdx.x == 0) S->t0_res = gtimer();
    const double step = S->step;
    GRID_STRIDE(i, n)
    {
        x[i] = __fma_rn(step, d[i], xp[i]);
        r[i] = -fext[i];
    }
}

// End of an iteration (LBFGS.h:150-170): stop on a non-finite residual or
// solution, on convergence (||r||_inf <= eps or <= eps ||x||_inf) or at the
// iteration limit; otherwise count the iteration and go on, up to `cap`
// iterations per launch.  Sets the iteration loop condition.
__global__ void k_iter_decide(Scalars* S, cudaGraphConditionalHandle h, double* hread)
{
    griddep_wait();
    if (threadIdx.x != 0) return;
    const double rinf = S->rinf, xinf = S->xinf;
    int st = kRunning;
    S->n_body++;
    if (S->perr != 0.0)
        st = kPrecondFail;
    else if (!isfinite(rinf) || !isfinite(xinf))
        st = kNonFinite;
    else if (rinf <= S->eps || rinf <= S->eps * xinf)
        st = kConverged;
    else if (S->max_iter != 0 && S->k >= S->max_iter)
        st = kMaxIters;
    else if (S->stall_iters > 0 && !(rinf < 0.5 * S->best_rinf) && S->k - S->best_k >= S->stall_iters)
        st = kStalled;
    else {
        if (rinf < 0.5 * S->best_rinf) {
            S->best_rinf = rinf;
            S->best_k = S->k;
        }
        S->k++;
        if (++S->launch_iters >= S->cap) st = kCapReached;
    }
    S->status = st;
    hread[kRdStatus] = st;
    hread[kRdK] = S->k;
    hread[kRdNExtra] = static_cast<double>(S->n_extra);
    hread[kRdNBody] = static_cast<double>(S->n_body);
    hread[kRdTPc] = static_cast<double>(S->t_pc);
    cudaGraphSetConditional(h, st == kRunning ? 1u : 0u);
}

__global__ void k_loop_start(Scalars* S) { S->launch_iters = 0; }

// options of the device-driven loop, and the iteration number it starts at
__global__ void k_loop_params(Scalars* S, double eps, int max_iter, int max_ls, int cap, int k, int stall_iters,
    double best_rinf)
{
    S->stall_iters = stall_iters;
    S->best_rinf = best_rinf;
    S->best_k = k;
    S->eps = eps;
    S->max_iter = max_iter;
    S->max_ls = max_ls;
    S->cap = cap;
    S->k = k;
    S->n_extra = 0;
    S->n_body = 0;
    S->t_pc = 0;
}

// counters, timers and trace of one solve (the initial residual is trace record 0, step 0);
// keep_trace: a second phase of the same solve, whose records follow the first phase's
__global__ void k_solve_init(Scalars* S, double* trace, int trace_cap, int keep_trace)
{
    S->n_res = 0;
    S->t_res = 0;
    S->t_pc = 0;
    S->n_extra = 0;
    S->n_body = 0;
    S->trace = trace;
    S->trace_cap = trace ? trace_cap : 0;
    S->step = 0.0;
    if (!keep_trace) {
        S->tr_i = 0;
        S->tr_evals = 0;
        S->t_start = gtimer();
    }
}

// vector kernels are latency-bound at these sizes: about one element per thread
int grid_for(size_t n) { return static_cast<int>(std::min<size_t>(kMaxBlocks, std::max<size_t>(1, (n + kThreads - 1) / kThreads))); }
int row_blocks(size_t n) { return static_cast<int>(std::min<size_t>(kRowBlocks, std::max<size_t>(1, (n + 2 * kThreads - 1) / (2 * kThreads)))); }

}  // namespace

struct SolverWS {
    size_t n = 0;
    int m = 0;
    bool pdl = true;  // programmatic dependent launch in the captured iteration graphs (off if a capture refused it)
    double *r = nullptr, *xp = nullptr, *rp = nullptr, *d = nullptr, *q = nullptr;
    double *S = nullptr, *Y = nullptr;
    double* partials = nullptr;
    double* sums = nullptr;
    Scalars* sc = nullptr;
    double* h_read = nullptr;  // mapped pinned memory: kRdCount scalars written by the device
    double* trace = nullptr;   // [trace_cap][kTraceCols] convergence trace of the last solve
    int trace_cap = 0;
    int trace_n = 0;           // records the last solve produced (may exceed trace_cap)
    cudaEvent_t ev[4] = { nullptr, nullptr, nullptr, nullptr };  // solve start / end, initial H0 start / end
    cudaStream_t capture[3] = { nullptr, nullptr, nullptr };      // outer graph, loop body, line-search body
    struct Graphs {
        cudaGraphExec_t first = nullptr;  // iteration 1: line-search start + first trial
        cudaGraphExec_t loop = nullptr;   // iterations 2, 3, ... (device-driven)
        cudaGraphExec_t step = nullptr;   // one iteration (host-driven loop)
    };
    std::map<std::pair<double*, int>, Graphs> graphs;  // per (solution pointer, configuration)
    long long epoch = -1;                                // Model::epoch the graphs were captured at
};

__global__ void k_neg(double* __restrict__ r, const double* __restrict__ f, size_t n, unsigned long long* stamp)
{
    if (stamp && blockIdx.x == 0 && threadIdx.x == 0) *stamp = gtimer();
    GRID_STRIDE(i, n) r[i] = -f[i];
}

void launch_neg(double* r, const double* f, size_t n, cudaStream_t st, unsigned long long* stamp)
{
    k_neg<<<grid_for(n), kThreads, 0, st>>>(r, f, n, stamp);
}

static void drop_graphs(SolverWS& w)
{
    for (auto& kv : w.graphs) {
        if (kv.second.first) cudaGraphExecDestroy(kv.second.first);
        if (kv.second.loop) cudaGraphExecDestroy(kv.second.loop);
        if (kv.second.step) cudaGraphExecDestroy(kv.second.step);
    }
    w.graphs.clear();
}

void free_solver(Model& m)
{
    if (!m.ws) return;
    SolverWS& w = *m.ws;
    drop_graphs(w);
    dev_free(w.r);
    dev_free(w.xp);
    dev_free(w.rp);
    dev_free(w.d);
    dev_free(w.q);
    dev_free(w.S);
    dev_free(w.Y);
    dev_free(w.partials);
    dev_free(w.sums);
    dev_free(w.trace);
    if (w.sc) cudaFree(w.sc);
    if (w.h_read) cudaFreeHost(w.h_read);
    for (auto& e : w.ev)
        if (e) cudaEventDestroy(e);
    for (auto& c : w.capture)
        if (c) cudaStreamDestroy(c);
    delete m.ws;
    m.ws = nullptr;
}

static efem_status alloc_ws(Model& m)
{
    const size_t n = 3 * static_cast<size_t>(m.n_free);
    if (m.ws && m.ws->n == n && m.ws->m == m.opts.m) return EFEM_OK;
    free_solver(m);
    if (m.opts.m > kMaxHist) {
        set_error("history length m is limited to 64");
        return EFEM_ERR_ARG;
    }
    m.ws = new SolverWS();
    SolverWS& w = *m.ws;
    w.n = n;
    w.m = m.opts.m;
    efem_status s;
    for (double** p : { &w.r, &w.xp, &w.rp, &w.d, &w.q })
        if ((s = dev_alloc(p, n)) != EFEM_OK) return s;
    if ((s = dev_alloc(&w.S, n * w.m)) != EFEM_OK) return s;
    if ((s = dev_alloc(&w.Y, n * w.m)) != EFEM_OK) return s;
    const size_t np = std::max<size_t>(static_cast<size_t>(kMaxBlocks) * (3 * kMaxFast + 2),
        static_cast<size_t>(kRowBlocks) * (w.m + 1) * 3);
    if ((s = dev_alloc(&w.partials, np)) != EFEM_OK) return s;
    if ((s = dev_alloc(&w.sums, 3 * static_cast<size_t>(w.m + 1))) != EFEM_OK) return s;
    EFEM_CUDA(cudaMalloc(&w.sc, sizeof(Scalars)));
    EFEM_CUDA(cudaMemset(w.sc, 0, sizeof(Scalars)));
    EFEM_CUDA(cudaHostAlloc(&w.h_read, sizeof(double) * kRdCount, cudaHostAllocMapped));
    std::memset(w.h_read, 0, sizeof(double) * kRdCount);
    for (auto& e : w.ev) EFEM_CUDA(cudaEventCreate(&e));
    for (auto& c : w.capture) EFEM_CUDA(cudaStreamCreateWithFlags(&c, cudaStreamNonBlocking));
    return EFEM_OK;
}

namespace {

constexpr int kIterCap = 32;  // device-driven iterations per graph launch

double* mapped(double* h)
{
    void* d = nullptr;
    return cudaHostGetDevicePointer(&d, h, 0) == cudaSuccess ? static_cast<double*>(d) : h;
}

// the residual at the current trial x and the line-search reductions; inside
// the device-driven line search (h_ls given) r was started by k_pass4 or k_trial_dev and
// the reduction applies the accept / scale rule
efem_status enqueue_trial_tail(Model& m, SolverWS& w, double* x, cudaStream_t st,
    const cudaGraphConditionalHandle* h_ls = nullptr, bool init_r = true)
{
    const size_t n = w.n;
    efem_status s = launch_residual_on(m, x, w.r, st, &w.sc->t0_res, init_r);
    if (s != EFEM_OK) return s;
    launch_k(k_ls_reduce, grid_for(n), kThreads, 0, st, w.r, w.d, x, n, w.sc, w.partials, precond_error_flag(m),
        mapped(w.h_read), h_ls ? *h_ls : cudaGraphConditionalHandle(), h_ls ? 1 : 0);
    return EFEM_OK;
}

// iteration 1: line-search start and first trial along the initial direction
efem_status enqueue_first(Model& m, SolverWS& w, double* x, cudaStream_t st)
{
    k_ls_begin_trial<<<grid_for(w.n), kThreads, 0, st>>>(w.r, w.d, x, w.xp, w.rp, w.n, w.sc, w.partials);
    return enqueue_trial_tail(m, w, x, st);
}

// add_correction + two-loop with H0 + line-search start
efem_status enqueue_body(Model& m, SolverWS& w, double* x, bool use_factor, cudaStream_t st)
{
    const size_t n = w.n;
    const int mm = w.m;
    const dim3 g1(row_blocks(n), mm + 1), g3(row_blocks(n), mm);
    const size_t sm1 = sizeof(double) * (mm * mm + 2 * mm), sm3 = sizeof(double) * (mm * mm + 3 * mm);
    const int G = grid_for(n);
    switch (mm) {
#define P1(M) case M: k_pass1_m<M><<<G, kThreads, sm1, st>>>(x, w.xp, w.r, w.rp, w.S, w.Y, n, w.sc, w.partials); break;
        P1(1) P1(2) P1(3) P1(4) P1(5) P1(6) P1(7) P1(8)
#undef P1
    default: k_pass1<<<g1, kThreads, sm1, st>>>(x, w.xp, w.r, w.rp, w.S, w.Y, n, mm, w.sc, w.partials, w.sums);
    }
    int* clear = nullptr;
    int n_clear = 0;
    if (use_factor) precond_counters(m, &clear, &n_clear);
    launch_k(k_pass2, grid_for(n), kThreads, 0, st, w.q, w.r, w.Y, n, mm, use_factor ? 0 : 1, w.sc, clear, n_clear);
    if (use_factor) {
        efem_status s = precond_enqueue(m, w.q, st, false, &w.sc->t0_pc);
        if (s != EFEM_OK) return s;
    }
    switch (mm) {
#define P3(M) case M: launch_k(k_pass3_m<M>, G, kThreads, sm3, st, w.q, w.Y, n, w.sc, w.partials, use_factor ? 1 : 0); break;
        P3(1) P3(2) P3(3) P3(4) P3(5) P3(6) P3(7) P3(8)
#undef P3
    default: launch_k(k_pass3, g3, kThreads, sm3, st, w.q, w.Y, n, mm, w.sc, w.partials, w.sums, use_factor ? 1 : 0);
    }
    launch_k(k_pass4, grid_for(n), kThreads, 0, st, w.d, w.q, w.S, w.r, x, w.xp, w.rp, m.d_fext, n, w.sc, w.partials);
    return EFEM_OK;
}

efem_status instantiate(cudaGraph_t g, cudaGraphExec_t* out)
{
    const cudaError_t e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        set_error(std::string("graph instantiation: ") + cudaGetErrorString(e));
        return EFEM_ERR_CUDA;
    }
    return EFEM_OK;
}

// a while node appended to the work captured so far on `st`; returns its body graph
efem_status add_while(cudaStream_t st, cudaGraphConditionalHandle h, cudaGraph_t* body)
{
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    EFEM_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    EFEM_CUDA(cudaGraphAddNode(&node, g, deps, nd, &p));
    EFEM_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    *body = p.conditional.phGraph_out[0];
    return EFEM_OK;
}

// The device-driven iteration loop:
//   k_loop_start;
//   while (hIter) { passes + H0 + first trial; residual; reductions + decision (sets hLs);
//                   while (hLs) { trial; residual; reductions + decision }; k_iter_decide }
// launch_k uses programmatic dependent launch while one of these is alive
struct PdlScope {
    explicit PdlScope(bool on) { t_pdl = on; }
    ~PdlScope() { t_pdl = false; }
};

efem_status capture_loop(Model& m, SolverWS& w, double* x, bool use_factor, cudaGraphExec_t* out)
{
    std::lock_guard<std::mutex> lock(capture_mutex());
    PdlScope pdl(w.pdl);  // the first kernel of each body graph is a plain launch
    const long long launches = m.launches;  // capture launches nothing; replays are counted
    cudaStream_t s0 = w.capture[0], s1 = w.capture[1], s2 = w.capture[2];
    cudaGraph_t g = nullptr;
    efem_status s = EFEM_OK;
    EFEM_CUDA(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
    do {
        cudaGraph_t outer = nullptr;
        cudaStreamCaptureStatus cs;
        if (cudaStreamGetCaptureInfo(s0, &cs, nullptr, &outer, nullptr, nullptr) != cudaSuccess) {
            s = EFEM_ERR_CUDA;
            break;
        }
        cudaGraphConditionalHandle h_iter, h_ls;
        if (cudaGraphConditionalHandleCreate(&h_iter, outer, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
            s = EFEM_ERR_CUDA;
            break;
        }
        k_loop_start<<<1, 1, 0, s0>>>(w.sc);
        cudaGraph_t body = nullptr, ls_body = nullptr;
        if ((s = add_while(s0, h_iter, &body)) != EFEM_OK) break;
        if (cudaGraphConditionalHandleCreate(&h_ls, body, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
            s = EFEM_ERR_CUDA;
            break;
        }
        if (cudaStreamBeginCaptureToGraph(s1, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            s = EFEM_ERR_CUDA;
            break;
        }
        // passes, H0 and the first trial (pass 4), its residual and the line
        // search's decision, which sets hLs; then the further trials
        s = enqueue_body(m, w, x, use_factor, s1);
        if (s == EFEM_OK) s = enqueue_trial_tail(m, w, x, s1, &h_ls, false);
        if (s == EFEM_OK) s = add_while(s1, h_ls, &ls_body);
        if (s == EFEM_OK && cudaStreamBeginCaptureToGraph(s2, ls_body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            s = EFEM_ERR_CUDA;
        if (s == EFEM_OK) {
            k_trial_dev<<<grid_for(w.n), kThreads, 0, s2>>>(x, w.xp, w.d, w.r, m.d_fext, w.n, w.sc);
            s = enqueue_trial_tail(m, w, x, s2, &h_ls, false);
            cudaGraph_t tmp = nullptr;
            if (cudaStreamEndCapture(s2, &tmp) != cudaSuccess && s == EFEM_OK) s = EFEM_ERR_CUDA;
        }
        if (s == EFEM_OK) k_iter_decide<<<1, 32, 0, s1>>>(w.sc, h_iter, mapped(w.h_read));
        cudaGraph_t tmp = nullptr;
        if (cudaStreamEndCapture(s1, &tmp) != cudaSuccess && s == EFEM_OK) s = EFEM_ERR_CUDA;
    } while (false);
    const cudaError_t e = cudaStreamEndCapture(s0, &g);
    m.launches = launches;
    if (s != EFEM_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        if (s == EFEM_ERR_CUDA || e != cudaSuccess) set_error(std::string("capture of the iteration loop: ") +
            cudaGetErrorString(e != cudaSuccess ? e : cudaGetLastError()));
        return s != EFEM_OK ? s : EFEM_ERR_CUDA;
    }
    return instantiate(g, out);
}

// One iteration for the host-driven loop: the passes with H0 and the line
// search's first trial with its residual and reductions; the host applies the
// accept / scale rule and the convergence tests.
efem_status capture_step(Model& m, SolverWS& w, double* x, bool use_factor, cudaGraphExec_t* out)
{
    std::lock_guard<std::mutex> lock(capture_mutex());
    PdlScope pdl(w.pdl);
    const long long launches = m.launches;
    cudaStream_t s0 = w.capture[0];
    cudaGraph_t g = nullptr;
    EFEM_CUDA(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
    efem_status s = enqueue_body(m, w, x, use_factor, s0);
    if (s == EFEM_OK) s = enqueue_trial_tail(m, w, x, s0, nullptr, false);  // pass 4 started the first trial
    const cudaError_t e = cudaStreamEndCapture(s0, &g);
    m.launches = launches;
    if (s != EFEM_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        if (s == EFEM_OK) set_error(std::string("graph capture: ") + cudaGetErrorString(e));
        return s != EFEM_OK ? s : EFEM_ERR_CUDA;
    }
    return instantiate(g, out);
}

efem_status capture_first(Model& m, SolverWS& w, double* x, cudaGraphExec_t* out)
{
    std::lock_guard<std::mutex> lock(capture_mutex());
    const long long launches = m.launches;
    cudaGraph_t g = nullptr;
    EFEM_CUDA(cudaStreamBeginCapture(w.capture[0], cudaStreamCaptureModeThreadLocal));
    const efem_status s = enqueue_first(m, w, x, w.capture[0]);
    const cudaError_t e = cudaStreamEndCapture(w.capture[0], &g);
    m.launches = launches;
    if (s != EFEM_OK) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess) {
        set_error(std::string("graph capture: ") + cudaGetErrorString(e));
        return EFEM_ERR_CUDA;
    }
    return instantiate(g, out);
}

double elapsed_ms(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0.f;
    return cudaEventElapsedTime(&ms, a, b) == cudaSuccess ? static_cast<double>(ms) : 0.0;
}

}  // namespace

// One L-BFGS solve from x (LBFGSSolver::solve, LBFGS.h:96-174) with the
// model's element precision.  refactor: factor the approximate Jacobian
// (once per solve, LBFGS.h:122-124; a second phase reuses the factor, which
// does not depend on u).  stall_iters > 0: also end, with *stalled set, when
// the best ||r||_inf has not halved for that many iterations.  keep_trace:
// append to the trace of an earlier phase.
efem_status run_solve_phase(Model& m, double* x, efem_solve_info* info, bool refactor, int stall_iters,
    bool keep_trace, bool* stalled)
{
    *stalled = false;
    efem_status s = alloc_ws(m);
    if (s != EFEM_OK) return s;
    SolverWS& w = *m.ws;
    const size_t n = w.n;
    const int mm = w.m;
    const int G = grid_for(n);
    cudaStream_t st = m.stream;
    const double eps = m.opts.residual_criterion;
    std::memset(info, 0, sizeof(*info));
    const long long launches0 = m.launches;
    const long long per_res = 1 + static_cast<long long>(m.blocks.size() + m.faces.size()) + (m.opts.deterministic ? 1 : 0);
    double ms_pc = 0.0;
    double rinf = 0.0, xinf = 0.0;
    int k = 1;
    bool converged = false, ok = false;
    long long n_body = 0;
    volatile double* hr = w.h_read;
    if (m.opts.trace != w.trace_cap) {  // the buffer is read through Scalars, so graphs need no recapture
        EFEM_CUDA(cudaStreamSynchronize(st));
        dev_free(w.trace);
        w.trace_cap = 0;
        if (m.opts.trace > 0) {
            if ((s = dev_alloc(&w.trace, static_cast<size_t>(m.opts.trace) * kTraceCols)) != EFEM_OK) return s;
            w.trace_cap = m.opts.trace;
        }
    }
    if (!keep_trace) hr[kRdTrN] = 0.0;
    EFEM_CUDA(cudaEventRecord(w.ev[0], st));
    k_solve_init<<<1, 1, 0, st>>>(w.sc, w.trace, w.trace_cap, keep_trace ? 1 : 0);
    m.launches++;

    // host-driven line-search trial: x = xp + step d (step 0: x as is),
    // residual, reductions, read-back
    auto direct_trial = [&](double step) -> efem_status {
        if (step != 0.0) {
            k_trial<<<G, kThreads, 0, st>>>(x, w.xp, w.d, step, n, w.sc);
            m.launches++;
        }
        efem_status rs = enqueue_trial_tail(m, w, x, st);
        if (rs != EFEM_OK) return rs;
        m.launches++;
        EFEM_CUDA(cudaStreamSynchronize(st));
        return EFEM_OK;
    };

    // Line search after a first trial x = xp + d whose residual and r.d are in
    // the read-back slots: the reference's residual-projection rule
    // (LineSearchFEA.h:43-67), or with line_search = 1 the Armijo test
    // Pi(xp + a d) <= Pi(xp) + 1e-4 a r(xp).d on the total potential, halving a.
    const bool armijo = m.opts.line_search == 1;
    double pi_prev = 0.0;
    auto line_search = [&]() -> efem_status {
        const double dg0 = hr[kRdDg0];
        double dg = hr[kRdDg], step = 1.0;
        if (!armijo) {
            for (int it = 1; it < m.opts.max_linesearch && !(std::fabs(dg) <= std::fabs(dg0)); it++) {
                step *= dg * dg0 > 0 ? 1.5 : 0.5;
                efem_status rs = direct_trial(step);
                if (rs != EFEM_OK) return rs;
                dg = hr[kRdDg];
            }
            return EFEM_OK;
        }
        double pi = 0.0;
        efem_status rs = total_potential(m, x, &pi);
        if (rs != EFEM_OK) return rs;
        for (int it = 1; it < m.opts.max_linesearch && !(pi <= pi_prev + 1e-4 * step * dg0); it++) {
            step *= 0.5;
            if ((rs = direct_trial(step)) != EFEM_OK) return rs;
            if ((rs = total_potential(m, x, &pi)) != EFEM_OK) return rs;
        }
        pi_prev = pi;
        return EFEM_OK;
    };
    if (armijo && m.n_faces > 0) {
        set_error("the Armijo line search needs conservative loads: pressure faces have no potential");
        return EFEM_ERR_UNSUPPORTED;
    }

    // initial residual and early exit (LBFGS.h:110-120); d = 0 so dg = 0 here
    EFEM_CUDA(cudaMemsetAsync(w.d, 0, n * sizeof(double), st));
    k_state_init<<<1, 1, 0, st>>>(w.sc, mm);
    m.launches++;
    if ((s = direct_trial(0.0)) != EFEM_OK) return s;
    rinf = hr[kRdRinf];
    xinf = hr[kRdXinf];
    if (!(std::isfinite(rinf))) goto nan_exit;
    if (rinf <= eps || rinf <= eps * std::sqrt(hr[kRdX2])) {
        converged = true;
        goto done;
    }
    if (armijo && (s = total_potential(m, x, &pi_prev)) != EFEM_OK) return s;
    // approximate-Jacobian factor, once per solve (LBFGS.h:122-124)
    if (m.opts.nl_solver == 0) {
        int okf = 0;
        double msf = 0;
        if ((s = precond_setup(m, refactor, &okf, &msf)) != EFEM_OK) return s;
        if ((s = precond_sync_grid(m)) != EFEM_OK) return s;
        ok = okf != 0;
        info->n_jacobian_evals = refactor ? 1 : 0;
        info->ms_factor = msf;
        if (!ok) info->flags |= EFEM_SOLVE_PRECOND_FALLBACK;
    }
    // initial direction d = -H0 r
    k_neg_copy<<<G, kThreads, 0, st>>>(w.d, w.r, n);
    m.launches++;
    if (ok) {
        EFEM_CUDA(cudaEventRecord(w.ev[2], st));
        if ((s = precond_apply(m, w.d)) != EFEM_OK) return s;
        EFEM_CUDA(cudaEventRecord(w.ev[3], st));
        if ((s = precond_check(m)) != EFEM_OK) return s;
        ms_pc += elapsed_ms(w.ev[2], w.ev[3]);
        info->n_precond_applies++;
    }
    {
        if (w.epoch != m.epoch) {  // blocks or factor rebuilt since the graphs were captured
            drop_graphs(w);
            w.epoch = m.epoch;
        }
        const bool host_loop = m.opts.host_loop != 0 || armijo;  // the Armijo test is applied from the host
        const auto key = std::make_pair(x, (ok ? 1 : 0) | (m.opts.precision << 1) | (host_loop ? 4 : 0)
            | (m.opts.deterministic ? 8 : 0));
        if (!w.graphs.count(key) && w.graphs.size() >= 8) drop_graphs(w);  // many distinct solution pointers
        SolverWS::Graphs& gr = w.graphs[key];
        if (!gr.first) {
            if ((s = capture_first(m, w, x, &gr.first)) != EFEM_OK) return s;
            for (int attempt = 0; attempt < 2; attempt++) {
                s = host_loop ? capture_step(m, w, x, ok, &gr.step) : capture_loop(m, w, x, ok, &gr.loop);
                if (s == EFEM_OK || !w.pdl) break;
                cudaGetLastError();
                w.pdl = false;  // capture again with plain launches
            }
            if (s != EFEM_OK) return s;
        }
        if (w.pdl) info->flags |= EFEM_SOLVE_PDL;
        // iteration 1 from the host
        EFEM_CUDA(cudaGraphLaunch(gr.first, st));
        EFEM_CUDA(cudaStreamSynchronize(st));
        m.launches += per_res + 2;
        if ((s = line_search()) != EFEM_OK) return s;
        rinf = hr[kRdRinf];
        xinf = hr[kRdXinf];
        if (!std::isfinite(rinf) || !std::isfinite(xinf)) goto nan_exit;
        if (rinf <= eps || rinf <= eps * xinf) {
            converged = true;
            goto done;
        }
        if (m.opts.max_iterations != 0 && k >= m.opts.max_iterations) {
            info->flags |= EFEM_SOLVE_MAX_ITERS;
            goto done;
        }
        k++;
        if (host_loop) {  // iterations 2, 3, ... one graph launch each, decisions on the host
            const long long per_step = 4 + (ok ? precond_launch_count(m) : 0) + (per_res - 1) + 1;
            double best = rinf;
            int best_k = k;
            for (;;) {
                EFEM_CUDA(cudaGraphLaunch(gr.step, st));
                EFEM_CUDA(cudaStreamSynchronize(st));
                m.launches += per_step;
                if (ok) info->n_precond_applies++;
                if (hr[kRdPerr] != 0.0) {
                    set_error("the triangular solve of the preconditioner gave up waiting for a front");
                    return EFEM_ERR_TIMEOUT;
                }
                if ((s = line_search()) != EFEM_OK) return s;
                rinf = hr[kRdRinf];
                xinf = hr[kRdXinf];
                if (!std::isfinite(rinf) || !std::isfinite(xinf)) goto nan_exit;
                if (rinf <= eps || rinf <= eps * xinf) {
                    converged = true;
                    break;
                }
                if (m.opts.max_iterations != 0 && k >= m.opts.max_iterations) {
                    info->flags |= EFEM_SOLVE_MAX_ITERS;
                    break;
                }
                if (rinf < 0.5 * best) {
                    best = rinf;
                    best_k = k;
                } else if (stall_iters > 0 && k - best_k >= stall_iters) {
                    *stalled = true;
                    break;
                }
                k++;
            }
            if (ok) ms_pc += hr[kRdTPc] * 1e-6;
            goto done;
        }
        // iterations 2, 3, ... on the device, kIterCap per graph launch
        k_loop_params<<<1, 1, 0, st>>>(w.sc, eps, m.opts.max_iterations, std::max(1, m.opts.max_linesearch),
            kIterCap, k, stall_iters, rinf);
        m.launches++;
        // passes, H0, trial (which starts r), residual, reductions, iteration decision
        // passes (pass 4 starts the first trial), H0, residual, reductions, iteration decision
        const long long per_body = 4 + (ok ? precond_launch_count(m) : 0) + (per_res - 1) + 2;
        const long long per_extra = per_res + 1;  // trial, residual, reductions
        long long n_extra = 0;
        int status = kRunning;
        for (;;) {
            EFEM_CUDA(cudaGraphLaunch(gr.loop, st));
            EFEM_CUDA(cudaStreamSynchronize(st));
            status = static_cast<int>(hr[kRdStatus]);
            const long long nb = static_cast<long long>(hr[kRdNBody]), ne = static_cast<long long>(hr[kRdNExtra]);
            m.launches += 1 + (nb - n_body) * per_body + (ne - n_extra) * per_extra;
            n_body = nb;
            n_extra = ne;
            if (status != kCapReached) break;
        }
        k = static_cast<int>(hr[kRdK]);
        rinf = hr[kRdRinf];
        xinf = hr[kRdXinf];
        if (ok) {
            info->n_precond_applies += static_cast<int>(n_body);
            ms_pc += hr[kRdTPc] * 1e-6;
        }
        if (status == kPrecondFail) {
            set_error("the triangular solve of the preconditioner gave up waiting for a front");
            return EFEM_ERR_TIMEOUT;
        }
        if (status == kNonFinite) goto nan_exit;
        if (status == kConverged) converged = true;
        if (status == kMaxIters) info->flags |= EFEM_SOLVE_MAX_ITERS;
        if (status == kStalled) *stalled = true;
    }
done:
    EFEM_CUDA(cudaEventRecord(w.ev[1], st));
    EFEM_CUDA(cudaEventSynchronize(w.ev[1]));
    info->ms_total = elapsed_ms(w.ev[0], w.ev[1]);
    info->ms_residual = hr[kRdTRes] * 1e-6;
    info->ms_precond = ms_pc;
    info->n_residual_evals = static_cast<int>(hr[kRdNRes]);
    info->niter = k;
    info->u_inf = xinf;
    info->r_inf = rinf;
    info->n_kernel_launches = m.launches - launches0;
    w.trace_n = static_cast<int>(hr[kRdTrN]);
    if (converged) info->flags |= EFEM_SOLVE_CONVERGED;
    if (xinf < m.opts.dx_criterion) info->flags |= EFEM_SOLVE_DX_CONVERGED;
    return EFEM_OK;
nan_exit:
    // Integrator::integral zeroes the solution when it is not finite (Integrator.cpp:28-34)
    EFEM_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), st));
    EFEM_CUDA(cudaStreamSynchronize(st));
    info->niter = k;
    info->u_inf = xinf;
    info->r_inf = rinf;
    info->n_residual_evals = static_cast<int>(hr[kRdNRes]);
    info->n_kernel_launches = m.launches - launches0;
    w.trace_n = static_cast<int>(hr[kRdTrN]);
    set_error("L-BFGS produced a non-finite residual or solution");
    return EFEM_ERR_NAN;
}

// iterations without a halving of the best ||r||_inf after which the FP32
// phase of a mixed-precision solve hands over to FP64 element kernels
constexpr int kStallIters = 24;
// the FP32 phase's residual target, as a fraction of the tolerance
constexpr double kFp32Target = 0.5;

// The solve behind efem_solve.  FP64: one phase.  Mixed precision: FP32
// element kernels until the residual passes the test or stops improving (the
// FP32 rounding floor of the element forces lies above the tolerance), then
// FP64 element kernels from that point, with a fresh L-BFGS history and the
// same factor, so that the residual read by the convergence test that ends
// the solve is always formed in FP64.  When the FP32 phase has converged the
// FP64 phase is one residual evaluation (its initial test).
efem_status run_solve(Model& m, double* x, efem_solve_info* info)
{
    bool stalled = false;
    if (m.opts.precision != EFEM_MIXED) return run_solve_phase(m, x, info, true, 0, false, &stalled);
    efem_solve_info a {};
    const efem_options keep = m.opts;
    // the FP32 phase aims below the tolerance, so that the FP64 test that
    // follows usually passes at once instead of restarting the history
    m.opts.residual_criterion = kFp32Target * keep.residual_criterion;
    efem_status s = run_solve_phase(m, x, &a, true, kStallIters, false, &stalled);
    m.opts = keep;
    if (s != EFEM_OK || (a.flags & EFEM_SOLVE_MAX_ITERS)) {
        *info = a;
        return s;
    }
    m.opts.precision = EFEM_FP64;
    if (keep.max_iterations != 0) m.opts.max_iterations = std::max(1, keep.max_iterations - a.niter);
    efem_solve_info b {};
    s = run_solve_phase(m, x, &b, false, 0, true, &stalled);
    m.opts = keep;
    const bool early = b.n_precond_applies == 0 && b.n_residual_evals <= 1;  // passed its initial test
    *info = b;
    info->niter = a.niter + (early ? 0 : b.niter);
    info->n_residual_evals = a.n_residual_evals + b.n_residual_evals;
    info->n_jacobian_evals = a.n_jacobian_evals;
    info->flags = b.flags | (a.flags & (EFEM_SOLVE_PRECOND_FALLBACK | EFEM_SOLVE_PDL)) | (early ? 0 : EFEM_SOLVE_REFINED);
    info->ms_total = a.ms_total + b.ms_total;
    info->ms_factor = a.ms_factor;
    info->ms_residual = a.ms_residual + b.ms_residual;
    info->ms_precond = a.ms_precond + b.ms_precond;
    info->n_kernel_launches = a.n_kernel_launches + b.n_kernel_launches;
    info->n_precond_applies = a.n_precond_applies + b.n_precond_applies;
    return s;
}

efem_status solve_trace(Model& m, double* out, int capacity, int* n_records)
{
    const int n = m.ws ? m.ws->trace_n : 0;
    if (n_records) *n_records = n;
    if (!out || capacity <= 0 || !m.ws || !m.ws->trace) return EFEM_OK;
    const int k = std::min(std::min(n, capacity), m.ws->trace_cap);
    if (k > 0) {
        EFEM_CUDA(cudaMemcpyAsync(out, m.ws->trace, sizeof(double) * kTraceCols * static_cast<size_t>(k),
            cudaMemcpyDeviceToHost, m.stream));
        EFEM_CUDA(cudaStreamSynchronize(m.stream));
    }
    return EFEM_OK;
}

}  // namespace efem
