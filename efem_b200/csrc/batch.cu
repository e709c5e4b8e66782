// Batched solves: many independent models solved as one union model.
//
// The reference solves one problem per process (Simulator::start,
// src/simulation/Simulator.cpp:20-41).  A batch of load cases or material
// samples is solved here in one stream of launches:
//
//  * The members' meshes are concatenated into a union model: disjoint bodies
//    (each member translated clear of the others, which changes nothing in a
//    Total-Lagrangian residual and lets the geometric dissection separate
//    them), every member's free DOFs a contiguous segment of the union's DOF
//    vector, in member order.  One element-kernel launch per element type and
//    one face-kernel launch per face type evaluate every member's residual,
//    with the tile sizes the set-up autotuner chose for the union.
//  * The union's approximate Jacobian is block diagonal, so its factor is the
//    forest of the members' elimination trees: one numeric factorisation and
//    one persistent triangular-solve launch (k_solve) apply every member's H0.
//  * The L-BFGS state (LBFGSSolver::solve, LBFGS.h:96-174: history, two-loop
//    recursion, line search LineSearchFEA.h:37-68, convergence test) is kept
//    per member.  The vector kernels below work on segments: every CTA takes
//    one chunk of one member's segment, and the last CTA of each member to
//    finish a reduction adds that member's partial sums in chunk order and
//    runs that member's small recursion, so every member follows exactly the
//    arithmetic of a single solve.
//  * One CUDA graph holds the iteration loop: a while node over iterations
//    whose body holds a while node over line-search trials; each condition
//    is set by a one-CTA kernel that reads every member's state, and both
//    loops are bounded there (kCap iterations per launch, max_line_search
//    trials per iteration) whatever that state holds.  A member that
//    converged (or stopped) is frozen: its x no longer moves and its
//    counters stop; the loop ends when no member is running.  The host checks
//    the state every kCap iterations.
//
// Mixed precision follows the single solve: FP32 element kernels until every
// member has converged or stalled, then FP64 element kernels (fresh history,
// same factor) finish every member whose FP64 residual fails the test.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "efem_internal.h"

namespace efem {

namespace {

constexpr int kT = 256;       // threads per CTA of the segmented vector kernels
constexpr int kChunk = 2048;  // vector entries per CTA; a chunk never spans two members
constexpr int kHist = 8;      // largest L-BFGS history of a batch
constexpr int kCap = 64;      // iterations per launch of the iteration graph
constexpr int kStall = 24;    // FP32 phase: iterations without halving the best ||r||_inf
constexpr double kFp32Target = 0.5;  // FP32 phase: residual target as a fraction of the tolerance

enum { kRun = 0, kDone = 1, kMaxIt = 2, kNaN = 3, kStalled = 4, kPcFail = 5 };

// per member: the L-BFGS state of LBFGSSolver / LBFGSMat / LineSearchFEA
struct Seg {
    double G[kHist][kHist];  // G[a][b] = s_a . y_b
    double ys[kHist], alpha[kHist], coef[kHist];
    double theta;
    double dg, dg0, rinf, xinf, x2, step;
    double eps, best;
    int ptr, ncorr, first;   // first: no pair to add yet (iteration 1)
    int max_iter, max_ls, k, ls_t, trial, state, best_k, stall;
    int n_res;               // residual evaluations while running
    unsigned int cnt;        // CTAs of this member done with the current reduction
    int c0, c1;              // the member's chunks
};

struct Glob {
    int ls_round;            // line-search trials of the current iteration
    int launch_iters, cap;
    int n_running;
    int pc_fail;
    long long body_iters;    // loop bodies run (for the launch count)
    long long trials;        // extra line-search trials run
};

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

// CTA reduction of NV values (bit k of maxmask: max, else sum); result in every thread
template <int NV>
__device__ void cta_reduce(double* v, unsigned maxmask)
{
    __shared__ double sh[NV][kT / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        v[k] = (maxmask >> k) & 1u ? warp_max(v[k]) : warp_sum(v[k]);
        if (lane == 0) sh[k][w] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double a = 0.0;
        for (int q = 0; q < kT / 32; q++) a = (maxmask >> k) & 1u ? nan_max(a, sh[k][q]) : a + sh[k][q];
        v[k] = a;
    }
    __syncthreads();
}

// The member's sums over its chunks in chunk order: every CTA stores its NV
// partials; the member's last CTA adds them and returns true (all its
// threads), with the totals in v.
template <int NV>
__device__ bool seg_finish(double* v, unsigned maxmask, Seg* sg, double* partials)
{
    __shared__ bool last;
    cta_reduce<NV>(v, maxmask);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) partials[static_cast<size_t>(blockIdx.x) * NV + k] = v[k];
        __threadfence();
        last = atomicAdd(&sg->cnt, 1u) == static_cast<unsigned>(sg->c1 - sg->c0 - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) acc[k] = 0.0;
    for (int b = sg->c0 + static_cast<int>(threadIdx.x); b < sg->c1; b += kT) {
        const volatile double* pb = partials + static_cast<size_t>(b) * NV;
#pragma unroll
        for (int k = 0; k < NV; k++) acc[k] = (maxmask >> k) & 1u ? nan_max(acc[k], pb[k]) : acc[k] + pb[k];
    }
    cta_reduce<NV>(acc, maxmask);
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = acc[k];
    if (threadIdx.x == 0) sg->cnt = 0u;
    return true;
}

// the chunk of this CTA: member, entries [a, b)
struct Chunk {
    int seg, a, b, pad;
};

__device__ __forceinline__ int ring(int i, int m) { return ((i % m) + m) % m; }

__global__ void kb_init(Seg* S, const int* c0, const double* eps, const int* max_iter, int max_ls, int m, int nseg,
    int stall, const int* keep, int* frozen)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nseg) return;
    Seg& s = S[i];
    frozen[i] = keep && keep[i] ? 1 : 0;
    if (keep && keep[i]) return;  // a member whose earlier phase ended for good
    s.theta = 1.0;
    s.ptr = m;  // ptr % m == 0 on the first correction (LBFGSMat.h:68)
    s.ncorr = 0;
    s.first = 1;
    s.eps = eps[i];
    s.max_iter = max_iter[i];
    s.max_ls = max_ls;
    s.k = 1;
    s.ls_t = 0;
    s.trial = 0;
    s.state = kRun;
    s.best = INFINITY;
    s.best_k = 1;
    s.stall = stall;
    s.n_res = 0;
    s.cnt = 0u;
    s.c0 = c0[i];
    s.c1 = c0[i + 1];
    s.step = 0.0;
    s.dg = s.dg0 = 0.0;
}

__global__ void kb_glob_init(Glob* G, int cap)
{
    G->ls_round = 0;
    G->launch_iters = 0;
    G->cap = cap;
    G->n_running = 0;
    G->pc_fail = 0;
    G->body_iters = 0;
    G->trials = 0;
}

__global__ void kb_loop_start(Glob* G)
{
    G->launch_iters = 0;
    G->ls_round = 0;
}

// the initial residual's norms and the early exit (LBFGS.h:110-120) of every running member
__global__ void __launch_bounds__(kT) kb_initial(const double* __restrict__ r, const double* __restrict__ x,
    const Chunk* __restrict__ ch, Seg* S, double* partials, int* frozen)
{
    const Chunk c = ch[blockIdx.x];
    Seg* sg = S + c.seg;
    double v[3] = { 0, 0, 0 };
    for (int i = c.a + threadIdx.x; i < c.b; i += kT) {
        v[0] = nan_max(v[0], fabs(r[i]));
        v[1] = nan_max(v[1], fabs(x[i]));
        v[2] += x[i] * x[i];
    }
    if (!seg_finish<3>(v, 3u, sg, partials) || threadIdx.x != 0) return;
    if (sg->state != kRun) return;
    sg->rinf = v[0];
    sg->xinf = v[1];
    sg->x2 = v[2];
    sg->n_res = 1;
    if (!isfinite(v[0]))
        sg->state = kNaN;
    else if (v[0] <= sg->eps || v[0] <= sg->eps * sqrt(v[2]))
        sg->state = kDone;
    frozen[c.seg] = sg->state != kRun;
}

// Pass 1 (LBFGSMat::add_correction, LBFGSMat.h:81-98, and the first loop's
// dot products, LBFGSMat.h:106-113) of every running member with a pair to
// add: the new pair s = x - xp, y = r - rp into the member's slot, its row
// and column of G, s_j . q0; the member's last CTA runs the first loop.
template <int M>
__global__ void __launch_bounds__(kT) kb_pass1(const double* __restrict__ x, const double* __restrict__ xp,
    const double* __restrict__ r, const double* __restrict__ rp, double* __restrict__ Sh, double* __restrict__ Yh,
    size_t n, const Chunk* __restrict__ ch, Seg* S, double* partials)
{
    constexpr int NV = 3 * M + 2;
    const Chunk c = ch[blockIdx.x];
    Seg* sg = S + c.seg;
    const bool act = sg->state == kRun && !sg->first;
    const int loc = sg->ptr % M;
    const int ncorr = sg->ncorr < M ? sg->ncorr + 1 : M;
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = 0.0;
    if (act) {
        double* snew = Sh + static_cast<size_t>(loc) * n;
        double* ynew = Yh + static_cast<size_t>(loc) * n;
        for (int i = c.a + threadIdx.x; i < c.b; i += kT) {
            const double si = x[i] - xp[i], ri = r[i], yi = ri - rp[i];
            snew[i] = si;
            ynew[i] = yi;
            v[3 * M] += si * yi;
            v[3 * M + 1] += yi * yi;
#pragma unroll
            for (int j = 0; j < M; j++)
                if (j < ncorr) {
                    const bool self = j == loc;
                    const double sj = self ? si : Sh[static_cast<size_t>(j) * n + i];
                    const double yj = self ? yi : Yh[static_cast<size_t>(j) * n + i];
                    v[3 * j] += si * yj;
                    v[3 * j + 1] += sj * yi;
                    v[3 * j + 2] -= sj * ri;
                }
        }
    }
    if (!seg_finish<NV>(v, 0u, sg, partials)) return;
    if (threadIdx.x != 0) return;
    if (sg->state != kRun) return;
    if (sg->first) {  // iteration 1: d = -H0 r, no pair yet
        sg->first = 0;
        sg->ncorr = 0;
        return;
    }
    const double ys = v[3 * M], yy = v[3 * M + 1];
    for (int j = 0; j < ncorr; j++) {
        sg->G[loc][j] = v[3 * j];
        sg->G[j][loc] = v[3 * j + 1];
    }
    sg->G[loc][loc] = ys;
    sg->ys[loc] = ys;
    double al[M];
    for (int i = 0; i < ncorr; i++) {  // newest slot first
        const int j = ring(loc - i, M);
        double t = v[3 * j + 2];
        for (int q = 0; q < i; q++) {
            const int jq = ring(loc - q, M);
            t -= al[jq] * sg->G[j][jq];
        }
        al[j] = t / sg->ys[j];
    }
    for (int j = 0; j < ncorr; j++) sg->alpha[j] = al[j];
    sg->theta = yy / ys;
    sg->ptr = loc + 1;
    sg->ncorr = ncorr;
}

// Pass 2: q = -r - sum_j alpha_j y_j for running members (0 elsewhere); also
// clears the triangular solve's counters for the H0 application that follows
__global__ void __launch_bounds__(kT) kb_pass2(double* __restrict__ q, const double* __restrict__ r,
    const double* __restrict__ Yh, size_t n, const Chunk* __restrict__ ch, const Seg* S, int* clear, int n_clear)
{
    const Chunk c = ch[blockIdx.x];
    const Seg* sg = S + c.seg;
    __shared__ double al[kHist];
    const bool act = sg->state == kRun;
    const int ncorr = act ? sg->ncorr : 0;
    if (threadIdx.x < kHist) al[threadIdx.x] = static_cast<int>(threadIdx.x) < ncorr ? sg->alpha[threadIdx.x] : 0.0;
    __syncthreads();
    for (int i = c.a + threadIdx.x; i < c.b; i += kT) {
        double qi = act ? -r[i] : 0.0;
        for (int j = 0; j < ncorr; j++) qi -= al[j] * Yh[static_cast<size_t>(j) * n + i];
        q[i] = qi;
    }
    if (clear)
        for (int k = blockIdx.x * kT + threadIdx.x; k < n_clear; k += gridDim.x * kT) clear[k] = 0;
}

// Pass 3: y_j . z for every slot; the member's last CTA runs the second loop
// (LBFGSMat.h:121-128), oldest pair first
template <int M>
__global__ void __launch_bounds__(kT) kb_pass3(const double* __restrict__ z, const double* __restrict__ Yh, size_t n,
    const Chunk* __restrict__ ch, Seg* S, double* partials)
{
    const Chunk c = ch[blockIdx.x];
    Seg* sg = S + c.seg;
    const int ncorr = sg->state == kRun ? sg->ncorr : 0;
    double v[M];
#pragma unroll
    for (int k = 0; k < M; k++) v[k] = 0.0;
    for (int i = c.a + threadIdx.x; i < c.b; i += kT) {
        const double zi = z[i];
#pragma unroll
        for (int j = 0; j < M; j++)
            if (j < ncorr) v[j] += Yh[static_cast<size_t>(j) * n + i] * zi;
    }
    if (!seg_finish<M>(v, 0u, sg, partials)) return;
    if (threadIdx.x != 0 || sg->state != kRun) return;
    const int ptr = sg->ptr;
    double cf[M];
    for (int o = 0; o < ncorr; o++) {
        const int j = ring(ptr - ncorr + o, M);
        double t = v[j];
        for (int p = 0; p < o; p++) {
            const int jp = ring(ptr - ncorr + p, M);
            t += cf[jp] * sg->G[jp][j];
        }
        cf[j] = sg->alpha[j] - t / sg->ys[j];
    }
    for (int j = 0; j < ncorr; j++) sg->coef[j] = cf[j];
}

// Pass 4: d = z + sum_j coef_j s_j and the start of the line search of every
// running member (dg0 = r.d, xp = x, rp = r, step 1) with its first trial
// x = xp + d; r = -f_ext everywhere for the residual that follows
__global__ void __launch_bounds__(kT) kb_pass4(double* __restrict__ d, const double* __restrict__ z,
    const double* __restrict__ Sh, double* __restrict__ r, double* __restrict__ x, double* __restrict__ xp,
    double* __restrict__ rp, const double* __restrict__ fext, size_t n, const Chunk* __restrict__ ch, Seg* S,
    double* partials)
{
    const Chunk c = ch[blockIdx.x];
    Seg* sg = S + c.seg;
    const bool act = sg->state == kRun;
    const int ncorr = act ? sg->ncorr : 0;
    __shared__ double cf[kHist];
    if (threadIdx.x < kHist) cf[threadIdx.x] = static_cast<int>(threadIdx.x) < ncorr ? sg->coef[threadIdx.x] : 0.0;
    __syncthreads();
    double v[1] = { 0.0 };
    for (int i = c.a + threadIdx.x; i < c.b; i += kT) {
        const double ri = r[i];
        if (act) {
            double di = z[i];
            for (int j = 0; j < ncorr; j++) di += cf[j] * Sh[static_cast<size_t>(j) * n + i];
            d[i] = di;
            const double xi = x[i];
            v[0] += ri * di;
            xp[i] = xi;
            rp[i] = ri;
            x[i] = xi + di;
        }
        r[i] = -fext[i];
    }
    if (!seg_finish<1>(v, 0u, sg, partials)) return;
    if (threadIdx.x != 0 || sg->state != kRun) return;
    sg->dg0 = v[0];
    sg->step = 1.0;
    sg->ls_t = 0;
    sg->trial = 1;
}

// After a trial's residual: r.d, ||r||_inf, ||x||_inf, ||x||^2 of every
// member in its line search, which applies the reference's rule (accept when
// |r.d| <= |r0.d|, else step x1.5 if (r.d)(r0.d) > 0, x0.5 otherwise, at
// most max_line_search trials, LineSearchFEA.h:43-67).
__global__ void __launch_bounds__(kT) kb_ls_reduce(const double* __restrict__ r, const double* __restrict__ d,
    const double* __restrict__ x, const Chunk* __restrict__ ch, Seg* S, double* partials)
{
    const Chunk c = ch[blockIdx.x];
    Seg* sg = S + c.seg;
    const bool act = sg->state == kRun && sg->trial;
    double v[4] = { 0, 0, 0, 0 };
    if (act)
        for (int i = c.a + threadIdx.x; i < c.b; i += kT) {
            const double ri = r[i], xi = x[i];
            v[0] += ri * d[i];
            v[1] = nan_max(v[1], fabs(ri));
            v[2] = nan_max(v[2], fabs(xi));
            v[3] += xi * xi;
        }
    if (!seg_finish<4>(v, 6u, sg, partials)) return;
    if (threadIdx.x != 0) return;
    if (act) {
        sg->dg = v[0];
        sg->rinf = v[1];
        sg->xinf = v[2];
        sg->x2 = v[3];
        sg->n_res++;
        const int t = ++sg->ls_t;
        const bool again = !(fabs(v[0]) <= fabs(sg->dg0)) && t < sg->max_ls;
        if (again) sg->step *= v[0] * sg->dg0 > 0 ? 1.5 : 0.5;
        sg->trial = again ? 1 : 0;
    }
}

// The trial loop's condition: some member wants another trial.  The loop
// is also bounded here, whatever the members' state: after max_ls trials of
// one iteration every line search ends.
__global__ void __launch_bounds__(1024) kb_ls_decide(Seg* S, int nseg, int max_ls, Glob* G,
    cudaGraphConditionalHandle h)
{
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    const bool stop = G->ls_round + 1 >= max_ls;
    int mine = 0;
    for (int i = threadIdx.x; i < nseg; i += blockDim.x) {
        Seg& s = S[i];
        if (s.state != kRun || !s.trial) continue;
        if (stop)
            s.trial = 0;
        else
            mine = 1;
    }
    if (mine) atomicOr(&any, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        G->ls_round++;
        if (any) G->trials++;
        cudaGraphSetConditional(h, any ? 1u : 0u);
    }
}

// a further trial: x = xp + step d for the members still in their line search; r = -f_ext everywhere
__global__ void __launch_bounds__(kT) kb_trial(double* __restrict__ x, const double* __restrict__ xp,
    const double* __restrict__ d, double* __restrict__ r, const double* __restrict__ fext,
    const Chunk* __restrict__ ch, const Seg* S)
{
    const Chunk c = ch[blockIdx.x];
    const Seg* sg = S + c.seg;
    const bool act = sg->state == kRun && sg->trial;
    const double step = sg->step;
    for (int i = c.a + threadIdx.x; i < c.b; i += kT) {
        if (act) x[i] = __fma_rn(step, d[i], xp[i]);
        r[i] = -fext[i];
    }
}

// End of an iteration for every running member (LBFGS.h:150-170): stop on a
// non-finite residual or solution, on convergence (||r||_inf <= eps or
// <= eps ||x||_inf), at the iteration limit, or (FP32 phase) when the best
// ||r||_inf has not halved for `stall` iterations; else count the iteration.
// Sets the iteration loop's condition: some member runs and the launch has
// iterations left.
__global__ void __launch_bounds__(1024) kb_decide(Seg* S, int nseg, Glob* G, const int* perr, int* frozen,
    cudaGraphConditionalHandle h)
{
    __shared__ int running;
    if (threadIdx.x == 0) running = 0;
    __syncthreads();
    const bool pc_fail = perr && *reinterpret_cast<const volatile int*>(perr) != 0;
    int mine = 0;
    for (int i = threadIdx.x; i < nseg; i += blockDim.x) {
        Seg& s = S[i];
        if (s.state != kRun) continue;
        const double rinf = s.rinf, xinf = s.xinf;
        if (pc_fail)
            s.state = kPcFail;
        else if (!isfinite(rinf) || !isfinite(xinf))
            s.state = kNaN;
        else if (rinf <= s.eps || rinf <= s.eps * xinf)
            s.state = kDone;
        else if (s.max_iter != 0 && s.k >= s.max_iter)
            s.state = kMaxIt;
        else if (s.stall > 0 && !(rinf < 0.5 * s.best) && s.k - s.best_k >= s.stall)
            s.state = kStalled;
        else {
            if (rinf < 0.5 * s.best) {
                s.best = rinf;
                s.best_k = s.k;
            }
            s.k++;
            mine++;
        }
        if (s.state != kRun) frozen[i] = 1;  // the triangular solve skips its items from now on
    }
    if (mine) atomicAdd(&running, mine);
    __syncthreads();
    if (threadIdx.x == 0) {
        G->n_running = running;
        G->body_iters++;
        G->ls_round = 0;
        if (pc_fail) G->pc_fail = 1;
        const bool more = running > 0 && ++G->launch_iters < G->cap;
        cudaGraphSetConditional(h, more ? 1u : 0u);
    }
}

efem_status add_while_node(cudaStream_t st, cudaGraphConditionalHandle h, cudaGraph_t* body)
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

// One union of batch members, cached between calls with the same members.
struct Union {
    std::vector<Model*> members;
    std::vector<std::vector<char>> opts_seen;  // the members' options when the union was built
    std::vector<long long> epoch_seen;
    std::unique_ptr<Model> uni;
    int nseg = 0, nchunk = 0, m = 6;
    size_t n = 0;
    std::vector<size_t> off;                // DOF offset of every member (n_seg + 1)
    std::vector<int> c0;                    // first chunk of every member (n_seg + 1)
    Chunk* d_chunks = nullptr;
    int* d_c0 = nullptr;
    double* d_eps = nullptr;
    int* d_maxit = nullptr;
    int* d_keep = nullptr;
    int* d_frozen = nullptr;  // per member: 1 = no longer iterating (the triangular solve skips it)
    Seg* d_seg = nullptr;
    Glob* d_glob = nullptr;
    double *x = nullptr, *xp = nullptr, *r = nullptr, *rp = nullptr, *d = nullptr, *q = nullptr, *Sh = nullptr,
           *Yh = nullptr, *partials = nullptr;
    cudaStream_t cap[3] = { nullptr, nullptr, nullptr };
    cudaGraphExec_t loop[2] = { nullptr, nullptr };  // per element precision (FP64, FP32)
    long long loop_epoch[2] = { -1, -1 };
    long long per_res = 0;
    ~Union();
};

Union::~Union()
{
    if (uni && uni->device >= 0) cudaSetDevice(uni->device);
    for (auto& g : loop)
        if (g) cudaGraphExecDestroy(g);
    for (auto& s : cap)
        if (s) cudaStreamDestroy(s);
    for (double** p : { &x, &xp, &r, &rp, &d, &q, &Sh, &Yh, &partials, &d_eps }) dev_free(*p);
    dev_free(d_chunks);
    dev_free(d_c0);
    dev_free(d_maxit);
    dev_free(d_keep);
    dev_free(d_frozen);
    dev_free(d_seg);
    dev_free(d_glob);
}

std::mutex g_union_mutex;
std::vector<std::unique_ptr<Union>> g_unions;  // a few recent batches

std::vector<char> opts_bytes(const efem_options& o)
{
    std::vector<char> b(sizeof(o));
    std::memcpy(b.data(), &o, sizeof(o));
    return b;
}

// Can these models share one union?  The union takes its element precision,
// integration, solver and line-search settings from the first member.
bool union_eligible(Model** ms, int n, std::string* why)
{
    if (n < 2) return *why = "one model", false;
    const efem_options& o = ms[0]->opts;
    for (int i = 0; i < n; i++) {
        const Model& m = *ms[i];
        const efem_options& p = m.opts;
        if (p.precision != o.precision || p.integration != o.integration || p.m != o.m || p.m > kHist
            || p.max_linesearch != o.max_linesearch || p.nl_solver != 0 || p.deterministic || p.host_loop
            || p.line_search != 0 || p.wait_test || p.wait_limit != o.wait_limit)
            return *why = "member options differ or are not supported in a union", false;
        if (m.has_gravity) return *why = "gravity loads", false;
        if (m.device >= 0 && ms[0]->device >= 0 && m.device != ms[0]->device) return *why = "different devices", false;
        for (int j = 0; j < i; j++)
            if (ms[j] == ms[i]) return *why = "a model appears twice", false;
    }
    return true;
}

// Build the union model's input from the members' kept input.
efem_status build_union(Union& U)
{
    ModelInput in;
    in.opts = U.members[0]->opts;
    in.opts.residual_criterion = 1e-6;  // per member, in Seg
    in.opts.max_iterations = 0;
    in.opts.device = U.members[0]->device >= 0 ? U.members[0]->device : U.members[0]->opts.device;
    int node0 = 0, mat0 = 0;
    double shift = 0.0;
    std::vector<HostBlock> by_nen(21);
    for (Model* mp : U.members) {
        const Model& m = *mp;
        double lo = 1e300, hi = -1e300;
        for (int i = 0; i < m.n_nodes; i++) {
            lo = std::min(lo, m.X[3 * static_cast<size_t>(i)]);
            hi = std::max(hi, m.X[3 * static_cast<size_t>(i)]);
        }
        const double dx = shift - lo;  // place this member's bodies right of the previous ones
        for (int i = 0; i < m.n_nodes; i++) {
            in.X.push_back(m.X[3 * static_cast<size_t>(i)] + dx);
            in.X.push_back(m.X[3 * static_cast<size_t>(i) + 1]);
            in.X.push_back(m.X[3 * static_cast<size_t>(i) + 2]);
        }
        shift += (hi - lo) * 1.5 + 1.0;
        for (size_t s = 0; s < m.materials_used.size(); s++) {
            HostMaterial hm = m.materials_used[s];
            hm.id = mat0 + static_cast<int>(s);
            in.materials.push_back(hm);
        }
        for (const HostBlock& hb : m.in_blocks) {
            HostBlock& ub = by_nen[hb.nen];
            ub.nen = hb.nen;
            for (int v : hb.conn) ub.conn.push_back(v + node0);
            for (int s : hb.mat_id) ub.mat_id.push_back(s + mat0);
        }
        for (const HostLoad& L : m.in_loads) {
            HostLoad u = L;
            for (int& v : u.nodes) v += node0;
            in.loads.push_back(std::move(u));
        }
        node0 += m.n_nodes;
        mat0 += static_cast<int>(m.materials_used.size());
    }
    for (auto& b : by_nen)
        if (!b.mat_id.empty()) in.blocks.push_back(std::move(b));
    U.uni = std::make_unique<Model>();
    efem_status s = build_model(in, *U.uni);
    if (s != EFEM_OK) return s;
    // every member's free DOFs form one segment, in member order
    U.nseg = static_cast<int>(U.members.size());
    U.off.assign(1, 0);
    for (Model* mp : U.members) U.off.push_back(U.off.back() + 3 * static_cast<size_t>(mp->n_free));
    U.n = U.off.back();
    if (U.n != 3 * static_cast<size_t>(U.uni->n_free)) {
        set_error("batch union: DOF count mismatch");
        return EFEM_ERR_ARG;
    }
    return EFEM_OK;
}

efem_status setup_union(Union& U)
{
    Model& M = *U.uni;
    efem_status s = ensure_device(M);
    if (s != EFEM_OK) return s;
    U.m = M.opts.m;
    std::vector<Chunk> ch;
    U.c0.assign(1, 0);
    for (int i = 0; i < U.nseg; i++) {
        for (size_t a = U.off[i]; a < U.off[i + 1]; a += kChunk)
            ch.push_back({ i, static_cast<int>(a), static_cast<int>(std::min(U.off[i + 1], a + kChunk)), 0 });
        if (U.off[i + 1] == U.off[i]) ch.push_back({ i, static_cast<int>(U.off[i]), static_cast<int>(U.off[i]), 0 });
        U.c0.push_back(static_cast<int>(ch.size()));
    }
    U.nchunk = static_cast<int>(ch.size());
    if ((s = dev_upload(&U.d_chunks, ch)) != EFEM_OK) return s;
    if ((s = dev_upload(&U.d_c0, U.c0)) != EFEM_OK) return s;
    for (double** p : { &U.x, &U.xp, &U.r, &U.rp, &U.d, &U.q })
        if ((s = dev_alloc(p, std::max<size_t>(U.n, 1))) != EFEM_OK) return s;
    if ((s = dev_alloc(&U.Sh, std::max<size_t>(U.n, 1) * U.m)) != EFEM_OK) return s;
    if ((s = dev_alloc(&U.Yh, std::max<size_t>(U.n, 1) * U.m)) != EFEM_OK) return s;
    if ((s = dev_alloc(&U.partials, static_cast<size_t>(U.nchunk) * (3 * kHist + 2))) != EFEM_OK) return s;
    if ((s = dev_alloc(&U.d_eps, U.nseg)) != EFEM_OK) return s;
    if ((s = dev_alloc(&U.d_maxit, U.nseg)) != EFEM_OK) return s;
    if ((s = dev_alloc(&U.d_keep, U.nseg)) != EFEM_OK) return s;
    if ((s = dev_alloc(&U.d_frozen, U.nseg)) != EFEM_OK) return s;
    if ((s = dev_alloc(&U.d_seg, U.nseg)) != EFEM_OK) return s;
    if ((s = dev_alloc(&U.d_glob, 1)) != EFEM_OK) return s;
    EFEM_CUDA(cudaMemset(U.d_seg, 0, sizeof(Seg) * U.nseg));
    EFEM_CUDA(cudaMemset(U.d_frozen, 0, sizeof(int) * U.nseg));
    // members that stop iterating drop out of the element kernels: the
    // member of every element, block by block (members' elements are
    // concatenated in member order within each element type)
    for (auto& b : M.blocks) {
        std::vector<int> eg;
        eg.reserve(b.n);
        for (int i = 0; i < U.nseg; i++)
            for (const HostBlock& hb : U.members[i]->in_blocks)
                if (hb.nen == b.nen) eg.insert(eg.end(), hb.mat_id.size(), i);
        if (static_cast<int>(eg.size()) != b.n) {
            set_error("batch union: element count mismatch");
            return EFEM_ERR_ARG;
        }
        if ((s = dev_upload(&b.egroup, eg)) != EFEM_OK) return s;
    }
    M.d_frozen_groups = U.d_frozen;
    for (auto& c : U.cap) EFEM_CUDA(cudaStreamCreateWithFlags(&c, cudaStreamNonBlocking));
    U.per_res = 1 + static_cast<long long>(M.blocks.size() + M.faces.size());
    return EFEM_OK;
}

// the iteration graph: while (iterate) { passes, H0, first trial, residual,
// line-search reduction; while (trial) { trial, residual, reduction }; decide }
efem_status capture_union_loop(Union& U, cudaGraphExec_t* out)
{
    Model& M = *U.uni;
    std::lock_guard<std::mutex> lock(capture_mutex());
    cudaStream_t s0 = U.cap[0], s1 = U.cap[1], s2 = U.cap[2];
    const int nb = U.nchunk;
    cudaGraph_t g = nullptr;
    efem_status s = EFEM_OK;
    const long long launches = M.launches;
    EFEM_CUDA(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
    do {
        cudaGraph_t outer = nullptr;
        cudaStreamCaptureStatus cs;
        if (cudaStreamGetCaptureInfo(s0, &cs, nullptr, &outer, nullptr, nullptr) != cudaSuccess) {
            s = EFEM_ERR_CUDA;
            break;
        }
        cudaGraphConditionalHandle h_it, h_ls;
        if (cudaGraphConditionalHandleCreate(&h_it, outer, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
            s = EFEM_ERR_CUDA;
            break;
        }
        kb_loop_start<<<1, 1, 0, s0>>>(U.d_glob);
        cudaGraph_t body = nullptr, ls_body = nullptr;
        if ((s = add_while_node(s0, h_it, &body)) != EFEM_OK) break;
        if (cudaGraphConditionalHandleCreate(&h_ls, body, 1, cudaGraphCondAssignDefault) != cudaSuccess
            || cudaStreamBeginCaptureToGraph(s1, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            s = EFEM_ERR_CUDA;
            break;
        }
        switch (U.m) {
#define P1(K) case K: kb_pass1<K><<<nb, kT, 0, s1>>>(U.x, U.xp, U.r, U.rp, U.Sh, U.Yh, U.n, U.d_chunks, U.d_seg, U.partials); break;
            P1(1) P1(2) P1(3) P1(4) P1(5) P1(6) P1(7) P1(8)
#undef P1
        }
        int* clear = nullptr;
        int n_clear = 0;
        precond_counters(M, &clear, &n_clear);
        kb_pass2<<<nb, kT, 0, s1>>>(U.q, U.r, U.Yh, U.n, U.d_chunks, U.d_seg, clear, n_clear);
        if ((s = precond_enqueue(M, U.q, s1, false)) != EFEM_OK) break;
        switch (U.m) {
#define P3(K) case K: kb_pass3<K><<<nb, kT, 0, s1>>>(U.q, U.Yh, U.n, U.d_chunks, U.d_seg, U.partials); break;
            P3(1) P3(2) P3(3) P3(4) P3(5) P3(6) P3(7) P3(8)
#undef P3
        }
        kb_pass4<<<nb, kT, 0, s1>>>(U.d, U.q, U.Sh, U.r, U.x, U.xp, U.rp, M.d_fext, U.n, U.d_chunks, U.d_seg,
            U.partials);
        if ((s = launch_residual_on(M, U.x, U.r, s1, nullptr, false)) != EFEM_OK) break;
        kb_ls_reduce<<<nb, kT, 0, s1>>>(U.r, U.d, U.x, U.d_chunks, U.d_seg, U.partials);
        kb_ls_decide<<<1, 1024, 0, s1>>>(U.d_seg, U.nseg, std::max(1, M.opts.max_linesearch), U.d_glob, h_ls);
        if ((s = add_while_node(s1, h_ls, &ls_body)) != EFEM_OK) break;
        if (cudaStreamBeginCaptureToGraph(s2, ls_body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            s = EFEM_ERR_CUDA;
            break;
        }
        kb_trial<<<nb, kT, 0, s2>>>(U.x, U.xp, U.d, U.r, M.d_fext, U.d_chunks, U.d_seg);
        s = launch_residual_on(M, U.x, U.r, s2, nullptr, false);
        kb_ls_reduce<<<nb, kT, 0, s2>>>(U.r, U.d, U.x, U.d_chunks, U.d_seg, U.partials);
        kb_ls_decide<<<1, 1024, 0, s2>>>(U.d_seg, U.nseg, std::max(1, M.opts.max_linesearch), U.d_glob, h_ls);
        cudaGraph_t tmp = nullptr;
        if (cudaStreamEndCapture(s2, &tmp) != cudaSuccess && s == EFEM_OK) s = EFEM_ERR_CUDA;
        if (s != EFEM_OK) break;
        kb_decide<<<1, 1024, 0, s1>>>(U.d_seg, U.nseg, U.d_glob, precond_error_flag(M), U.d_frozen, h_it);
        if (cudaStreamEndCapture(s1, &tmp) != cudaSuccess) s = EFEM_ERR_CUDA;
    } while (false);
    const cudaError_t e = cudaStreamEndCapture(s0, &g);
    M.launches = launches;
    if (s != EFEM_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        if (s == EFEM_ERR_CUDA || e != cudaSuccess)
            set_error(std::string("capture of the batch iteration loop: ")
                + cudaGetErrorString(e != cudaSuccess ? e : cudaGetLastError()));
        return s != EFEM_OK ? s : EFEM_ERR_CUDA;
    }
    const cudaError_t ei = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        set_error(std::string("batch graph instantiation: ") + cudaGetErrorString(ei));
        return EFEM_ERR_CUDA;
    }
    return EFEM_OK;
}

// One phase: every member not marked in keep starts from x with a fresh
// history; the initial residual, the early exits, then the iteration graph
// until no member runs.  stall > 0: the FP32 phase's stall test.
efem_status run_union_phase(Union& U, int stall, const std::vector<int>& keep, long long* launches,
    double* ms_factor, bool refactor)
{
    Model& M = *U.uni;
    cudaStream_t st = M.stream;
    std::vector<double> eps(U.nseg);
    std::vector<int> maxit(U.nseg);
    // the FP32 phase aims below each tolerance, so that the FP64 test that
    // follows usually passes at once
    const double target = stall > 0 ? kFp32Target : 1.0;
    for (int i = 0; i < U.nseg; i++) {
        eps[i] = target * U.members[i]->opts.residual_criterion;
        maxit[i] = U.members[i]->opts.max_iterations;
    }
    EFEM_CUDA(cudaMemcpyAsync(U.d_eps, eps.data(), sizeof(double) * U.nseg, cudaMemcpyHostToDevice, st));
    EFEM_CUDA(cudaMemcpyAsync(U.d_maxit, maxit.data(), sizeof(int) * U.nseg, cudaMemcpyHostToDevice, st));
    EFEM_CUDA(cudaMemcpyAsync(U.d_keep, keep.data(), sizeof(int) * U.nseg, cudaMemcpyHostToDevice, st));
    kb_init<<<(U.nseg + 127) / 128, 128, 0, st>>>(U.d_seg, U.d_c0, U.d_eps, U.d_maxit, M.opts.max_linesearch, U.m,
        U.nseg, stall, U.d_keep, U.d_frozen);
    kb_glob_init<<<1, 1, 0, st>>>(U.d_glob, kCap);
    efem_status s = launch_residual_on(M, U.x, U.r, st);
    if (s != EFEM_OK) return s;
    kb_initial<<<U.nchunk, kT, 0, st>>>(U.r, U.x, U.d_chunks, U.d_seg, U.partials, U.d_frozen);
    *launches += 4 + U.per_res;
    // the approximate Jacobian's factor (LBFGS.h:122-124): the forest of the members' trees
    int ok = 0;
    double msf = 0.0;
    if ((s = precond_setup(M, refactor, &ok, &msf)) != EFEM_OK) return s;
    if (refactor) *ms_factor = msf;
    if (!ok) {
        set_error("batch union: an approximate Jacobian is not positive definite");
        return EFEM_ERR_UNSUPPORTED;
    }
    if (!precond_has_groups(M)) {  // members that stop iterating drop out of the triangular solve
        std::vector<int> group(M.n_free);
        for (int i = 0; i < U.nseg; i++)
            for (size_t q = U.off[i] / 3; q < U.off[i + 1] / 3; q++) group[q] = i;
        if ((s = precond_set_groups(M, group, U.d_frozen)) != EFEM_OK) return s;
    }
    const int slot = M.opts.precision == EFEM_MIXED ? 1 : 0;
    if (!U.loop[slot] || U.loop_epoch[slot] != M.epoch) {
        if (U.loop[slot]) cudaGraphExecDestroy(U.loop[slot]);
        U.loop[slot] = nullptr;
        if ((s = capture_union_loop(U, &U.loop[slot])) != EFEM_OK) return s;
        U.loop_epoch[slot] = M.epoch;
    }
    Glob g {};
    long long body0 = 0, trials0 = 0;
    // per loop body: passes 1-4, H0, residual, reduction, decision; per extra trial: trial, residual, reduction
    const long long per_body = 7 + precond_launch_count(M) + (U.per_res - 1) + 1;
    const long long per_trial = 3 + (U.per_res - 1);
    for (;;) {
        EFEM_CUDA(cudaGraphLaunch(U.loop[slot], st));
        EFEM_CUDA(cudaMemcpyAsync(&g, U.d_glob, sizeof(Glob), cudaMemcpyDeviceToHost, st));
        EFEM_CUDA(cudaStreamSynchronize(st));
        *launches += 1 + (g.body_iters - body0) * per_body + (g.trials - trials0) * per_trial;
        body0 = g.body_iters;
        trials0 = g.trials;
        if (g.pc_fail) {
            set_error("the triangular solve of the preconditioner gave up waiting for a front");
            return EFEM_ERR_TIMEOUT;
        }
        if (g.n_running == 0) break;
    }
    return EFEM_OK;
}

}  // namespace

void batch_forget(const Model* m)
{
    // Unions that hold m are moved out under the lock and destroyed after it
    // is released: a union's own model calls this function from its
    // destructor, and the lock is not recursive.
    std::vector<std::unique_ptr<Union>> dead;
    {
        std::lock_guard<std::mutex> lock(g_union_mutex);
        for (auto& u : g_unions)
            if (std::find(u->members.begin(), u->members.end(), m) != u->members.end()) dead.push_back(std::move(u));
        g_unions.erase(std::remove(g_unions.begin(), g_unions.end(), nullptr), g_unions.end());
    }
}

efem_status batch_union_solve(Model** ms, int n, double* const* u, efem_solve_info* infos)
{
    std::string why;
    if (!union_eligible(ms, n, &why)) {
        set_error("batch union: " + why);
        return EFEM_ERR_UNSUPPORTED;
    }
    for (int i = 0; i < n; i++) {
        efem_status s = ensure_device(*ms[i]);
        if (s != EFEM_OK) return s;
    }
    std::unique_ptr<Union> evicted;  // declared before the lock: destroyed after it is released
    std::lock_guard<std::mutex> lock(g_union_mutex);
    Union* U = nullptr;
    for (auto& cand : g_unions) {
        if (static_cast<int>(cand->members.size()) != n) continue;
        bool same = true;
        for (int i = 0; i < n && same; i++)
            same = cand->members[i] == ms[i] && cand->opts_seen[i] == opts_bytes(ms[i]->opts)
                && cand->epoch_seen[i] == ms[i]->epoch;
        if (same) {
            U = cand.get();
            break;
        }
    }
    if (!U) {
        auto nu = std::make_unique<Union>();
        nu->members.assign(ms, ms + n);
        for (int i = 0; i < n; i++) {
            nu->opts_seen.push_back(opts_bytes(ms[i]->opts));
            nu->epoch_seen.push_back(ms[i]->epoch);
        }
        efem_status s = build_union(*nu);
        if (s == EFEM_OK) s = setup_union(*nu);
        if (s != EFEM_OK) return s;
        if (g_unions.size() >= 4) {  // the oldest union goes; its destruction must not hold the lock
            evicted = std::move(g_unions.front());
            g_unions.erase(g_unions.begin());
        }
        g_unions.push_back(std::move(nu));
        U = g_unions.back().get();
    }
    Model& M = *U->uni;
    EFEM_CUDA(cudaSetDevice(M.device));
    cudaStream_t st = M.stream;
    cudaEvent_t e0, e1;
    EFEM_CUDA(cudaEventCreate(&e0));
    EFEM_CUDA(cudaEventCreate(&e1));
    // the members' start vectors into the union's x
    for (int i = 0; i < n; i++) {
        const size_t len = U->off[i + 1] - U->off[i];
        if (len == 0) continue;
        const bool dev = ms[i]->opts.device_ptrs != 0;
        EFEM_CUDA(cudaMemcpyAsync(U->x + U->off[i], u[i], sizeof(double) * len,
            dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    }
    EFEM_CUDA(cudaEventRecord(e0, st));
    long long launches = 0;
    double ms_factor = 0.0;
    std::vector<int> keep(U->nseg, 0);
    const bool mixed = M.opts.precision == EFEM_MIXED;
    efem_status s = run_union_phase(*U, mixed ? kStall : 0, keep, &launches, &ms_factor, true);
    std::vector<Seg> sg1(U->nseg), sg(U->nseg);
    if (s == EFEM_OK) {
        EFEM_CUDA(cudaMemcpy(sg1.data(), U->d_seg, sizeof(Seg) * U->nseg, cudaMemcpyDeviceToHost));
        sg = sg1;
    }
    if (s == EFEM_OK && mixed) {
        // FP64 element kernels finish every member the FP32 phase left converged or stalled
        for (int i = 0; i < U->nseg; i++) keep[i] = sg1[i].state == kDone || sg1[i].state == kStalled ? 0 : 1;
        M.opts.precision = EFEM_FP64;
        s = run_union_phase(*U, 0, keep, &launches, &ms_factor, false);
        M.opts.precision = EFEM_MIXED;
        if (s == EFEM_OK) EFEM_CUDA(cudaMemcpy(sg.data(), U->d_seg, sizeof(Seg) * U->nseg, cudaMemcpyDeviceToHost));
    }
    EFEM_CUDA(cudaEventRecord(e1, st));
    if (s != EFEM_OK) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return s;
    }
    // results back to the members
    for (int i = 0; i < n; i++) {
        const size_t len = U->off[i + 1] - U->off[i];
        if (len == 0) continue;
        const bool dev = ms[i]->opts.device_ptrs != 0;
        if (sg[i].state == kNaN)  // Integrator::integral zeroes a non-finite solution (Integrator.cpp:28-34)
            EFEM_CUDA(cudaMemsetAsync(U->x + U->off[i], 0, sizeof(double) * len, st));
        EFEM_CUDA(cudaMemcpyAsync(u[i], U->x + U->off[i], sizeof(double) * len,
            dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    }
    EFEM_CUDA(cudaStreamSynchronize(st));
    float ms_total = 0.f;
    cudaEventElapsedTime(&ms_total, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (int i = 0; i < n && infos; i++) {
        efem_solve_info& f = infos[i];
        std::memset(&f, 0, sizeof(f));
        const Seg& a = sg1[i];
        const Seg& b = sg[i];
        const bool second = mixed && (a.state == kDone || a.state == kStalled);  // ran the FP64 phase
        const bool refined = second && b.n_res > 1;
        f.niter = mixed ? a.k + (refined ? b.k : 0) : b.k;
        f.n_residual_evals = a.n_res + (second ? b.n_res : 0);
        f.n_jacobian_evals = 1;
        f.flags = (b.state == kDone ? EFEM_SOLVE_CONVERGED : 0) | (b.state == kMaxIt ? EFEM_SOLVE_MAX_ITERS : 0)
            | (refined ? EFEM_SOLVE_REFINED : 0) | (b.xinf < ms[i]->opts.dx_criterion ? EFEM_SOLVE_DX_CONVERGED : 0)
            | EFEM_SOLVE_BATCHED;
        f.u_inf = b.xinf;
        f.r_inf = b.rinf;
        f.ms_total = ms_total;  // the whole batch's device time
        f.ms_factor = ms_factor;
        f.n_kernel_launches = launches;
        f.n_precond_applies = f.niter;
    }
    for (int i = 0; i < n; i++)
        if (sg[i].state == kNaN) {
            set_error("model " + std::to_string(i) + ": L-BFGS produced a non-finite residual or solution");
            return EFEM_ERR_NAN;
        }
    return EFEM_OK;
}

}  // namespace efem
