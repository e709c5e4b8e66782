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
// One iteration's common path -- add_correction, the two-loop recursion with
// H0, the start of the line search, its first trial x = xp + d, the residual
// and the line-search reductions, plus the read-back of five scalars -- is
// captured once as a CUDA graph and replayed, so an iteration costs one graph
// launch and one host wait.  The host then makes the reference's
// accept / scale decision; the rare further trials are launched directly.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>

#include "efem_internal.h"

namespace efem {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 296;  // 2 x 148 SMs
constexpr int kMaxHist = 64;

// device-resident solver state; the first five doubles are read by the host
struct Scalars {
    double dg, rinf, xinf, x2;  // line-search reads (r.d, ||r||_inf, ||x||_inf, ||x||_2^2)
    double dg0;                 // r.d at the start of the line search
    double perr;                // the preconditioner's solve gave up waiting (nonzero)
    double theta;
    double ys[kMaxHist];
    double alpha[kMaxHist];
    double coef[kMaxHist];
    int ptr, ncorr;             // LBFGSMat::m_ptr, m_ncorr
    int ptr_next, ncorr_next;
    unsigned int counter[8];
};

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
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
            acc[k] = ops[k] ? fmax(acc[k], p) : acc[k] + p;
        }
    block_reduce<NV>(acc, ops);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) v[k] = acc[k];
        *counter = 0u;
    }
    return threadIdx.x == 0;
}

#define GRID_STRIDE(i, n) for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

__global__ void k_scale(double* v, double s, size_t n)
{
    GRID_STRIDE(i, n) v[i] *= s;
}

__global__ void k_state_init(Scalars* S, int m)
{
    S->ptr = m;  // makes ptr % m == 0 on the first correction (LBFGSMat.h:68)
    S->ncorr = 0;
    S->theta = 1.0;
}

// x = xp + step d
__global__ void k_trial(double* __restrict__ x, const double* __restrict__ xp, const double* __restrict__ d, double step, size_t n)
{
    GRID_STRIDE(i, n) x[i] = xp[i] + step * d[i];
}

// line-search scalars: dg = r.d, rinf = ||r||_inf, xinf = ||x||_inf, x2 = ||x||^2
__global__ void __launch_bounds__(kThreads) k_ls_reduce(const double* __restrict__ r, const double* __restrict__ d,
    const double* __restrict__ x, size_t n, Scalars* S, double* partials, const int* perr)
{
    double v[4] = { 0, 0, 0, 0 };
    const int ops[4] = { 0, 1, 1, 0 };
    GRID_STRIDE(i, n)
    {
        const double ri = r[i], xi = x[i];
        v[0] += ri * d[i];
        v[1] = fmax(v[1], fabs(ri));
        v[2] = fmax(v[2], fabs(xi));
        v[3] += xi * xi;
    }
    block_reduce<4>(v, ops);
    if (grid_finish<4>(v, ops, partials, &S->counter[0])) {
        S->dg = v[0];
        S->rinf = v[1];
        S->xinf = v[2];
        S->x2 = v[3];
        S->perr = perr ? static_cast<double>(*perr) : 0.0;
    }
}

// dg0 = r.d (the line search's initial projection) and xp = x, rp = r
__global__ void __launch_bounds__(kThreads) k_ls_begin(const double* __restrict__ r, const double* __restrict__ d,
    const double* __restrict__ x, double* __restrict__ xp, double* __restrict__ rp, size_t n, Scalars* S,
    double* partials)
{
    double v[1] = { 0 };
    const int ops[1] = { 0 };
    GRID_STRIDE(i, n)
    {
        const double ri = r[i];
        v[0] += ri * d[i];
        xp[i] = x[i];
        rp[i] = ri;
    }
    block_reduce<1>(v, ops);
    if (grid_finish<1>(v, ops, partials, &S->counter[1])) S->dg0 = v[0];
}

// add_correction (LBFGSMat.h:81-98): s = x - xp, y = r - rp into slot ptr % m;
// ys, theta = yy/ys; the new pointer and count take effect in k_advance_neg.
__global__ void __launch_bounds__(kThreads) k_correction(const double* __restrict__ x, const double* __restrict__ xp,
    const double* __restrict__ r, const double* __restrict__ rp, double* __restrict__ Sh, double* __restrict__ Yh,
    size_t n, int m, Scalars* S, double* partials)
{
    const int loc = S->ptr % m;
    double* s = Sh + loc * n;
    double* y = Yh + loc * n;
    double v[2] = { 0, 0 };
    const int ops[2] = { 0, 0 };
    GRID_STRIDE(i, n)
    {
        const double si = x[i] - xp[i], yi = r[i] - rp[i];
        s[i] = si;
        y[i] = yi;
        v[0] += si * yi;
        v[1] += yi * yi;
    }
    block_reduce<2>(v, ops);
    if (grid_finish<2>(v, ops, partials, &S->counter[2])) {
        S->ys[loc] = v[0];
        S->theta = v[1] / v[0];
        S->ptr_next = loc + 1;
        S->ncorr_next = S->ncorr < m ? S->ncorr + 1 : m;
    }
}

// commit the new history pointer / count, and start the two-loop with q = -r
__global__ void k_advance_neg(double* __restrict__ q, const double* __restrict__ r, size_t n, Scalars* S)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        S->ptr = S->ptr_next;
        S->ncorr = S->ncorr_next;
    }
    GRID_STRIDE(i, n) q[i] = -r[i];
}

__global__ void k_neg_copy(double* __restrict__ q, const double* __restrict__ r, size_t n)
{
    GRID_STRIDE(i, n) q[i] = -r[i];
}

// first loop, step i (newest history first), fused with step i-1's update:
//   q -= alpha[j_{i-1}] y_{j_{i-1}};  alpha[j_i] = s_{j_i} . q / ys[j_i]
// j_i = (ptr - 1 - i) mod m; a step beyond ncorr does nothing
__global__ void __launch_bounds__(kThreads) k_loop1(double* __restrict__ q, const double* __restrict__ Sh,
    const double* __restrict__ Yh, int i, int m, size_t n, Scalars* S, double* partials)
{
    const int ncorr = S->ncorr, ptr = S->ptr;
    if (i >= ncorr) return;
    const int j = ((ptr - 1 - i) % m + m) % m;
    const int jp = ((ptr - i) % m + m) % m;
    const double ap = i > 0 ? S->alpha[jp] : 0.0;
    const double* yp = Yh + jp * n;
    const double* sj = Sh + j * n;
    double v[1] = { 0 };
    const int ops[1] = { 0 };
    GRID_STRIDE(t, n)
    {
        double qi = q[t];
        if (i > 0) {
            qi -= ap * yp[t];
            q[t] = qi;
        }
        v[0] += sj[t] * qi;
    }
    block_reduce<1>(v, ops);
    if (grid_finish<1>(v, ops, partials, &S->counter[3])) S->alpha[j] = v[0] / S->ys[j];
}

// last update of the first loop; H0 = I/theta when there is no factor
__global__ void k_loop1_tail(double* __restrict__ q, const double* __restrict__ Yh, int m, int divide_theta, size_t n,
    const Scalars* S)
{
    const int ncorr = S->ncorr, ptr = S->ptr;
    const int jl = ((ptr - ncorr) % m + m) % m;  // j of step ncorr - 1 (the oldest)
    const double al = ncorr > 0 ? S->alpha[jl] : 0.0;
    const double* yl = Yh + jl * n;
    const double th = S->theta;
    GRID_STRIDE(t, n)
    {
        double qi = q[t];
        if (ncorr > 0) qi -= al * yl[t];
        if (divide_theta) qi = qi / th;
        q[t] = qi;
    }
}

// second loop, step i (oldest first), fused with step i-1's update:
//   q += coef[j_{i-1}] s_{j_{i-1}};  coef[j_i] = alpha[j_i] - y_{j_i} . q / ys[j_i]
// j_i = (ptr - ncorr + i) mod m
__global__ void __launch_bounds__(kThreads) k_loop2(double* __restrict__ q, const double* __restrict__ Sh,
    const double* __restrict__ Yh, int i, int m, size_t n, Scalars* S, double* partials)
{
    const int ncorr = S->ncorr, ptr = S->ptr;
    if (i >= ncorr) return;
    const int j = ((ptr - ncorr + i) % m + m) % m;
    const int jp = ((ptr - ncorr + i - 1) % m + m) % m;
    const double cp = i > 0 ? S->coef[jp] : 0.0;
    const double* sp = Sh + jp * n;
    const double* yj = Yh + j * n;
    double v[1] = { 0 };
    const int ops[1] = { 0 };
    GRID_STRIDE(t, n)
    {
        double qi = q[t];
        if (i > 0) {
            qi += cp * sp[t];
            q[t] = qi;
        }
        v[0] += yj[t] * qi;
    }
    block_reduce<1>(v, ops);
    if (grid_finish<1>(v, ops, partials, &S->counter[4])) S->coef[j] = S->alpha[j] - v[0] / S->ys[j];
}

// d = q + coef[j_last] s_{j_last}, j_last the newest slot
__global__ void k_loop2_tail(double* __restrict__ d, const double* __restrict__ q, const double* __restrict__ Sh, int m,
    size_t n, const Scalars* S)
{
    const int ncorr = S->ncorr, ptr = S->ptr;
    const int jl = ((ptr - 1) % m + m) % m;
    const double cl = ncorr > 0 ? S->coef[jl] : 0.0;
    const double* sl = Sh + jl * n;
    GRID_STRIDE(t, n) d[t] = ncorr > 0 ? q[t] + cl * sl[t] : q[t];
}

int grid_for(size_t n) { return static_cast<int>(std::min<size_t>(kMaxBlocks, std::max<size_t>(1, (n + kThreads * 4 - 1) / (kThreads * 4)))); }

}  // namespace

struct SolverWS {
    size_t n = 0;
    int m = 0;
    double *r = nullptr, *xp = nullptr, *rp = nullptr, *d = nullptr, *q = nullptr;
    double *S = nullptr, *Y = nullptr;
    double* partials = nullptr;
    Scalars* sc = nullptr;
    double* h_read = nullptr;  // pinned: the five line-search scalars
    cudaEvent_t ev[2] = { nullptr, nullptr };
    // event pairs around the residual and H0, recorded inside the graphs too
    cudaEvent_t gev[4] = { nullptr, nullptr, nullptr, nullptr };
    cudaStream_t capture = nullptr;
    struct Graphs {
        cudaGraphExec_t first = nullptr;  // line-search start + first trial (iteration 1)
        cudaGraphExec_t body = nullptr;   // correction + two-loop + H0 + line-search start + first trial
    };
    std::map<std::pair<double*, int>, Graphs> graphs;  // per (solution pointer, configuration)
    long long epoch = -1;                                // Model::epoch the graphs were captured at
};

void launch_scale(double* v, double s, size_t n, cudaStream_t st)
{
    k_scale<<<grid_for(n), kThreads, 0, st>>>(v, s, n);
}

static void drop_graphs(SolverWS& w)
{
    for (auto& kv : w.graphs) {
        if (kv.second.first) cudaGraphExecDestroy(kv.second.first);
        if (kv.second.body) cudaGraphExecDestroy(kv.second.body);
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
    if (w.sc) cudaFree(w.sc);
    if (w.h_read) cudaFreeHost(w.h_read);
    for (auto& e : w.ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : w.gev)
        if (e) cudaEventDestroy(e);
    if (w.capture) cudaStreamDestroy(w.capture);
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
    if ((s = dev_alloc(&w.partials, static_cast<size_t>(kMaxBlocks) * 4)) != EFEM_OK) return s;
    EFEM_CUDA(cudaMalloc(&w.sc, sizeof(Scalars)));
    EFEM_CUDA(cudaMemset(w.sc, 0, sizeof(Scalars)));
    EFEM_CUDA(cudaMallocHost(&w.h_read, sizeof(double) * 8));
    for (auto& e : w.ev) EFEM_CUDA(cudaEventCreate(&e));
    for (auto& e : w.gev) EFEM_CUDA(cudaEventCreate(&e));
    EFEM_CUDA(cudaStreamCreateWithFlags(&w.capture, cudaStreamNonBlocking));
    return EFEM_OK;
}

namespace {

// one line-search trial with step 1 (after xp = x, rp = r, dg0 = r.d), its
// residual and reductions, and the scalar read-back
efem_status enqueue_first_trial(Model& m, SolverWS& w, double* x, cudaStream_t st)
{
    const size_t n = w.n;
    const int G = grid_for(n);
    k_ls_begin<<<G, kThreads, 0, st>>>(w.r, w.d, x, w.xp, w.rp, n, w.sc, w.partials);
    k_trial<<<G, kThreads, 0, st>>>(x, w.xp, w.d, 1.0, n);
    EFEM_CUDA(cudaEventRecordWithFlags(w.gev[0], st, cudaEventRecordExternal));
    efem_status s = launch_residual_on(m, x, w.r, st);
    if (s != EFEM_OK) return s;
    EFEM_CUDA(cudaEventRecordWithFlags(w.gev[1], st, cudaEventRecordExternal));
    k_ls_reduce<<<G, kThreads, 0, st>>>(w.r, w.d, x, n, w.sc, w.partials, precond_error_flag(m));
    EFEM_CUDA(cudaMemcpyAsync(w.h_read, w.sc, sizeof(double) * 6, cudaMemcpyDeviceToHost, st));
    return EFEM_OK;
}

// add_correction + two-loop + H0, leaving the new direction in w.d
efem_status enqueue_direction(Model& m, SolverWS& w, double* x, bool use_factor, cudaStream_t st)
{
    const size_t n = w.n;
    const int G = grid_for(n), mm = w.m;
    k_correction<<<G, kThreads, 0, st>>>(x, w.xp, w.r, w.rp, w.S, w.Y, n, mm, w.sc, w.partials);
    k_advance_neg<<<G, kThreads, 0, st>>>(w.q, w.r, n, w.sc);
    for (int i = 0; i < mm; i++) k_loop1<<<G, kThreads, 0, st>>>(w.q, w.S, w.Y, i, mm, n, w.sc, w.partials);
    k_loop1_tail<<<G, kThreads, 0, st>>>(w.q, w.Y, mm, use_factor ? 0 : 1, n, w.sc);
    if (use_factor) {
        EFEM_CUDA(cudaEventRecordWithFlags(w.gev[2], st, cudaEventRecordExternal));
        efem_status s = precond_enqueue(m, w.q, st);
        if (s != EFEM_OK) return s;
        EFEM_CUDA(cudaEventRecordWithFlags(w.gev[3], st, cudaEventRecordExternal));
    }
    for (int i = 0; i < mm; i++) k_loop2<<<G, kThreads, 0, st>>>(w.q, w.S, w.Y, i, mm, n, w.sc, w.partials);
    k_loop2_tail<<<G, kThreads, 0, st>>>(w.d, w.q, w.S, mm, n, w.sc);
    return EFEM_OK;
}

efem_status capture(Model& m, SolverWS& w, double* x, bool use_factor, bool with_direction, cudaGraphExec_t* out)
{
    const long long launches = m.launches;  // capture launches nothing; replays are counted
    cudaGraph_t g = nullptr;
    EFEM_CUDA(cudaStreamBeginCapture(w.capture, cudaStreamCaptureModeThreadLocal));
    efem_status s = EFEM_OK;
    if (with_direction) s = enqueue_direction(m, w, x, use_factor, w.capture);
    if (s == EFEM_OK) s = enqueue_first_trial(m, w, x, w.capture);
    const cudaError_t e = cudaStreamEndCapture(w.capture, &g);
    m.launches = launches;
    if (s != EFEM_OK) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess) {
        set_error(std::string("graph capture: ") + cudaGetErrorString(e));
        return EFEM_ERR_CUDA;
    }
    EFEM_CUDA(cudaGraphInstantiate(out, g, 0));
    cudaGraphDestroy(g);
    return EFEM_OK;
}

double elapsed_ms(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0.f;
    return cudaEventElapsedTime(&ms, a, b) == cudaSuccess ? static_cast<double>(ms) : 0.0;
}

}  // namespace

efem_status run_solve(Model& m, double* x, efem_solve_info* info)
{
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
    const long long per_res = 1 + static_cast<long long>(m.blocks.size() + m.faces.size());
    double ms_res = 0.0, ms_pc = 0.0;
    double rinf = 0.0, xinf = 0.0;
    int k = 1;
    bool converged = false, ok = false;
    EFEM_CUDA(cudaEventRecord(w.ev[0], st));

    // direct (non-graph) line-search trial: x = xp + step d (step 0: x as is),
    // residual, reductions, read-back
    auto direct_trial = [&](double step) -> efem_status {
        if (step != 0.0) {
            k_trial<<<G, kThreads, 0, st>>>(x, w.xp, w.d, step, n);
            m.launches++;
        }
        EFEM_CUDA(cudaEventRecord(w.gev[0], st));
        efem_status rs = launch_residual_on(m, x, w.r, st);
        if (rs != EFEM_OK) return rs;
        EFEM_CUDA(cudaEventRecord(w.gev[1], st));
        info->n_residual_evals++;
        k_ls_reduce<<<G, kThreads, 0, st>>>(w.r, w.d, x, n, w.sc, w.partials, precond_error_flag(m));
        m.launches++;
        EFEM_CUDA(cudaMemcpyAsync(w.h_read, w.sc, sizeof(double) * 6, cudaMemcpyDeviceToHost, st));
        EFEM_CUDA(cudaStreamSynchronize(st));
        ms_res += elapsed_ms(w.gev[0], w.gev[1]);
        return EFEM_OK;
    };

    // initial residual and early exit (LBFGS.h:110-120); d = 0 so dg = 0 here
    EFEM_CUDA(cudaMemsetAsync(w.d, 0, n * sizeof(double), st));
    k_state_init<<<1, 1, 0, st>>>(w.sc, mm);
    m.launches++;
    if ((s = direct_trial(0.0)) != EFEM_OK) return s;
    rinf = w.h_read[1];
    xinf = w.h_read[2];
    if (!(std::isfinite(rinf))) goto nan_exit;
    if (rinf <= eps || rinf <= eps * std::sqrt(w.h_read[3])) {
        converged = true;
        goto done;
    }
    // approximate-Jacobian factor, once per solve (LBFGS.h:122-124)
    if (m.opts.nl_solver == 0) {
        int okf = 0;
        double msf = 0;
        if ((s = precond_setup(m, true, &okf, &msf)) != EFEM_OK) return s;
        ok = okf != 0;
        info->n_jacobian_evals = 1;
        info->ms_factor = msf;
        if (!ok) info->flags |= EFEM_SOLVE_PRECOND_FALLBACK;
    }
    // initial direction d = -H0 r
    k_neg_copy<<<G, kThreads, 0, st>>>(w.d, w.r, n);
    m.launches++;
    if (ok) {
        EFEM_CUDA(cudaEventRecord(w.gev[2], st));
        if ((s = precond_apply(m, w.d)) != EFEM_OK) return s;
        EFEM_CUDA(cudaEventRecord(w.gev[3], st));
        EFEM_CUDA(cudaStreamSynchronize(st));
        ms_pc += elapsed_ms(w.gev[2], w.gev[3]);
        info->n_precond_applies++;
    }
    {
        if (w.epoch != m.epoch) {  // blocks or factor rebuilt since the graphs were captured
            drop_graphs(w);
            w.epoch = m.epoch;
        }
        const auto key = std::make_pair(x, (ok ? 1 : 0) | (m.opts.precision << 1));
        if (!w.graphs.count(key) && w.graphs.size() >= 8) drop_graphs(w);  // many distinct solution pointers
        SolverWS::Graphs& gr = w.graphs[key];
        if (!gr.first) {
            if ((s = capture(m, w, x, ok, false, &gr.first)) != EFEM_OK) return s;
            if ((s = capture(m, w, x, ok, true, &gr.body)) != EFEM_OK) return s;
        }
        const long long per_dir = 5 + 2LL * mm + (ok ? precond_launch_count(m) : 0);
        bool first = true;
        for (;;) {
            // common path: one graph launch, one wait
            EFEM_CUDA(cudaGraphLaunch(first ? gr.first : gr.body, st));
            EFEM_CUDA(cudaStreamSynchronize(st));
            m.launches += 3 + per_res + (first ? 0 : per_dir);
            ms_res += elapsed_ms(w.gev[0], w.gev[1]);
            if (!first && ok) {
                ms_pc += elapsed_ms(w.gev[2], w.gev[3]);
                info->n_precond_applies++;
            }
            info->n_residual_evals++;
            first = false;
            // residual-projection line search (LineSearchFEA.h:43-67); trial 1 done
            const double dg0 = w.h_read[4];
            double dg = w.h_read[0], step = 1.0;
            for (int it = 1; it < m.opts.max_linesearch && !(std::fabs(dg) <= std::fabs(dg0)); it++) {
                step *= dg * dg0 > 0 ? 1.5 : 0.5;
                if ((s = direct_trial(step)) != EFEM_OK) return s;
                dg = w.h_read[0];
            }
            rinf = w.h_read[1];
            xinf = w.h_read[2];
            if (!std::isfinite(rinf) || !std::isfinite(xinf)) goto nan_exit;
            if (rinf <= eps || rinf <= eps * xinf) {
                converged = true;
                break;
            }
            if (m.opts.max_iterations != 0 && k >= m.opts.max_iterations) {
                info->flags |= EFEM_SOLVE_MAX_ITERS;
                break;
            }
            k++;
        }
    }
done:
    EFEM_CUDA(cudaEventRecord(w.ev[1], st));
    EFEM_CUDA(cudaEventSynchronize(w.ev[1]));
    info->ms_total = elapsed_ms(w.ev[0], w.ev[1]);
    info->ms_residual = ms_res;
    info->ms_precond = ms_pc;
    info->niter = k;
    info->u_inf = xinf;
    info->r_inf = rinf;
    info->n_kernel_launches = m.launches - launches0;
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
    info->n_kernel_launches = m.launches - launches0;
    set_error("L-BFGS produced a non-finite residual or solution");
    return EFEM_ERR_NAN;
}

}  // namespace efem
