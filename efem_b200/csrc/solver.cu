// L-BFGS solve on the GPU: the reference's solver semantics
// (src/simulation/nlsolver/LBFGS.h:96-174, LBFGSMat.h:59-131,
// LineSearchFEA.h:37-68) with every vector operation on the device.
//
// Vector work is done by grid-stride kernels; dot products and max-norms use a
// deterministic two-level reduction (per-CTA partials, the last CTA to finish
// combines them in a fixed order), so results are bitwise repeatable.  The
// L-BFGS scalars (alpha_j, ys_j, theta) live in device memory and are produced
// and consumed by kernels without host round trips.  The only host reads are
// the three line-search scalars (r.d, ||r||_inf, ||x||_inf) after each residual
// evaluation, which drive the reference's accept / scale decision.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "efem_internal.h"

namespace efem {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 296;  // 2 x 148 SMs

// device-resident solver scalars
struct Scalars {
    double dg, rinf, xinf;   // line-search reads (slots 0..2, read by the host)
    double x2;               // ||x||_2^2
    double dg0;
    double theta;
    double yy;
    double tmp;
    double ys[64];
    double alpha[64];
    double coef[64];
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
            double x = lane < kThreads / 32 ? sh[k][lane] : (ops[k] ? 0.0 : 0.0);
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

__global__ void k_scale(double* v, double s, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) v[i] *= s;
}

// x = xp + step d
__global__ void k_trial(double* __restrict__ x, const double* __restrict__ xp, const double* __restrict__ d, double step, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        x[i] = xp[i] + step * d[i];
}

// line-search scalars: dg = r.d, rinf = ||r||_inf, xinf = ||x||_inf, x2 = ||x||^2
__global__ void __launch_bounds__(kThreads) k_ls_reduce(const double* __restrict__ r, const double* __restrict__ d,
    const double* __restrict__ x, size_t n, Scalars* S, double* partials)
{
    double v[4] = { 0, 0, 0, 0 };
    const int ops[4] = { 0, 1, 1, 0 };
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
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
    }
}

// dg0 = r.d (the line search's initial projection) and xp = x, rp = r
__global__ void __launch_bounds__(kThreads) k_ls_begin(const double* __restrict__ r, const double* __restrict__ d,
    const double* __restrict__ x, double* __restrict__ xp, double* __restrict__ rp, size_t n, Scalars* S,
    double* partials)
{
    double v[1] = { 0 };
    const int ops[1] = { 0 };
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double ri = r[i];
        v[0] += ri * d[i];
        xp[i] = x[i];
        rp[i] = ri;
    }
    block_reduce<1>(v, ops);
    if (grid_finish<1>(v, ops, partials, &S->counter[1])) S->dg0 = v[0];
}

// add_correction: s = x - xp, y = r - rp into history slot loc; ys, theta = yy/ys
__global__ void __launch_bounds__(kThreads) k_correction(const double* __restrict__ x, const double* __restrict__ xp,
    const double* __restrict__ r, const double* __restrict__ rp, double* __restrict__ s, double* __restrict__ y, size_t n,
    int loc, Scalars* S, double* partials)
{
    double v[2] = { 0, 0 };
    const int ops[2] = { 0, 0 };
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double si = x[i] - xp[i], yi = r[i] - rp[i];
        s[i] = si;
        y[i] = yi;
        v[0] += si * yi;
        v[1] += yi * yi;
    }
    block_reduce<2>(v, ops);
    if (grid_finish<2>(v, ops, partials, &S->counter[2])) {
        S->ys[loc] = v[0];
        S->yy = v[1];
        S->theta = v[1] / v[0];
    }
}

// q = a * v (first use) -- here a = -1 and v = r
__global__ void k_neg_copy(double* __restrict__ q, const double* __restrict__ r, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) q[i] = -r[i];
}

// Two-loop step of the first loop, fused with the previous update:
//   q -= alpha[prev] * y_prev   (if prev >= 0),   alpha[j] = s_j . q / ys[j]
__global__ void __launch_bounds__(kThreads) k_loop1(double* __restrict__ q, const double* __restrict__ yprev, int prev,
    const double* __restrict__ sj, int j, size_t n, Scalars* S, double* partials)
{
    const double ap = prev >= 0 ? S->alpha[prev] : 0.0;
    double v[1] = { 0 };
    const int ops[1] = { 0 };
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double qi = q[i];
        if (prev >= 0) {
            qi -= ap * yprev[i];
            q[i] = qi;
        }
        v[0] += sj[i] * qi;
    }
    block_reduce<1>(v, ops);
    if (grid_finish<1>(v, ops, partials, &S->counter[3])) S->alpha[j] = v[0] / S->ys[j];
}

// last update of the first loop, then H0 = I/theta when there is no factor
__global__ void k_loop1_tail(double* __restrict__ q, const double* __restrict__ yprev, int prev, int divide_theta, size_t n,
    const Scalars* S)
{
    const double ap = prev >= 0 ? S->alpha[prev] : 0.0;
    const double it = divide_theta ? 1.0 / S->theta : 1.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double qi = q[i];
        if (prev >= 0) qi -= ap * yprev[i];
        if (divide_theta) qi = qi / S->theta;
        q[i] = qi;
    }
    (void)it;
}

// Second loop step, fused with the previous update:
//   q += coef[prev] * s_prev (if prev >= 0),  coef[j] = alpha[j] - y_j . q / ys[j]
__global__ void __launch_bounds__(kThreads) k_loop2(double* __restrict__ q, const double* __restrict__ sprev, int prev,
    const double* __restrict__ yj, int j, size_t n, Scalars* S, double* partials)
{
    const double cp = prev >= 0 ? S->coef[prev] : 0.0;
    double v[1] = { 0 };
    const int ops[1] = { 0 };
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double qi = q[i];
        if (prev >= 0) {
            qi += cp * sprev[i];
            q[i] = qi;
        }
        v[0] += yj[i] * qi;
    }
    block_reduce<1>(v, ops);
    if (grid_finish<1>(v, ops, partials, &S->counter[4])) S->coef[j] = S->alpha[j] - v[0] / S->ys[j];
}

// d = q + coef[prev] s_prev
__global__ void k_loop2_tail(double* __restrict__ d, const double* __restrict__ q, const double* __restrict__ sprev, int prev,
    size_t n, const Scalars* S)
{
    const double cp = prev >= 0 ? S->coef[prev] : 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        d[i] = prev >= 0 ? q[i] + cp * sprev[i] : q[i];
}

int grid_for(size_t n) { return static_cast<int>(std::min<size_t>(kMaxBlocks, std::max<size_t>(1, (n + kThreads * 4 - 1) / (kThreads * 4)))); }

}  // namespace

// CUDA-event timing of the solve's phases: a pair of events around each
// residual evaluation / H0 application, harvested after the host syncs the
// line search already needs.
struct PhaseTimer {
    static constexpr int kPairs = 32;
    cudaEvent_t ev[2 * kPairs] = {};
    int kind[kPairs] = {};
    int used = 0;
    double acc[2] = { 0, 0 };
    cudaError_t init()
    {
        for (auto& e : ev)
            if (!e) {
                cudaError_t s = cudaEventCreate(&e);
                if (s != cudaSuccess) return s;
            }
        return cudaSuccess;
    }
    void destroy()
    {
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
    int begin(int k, cudaStream_t st)
    {
        if (used == kPairs) return -1;  // pool full: this phase goes unmeasured
        kind[used] = k;
        cudaEventRecord(ev[2 * used], st);
        return used++;
    }
    void end(int slot, cudaStream_t st)
    {
        if (slot >= 0) cudaEventRecord(ev[2 * slot + 1], st);
    }
    void harvest()  // call only after the stream has been synchronised
    {
        for (int i = 0; i < used; i++) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]) == cudaSuccess) acc[kind[i]] += ms;
        }
        used = 0;
    }
};

struct SolverWS {
    PhaseTimer timer;
    size_t n = 0;
    int m = 0;
    double *r = nullptr, *xp = nullptr, *rp = nullptr, *d = nullptr, *q = nullptr;
    double *S = nullptr, *Y = nullptr;
    double* partials = nullptr;
    Scalars* sc = nullptr;
    double* h_read = nullptr;  // pinned
    cudaEvent_t ev[4] = { nullptr, nullptr, nullptr, nullptr };
};

void launch_scale(double* v, double s, size_t n, cudaStream_t st)
{
    k_scale<<<grid_for(n), kThreads, 0, st>>>(v, s, n);
}

void free_solver(Model& m)
{
    if (!m.ws) return;
    SolverWS& w = *m.ws;
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
    w.timer.destroy();
    delete m.ws;
    m.ws = nullptr;
}

static efem_status alloc_ws(Model& m)
{
    const size_t n = 3 * static_cast<size_t>(m.n_free);
    if (m.ws && m.ws->n == n && m.ws->m == m.opts.m) return EFEM_OK;
    free_solver(m);
    if (m.opts.m > 64) {
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
    EFEM_CUDA(w.timer.init());
    return EFEM_OK;
}

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
    EFEM_CUDA(cudaEventRecord(w.ev[0], st));
    float ms_res = 0.f;

    w.timer.used = 0;
    w.timer.acc[0] = w.timer.acc[1] = 0;
    auto residual = [&](const double* xx) -> efem_status {
        info->n_residual_evals++;
        const int t = w.timer.begin(0, st);
        efem_status rs = launch_residual(m, xx, w.r);
        w.timer.end(t, st);
        return rs;
    };
    auto precond = [&](double* v) -> efem_status {
        info->n_precond_applies++;
        const int t = w.timer.begin(1, st);
        efem_status rs = precond_apply(m, v);
        w.timer.end(t, st);
        return rs;
    };
    auto read_ls = [&]() -> efem_status {
        m.launches++;
        k_ls_reduce<<<G, kThreads, 0, st>>>(w.r, w.d, x, n, w.sc, w.partials);
        EFEM_CUDA(cudaMemcpyAsync(w.h_read, w.sc, sizeof(double) * 4, cudaMemcpyDeviceToHost, st));
        EFEM_CUDA(cudaStreamSynchronize(st));
        w.timer.harvest();
        return EFEM_OK;
    };

    // initial residual and early exit (LBFGS.h:110-120); d = 0 so dg = 0 here
    EFEM_CUDA(cudaMemsetAsync(w.d, 0, n * sizeof(double), st));
    if ((s = residual(x)) != EFEM_OK) return s;
    if ((s = read_ls()) != EFEM_OK) return s;
    double rinf = w.h_read[1], xinf = w.h_read[2];
    int k = 1;
    bool converged = false, ok = false;
    if (!(std::isfinite(rinf))) goto nan_exit;
    if (rinf <= eps || rinf <= eps * std::sqrt(w.h_read[3])) {
        converged = true;
        goto done;
    }
    // approximate-Jacobian factor, once (LBFGS.h:122-124)
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
    m.launches++;
    k_neg_copy<<<G, kThreads, 0, st>>>(w.d, w.r, n);
    if (ok && (s = precond(w.d)) != EFEM_OK) return s;
    {
        int ncorr = 0, ptr = mm;
        for (;;) {
            m.launches++;
            k_ls_begin<<<G, kThreads, 0, st>>>(w.r, w.d, x, w.xp, w.rp, n, w.sc, w.partials);
            EFEM_CUDA(cudaMemcpyAsync(w.h_read + 4, &w.sc->dg0, sizeof(double), cudaMemcpyDeviceToHost, st));
            // residual-projection line search (LineSearchFEA.h:43-67); dg0 is read
            // together with the first trial's scalars
            double step = 1.0;
            for (int it = 0; it < m.opts.max_linesearch; it++) {
                m.launches++;
                k_trial<<<G, kThreads, 0, st>>>(x, w.xp, w.d, step, n);
                if ((s = residual(x)) != EFEM_OK) return s;
                if ((s = read_ls()) != EFEM_OK) return s;
                const double dg = w.h_read[0], dg0 = w.h_read[4];
                if (std::fabs(dg) <= std::fabs(dg0)) break;
                step *= dg * dg0 > 0 ? 1.5 : 0.5;
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
            // add_correction (LBFGSMat.h:81-98)
            const int loc = ptr % mm;
            m.launches++;
            k_correction<<<G, kThreads, 0, st>>>(x, w.xp, w.r, w.rp, w.S + loc * n, w.Y + loc * n, n, loc, w.sc, w.partials);
            if (ncorr < mm) ncorr++;
            ptr = loc + 1;
            // d = -H r, two-loop recursion (LBFGSMat.h:103-131)
            m.launches++;
            k_neg_copy<<<G, kThreads, 0, st>>>(w.q, w.r, n);
            int j = ptr % mm, prev = -1;
            for (int i = 0; i < ncorr; i++) {
                j = (j + mm - 1) % mm;
                m.launches++;
                k_loop1<<<G, kThreads, 0, st>>>(w.q, prev >= 0 ? w.Y + prev * n : nullptr, prev, w.S + j * n, j, n, w.sc, w.partials);
                prev = j;
            }
            m.launches++;
            k_loop1_tail<<<G, kThreads, 0, st>>>(w.q, prev >= 0 ? w.Y + prev * n : nullptr, prev, ok ? 0 : 1, n, w.sc);
            if (ok && (s = precond(w.q)) != EFEM_OK) return s;
            prev = -1;
            for (int i = 0; i < ncorr; i++) {
                m.launches++;
                k_loop2<<<G, kThreads, 0, st>>>(w.q, prev >= 0 ? w.S + prev * n : nullptr, prev, w.Y + j * n, j, n, w.sc, w.partials);
                prev = j;
                j = (j + 1) % mm;
            }
            m.launches++;
            k_loop2_tail<<<G, kThreads, 0, st>>>(w.d, w.q, prev >= 0 ? w.S + prev * n : nullptr, prev, n, w.sc);
            EFEM_CUDA(cudaGetLastError());
            k++;
        }
    }
done:
    EFEM_CUDA(cudaEventRecord(w.ev[1], st));
    EFEM_CUDA(cudaEventSynchronize(w.ev[1]));
    w.timer.harvest();
    {
        float ms = 0;
        cudaEventElapsedTime(&ms, w.ev[0], w.ev[1]);
        info->ms_total = ms;
    }
    info->ms_residual = w.timer.acc[0];
    info->ms_precond = w.timer.acc[1];
    (void)ms_res;
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
    set_error("L-BFGS produced a non-finite residual or solution");
    return EFEM_ERR_NAN;
}

}  // namespace efem
