// Residual R(u) = f_int(u) - f_ext(u) on the GPU.
//
//   element internal force   r_e = V_e sum_g w_g P(F_g) T_g
//                            (src/fe/ElementConstraint.cpp:139-162)
//   follower pressure        f_i = p sum_g w_g N_i(xi_g) cof(F_g) A0, r_i -= f_i
//   directed pressure        f_i = v sum_g w_g N_i(xi_g) |cof(F_g) A0|
//                            (src/fe/ExternalConstraint.cpp:829-959)
//   nodal forces             r starts from -f_ext (:149-167)
//
// Element kernel: one CTA processes EPB elements in three phases.
//   1. stage: threads (element, node) load conn (SoA, coalesced over elements)
//      and gather u, relative to the element's first node, into shared memory;
//   2. Gauss point: thread (element, gp) forms H = (u . dN) J0^{-1}, P(I+H) and
//      S_g = V_e w_g P J0^{-T} (3x3) into shared memory;
//   3. node: thread (element, node) reduces r_a = sum_g S_g dN_ga and adds it
//      to the global residual with FP64 atomics (red.global.add.f64) or, in
//      deterministic mode (opts.deterministic), stores it in its own slot of a
//      contribution buffer that k_gather then sums per node in ascending slot
//      order, so the residual is bitwise repeatable.
// The arithmetic type T is double (FP64 path) or float (mixed path); the
// global residual is always accumulated in FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <vector>

#include "efem_internal.h"
#include "mechanics.cuh"

namespace efem {

namespace {

constexpr int kBlock = 128;

template <typename T>
struct ElemArgs {
    int n, n_free;
    const int* __restrict__ conn;     // [NEN][n]
    const int* __restrict__ mat;      // [n]
    const T* __restrict__ vol;        // [n]
    const T* __restrict__ J0inv;      // [n][NGP][9]
    const T* __restrict__ dN;         // [NGP][NEN][3]
    const T* __restrict__ gw;         // [NGP]
    const MatParams<T>* __restrict__ mats;
    const double* __restrict__ u;     // [3*n_free]
    double* __restrict__ r;           // [3*n_free]
    double* __restrict__ contrib;     // deterministic scatter: [3][n_slots], or null for atomics
    size_t n_slots, slot0;
    const int* __restrict__ egroup;   // batch unions: the member of every element
    const int* frozen;                // batch unions: 1 for a member that no longer iterates (null: none)
};

// where an (element or face, node) pair's nodal force goes
struct Scatter {
    double* contrib = nullptr;
    size_t n_slots = 0, slot0 = 0;
};

// BLK threads per CTA (64, 128 or 256, picked per element block by the
// autotuner in tune_element_blocks); EPB = BLK / NGP elements per CTA, at
// most 128 (shared memory)
template <int NGP, int BLK>
constexpr int elems_per_cta() { return (BLK / NGP) < 1 ? 1 : ((BLK / NGP) > 128 ? 128 : BLK / NGP); }

// MT: the block's one material law, or -1 when its elements mix laws
template <int NEN, int NGP, typename T, int BLK, int MT>
__global__ void __launch_bounds__(BLK) k_elem_residual(ElemArgs<T> a)
{
    griddep_wait();
    constexpr int EPB = elems_per_cta<NGP, BLK>();
    // per-element rows padded to an odd length, so that threads on
    // consecutive elements (phases 1 and 3) or Gauss points (phase 2) read
    // different shared-memory banks
    constexpr int SU = (NEN * 3) | 1, SS = (NGP * 9) | 1, SD = (NEN * 3) | 1, SN = NEN | 1;
    __shared__ T s_u[EPB][SU];     // [element][node * 3 + component]
    __shared__ T s_S[EPB][SS];     // [element][gp * 9 + 3 i + j]
    __shared__ T s_dN[NGP][SD];    // [gp][node * 3 + k]
    __shared__ int s_node[EPB][SN];

    const int tid = threadIdx.x;
    const int e0 = blockIdx.x * EPB;
    if (a.frozen) {  // a batch union: skip the CTA when every member it covers has stopped iterating
        const int e1 = min(a.n, e0 + EPB) - 1;
        bool act = false;
        for (int g = __ldg(a.egroup + e0); g <= __ldg(a.egroup + e1); g++) act = act || !a.frozen[g];
        if (!act) {
            griddep_launch();
            return;
        }
    }
    for (int i = tid; i < NGP * NEN * 3; i += BLK) s_dN[i / (NEN * 3)][i % (NEN * 3)] = a.dN[i];

    // phase 1: stage node displacements relative to the element's first node,
    // formed in FP64 (H only sees differences, since sum_a dN_a = 0, and FP32
    // would lose the differences of nearly equal displacements)
    for (int i = tid; i < EPB * NEN; i += BLK) {
        const int el = i % EPB, nd = i / EPB, e = e0 + el;
        int node = a.n_free;  // out-of-range marker
        T v0 = 0, v1 = 0, v2 = 0;
        if (e < a.n) {
            node = __ldg(a.conn + static_cast<size_t>(nd) * a.n + e);
            const int n0 = __ldg(a.conn + e);
            double w0 = 0.0, w1 = 0.0, w2 = 0.0, z0 = 0.0, z1 = 0.0, z2 = 0.0;
            if (node < a.n_free) {
                w0 = __ldg(a.u + 3 * node);
                w1 = __ldg(a.u + 3 * node + 1);
                w2 = __ldg(a.u + 3 * node + 2);
            }
            if (n0 < a.n_free) {
                z0 = __ldg(a.u + 3 * n0);
                z1 = __ldg(a.u + 3 * n0 + 1);
                z2 = __ldg(a.u + 3 * n0 + 2);
            }
            v0 = static_cast<T>(w0 - z0);
            v1 = static_cast<T>(w1 - z1);
            v2 = static_cast<T>(w2 - z2);
        }
        s_node[el][nd] = node;
        s_u[el][3 * nd] = v0;
        s_u[el][3 * nd + 1] = v1;
        s_u[el][3 * nd + 2] = v2;
    }
    __syncthreads();

    // phase 2: one thread per (element, Gauss point)
    if (tid < EPB * NGP) {
        const int el = tid / NGP, g = tid % NGP, e = e0 + el;
        if (e < a.n) {
            T A[9];
#pragma unroll
            for (int k = 0; k < 9; k++) A[k] = 0;
#pragma unroll 4
            for (int q = 0; q < NEN; q++) {
                const T u0 = s_u[el][3 * q], u1 = s_u[el][3 * q + 1], u2 = s_u[el][3 * q + 2];
                const T d0 = s_dN[g][3 * q], d1 = s_dN[g][3 * q + 1], d2 = s_dN[g][3 * q + 2];
                A[0] += u0 * d0; A[1] += u0 * d1; A[2] += u0 * d2;
                A[3] += u1 * d0; A[4] += u1 * d1; A[5] += u1 * d2;
                A[6] += u2 * d0; A[7] += u2 * d1; A[8] += u2 * d2;
            }
            const T* Jp = a.J0inv + (static_cast<size_t>(e) * NGP + g) * 9;
            T H[9];
            {
                T Ji[9];
#pragma unroll
                for (int k = 0; k < 9; k++) Ji[k] = __ldg(Jp + k);
#pragma unroll
                for (int i = 0; i < 3; i++)
#pragma unroll
                    for (int j = 0; j < 3; j++)
                        H[3 * i + j] = A[3 * i] * Ji[j] + A[3 * i + 1] * Ji[3 + j] + A[3 * i + 2] * Ji[6 + j];
            }
            const MatParams<T> mp = a.mats[__ldg(a.mat + e)];
            T P[9];
            piola<T, MT>(mp, H, P);
            const T wv = __ldg(a.vol + e) * a.gw[g];
            // S = wv P J0^{-T}; J0^{-1} read again (an L1 hit) rather than
            // kept in registers through the stress law
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const T j0 = __ldg(Jp + 3 * j), j1 = __ldg(Jp + 3 * j + 1), j2 = __ldg(Jp + 3 * j + 2);
#pragma unroll
                for (int i = 0; i < 3; i++) s_S[el][9 * g + 3 * i + j] = wv * (P[3 * i] * j0 + P[3 * i + 1] * j1 + P[3 * i + 2] * j2);
            }
        }
    }
    __syncthreads();

    // phase 3: one thread per (element, node): r_a = sum_g S_g dN_ga
    for (int i = tid; i < EPB * NEN; i += BLK) {
        const int el = i % EPB, nd = i / EPB, e = e0 + el;
        if (e >= a.n) continue;
        const int node = s_node[el][nd];
        if (node >= a.n_free) continue;
        T r0 = 0, r1 = 0, r2 = 0;
#pragma unroll 4
        for (int g = 0; g < NGP; g++) {
            const T d0 = s_dN[g][3 * nd], d1 = s_dN[g][3 * nd + 1], d2 = s_dN[g][3 * nd + 2];
            const T* S = &s_S[el][9 * g];
            r0 += S[0] * d0 + S[1] * d1 + S[2] * d2;
            r1 += S[3] * d0 + S[4] * d1 + S[5] * d2;
            r2 += S[6] * d0 + S[7] * d1 + S[8] * d2;
        }
        if (a.contrib) {  // consecutive threads: consecutive elements, consecutive slots
            const size_t sl = a.slot0 + static_cast<size_t>(nd) * a.n + e;
            a.contrib[sl] = static_cast<double>(r0);
            a.contrib[a.n_slots + sl] = static_cast<double>(r1);
            a.contrib[2 * a.n_slots + sl] = static_cast<double>(r2);
        } else {
            atomicAdd(a.r + 3 * node, static_cast<double>(r0));
            atomicAdd(a.r + 3 * node + 1, static_cast<double>(r1));
            atomicAdd(a.r + 3 * node + 2, static_cast<double>(r2));
        }
    }
    griddep_launch();
}

template <typename T>
struct FaceArgs {
    int n, n_free;
    const int* __restrict__ conn;     // [NEN][n]
    const int* __restrict__ table;    // [n]
    const double* __restrict__ A0;    // [n][3]
    const T* __restrict__ J0inv;      // [n][MAX_FGP][9]
    const double* __restrict__ load;  // [n][4]
    const int* __restrict__ t_ngp;
    const T* __restrict__ t_w;        // [t][MAX_FGP]
    const T* __restrict__ t_N;        // [t][MAX_FGP][NEN]
    const T* __restrict__ t_dN;       // [t][MAX_FGP][NEN][3]
    const double* __restrict__ u;
    double* __restrict__ r;
    double* __restrict__ contrib;     // deterministic scatter: [3][n_slots], or null for atomics
    size_t n_slots, slot0;
};

// One thread per face: cof(F_g) A0 at every face point, then the nodal forces
// of all element nodes.
template <int NEN, typename T>
__global__ void __launch_bounds__(kBlock) k_face_residual(FaceArgs<T> a)
{
    griddep_wait();
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= a.n) return;
    const int t = a.table[f];
    const int ngp = a.t_ngp[t];
    int node[NEN];
    T uu[NEN][3];
    double u0[3] = { 0.0, 0.0, 0.0 };  // displacements relative to the parent's first node, as in the element kernel
    {
        const int n0 = a.conn[f];
        if (n0 < a.n_free)
            for (int c = 0; c < 3; c++) u0[c] = a.u[3 * n0 + c];
    }
#pragma unroll
    for (int q = 0; q < NEN; q++) {
        node[q] = a.conn[static_cast<size_t>(q) * a.n + f];
        const bool fr = node[q] < a.n_free;
        uu[q][0] = static_cast<T>((fr ? a.u[3 * node[q]] : 0.0) - u0[0]);
        uu[q][1] = static_cast<T>((fr ? a.u[3 * node[q] + 1] : 0.0) - u0[1]);
        uu[q][2] = static_cast<T>((fr ? a.u[3 * node[q] + 2] : 0.0) - u0[2]);
    }
    const T A0[3] = { static_cast<T>(a.A0[3 * f]), static_cast<T>(a.A0[3 * f + 1]), static_cast<T>(a.A0[3 * f + 2]) };
    const bool directed = a.load[4 * f] != 0.0;
    T cA[MAX_FGP][3];
    for (int g = 0; g < ngp; g++) {
        const T* dN = a.t_dN + (static_cast<size_t>(t) * MAX_FGP + g) * NEN * 3;
        T A[9] = { 0, 0, 0, 0, 0, 0, 0, 0, 0 };
        for (int q = 0; q < NEN; q++)
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int k = 0; k < 3; k++) A[3 * i + k] += uu[q][i] * dN[3 * q + k];
        const T* Ji = a.J0inv + (static_cast<size_t>(f) * MAX_FGP + g) * 9;
        T H[9];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) H[3 * i + j] = A[3 * i] * Ji[j] + A[3 * i + 1] * Ji[3 + j] + A[3 * i + 2] * Ji[6 + j];
        Kin<T> k;
        kinematics(H, k);
        // cof F A0 = (I + B) A0
#pragma unroll
        for (int i = 0; i < 3; i++)
            cA[g][i] = A0[i] + k.B[3 * i] * A0[0] + k.B[3 * i + 1] * A0[1] + k.B[3 * i + 2] * A0[2];
        if (directed) {
            const T nrm = sqrt(cA[g][0] * cA[g][0] + cA[g][1] * cA[g][1] + cA[g][2] * cA[g][2]);
            cA[g][0] = nrm;
        }
    }
    const double* L = a.load + 4 * f;
    for (int q = 0; q < NEN; q++) {
        if (node[q] >= a.n_free) continue;
        T v0 = 0, v1 = 0, v2 = 0;
        for (int g = 0; g < ngp; g++) {
            const T wn = a.t_w[t * MAX_FGP + g] * a.t_N[(static_cast<size_t>(t) * MAX_FGP + g) * NEN + q];
            if (directed) {
                v0 += wn * cA[g][0];
            } else {
                v0 += wn * cA[g][0];
                v1 += wn * cA[g][1];
                v2 += wn * cA[g][2];
            }
        }
        double f0, f1, f2;
        if (directed) {
            f0 = L[1] * static_cast<double>(v0);
            f1 = L[2] * static_cast<double>(v0);
            f2 = L[3] * static_cast<double>(v0);
        } else {
            f0 = L[1] * static_cast<double>(v0);
            f1 = L[1] * static_cast<double>(v1);
            f2 = L[1] * static_cast<double>(v2);
        }
        if (a.contrib) {
            const size_t sl = a.slot0 + static_cast<size_t>(q) * a.n + f;
            a.contrib[sl] = -f0;
            a.contrib[a.n_slots + sl] = -f1;
            a.contrib[2 * a.n_slots + sl] = -f2;
        } else {
            atomicAdd(a.r + 3 * node[q], -f0);
            atomicAdd(a.r + 3 * node[q] + 1, -f1);
            atomicAdd(a.r + 3 * node[q] + 2, -f2);
        }
    }
}

// Deterministic scatter, second half: free node i adds its contributions in
// ascending slot order, r_i += sum_k contrib[gidx[k]], one thread per node
__global__ void __launch_bounds__(kBlock) k_gather(int n_free, const int* __restrict__ gptr,
    const int* __restrict__ gidx, const double* __restrict__ contrib, size_t n_slots, double* __restrict__ r)
{
    griddep_wait();
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= n_free) return;
    double s0 = r[3 * i], s1 = r[3 * i + 1], s2 = r[3 * i + 2];
    for (int k = gptr[i]; k < gptr[i + 1]; k++) {
        const size_t sl = static_cast<size_t>(__ldg(gidx + k));
        s0 += __ldg(contrib + sl);
        s1 += __ldg(contrib + n_slots + sl);
        s2 += __ldg(contrib + 2 * n_slots + sl);
    }
    r[3 * i] = s0;
    r[3 * i + 1] = s1;
    r[3 * i + 2] = s2;
}

template <int NEN, int NGP, typename T, int BLK>
void launch_elem_blk(const ElemArgs<T>& a, int mt, cudaStream_t st)
{
    constexpr int EPB = elems_per_cta<NGP, BLK>();
    const int grid = (a.n + EPB - 1) / EPB;
    switch (mt) {
    case EFEM_NEO_HOOKEAN: launch_k(k_elem_residual<NEN, NGP, T, BLK, EFEM_NEO_HOOKEAN>, grid, BLK, 0, st, a); break;
    case EFEM_MOONEY_RIVLIN: launch_k(k_elem_residual<NEN, NGP, T, BLK, EFEM_MOONEY_RIVLIN>, grid, BLK, 0, st, a); break;
    case EFEM_YEOH: launch_k(k_elem_residual<NEN, NGP, T, BLK, EFEM_YEOH>, grid, BLK, 0, st, a); break;
    default: launch_k(k_elem_residual<NEN, NGP, T, BLK, -1>, grid, BLK, 0, st, a); break;
    }
}

template <int NEN, int NGP, typename T>
void launch_elem(const DevBlock& b, const MatParams<T>* mats, const T* vol, const T* J0, const T* dN, const T* gw,
    int n_free, const double* u, double* r, cudaStream_t st, int threads, const Scatter& sc, const int* frozen)
{
    ElemArgs<T> a { b.n, n_free, b.conn, b.mat, vol, J0, dN, gw, mats, u, r, sc.contrib, sc.n_slots, sc.slot0,
        b.egroup, b.egroup ? frozen : nullptr };
    if (threads == 64) launch_elem_blk<NEN, NGP, T, 64>(a, b.mat_type, st);
    else if (threads == 256) launch_elem_blk<NEN, NGP, T, 256>(a, b.mat_type, st);
    else launch_elem_blk<NEN, NGP, T, 128>(a, b.mat_type, st);
}

template <typename T>
void dispatch_elem(const DevBlock& b, const MatParams<T>* mats, const T* vol, const T* J0, const T* dN, const T* gw,
    int n_free, const double* u, double* r, cudaStream_t st, int threads, const Scatter& sc = Scatter(),
    const int* frozen = nullptr)
{
#define CASE(NEN, NGP)                                                                             \
    if (b.nen == NEN && b.ngp == NGP) {                                                            \
        launch_elem<NEN, NGP, T>(b, mats, vol, J0, dN, gw, n_free, u, r, st, threads, sc, frozen); \
        return;                                                                                    \
    }
    CASE(4, 1)
    CASE(10, 4)
    CASE(10, 1)
    CASE(8, 8)
    CASE(8, 1)
    CASE(20, 27)
    CASE(20, 8)
#undef CASE
}

template <typename T>
void dispatch_face(const DevFaces& f, const T* J0, const T* tw, const T* tN, const T* tdN, int n_free, const double* u,
    double* r, cudaStream_t st, const Scatter& sc)
{
    FaceArgs<T> a { f.n, n_free, f.conn, f.table, f.A0, J0, f.load, f.t_ngp, tw, tN, tdN, u, r, sc.contrib, sc.n_slots,
        sc.slot0 };
    const int grid = (f.n + kBlock - 1) / kBlock;
    switch (f.nen) {
    case 4: launch_k(k_face_residual<4, T>, grid, kBlock, 0, st, a); break;
    case 8: launch_k(k_face_residual<8, T>, grid, kBlock, 0, st, a); break;
    case 10: launch_k(k_face_residual<10, T>, grid, kBlock, 0, st, a); break;
    case 20: launch_k(k_face_residual<20, T>, grid, kBlock, 0, st, a); break;
    }
}

}  // namespace

// Autotuner of the element kernels' CTA size: for every element block and
// both precisions, time the 64-, 128- and 256-thread variants (2 warm-up and
// 5 timed launches each, CUDA events on the model's stream, at u = 0: the
// kernels' work does not depend on the values) and keep the fastest.
// opts.elem_threads = 64 / 128 / 256 forces one variant instead; so does
// deterministic mode (128 unless forced), so that every model and every solve
// runs the same instantiation and the results repeat bitwise whatever the
// timings.
int element_tune_key(const Model& m) { return m.opts.elem_threads | (m.opts.deterministic ? 0x400 : 0); }
efem_status tune_element_blocks(Model& m)
{
    const int forced = m.opts.elem_threads ? m.opts.elem_threads : (m.opts.deterministic ? 128 : 0);
    const size_t n = 3 * static_cast<size_t>(std::max(m.n_free, 1));
    EFEM_CUDA(cudaMemsetAsync(m.d_u, 0, n * sizeof(double), m.stream));
    cudaEvent_t e0, e1;
    EFEM_CUDA(cudaEventCreate(&e0));
    EFEM_CUDA(cudaEventCreate(&e1));
    for (auto& b : m.blocks) {
        for (int prec = 0; prec < 2; prec++) {
            if (forced == 64 || forced == 128 || forced == 256) {
                b.threads[prec] = forced;
                continue;
            }
            if (b.n == 0) {
                b.threads[prec] = 128;
                continue;
            }
            float best = 1e30f;
            for (int t : { 64, 128, 256 }) {
                for (int rep = 0; rep < 7; rep++) {
                    if (rep == 2) EFEM_CUDA(cudaEventRecord(e0, m.stream));
                    if (prec == 1)
                        dispatch_elem<float>(b, m.d_mats_f, b.vol_f, b.J0inv_f, b.dN_f, b.gw_f, m.n_free, m.d_u, m.d_r,
                            m.stream, t);
                    else
                        dispatch_elem<double>(b, m.d_mats, b.vol, b.J0inv, b.dN, b.gw, m.n_free, m.d_u, m.d_r, m.stream, t);
                }
                EFEM_CUDA(cudaEventRecord(e1, m.stream));
                EFEM_CUDA(cudaEventSynchronize(e1));
                float ms = 0.f;
                EFEM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                if (ms < best) {
                    best = ms;
                    b.threads[prec] = t;
                }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    EFEM_CUDA(cudaGetLastError());
    m.tuned_threads = element_tune_key(m);
    return EFEM_OK;
}

efem_status launch_residual(Model& m, const double* d_u, double* d_r)
{
    return launch_residual_on(m, d_u, d_r, m.stream);
}

efem_status launch_residual_on(Model& m, const double* d_u, double* d_r, cudaStream_t stream,
    unsigned long long* stamp, bool init_r)
{
    const size_t n = 3 * static_cast<size_t>(m.n_free);
    if (n == 0) return EFEM_OK;
    // r = -f_ext (its first thread stores the start time in *stamp when given)
    extern void launch_neg(double* r, const double* f, size_t n, cudaStream_t st, unsigned long long* stamp);
    if (init_r) {
        launch_neg(d_r, m.d_fext, n, stream, stamp);
        m.launches++;
    }
    const bool mixed = m.opts.precision == EFEM_MIXED;
    const bool det = m.opts.deterministic != 0;
    if (det && !m.d_contrib) {
        set_error("deterministic scatter requested but its tables are not built");
        return EFEM_ERR_ARG;
    }
    for (auto& b : m.blocks) {
        if (b.n == 0) continue;
        m.launches++;
        Scatter sc;
        if (det) sc = Scatter { m.d_contrib, m.n_slots, b.slot0 };
        if (mixed)
            dispatch_elem<float>(b, m.d_mats_f, b.vol_f, b.J0inv_f, b.dN_f, b.gw_f, m.n_free, d_u, d_r, stream,
                b.threads[1], sc, m.d_frozen_groups);
        else
            dispatch_elem<double>(b, m.d_mats, b.vol, b.J0inv, b.dN, b.gw, m.n_free, d_u, d_r, stream, b.threads[0], sc,
                m.d_frozen_groups);
    }
    for (auto& f : m.faces) {
        if (f.n == 0) continue;
        m.launches++;
        Scatter sc;
        if (det) sc = Scatter { m.d_contrib, m.n_slots, f.slot0 };
        if (mixed)
            dispatch_face<float>(f, f.J0inv_f, f.t_w_f, f.t_N_f, f.t_dN_f, m.n_free, d_u, d_r, stream, sc);
        else
            dispatch_face<double>(f, f.J0inv, f.t_w, f.t_N, f.t_dN, m.n_free, d_u, d_r, stream, sc);
    }
    if (det) {
        launch_k(k_gather, (m.n_free + kBlock - 1) / kBlock, kBlock, 0, stream, m.n_free, m.d_gptr, m.d_gidx,
            m.d_contrib, m.n_slots, d_r);
        m.launches++;
    }
    EFEM_CUDA(cudaGetLastError());
    return EFEM_OK;
}

void free_gather(Model& m)
{
    dev_free(m.d_contrib);
    dev_free(m.d_gptr);
    dev_free(m.d_gidx);
    m.n_slots = 0;
}

// Slots of the deterministic scatter: element block b owns slots
// [slot0, slot0 + nen n) in node-major order, then each face group likewise;
// the gather lists of every free node are sorted by slot, so each node's sum
// has one fixed order whatever the launch configuration.
efem_status build_gather(Model& m)
{
    free_gather(m);
    size_t slots = 0;
    for (auto& b : m.blocks) {
        b.slot0 = slots;
        slots += static_cast<size_t>(b.nen) * b.n;
    }
    for (auto& f : m.faces) {
        f.slot0 = slots;
        slots += static_cast<size_t>(f.nen) * f.n;
    }
    if (slots >= static_cast<size_t>(INT_MAX)) {
        set_error("too many element-node pairs for the deterministic scatter");
        return EFEM_ERR_ARG;
    }
    std::vector<int> cnt(static_cast<size_t>(m.n_free) + 1, 0);
    auto node_of_slot = [&](auto&& visit) {
        for (auto& b : m.blocks)
            for (int a = 0; a < b.nen; a++)
                for (int e = 0; e < b.n; e++)
                    visit(b.h_conn[static_cast<size_t>(e) * b.nen + a], b.slot0 + static_cast<size_t>(a) * b.n + e);
        for (auto& f : m.faces)
            for (int q = 0; q < f.nen; q++)
                for (int k = 0; k < f.n; k++)
                    visit(f.h_conn[static_cast<size_t>(q) * f.n + k], f.slot0 + static_cast<size_t>(q) * f.n + k);
    };
    node_of_slot([&](int node, size_t) {
        if (node < m.n_free) cnt[node + 1]++;
    });
    for (int i = 0; i < m.n_free; i++) cnt[i + 1] += cnt[i];
    std::vector<int> idx(static_cast<size_t>(cnt[m.n_free]));
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    node_of_slot([&](int node, size_t sl) {  // visited in ascending slot order
        if (node < m.n_free) idx[fill[node]++] = static_cast<int>(sl);
    });
    for (int i = 0; i < m.n_free; i++) std::sort(idx.begin() + cnt[i], idx.begin() + cnt[i + 1]);
    efem_status s;
    if ((s = dev_alloc(&m.d_contrib, 3 * std::max<size_t>(slots, 1))) != EFEM_OK) return s;
    if ((s = dev_upload(&m.d_gptr, cnt)) != EFEM_OK) return s;
    if (idx.empty()) idx.push_back(0);
    if ((s = dev_upload(&m.d_gidx, idx)) != EFEM_OK) return s;
    m.n_slots = slots;
    return EFEM_OK;
}

}  // namespace efem
