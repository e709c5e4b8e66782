// Internal data model of the B200 EFEM library.
//
// Device layout (one model = one problem on one GPU):
//   * node numbering: free nodes first, in the reference's DOF order
//     (src/fe/Constraint.cpp:61-72), then fixed nodes.  A solver vector u of
//     length 3*n_free is indexed u[3*dnode + c] for dnode < n_free.
//   * element blocks, one per node count: connectivity SoA conn[a][e] (dnode
//     ids), material index, V_e, and J0^{-1} per Gauss point AoS
//     [e][g][9] (row-major 3x3), in FP64 and (for the mixed path) FP32.
//   * pressure faces grouped by parent element kind: parent connectivity SoA,
//     A0, J0^{-1} at each face point, and an index into small face tables
//     (weights, N, dN/dxi at the face points).
//   * f_ext: the nodal-force vector; every residual starts from r = -f_ext.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/efem_gpu.h"
#include "elements.h"

namespace efem {

// ------------------------------------------------------------------ host input
struct HostMaterial {
    int type, id;
    double C10, C01, C20, C30, D1, density;
};

struct HostBlock {
    int nen = 0;
    std::vector<int> conn;    // row-major (n, nen), original node ids
    std::vector<int> mat_id;  // material id per element
};

struct HostLoad {
    int type = 0;                   // efem_load_type
    std::vector<int> nodes;         // FIX / FORCE nodes, or face nodes
    std::vector<int> face_ptr;      // faces (CSR), PRESSURE / DPRESSURE
    double value[3] = { 0, 0, 0 };
};

struct ModelInput {
    std::vector<double> X;          // (n, 3)
    std::vector<HostBlock> blocks;
    std::vector<int> cell_ptr, cell_nodes;  // every element in input order (bodies, then file order), for output
    std::vector<HostMaterial> materials;
    std::vector<HostLoad> loads;
    efem_options opts;
};

// ------------------------------------------------------------------ device
// Material parameters as the kernels see them.
template <typename T>
struct MatParams {
    int type;
    T C10, C01, C20, C30, D1;
};

constexpr int MAX_MATS = 16;

struct DevBlock {
    int kind = 0, nen = 0, ngp = 0, n = 0;
    int threads[2] = { 128, 128 };  // element-kernel CTA size per precision (FP64, FP32), from the autotuner
    int mat_type = -1;            // the one material law of every element, or -1 when they mix laws
    size_t slot0 = 0;             // deterministic scatter: first contribution slot, slot = slot0 + a * n + e
    int* conn = nullptr;          // [nen][n]
    int* mat = nullptr;           // [n]
    double* vol = nullptr;        // [n]
    float* vol_f = nullptr;
    double* J0inv = nullptr;      // [n][ngp][9]
    float* J0inv_f = nullptr;
    double* dN = nullptr;         // [ngp][nen][3]
    float* dN_f = nullptr;
    double* gw = nullptr;         // [ngp]
    float* gw_f = nullptr;
    int* egroup = nullptr;        // batch unions: member of every element (null otherwise)
    // host copies used by set-up (Jacobian assembly, tests)
    std::vector<int> h_conn;      // row-major (n, nen), dnode ids
    std::vector<int> h_mat;
    std::vector<double> h_vol, h_J0inv, h_dN, h_gw;
};

struct DevFaces {
    int kind = 0, nen = 0, n = 0;
    int* conn = nullptr;          // [nen][n] parent element nodes (dnode)
    int* table = nullptr;         // [n]
    double* A0 = nullptr;         // [n][3]
    double* J0inv = nullptr;      // [n][MAX_FGP][9]
    float* J0inv_f = nullptr;
    double* load = nullptr;       // [n][4]: directed flag, value / vector
    int* load_idx = nullptr;      // [n]: index of the face's load among the pressure loads
    size_t slot0 = 0;             // deterministic scatter: first contribution slot, slot = slot0 + q * n + f
    // face tables for this element kind
    int n_tables = 0;
    int* t_ngp = nullptr;         // [n_tables]
    double* t_w = nullptr;        // [n_tables][MAX_FGP]
    double* t_N = nullptr;        // [n_tables][MAX_FGP][nen]
    double* t_dN = nullptr;       // [n_tables][MAX_FGP][nen][3]
    float* t_w_f = nullptr;
    float* t_N_f = nullptr;
    float* t_dN_f = nullptr;
    // host copies (set-up output; uploaded by ensure_device)
    std::vector<int> h_conn, h_table, h_ngp;
    std::vector<double> h_A0, h_J0inv, h_load, h_w, h_N, h_dN;
    std::vector<int> h_load_idx;
};

struct Precond;   // Cholesky preconditioner (chol.cu)
struct SolverWS;  // L-BFGS workspace (solver.cu)
struct AdjointWS; // tangent / adjoint workspace (adjoint.cu)

struct Model {
    efem_options opts;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;          // false: the caller's stream (efem_set_stream)

    int n_nodes = 0, n_free = 0, n_elements = 0, n_skipped = 0, n_force_nodes = 0;
    std::vector<int> node_of_dnode;   // dnode -> original node
    std::vector<int> dnode_of_node;   // original node -> dnode
    std::vector<double> X;            // original order (n,3)

    std::vector<int> cell_ptr, cell_nodes;     // every input element (output meshes), original node ids
    std::vector<HostMaterial> materials_used;  // index = material slot
    std::vector<double> kappa;                 // elasticity_coeff per slot

    // element input kept for rebuilding the integration tables
    std::vector<HostBlock> in_blocks;
    std::vector<HostLoad> in_loads;   // the constraints as given (batch solves rebuild them in a union model)
    int built_integration = -1;
    std::vector<DevBlock> blocks;
    std::vector<DevFaces> faces;
    int n_faces = 0;
    int n_pressure_loads = 0;         // follower and directed pressure loads, in input order

    MatParams<double>* d_mats = nullptr;
    MatParams<float>* d_mats_f = nullptr;
    std::vector<double> h_fext;       // [3*n_free]: nodal forces + M g
    std::vector<double> h_fnodal;     // [3*n_free]: nodal forces alone
    double gravity[3] = { 0, 0, 0 };  // summed EFEM_LOAD_GRAVITY accelerations
    bool has_gravity = false;
    bool on_device = false;
    double* d_fext = nullptr;         // [3*n_free]
    const int* d_frozen_groups = nullptr;  // batch unions: per member, 1 = its elements are skipped
    double* d_u = nullptr;            // staging for host-pointer calls
    double* d_r = nullptr;
    // deterministic scatter (opts.deterministic): nodal contributions of every
    // (element, node) and (face, node) pair in contrib[3][n_slots]; free node i
    // sums slots gidx[gptr[i] .. gptr[i+1]) in ascending slot order
    double* d_contrib = nullptr;
    int* d_gptr = nullptr;
    int* d_gidx = nullptr;
    size_t n_slots = 0;

    long long launches = 0;           // kernels launched by this model (diagnostics)
    long long epoch = 0;              // bumped when device arrays that captured graphs point to are rebuilt
    int tuned_threads = -1;           // opts.elem_threads the element kernels were tuned for (-1: not yet)
    Precond* precond = nullptr;   // owned; freed by free_precond
    SolverWS* ws = nullptr;       // owned; freed by free_solver
    AdjointWS* aws = nullptr;     // owned; freed by free_adjoint

    ~Model();
};

// ------------------------------------------------------------------ errors
void set_error(const std::string& msg);
const std::string& get_error();

// Programmatic dependent launch inside the solver's graph captures: while
// t_pdl is set, kernels launched through launch_k may be scheduled while the
// kernel before them in the stream is still finishing (their CTAs become
// resident and wait), which takes the launch gap off the iteration's chain.
// Every kernel launched this way calls griddep_wait() before it touches
// memory; kernels call griddep_launch() once their main work is issued.
// Outside such captures launch_k is a plain launch.
extern thread_local bool t_pdl;

#ifdef __CUDACC__
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... P, typename... A>
inline void launch_k(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A&&... args)
{
    if (!t_pdl) {
        kernel<<<grid, block, smem, st>>>(std::forward<A>(args)...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}
#endif

#define EFEM_CUDA(call)                                                                          \
    do {                                                                                         \
        cudaError_t _e = (call);                                                                 \
        if (_e != cudaSuccess) {                                                                 \
            efem::set_error(std::string(#call) + ": " + cudaGetErrorString(_e));                 \
            return EFEM_ERR_CUDA;                                                                \
        }                                                                                        \
    } while (0)

template <typename T>
efem_status dev_alloc(T** p, size_t n)
{
    *p = nullptr;
    if (n == 0) return EFEM_OK;
    EFEM_CUDA(cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T)));
    return EFEM_OK;
}

template <typename T>
efem_status dev_upload(T** p, const std::vector<T>& h)
{
    efem_status s = dev_alloc(p, h.size());
    if (s != EFEM_OK) return s;
    if (!h.empty()) EFEM_CUDA(cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return EFEM_OK;
}

template <typename T>
void dev_free(T*& p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

// ------------------------------------------------------------------ set-up
efem_status read_json_config(const char* path, ModelInput& in);
efem_status build_model(ModelInput& in, Model& m);
efem_status build_blocks(Model& m);   // (re)build the integration tables for opts.integration (host)
// one residual evaluation's algorithmic bytes and flops (pressure faces included when faces is set)
void residual_work(const Model& m, int sz, long long* bytes, double* flops, bool faces);
efem_status ensure_device(Model& m);  // create the stream and upload everything not yet on the device

// ------------------------------------------------------------------ kernels (residual.cu)
// r = R(u) on the model's stream; u, r device pointers of length 3*n_free.
efem_status launch_residual(Model& m, const double* d_u, double* d_r);
int element_tune_key(const Model& m);  // what the element kernels' CTA sizes were tuned for
efem_status tune_element_blocks(Model& m);  // autotuner of the element kernels' CTA size
// the same on `stream`; with `stamp`, the GPU's global timer at the start is
// stored there; init_r = false when the caller has already set r = -f_ext
efem_status launch_residual_on(Model& m, const double* d_u, double* d_r, cudaStream_t stream,
    unsigned long long* stamp = nullptr, bool init_r = true);

// ------------------------------------------------------------------ solver (solver.cu)
efem_status run_solve(Model& m, double* d_u, efem_solve_info* info);
efem_status build_gather(Model& m);
void free_gather(Model& m);
efem_status solve_trace(Model& m, double* out, int capacity, int* n_records);
void free_solver(Model& m);
// Held while a CUDA graph is captured and instantiated, so that solves of
// different models running in parallel host threads never overlap a capture
// with an allocation or free (which may synchronise the device).
std::mutex& capture_mutex();
void free_adjoint(Model& m);

// ------------------------------------------------------------------ sensitivities (adjoint.cu)
int n_params(const Model& m);
// out = K(u) v (transpose: K(u)^T v); device pointers
efem_status hvp(Model& m, const double* d_u, const double* d_v, double* d_out, bool transpose);
efem_status residual_param_derivative(Model& m, const double* d_u, int k, double* d_out);
efem_status adjoint(Model& m, const double* d_u, const double* d_dJdu, double* dJdtheta, double* d_lambda,
    efem_adjoint_info* info);
efem_status adjoint_io(Model& m, double** io);  // an n_dof device buffer for host-pointer calls
efem_status strain_energy_sum(Model& m, const double* d_u, double* energy);  // energy.cu
efem_status total_potential(Model& m, const double* d_u, double* pi);       // energy.cu: E(u) - f_ext.u

// ------------------------------------------------------------------ preconditioner (chol.cu)
// Build (once) the scalar approximate Jacobian L and its Cholesky factor.
// Returns EFEM_OK with *ok = 0 when L is not positive definite.
efem_status precond_setup(Model& m, bool refactor, int* ok, double* ms_factor);
// v <- (L (x) I3)^{-1} v in place on the device (v: 3*n_free interleaved).
efem_status precond_apply(Model& m, double* d_v);
// The same H0 application enqueued on `stream` (for capture into a larger
// graph); clear = false when the caller has zeroed precond_counters itself.
// With `stamp`, the solve's first CTA stores the GPU's global timer there.
efem_status precond_enqueue(Model& m, double* d_v, cudaStream_t stream, bool clear = true,
    unsigned long long* stamp = nullptr);
void precond_counters(const Model& m, int** cnt, int* n);  // the solve's counters, cleared before each H0 v
// Batch unions: group_of_free_node[i] = the member free node i belongs to;
// items of member g are skipped while d_frozen[g] != 0 (a member's fronts
// form trees of their own, so nothing else waits on them).
efem_status precond_set_groups(Model& m, const std::vector<int>& group_of_free_node, const int* d_frozen);
bool precond_has_groups(const Model& m);
long long precond_launch_count(const Model& m);  // kernels per H0 application
const int* precond_error_flag(const Model& m);   // device flag: a solve gave up waiting (nullptr before set-up)
efem_status precond_check(Model& m);             // wait for the stream and report that flag
void free_precond(Model& m);
void precond_drop_graphs(Model& m);  // forget captured H0 solves (new wait limits); the factor stays
// ------------------------------------------------------------------ batches (batch.cu)
// Solve n models as one union model (see batch.cu); EFEM_ERR_UNSUPPORTED when
// the models cannot share one (different devices or options, gravity, an
// approximate Jacobian that is not positive definite): the caller then solves
// them one by one.
efem_status batch_union_solve(Model** models, int n, double* const* u, efem_solve_info* infos);
void batch_forget(const Model* m);  // drop cached unions that hold m (m is being destroyed)
void precond_info(const Model& m, efem_model_info* info);
// The persistent triangular solve's grid: every CTA that fits on the device
// (one solve at a time), or, while t_batch > 0 (the batch solve's worker
// threads, t_batch solves in flight), that many CTAs divided among the
// solves: CTAs waiting on a front's dependencies would otherwise hold the
// SMs the other solves need.  A change drops the graphs that captured the
// old grid.
extern thread_local int t_batch;
efem_status precond_sync_grid(Model& m);
// Host assembly of L in CSR over free nodes (upper and lower triangle).
void assemble_L_csr(const Model& m, std::vector<int>& rowptr, std::vector<int>& col, std::vector<double>& val);

}  // namespace efem
