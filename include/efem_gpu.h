/*
 * efem_gpu.h -- C ABI of the B200 (sm_100a) implementation of EFEM's hot path:
 * the Total-Lagrangian hyperelastic residual, the L-BFGS solve preconditioned
 * by the approximate-Jacobian Cholesky factor, and its adjoint.
 *
 * Plain C types only; every call returns an efem_status (0 = success) and
 * never throws.  A model owns all of its device memory and one CUDA stream.
 * Calls on different models may run from different threads; calls on one
 * model must not overlap.
 *
 * Vectors u, r, ... are in the reference's free-DOF order: entry 3*id + c,
 * id = the node's position among the non-fixed nodes in node-file order
 * (src/fe/Constraint.cpp:61-72).  By default they are host pointers; with
 * efem_options.device_ptrs = 1 they are device pointers on the model's GPU.
 */
#ifndef EFEM_GPU_H
#define EFEM_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    EFEM_OK = 0,
    EFEM_ERR_ARG = 1,          /* bad argument / handle */
    EFEM_ERR_CONFIG = 2,       /* JSON config unreadable or invalid (reference: std::terminate, src/io/IO.cpp:47-59) */
    EFEM_ERR_MESH = 3,         /* mesh / constraint file missing or malformed */
    EFEM_ERR_CUDA = 4,         /* a CUDA call failed; efem_last_error() has the text */
    EFEM_ERR_NAN = 5,          /* solution or residual not finite (reference: Integrator.cpp:28-34) */
    EFEM_ERR_TIMEOUT = 6,      /* a bounded device-side wait ran out */
    EFEM_ERR_UNSUPPORTED = 7,  /* a feature outside this library's scope */
    EFEM_ERR_NO_DEVICE = 8,    /* no CUDA device: the library has no CPU fallback */
    EFEM_ERR_FACE = 9          /* a pressure face does not lie on exactly one element */
} efem_status;

/* element material models, src/material/Material.h:9-16 */
typedef enum { EFEM_NEO_HOOKEAN = 0, EFEM_MOONEY_RIVLIN = 1, EFEM_YEOH = 2 } efem_material_type;

typedef struct {
    int type;      /* efem_material_type */
    int id;        /* material id matched against each element's id (-1 = default) */
    double C10, C01, C20, C30, D1, density;
} efem_material;

/* One block of elements that share a node count (4 = C3D4, 8 = C3D8,
 * 10 = C3D10, 20 = C3D20).  conn is row-major (n_elem, nen), 0-based. */
typedef struct {
    int nen;
    int n_elem;
    const int* conn;
    const int* material_id;  /* n_elem ids, or NULL for -1 */
} efem_element_block;

typedef struct {
    int n_nodes;
    const double* X;         /* (n_nodes, 3) reference coordinates */
    int n_blocks;
    const efem_element_block* blocks;
} efem_mesh_desc;

typedef enum {
    EFEM_LOAD_FIX = 0,
    EFEM_LOAD_FORCE = 1,
    EFEM_LOAD_PRESSURE = 2,
    EFEM_LOAD_DPRESSURE = 3,
    EFEM_LOAD_GRAVITY = 4
} efem_load_type;

/* A constraint as the reference's "constraint" JSON entries describe it
 * (src/fe/ExternalConstraint.cpp:13-247).
 *   FIX:       nodes[n]                      (0-based)
 *   FORCE:     nodes[n], value[3]            (each listed occurrence adds value)
 *   PRESSURE:  faces in CSR form, value[0] = follower pressure (> 0)
 *   DPRESSURE: faces in CSR form, value[0..2] = directed pressure vector
 *   GRAVITY:   value[0..2] = acceleration (the config's "gravity": "-z" is
 *              (0, 0, -9.8)); nodes / n unused.  Adds M g to the external
 *              load, M the consistent or lumped mass from the materials'
 *              density (efem_options.consistent_inertia), as the reference's
 *              inertia constraint does (src/fe/InertiaConstraint.cpp:34-84). */
typedef struct {
    int type;                /* efem_load_type */
    int n;                   /* nodes (FIX, FORCE) or faces (PRESSURE, DPRESSURE) */
    const int* nodes;        /* FIX / FORCE node list, or the concatenated face nodes */
    const int* face_ptr;     /* n+1 offsets into nodes, PRESSURE / DPRESSURE only */
    double value[3];
} efem_load_desc;

/* EFEM_MIXED: FP32 element kernels (FP32 arithmetic, FP64 accumulation of
 * the nodal forces) with the factor, its solves, the L-BFGS vectors and the
 * norms in FP64.  The FP32 phase runs until the residual is below half the
 * tolerance or stops improving; FP64 element kernels then finish the solve from there
 * (EFEM_SOLVE_REFINED), so the test that ends every solve reads an FP64
 * residual. */
typedef enum { EFEM_FP64 = 0, EFEM_MIXED = 1 } efem_precision;

typedef struct {
    int precision;            /* efem_precision: element kernels in FP64 or FP32 */
    int integration;          /* 0 full, 1 reduced (C3D4R/C3D10R/C3D8R/C3D20R rules) */
    int nl_solver;            /* 0 "lbfgs_ah": H0 = approximate-Jacobian Cholesky;
                                 1 "lbfgs": H0 = I/theta  (src/io/Config.cpp:25-33) */
    int m;                    /* L-BFGS history length (src/simulation/nlsolver/Param.h:102) */
    int max_iterations;       /* 0 = unlimited ("max_solver_iters"; "max_optim_iters" is accepted too) */
    int max_linesearch;       /* trials per line search ("max_line_search") */
    double residual_criterion;/* ||r||_inf <= eps or <= eps*||u||_inf ends the solve */
    double dx_criterion;      /* reported flag only, as in src/simulation/Integrator.cpp:36 */
    int device_ptrs;          /* 1: vector arguments are device pointers */
    int deterministic;        /* 1: element scatter by ordered gather (bitwise repeatable) */
    int device;               /* CUDA ordinal; -1 = current device */
    int host_loop;            /* 1: L-BFGS iterations driven from the host, one graph launch per
                                 iteration (same kernels; for profilers that do not see kernels
                                 inside conditional graph nodes); 0: the iteration loop runs on
                                 the device */
    double adjoint_tolerance; /* relative residual of the adjoint solve (default 1e-8) */
    int adjoint_max_iterations; /* GMRES iteration limit of the adjoint solve (default 2000) */
    int elem_threads;         /* element-kernel CTA size: 0 = chosen per element block by the autotuner
                                 at set-up (64, 128 or 256 threads, timed); 64 / 128 / 256 = forced */
    int consistent_inertia;   /* gravity loads: 1 consistent mass, 0 lumped (analysis "consistent_inertia",
                                 src/io/Config.cpp:63-65) */
    int trace;                /* > 0: keep a convergence trace of up to this many records per solve
                                 (efem_solve_trace); 0: off */
    int solve_subtree_levels; /* H0 triangular solves: fronts on the lowest k levels of the elimination
                                 tree are solved one subtree per CTA, the levels above by the dataflow
                                 kernel; 0 or -1 (default) = none, the dataflow kernel for every level */
    int line_search;          /* 0: the reference's residual-projection test |r.d| <= |r0.d| (default,
                                 LineSearchFEA.h:43-67); 1: Armijo test on the total potential
                                 Pi(u) = E(u) - f_ext.u (FP64 strain-energy sum), halving the step;
                                 needs conservative loads (no pressure faces), runs the iterations
                                 from the host */
    int wait_limit;           /* polls of one device-side wait of the preconditioner's triangular solve
                                 (a front waiting for the fronts it depends on) before the solve gives
                                 up with EFEM_ERR_TIMEOUT and leaves NaN in its output; 0 = default
                                 (2^22 polls, about half a second) */
    int wait_test;            /* test aid, 0 = off: 1 makes one wait of every H0 application wait for
                                 a count that no work item produces, so it runs out after wait_limit
                                 polls -- the timeout path without a GPU fault */
} efem_options;

enum {
    EFEM_SOLVE_CONVERGED = 1,      /* residual test passed */
    EFEM_SOLVE_PRECOND_FALLBACK = 2,/* factorisation failed; H0 = I/theta used (LBFGS.h:76-79) */
    EFEM_SOLVE_DX_CONVERGED = 4,   /* ||u||_inf < dx_criterion (the reference's return flag) */
    EFEM_SOLVE_MAX_ITERS = 8,
    EFEM_SOLVE_PDL = 16,           /* the captured iterations chain their kernels with programmatic
                                      dependent launch (a capture that refuses it falls back to plain launches) */
    EFEM_SOLVE_REFINED = 32,       /* mixed precision: the FP32 element kernels stopped short of the
                                      tolerance (their rounding floor) and FP64 element kernels finished
                                      the solve from that point */
    EFEM_SOLVE_BATCHED = 64        /* efem_batch_solve: solved inside one union model with the rest of the
                                      batch (ms_total, ms_factor and n_kernel_launches are the whole batch's) */
};

typedef struct {
    int niter;                /* L-BFGS iterations (LBFGS.h:96-174 return value) */
    int n_residual_evals;     /* SoftObjective::r_evalutes */
    int n_jacobian_evals;     /* SoftObjective::j_evalutes */
    int flags;                /* EFEM_SOLVE_* bits */
    double u_inf, r_inf;      /* final ||u||_inf and ||r||_inf (Integrator.cpp:37-40) */
    double ms_total;          /* device time of the whole solve (CUDA events on the model's stream) */
    double ms_factor;         /* numeric factorisation of the approximate Jacobian */
    double ms_residual;       /* all residual evaluations (GPU global timer, summed on the device) */
    double ms_precond;        /* all H0 applications (GPU global timer; the first one by CUDA events) */
    long long n_kernel_launches;  /* this library's kernels launched by the solve */
    int n_precond_applies;        /* H0 applications (ms_precond covers them) */
} efem_solve_info;

typedef struct {
    int n_nodes, n_free_nodes, n_dof;
    int n_elements, n_elements_skipped;   /* skipped: undefined material id */
    int n_faces, n_force_nodes;
    int n_blocks;
    long long factor_nnz;                 /* scalar Cholesky factor entries (0 before the first solve) */
    int n_supernodes, n_levels;
    double factor_gflop;
    long long factor_dinv_nnz;            /* entries of the inverted diagonal blocks (lower triangles) */
    long long residual_bytes;             /* algorithmic bytes of one residual evaluation */
    double residual_flops;                /* algorithmic flops of one residual evaluation */
    int n_params;                         /* sensitivity parameters (efem_adjoint): 5 per material slot
                                             (C10, C01, C20, C30, D1), then 1 per pressure load */
    int elem_threads_fp64, elem_threads_fp32;  /* the first element block's CTA size (autotuner) */
    int solve_subtree_levels, n_solve_subtrees; /* H0 solve schedule: levels solved per subtree, subtrees */
    int solve_ctas;                             /* CTAs of the persistent triangular solve */
    int solve_smem_bytes;                       /* its dynamic shared memory per CTA */
} efem_model_info;

typedef struct {
    int iterations;           /* GMRES iterations of the adjoint solve */
    int flags;                /* EFEM_SOLVE_CONVERGED: relative residual <= adjoint_tolerance */
    double rel_residual;      /* ||K(u)^T lambda - dJ/du|| / ||dJ/du|| (GMRES estimate) */
    double ms_total;          /* wall time of the call */
    double ms_solve;          /* the adjoint solve */
    double ms_params;         /* the parameter sensitivities */
    long long n_kernel_launches; /* kernels the call launched */
    double solve_bytes;       /* algorithmic bytes of the adjoint solve: per Krylov iteration the basis
                                 copy, one H0 application (16 nnz(L) + 40 n_dof, as for the solve), the
                                 transpose tangent (the FP64 residual's bytes, v and the zeroed output,
                                 the stored tangents) and two Gram-Schmidt passes over the basis */
} efem_adjoint_info;

/* --------------------------------------------------------------- lifetime */

/* Fill *o with the reference's defaults (Config.h:18-48, Param.h:92-103). */
efem_status efem_default_options(efem_options* o);

/* Replaces `EFEM -f cfg.json` set-up: Simulator::initial(path)
 * (src/simulation/Simulator.cpp:6-18) -> Config, Model, Constraint.
 * Same keys and files; paths relative to the config file's directory. */
efem_status efem_model_create_from_json(const char* cfg_path, void** model);

/* Array form of the same set-up (ElementConstraintConfig / ExternalConstraintConfig,
 * src/fe/ElementConstraint.cpp:11-67, src/fe/ExternalConstraint.cpp:13-247). */
efem_status efem_model_create(const efem_mesh_desc* mesh, const efem_material* materials, int n_materials,
    const efem_load_desc* loads, int n_loads, const efem_options* options, void** model);

efem_status efem_model_destroy(void* model);

efem_status efem_get_options(void* model, efem_options* o);
efem_status efem_set_options(void* model, const efem_options* o);
efem_status efem_get_model_info(void* model, efem_model_info* info);

/* node_of_dof[id] = node index of free node id (length n_free_nodes). */
efem_status efem_dof_map(void* model, int* node_of_dof);

/* f[3 n_free_nodes] (host memory) = the displacement-independent external
 * load: nodal forces plus, under gravity, M g (the inertia constraint's
 * -M g term of the residual, src/fe/InertiaConstraint.cpp:34-50, with the
 * nodal forces of src/fe/ExternalConstraint.cpp:149-167).  Pressure faces
 * follow the deformation and are not part of it.  Needs no GPU. */
efem_status efem_external_load(void* model, double* f);

/* --------------------------------------------------------------- hot path */

/* r = R(u): replaces SoftObjective::residual -> Constraint::assignDx +
 * Constraint::getResidual (src/simulation/Integrator.cpp:49-55,
 * src/fe/Constraint.cpp:93-126): element internal force, follower / directed
 * pressure and nodal forces. */
efem_status efem_residual(void* model, const double* u, double* r);

/* Scalar approximate Jacobian L (K~ = L (x) I3) in CSR over free nodes:
 * replaces Constraint::getJacobi triplets (src/fe/ElementConstraint.cpp:164-205,
 * src/simulation/Integrator.cpp:57-70).  Call with vals == NULL to get nnz in
 * *nnz; then with arrays of n_free_nodes+1 / nnz / nnz entries. */
efem_status efem_approx_jacobian_csr(void* model, long long* nnz, int* rowptr, int* colidx, double* vals);

/* Apply H0 = K~^{-1} (the Cholesky-preconditioner solve, LBFGSMat.h:119-120)
 * to v in place.  Factorises on first use. */
efem_status efem_precond_apply(void* model, double* v);

/* H0 v like efem_precond_apply, for callers that cannot allocate device
 * memory at call time (inside a CUDA stream capture, under another
 * framework's caching allocator).  No counterpart in the reference.  It calls
 * no cudaMalloc or cudaFree: its working memory lives in a fixed 16 MiB
 * device array that every GPU loading this library keeps until exit.
 * Requirements: the model's factor exists (efem_solve or efem_precond_apply
 * ran once) and 6 * free nodes + the factor's update-vector length
 * + 2 * fronts + 1 <= 2^21 doubles (EFEM_ERR_ARG otherwise, with the sizes in
 * efem_last_error; a model with more than 349 525 free nodes is refused
 * before anything else is checked); d_v is a device pointer, overwritten in
 * place.  Outside a capture the call waits for the result on the model's
 * stream and reports a solve that gave up waiting (EFEM_ERR_TIMEOUT).  Inside
 * a capture it only records the work, and the capture must be on the model's
 * stream (efem_set_stream with the capturing stream): a replay whose solve
 * gives up cannot report it, so it leaves NaN in every entry of d_v.  The
 * first call on a device looks up the array's device address and must come
 * before any stream capture (a first call inside a capture is refused with
 * EFEM_ERR_ARG).  All calls share the array: calls that overlap on the GPU
 * race and must be serialised by the caller. */
efem_status efem_precond_apply_noalloc(void* model, double* d_v);

/* Solve R(u) = 0 from u_inout: replaces Integrator::integral
 * (src/simulation/Integrator.cpp:22-42) -> LBFGSSolver::solve (LBFGS.h:96-174). */
efem_status efem_solve(void* model, double* u_inout, efem_solve_info* info);

/* The convergence trace of the model's last solve (options.trace > 0), the
 * reference's benchmark record (src/simulation/nlsolver/LBFGS.h:107-147,
 * printBenchmark :176-189) kept on the device: record 0 is the initial
 * residual, record i the state after iteration i's line search.  Each record
 * is 5 doubles: seconds since the solve started (GPU timer), ||r||_2,
 * ||r||_inf, the accepted step, residual evaluations in that iteration.
 * Copies min(records, capacity, options.trace) records to out (host memory;
 * out may be NULL) and sets *n_records to the number the solve produced. */
efem_status efem_solve_trace(void* model, double* out, int capacity, int* n_records);

/* --------------------------------------------------------------- sensitivities
 * None of these has a counterpart in the reference, which only forms the
 * approximate Jacobian (src/fe/ElementConstraint.cpp:164-205).  They extend
 * its residual (SoftObjective::residual, src/simulation/Integrator.cpp:49-55)
 * with derivatives, for gradient-based design and fitting.  Vectors follow
 * efem_options.device_ptrs like efem_residual. */

/* Kv = K(u) v, the true tangent dR/du at u applied to v (forward-mode
 * derivative of the residual, exact to rounding). */
efem_status efem_hvp(void* model, const double* u, const double* v, double* Kv);

/* KTw = K(u)^T w.  The element part of K is symmetric; the pressure part is
 * transposed face by face. */
efem_status efem_hvp_transpose(void* model, const double* u, const double* w, double* KTw);

/* dR = dR/dtheta_k at u for parameter k < efem_model_info.n_params: for
 * material slot s (the model's material table order) k = 5 s + {0 C10,
 * 1 C01, 2 C20, 3 C30, 4 D1}; then one scale per pressure load in input
 * order (a follower load's pressure, a directed load's vector scale). */
efem_status efem_residual_param_derivative(void* model, const double* u, int k, double* dR);

/* Adjoint sensitivities of J(u(theta)) at an equilibrium u (efem_solve's
 * result): solves K(u)^T lambda = dJ/du by restarted GMRES preconditioned
 * with the approximate-Jacobian factor, then dJdtheta[k] = -lambda .
 * dR/dtheta_k for every parameter (n_params values, host memory).  lambda
 * (may be NULL) receives the adjoint vector. */
efem_status efem_adjoint(void* model, const double* u, const double* dJdu, double* dJdtheta, double* lambda,
    efem_adjoint_info* info);

/* Write the mesh as a legacy ASCII VTK unstructured grid: every node at X + u
 * (u NULL: the reference configuration; fixed nodes stay at X) and every
 * element with its VTK cell type -- the content of Model::saveVTK
 * (src/model/Model.cpp:50-117), written without VTK.  u follows
 * efem_options.device_ptrs. */
efem_status efem_write_vtk(void* model, const double* u, const char* path);

/* Stored strain energy E(u) = sum_e V_e sum_g w_g W(F_g), summed in FP64 in a
 * fixed order; dE/du is the element part of R (the laws' energy functions
 * whose derivative is the reference's P(F)).  No reference counterpart. */
efem_status efem_strain_energy(void* model, const double* u, double* energy);

/* Solve n independent models (load cases, material samples, meshes of any
 * size) at once.  The reference solves one problem per process
 * (Simulator::start, src/simulation/Simulator.cpp:20-41).
 * When the models share their element precision, integration rule, history
 * length, line-search limit and device, use the approximate-Jacobian
 * preconditioner, the default line search and no gravity, they are solved as
 * one union model: one element-kernel launch per element type evaluates
 * every model's residual, one factorisation and one persistent triangular
 * solve apply every model's H0, and segmented L-BFGS kernels keep each
 * model's history, line search and convergence test apart, all inside one
 * CUDA graph of the iteration loop (EFEM_SOLVE_BATCHED in each info; each
 * model keeps its own residual_criterion and max_iterations; the union is
 * cached for further calls with the same models and options).  Otherwise
 * each model's solve runs on its own CUDA stream from a pool of max_threads
 * host threads (<= 0: one per hardware thread), and the CTAs of the
 * persistent triangular solve are divided among the solves in flight.  u[i]
 * is model i's u_inout (host or device per that model's device_ptrs); infos
 * may be NULL or hold n entries.  Returns the first failing model's status,
 * with its index in the error message. */
efem_status efem_batch_solve(void** models, int n, double* const* u, efem_solve_info* infos, int max_threads);

/* Run the model's device work on the caller's CUDA stream (a cudaStream_t);
 * NULL gives the model its own stream again.  The reference has no streams;
 * this lets a caller order the library's kernels with its own work. */
efem_status efem_set_stream(void* model, void* cuda_stream);

/* --------------------------------------------------------------- diagnostics */

/* Copy the last error message of this thread into buf. */
efem_status efem_last_error(char* buf, size_t len);

/* Library version string. */
const char* efem_version(void);

/* Measured CUDA-core FMA throughput of the current device in GFLOP/s (an FMA
 * counts 2): FP64 (fp32 = 0) or FP32 (fp32 = 1), the compute roof of the
 * element residual kernels.  Runs a short microbenchmark (a few ms).  No
 * reference counterpart; a measurement helper for roofline figures. */
efem_status efem_fma_peak(int fp32, double* gflops);

#ifdef __cplusplus
}
#endif
#endif
