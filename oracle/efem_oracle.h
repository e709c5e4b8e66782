/* Test infrastructure only: a plain-C restatement of the reference's hot path,
 * used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
 * the checker.  The product (efem_b200/) never links or calls it.
 *
 * Parity of this restatement is pinned against the reference itself: the
 * reference sources compiled unmodified (oracle/Makefile `ref` target) produce
 * the golden vectors in tests/golden/, and tests/test_oracle.py checks this
 * file against them.
 *
 * Conventions: node arrays are row-major (n,3); the free-DOF vector is
 * u[3*id + c] with id the free-node number in node order (fixed nodes skipped),
 * as src/fe/Constraint.cpp:61-72 numbers them.
 */
#ifndef EFEM_ORACLE_H
#define EFEM_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_NEO_HOOKEAN = 0, ORC_MOONEY_RIVLIN = 1, ORC_YEOH = 2 };

typedef struct orc_model orc_model;

typedef struct {
    double epsilon;      /* residual_criterion (absolute and relative) */
    int max_iterations;  /* 0 = unlimited */
    int max_linesearch;
    int m;               /* history length */
    int use_precond;     /* 1: H0 = approximate-Jacobian Cholesky, 0: H0 = I/theta */
} orc_params;

typedef struct {
    int niter, r_evals, precond_ok;
    double u_inf, r_inf;
} orc_info;

/* Build a model.  conn is flattened (n_elem * nen); all elements share one
 * node count nen (4, 8, 10 or 20).  elem_mat: material id per element.
 * mats: n_mat rows of {type, id, C10, C01, C20, C30, D1} (type/id as doubles).
 * fixed: n_nodes flags.  reduced: 1 selects the reduced integration rule. */
orc_model* orc_create(int n_nodes, const double* X, int n_elem, int nen, const int* conn,
    const int* elem_mat, int n_mat, const double* mats, const unsigned char* fixed, int reduced);
/* Follower (dvalue == NULL) or directed pressure on faces; faces flattened,
 * every face with face_nn nodes (3, 4, 6 or 8).  Returns 0 or a negative error. */
int orc_add_pressure(orc_model* m, int n_faces, int face_nn, const int* faces, double value,
    const double* dvalue);
/* Gravity as the reference's inertia constraint: the residual gains -M g,
 * M consistent (1) or lumped (0); g the acceleration, density per material
 * index (the order of orc_create's mats). */
int orc_add_gravity(orc_model* m, const double* g, int consistent, const double* density);
/* Nodal force f on each listed node (repeats accumulate). */
int orc_add_force(orc_model* m, int n, const int* nodes, const double* f);
int orc_n_dof(const orc_model* m);
int orc_n_elem_skipped(const orc_model* m);
void orc_residual(orc_model* m, const double* u, double* r);
/* Scalar approximate-Jacobian L (n_free x n_free, dense, row-major); the
 * reference's matrix is L (x) I3. */
void orc_approx_jacobian_dense(orc_model* m, double* L);
int orc_solve(orc_model* m, const orc_params* p, double* u, orc_info* info);
/* Record the next solves' convergence trace into buf (cap records of 5
 * doubles: 0, ||r||_2, ||r||_inf, step, residual evaluations); NULL: off.
 * orc_trace_count: records the last solve produced (may exceed cap). */
void orc_set_trace(orc_model* m, double* buf, int cap);
int orc_trace_count(const orc_model* m);
/* v <- (L (x) I3)^{-1} v (the preconditioner solve); 0 if L is not SPD. */
int orc_precond_apply(orc_model* m, double* v);
/* First Piola-Kirchhoff stress of one material at n column-major 3x3 F. */
void orc_piola(int type, const double* C, int n, const double* F, double* P);
double orc_elasticity_coeff(int type, const double* C);
void orc_destroy(orc_model* m);

#ifdef __cplusplus
}
#endif
#endif
