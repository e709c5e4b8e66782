/* Test infrastructure only -- the CPU checker for the CUDA path, never shipped
 * on the product path.  A plain-C restatement of the reference's algorithm;
 * each block cites the reference file:line it follows.  Parity of this file is
 * pinned against the reference compiled from its own sources (see
 * efem_oracle.h and tests/test_oracle.py). */
#include "efem_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXN 20
#define MAXG 27

/* ------------------------------------------------------------------ 3x3 helpers
 * Row-major: a[3*i+j] = A(i,j). */
static double det3(const double* a)
{
    return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6])
        + a[2] * (a[3] * a[7] - a[4] * a[6]);
}

static void inv3(const double* a, double* o)
{
    double d = det3(a);
    o[0] = (a[4] * a[8] - a[5] * a[7]) / d;
    o[1] = (a[2] * a[7] - a[1] * a[8]) / d;
    o[2] = (a[1] * a[5] - a[2] * a[4]) / d;
    o[3] = (a[5] * a[6] - a[3] * a[8]) / d;
    o[4] = (a[0] * a[8] - a[2] * a[6]) / d;
    o[5] = (a[2] * a[3] - a[0] * a[5]) / d;
    o[6] = (a[3] * a[7] - a[4] * a[6]) / d;
    o[7] = (a[1] * a[6] - a[0] * a[7]) / d;
    o[8] = (a[0] * a[4] - a[1] * a[3]) / d;
}

static void mul3(const double* a, const double* b, double* o)
{
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            o[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
}

/* ------------------------------------------------------------------ materials
 * First Piola-Kirchhoff stress, src/material/NeoHookean.cpp:4-20,
 * MooneyRivlin.cpp:4-24, Yeoh.cpp:4-19.  C = {C10, C01, C20, C30, D1}. */
static void piola(int type, const double* C, const double* F, double* P)
{
    double C10 = C[0], C01 = C[1], C20 = C[2], C30 = C[3], D1 = C[4];
    double J = det3(F);
    double Cm[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            Cm[3 * i + j] = F[i] * F[j] + F[3 + i] * F[3 + j] + F[6 + i] * F[6 + j];
    double I1 = Cm[0] + Cm[4] + Cm[8];
    double I3 = J * J;
    double I3c = pow(I3, 1.0 / 3.0);
    double I1bar = I1 / I3c;
    double Finv[9], dJdF[9];
    inv3(F, Finv);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            dJdF[3 * i + j] = J * Finv[3 * j + i];
    double c1;
    if (type == ORC_YEOH) {
        double t = I1bar - 3.0;
        c1 = C10 + 2.0 * C20 * t + 3.0 * C30 * pow(t, 2);
    } else {
        c1 = C10;
    }
    double vol = 2.0 / D1 * (J - 1.0);
    for (int k = 0; k < 9; k++)
        P[k] = c1 * (-2.0 * I1bar * dJdF[k] / (3.0 * J) + 2.0 * F[k] / I3c) + vol * dJdF[k];
    if (type == ORC_MOONEY_RIVLIN) {
        double CC = 0.0;
        for (int k = 0; k < 9; k++)
            CC += Cm[k] * Cm[k]; /* tr(C^T C) */
        double I2 = 0.5 * (pow(I1, 2) - CC);
        double I3c2 = pow(I3 * I3, 1.0 / 3.0);
        double I2bar = I2 / I3c2;
        double A[9]; /* I1*I - C */
        for (int k = 0; k < 9; k++)
            A[k] = -Cm[k];
        A[0] += I1;
        A[4] += I1;
        A[8] += I1;
        double FA[9];
        mul3(F, A, FA);
        for (int k = 0; k < 9; k++)
            P[k] += C01 * (-4.0 * I2bar * dJdF[k] / (3.0 * J) + 2.0 * FA[k] / I3c2);
    }
}

/* Preconditioner scale kappa, NeoHookean.cpp:41, MooneyRivlin.cpp:48, Yeoh.cpp:47. */
double orc_elasticity_coeff(int type, const double* C)
{
    if (type == ORC_MOONEY_RIVLIN)
        return 3.818 * C[1] + 2.94001 * C[0] + 2.0 / C[4];
    if (type == ORC_YEOH)
        return 2.94001 * C[0] + 3.51194 * C[2] + 3.3154 * C[3] + 2.0 / C[4];
    return 2.94001 * C[0] + 2.0 / C[4];
}

void orc_piola(int type, const double* C, int n, const double* F, double* P)
{
    for (int k = 0; k < n; k++) {
        double Fr[9], Pr[9];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                Fr[3 * i + j] = F[9 * k + i + 3 * j];
        piola(type, C, Fr, Pr);
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                P[9 * k + i + 3 * j] = Pr[3 * i + j];
    }
}

/* ------------------------------------------------------------------ elements
 * Shape functions, src/fe/element/TetrahedraElement.cpp:15-33 (C3D4),
 * :62-122 (C3D10); HexahedraElement.cpp:15-58 (C3D8), :147-238 (C3D20).
 * C3D20 is written in serendipity form with the reference's node coordinates
 * (corner 0 at (1,-1,1), ...), which is the same polynomial set. */
static const double HEX8_S[8][3] = { { -1, -1, -1 }, { 1, -1, -1 }, { 1, 1, -1 }, { -1, 1, -1 },
    { -1, -1, 1 }, { 1, -1, 1 }, { 1, 1, 1 }, { -1, 1, 1 } };
static const double HEX20_C[8][3] = { { 1, -1, 1 }, { 1, 1, 1 }, { 1, 1, -1 }, { 1, -1, -1 },
    { -1, -1, 1 }, { -1, 1, 1 }, { -1, 1, -1 }, { -1, -1, -1 } };
static const int HEX_EDGE[12][2] = { { 0, 1 }, { 1, 2 }, { 2, 3 }, { 3, 0 }, { 4, 5 }, { 5, 6 }, { 6, 7 },
    { 7, 4 }, { 0, 4 }, { 1, 5 }, { 2, 6 }, { 3, 7 } };

static void shape(int nen, const double* p, double* N, double* dN /* nen x 3 */)
{
    double x = p[0], y = p[1], z = p[2];
    if (nen == 4) {
        N[0] = x; N[1] = y; N[2] = z; N[3] = 1.0 - x - y - z;
        static const double g[12] = { 1, 0, 0, 0, 1, 0, 0, 0, 1, -1, -1, -1 };
        memcpy(dN, g, sizeof(g));
    } else if (nen == 10) {
        double L = 1.0 - x - y - z;
        N[0] = L * (2 * L - 1); N[1] = x * (2 * x - 1); N[2] = y * (2 * y - 1); N[3] = z * (2 * z - 1);
        N[4] = 4 * L * x; N[5] = 4 * x * y; N[6] = 4 * y * L; N[7] = 4 * z * L; N[8] = 4 * x * z; N[9] = 4 * y * z;
        double g[30] = { -(4 * L - 1), -(4 * L - 1), -(4 * L - 1),
            4 * x - 1, 0, 0,
            0, 4 * y - 1, 0,
            0, 0, 4 * z - 1,
            4 * L - 4 * x, -4 * x, -4 * x,
            4 * y, 4 * x, 0,
            -4 * y, 4 * L - 4 * y, -4 * y,
            -4 * z, -4 * z, 4 * L - 4 * z,
            4 * z, 0, 4 * x,
            0, 4 * z, 4 * y };
        memcpy(dN, g, sizeof(g));
    } else if (nen == 8) {
        for (int a = 0; a < 8; a++) {
            double sx = HEX8_S[a][0], sy = HEX8_S[a][1], sz = HEX8_S[a][2];
            double A = 1 + sx * x, B = 1 + sy * y, C = 1 + sz * z;
            N[a] = 0.125 * A * B * C;
            dN[3 * a] = 0.125 * sx * B * C;
            dN[3 * a + 1] = 0.125 * A * sy * C;
            dN[3 * a + 2] = 0.125 * A * B * sz;
        }
    } else {
        for (int a = 0; a < 8; a++) {
            double sx = HEX20_C[a][0], sy = HEX20_C[a][1], sz = HEX20_C[a][2];
            double A = 1 + sx * x, B = 1 + sy * y, C = 1 + sz * z;
            double s = sx * x + sy * y + sz * z;
            N[a] = 0.125 * A * B * C * (s - 2);
            dN[3 * a] = 0.125 * sx * B * C * (2 * sx * x + sy * y + sz * z - 1);
            dN[3 * a + 1] = 0.125 * sy * A * C * (sx * x + 2 * sy * y + sz * z - 1);
            dN[3 * a + 2] = 0.125 * sz * A * B * (sx * x + sy * y + 2 * sz * z - 1);
        }
        for (int e = 0; e < 12; e++) {
            int a = 8 + e;
            double c[3];
            for (int k = 0; k < 3; k++)
                c[k] = 0.5 * (HEX20_C[HEX_EDGE[e][0]][k] + HEX20_C[HEX_EDGE[e][1]][k]);
            /* exactly one local coordinate of a mid-edge node is zero */
            double A = 1 + c[0] * x, B = 1 + c[1] * y, C = 1 + c[2] * z;
            if (c[0] == 0) {
                N[a] = 0.25 * (1 - x * x) * B * C;
                dN[3 * a] = -0.5 * x * B * C;
                dN[3 * a + 1] = 0.25 * (1 - x * x) * c[1] * C;
                dN[3 * a + 2] = 0.25 * (1 - x * x) * B * c[2];
            } else if (c[1] == 0) {
                N[a] = 0.25 * A * (1 - y * y) * C;
                dN[3 * a] = 0.25 * c[0] * (1 - y * y) * C;
                dN[3 * a + 1] = -0.5 * y * A * C;
                dN[3 * a + 2] = 0.25 * A * (1 - y * y) * c[2];
            } else {
                N[a] = 0.25 * A * B * (1 - z * z);
                dN[3 * a] = 0.25 * c[0] * B * (1 - z * z);
                dN[3 * a + 1] = 0.25 * A * c[1] * (1 - z * z);
                dN[3 * a + 2] = -0.5 * z * A * B;
            }
        }
    }
}

/* Gauss rules with weights normalised to sum 1, src/fe/element/IntegralElement.inl:3-223.
 * The 4-point tet rule keeps the reference's 8-digit constants (:41-47). */
static int gauss(int nen, int reduced, double* pts, double* w)
{
    int rule; /* 1 tet1, 4 tet4, 101 hex1, 108 hex8, 127 hex27 */
    if (nen == 4)
        rule = 1;
    else if (nen == 10)
        rule = reduced ? 1 : 4;
    else if (nen == 8)
        rule = reduced ? 101 : 108;
    else
        rule = reduced ? 108 : 127;
    if (rule == 1) {
        pts[0] = pts[1] = pts[2] = 0.25;
        w[0] = 1.0;
        return 1;
    }
    if (rule == 4) {
        const double a = 0.58541020, b = 0.13819660;
        const double t[4][3] = { { a, b, b }, { b, a, b }, { b, b, a }, { b, b, b } };
        for (int g = 0; g < 4; g++) {
            memcpy(pts + 3 * g, t[g], sizeof(t[g]));
            w[g] = 0.25;
        }
        return 4;
    }
    if (rule == 101) {
        pts[0] = pts[1] = pts[2] = 0.0;
        w[0] = 1.0;
        return 1;
    }
    if (rule == 108) {
        double a = 1.0 / sqrt(3.0);
        for (int g = 0; g < 8; g++) {
            for (int k = 0; k < 3; k++)
                pts[3 * g + k] = a * HEX8_S[g][k];
            w[g] = 0.125;
        }
        return 8;
    }
    {
        double c = sqrt(3.0 / 5.0);
        const double q[3] = { -c, 0.0, c };
        const double qw[3] = { 5.0, 8.0, 5.0 };
        int g = 0;
        for (int k = 0; k < 3; k++)
            for (int j = 0; j < 3; j++)
                for (int i = 0; i < 3; i++, g++) {
                    pts[3 * g] = q[i];
                    pts[3 * g + 1] = q[j];
                    pts[3 * g + 2] = q[k];
                    w[g] = qw[i] * qw[j] * qw[k] / 5832.0;
                }
        return 27;
    }
}

/* ------------------------------------------------------------------ model */
typedef struct {
    int type, id;
    double C[5];
    double kappa;
} orc_mat;

typedef struct {
    int elem, ngp, directed;
    double value, dvalue[3];
    double A0[3];
    double w[9];
    double N[9][MAXN];
    double dN[9][MAXN * 3];
    double J0inv[9][9];
} orc_face;

struct orc_model {
    int n_nodes, n_elem, nen, ngp, n_free, reduced, n_skipped;
    double* X;
    int* conn;
    int* id;          /* node -> free id or -1 */
    int* elem_mat;    /* element -> index into mats, -1 = skipped */
    int n_mat;
    orc_mat* mats;
    double gw[MAXG], gdN[MAXG][MAXN * 3];
    double* J0inv;    /* n_elem * ngp * 9 */
    double* T;        /* n_elem * ngp * 3 * nen  (T[k*nen + a]) */
    double* vol;
    int n_faces;
    orc_face* faces;
    int n_force;
    int* force_node;
    double* force_val;
    double* gvec;     /* gravity load M g per free DOF, or NULL */
    double* trace;    /* caller's buffer for the solve trace, or NULL */
    int trace_cap, trace_n;
    /* incident elements per node (CSR) for the face -> element lookup */
    int* inc_ptr;
    int* inc;
};

/* Element volume from the corner nodes (see oracle/shim/model/Element.h):
 * tets |det|/6; hexahedra by the divergence theorem over the triangulated
 * corner faces (quad a-b-c-d -> a-b-c + a-c-d). */
static double elem_volume(const orc_model* m, const int* c)
{
    const double* X = m->X;
#define PX(i) (X + 3 * c[i])
    if (m->nen == 4 || m->nen == 10) {
        double a[3], b[3], d[3];
        for (int k = 0; k < 3; k++) {
            a[k] = PX(1)[k] - PX(0)[k];
            b[k] = PX(2)[k] - PX(0)[k];
            d[k] = PX(3)[k] - PX(0)[k];
        }
        double v = a[0] * (b[1] * d[2] - b[2] * d[1]) - a[1] * (b[0] * d[2] - b[2] * d[0])
            + a[2] * (b[0] * d[1] - b[1] * d[0]);
        return fabs(v) / 6.0;
    }
    static const int F[6][4] = { { 0, 3, 2, 1 }, { 4, 5, 6, 7 }, { 0, 1, 5, 4 }, { 1, 2, 6, 5 }, { 2, 3, 7, 6 }, { 3, 0, 4, 7 } };
    double v6 = 0.0;
    for (int f = 0; f < 6; f++) {
        const double *a = PX(F[f][0]), *b = PX(F[f][1]), *cc = PX(F[f][2]), *d = PX(F[f][3]);
        double bc[3] = { b[1] * cc[2] - b[2] * cc[1], b[2] * cc[0] - b[0] * cc[2], b[0] * cc[1] - b[1] * cc[0] };
        double cd[3] = { cc[1] * d[2] - cc[2] * d[1], cc[2] * d[0] - cc[0] * d[2], cc[0] * d[1] - cc[1] * d[0] };
        v6 += a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2] + a[0] * cd[0] + a[1] * cd[1] + a[2] * cd[2];
    }
#undef PX
    return fabs(v6) / 6.0;
}

/* J = Y . dN (3 x 3) for the element's nodal coordinates Y (nen x 3). */
static void jacobi(int nen, const double* Y, const double* dN, double* J)
{
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) {
            double s = 0.0;
            for (int a = 0; a < nen; a++)
                s += Y[3 * a + i] * dN[3 * a + k];
            J[3 * i + k] = s;
        }
}

orc_model* orc_create(int n_nodes, const double* X, int n_elem, int nen, const int* conn,
    const int* elem_mat, int n_mat, const double* mats, const unsigned char* fixed, int reduced)
{
    if (nen != 4 && nen != 8 && nen != 10 && nen != 20)
        return NULL;
    orc_model* m = calloc(1, sizeof(orc_model));
    m->n_nodes = n_nodes;
    m->n_elem = n_elem;
    m->nen = nen;
    m->reduced = reduced;
    m->X = malloc(sizeof(double) * 3 * n_nodes);
    memcpy(m->X, X, sizeof(double) * 3 * n_nodes);
    m->conn = malloc(sizeof(int) * nen * n_elem);
    memcpy(m->conn, conn, sizeof(int) * nen * n_elem);
    /* materials: the first definition of an id wins (unordered_map::insert,
     * src/fe/ElementConstraint.cpp:50-64); elements with an undefined id are
     * skipped (:23-26) */
    m->n_mat = n_mat;
    m->mats = calloc(n_mat > 0 ? n_mat : 1, sizeof(orc_mat));
    for (int i = 0; i < n_mat; i++) {
        m->mats[i].type = (int)mats[7 * i];
        m->mats[i].id = (int)mats[7 * i + 1];
        memcpy(m->mats[i].C, mats + 7 * i + 2, sizeof(double) * 5);
        m->mats[i].kappa = orc_elasticity_coeff(m->mats[i].type, m->mats[i].C);
    }
    m->elem_mat = malloc(sizeof(int) * n_elem);
    for (int e = 0; e < n_elem; e++) {
        m->elem_mat[e] = -1;
        for (int i = 0; i < n_mat; i++)
            if (m->mats[i].id == elem_mat[e]) {
                m->elem_mat[e] = i;
                break;
            }
        if (m->elem_mat[e] < 0)
            m->n_skipped++;
    }
    /* free-DOF numbering, src/fe/Constraint.cpp:61-72 */
    m->id = malloc(sizeof(int) * n_nodes);
    int nf = 0;
    for (int i = 0; i < n_nodes; i++)
        m->id[i] = fixed[i] ? -1 : nf++;
    m->n_free = nf;
    /* Gauss rule and per-gp reference geometry, IntegralElement.cpp:3-19 */
    double pts[3 * MAXG], Ntmp[MAXN];
    m->ngp = gauss(nen, reduced, pts, m->gw);
    for (int g = 0; g < m->ngp; g++)
        shape(nen, pts + 3 * g, Ntmp, m->gdN[g]);
    m->J0inv = malloc(sizeof(double) * 9 * m->ngp * n_elem);
    m->T = malloc(sizeof(double) * 3 * nen * m->ngp * n_elem);
    m->vol = malloc(sizeof(double) * n_elem);
    double Y[3 * MAXN];
    for (int e = 0; e < n_elem; e++) {
        const int* c = m->conn + nen * e;
        for (int a = 0; a < nen; a++)
            memcpy(Y + 3 * a, m->X + 3 * c[a], sizeof(double) * 3);
        m->vol[e] = elem_volume(m, c);
        for (int g = 0; g < m->ngp; g++) {
            double J0[9];
            double* Ji = m->J0inv + 9 * (m->ngp * e + g);
            double* T = m->T + 3 * nen * (m->ngp * e + g);
            jacobi(nen, Y, m->gdN[g], J0);
            inv3(J0, Ji);
            /* T = J0^{-T} (dN/dxi)^T */
            for (int k = 0; k < 3; k++)
                for (int a = 0; a < nen; a++)
                    T[k * nen + a] = Ji[k] * m->gdN[g][3 * a] + Ji[3 + k] * m->gdN[g][3 * a + 1]
                        + Ji[6 + k] * m->gdN[g][3 * a + 2];
        }
    }
    /* node -> incident elements */
    m->inc_ptr = calloc(n_nodes + 1, sizeof(int));
    for (int i = 0; i < nen * n_elem; i++)
        m->inc_ptr[m->conn[i] + 1]++;
    for (int i = 0; i < n_nodes; i++)
        m->inc_ptr[i + 1] += m->inc_ptr[i];
    m->inc = malloc(sizeof(int) * nen * n_elem);
    int* fill = calloc(n_nodes, sizeof(int));
    for (int e = 0; e < n_elem; e++)
        for (int a = 0; a < nen; a++) {
            int n = m->conn[nen * e + a];
            m->inc[m->inc_ptr[n] + fill[n]++] = e;
        }
    free(fill);
    return m;
}

int orc_n_dof(const orc_model* m) { return 3 * m->n_free; }
int orc_n_elem_skipped(const orc_model* m) { return m->n_skipped; }

static int elem_has(const orc_model* m, int e, int node)
{
    for (int a = 0; a < m->nen; a++)
        if (m->conn[m->nen * e + a] == node)
            return 1;
    return 0;
}

static int face_has(const int* face, int nn, int node)
{
    for (int i = 0; i < nn; i++)
        if (face[i] == node)
            return 1;
    return 0;
}

/* A0 = 1/2 (p2 - p0) x (p1 - p0), flipped to point towards `ref`. */
static void tri_area(const double* p0, const double* p1, const double* p2, double* A)
{
    double u[3] = { p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2] };
    double v[3] = { p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2] };
    A[0] = 0.5 * (u[1] * v[2] - u[2] * v[1]);
    A[1] = 0.5 * (u[2] * v[0] - u[0] * v[2]);
    A[2] = 0.5 * (u[0] * v[1] - u[1] * v[0]);
}

static void orient(double* A, const double* ref, const double* p0)
{
    double d = (ref[0] - p0[0]) * A[0] + (ref[1] - p0[1]) * A[1] + (ref[2] - p0[2]) * A[2];
    if (d < 0) {
        A[0] = -A[0];
        A[1] = -A[1];
        A[2] = -A[2];
    }
}

/* Pressure faces, src/fe/ExternalConstraint.cpp:184-247 (config), :255-287
 * (parent element), :290-827 (face Gauss points and A0). */
int orc_add_pressure(orc_model* m, int n_faces, int face_nn, const int* faces, double value,
    const double* dvalue)
{
    int directed = dvalue != NULL;
    if (!directed && value <= 0)
        return 0; /* non-positive follower pressure is ignored, :195-197 */
    if (directed && sqrt(dvalue[0] * dvalue[0] + dvalue[1] * dvalue[1] + dvalue[2] * dvalue[2]) <= 0)
        return 0;
    m->faces = realloc(m->faces, sizeof(orc_face) * (m->n_faces + n_faces));
    const double* X = m->X;
    for (int f = 0; f < n_faces; f++) {
        const int* fn = faces + face_nn * f;
        /* de-duplicate node list (:205-211) */
        int nd[8], nn = 0;
        for (int i = 0; i < face_nn; i++)
            if (!face_has(nd, nn, fn[i]))
                nd[nn++] = fn[i];
        /* parent: the unique element holding every face node */
        int parent = -1, count = 0;
        for (int k = m->inc_ptr[nd[0]]; k < m->inc_ptr[nd[0] + 1]; k++) {
            int e = m->inc[k], all = 1;
            for (int i = 1; i < nn; i++)
                if (!elem_has(m, e, nd[i])) {
                    all = 0;
                    break;
                }
            if (all) {
                parent = e;
                count++;
            }
        }
        if (count != 1)
            return -1;
        orc_face* F = &m->faces[m->n_faces + f];
        memset(F, 0, sizeof(*F));
        F->elem = parent;
        F->directed = directed;
        F->value = value;
        if (directed)
            memcpy(F->dvalue, dvalue, sizeof(double) * 3);
        const int* ec = m->conn + m->nen * parent;
        double lc[9][3];
        int ng = 0;
        if (nn == 3 || nn == 6) {
            int miss = -1;
            for (int k = 0; k < 4; k++)
                if (!face_has(nd, nn, ec[k])) {
                    miss = k;
                    break;
                }
            if (miss < 0)
                return -2;
            if (nn == 3) {
                ng = 1;
                F->w[0] = 1.0;
                for (int k = 0; k < 3; k++)
                    lc[0][k] = 1.0 / 3.0;
                if (miss < 3)
                    lc[0][miss] = 0.0;
            } else {
                ng = 3;
                for (int g = 0; g < 3; g++) {
                    F->w[g] = 1.0 / 3.0;
                    if (miss == 0) {
                        for (int k = 0; k < 3; k++)
                            lc[g][k] = (k == g) ? 2.0 / 3.0 : 1.0 / 6.0;
                    } else {
                        /* the zero coordinate is miss-1; the others run
                         * (2/3,1/6), (1/6,2/3), (1/6,1/6) in index order */
                        int z = miss - 1, o[2], q = 0;
                        for (int k = 0; k < 3; k++)
                            if (k != z)
                                o[q++] = k;
                        lc[g][z] = 0.0;
                        lc[g][o[0]] = g == 0 ? 2.0 / 3.0 : 1.0 / 6.0;
                        lc[g][o[1]] = g == 1 ? 2.0 / 3.0 : 1.0 / 6.0;
                    }
                }
            }
            tri_area(X + 3 * nd[0], X + 3 * nd[1], X + 3 * nd[2], F->A0);
            orient(F->A0, X + 3 * ec[miss], X + 3 * nd[0]);
        } else if (nn == 4 || nn == 8) {
            /* the face is identified by two element corners it does NOT hold */
            static const int pairs[6][2] = { { 0, 2 }, { 0, 5 }, { 0, 7 }, { 6, 3 }, { 6, 1 }, { 6, 4 } };
            /* fixed local axis and its sign, per pair, in each element's frame */
            static const int ax8[6][2] = { { 2, 1 }, { 1, 1 }, { 0, 1 }, { 1, -1 }, { 0, -1 }, { 2, -1 } };
            static const int ax20[6][2] = { { 0, -1 }, { 2, -1 }, { 1, 1 }, { 2, 1 }, { 1, -1 }, { 0, 1 } };
            int p = -1;
            for (int k = 0; k < 6; k++)
                if (!face_has(nd, nn, ec[pairs[k][0]]) && !face_has(nd, nn, ec[pairs[k][1]])) {
                    p = k;
                    break;
                }
            if (p < 0)
                return -2;
            int ax = (nn == 4 ? ax8 : ax20)[p][0];
            double sg = (nn == 4 ? ax8 : ax20)[p][1];
            int o0 = ax == 0 ? 1 : 0, o1 = ax == 2 ? 1 : 2;
            if (nn == 4) {
                double a = sqrt(1.0 / 3.0);
                const double pat[4][2] = { { -a, -a }, { a, -a }, { a, a }, { -a, a } };
                ng = 4;
                for (int g = 0; g < 4; g++) {
                    lc[g][ax] = sg;
                    lc[g][o0] = pat[g][0];
                    lc[g][o1] = pat[g][1];
                    F->w[g] = 0.25;
                }
            } else {
                double c = sqrt(0.6);
                const double q[3] = { -c, 0.0, c }, qw[3] = { 5.0, 8.0, 5.0 };
                ng = 9;
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++) {
                        int g = 3 * i + j;
                        lc[g][ax] = sg;
                        lc[g][o0] = q[i];
                        lc[g][o1] = q[j];
                        F->w[g] = 0.25 * qw[i] * qw[j] / 81.0;
                    }
            }
            const double* ref = X + 3 * ec[pairs[p][0]];
            double A1[3], A2[3];
            tri_area(X + 3 * nd[0], X + 3 * nd[1], X + 3 * nd[2], A1);
            /* 1/2 (p0 - p3) x (p2 - p3) */
            tri_area(X + 3 * nd[3], X + 3 * nd[2], X + 3 * nd[0], A2);
            orient(A1, ref, X + 3 * nd[0]);
            orient(A2, ref, X + 3 * nd[0]);
            for (int k = 0; k < 3; k++)
                F->A0[k] = A1[k] + A2[k];
        } else {
            return -3;
        }
        F->ngp = ng;
        double Y[3 * MAXN];
        for (int a = 0; a < m->nen; a++)
            memcpy(Y + 3 * a, X + 3 * ec[a], sizeof(double) * 3);
        for (int g = 0; g < ng; g++) {
            double J0[9];
            shape(m->nen, lc[g], F->N[g], F->dN[g]);
            jacobi(m->nen, Y, F->dN[g], J0);
            inv3(J0, F->J0inv[g]);
        }
    }
    m->n_faces += n_faces;
    return 0;
}

int orc_add_force(orc_model* m, int n, const int* nodes, const double* f)
{
    m->force_node = realloc(m->force_node, sizeof(int) * (m->n_force + n));
    m->force_val = realloc(m->force_val, sizeof(double) * 3 * (m->n_force + n));
    for (int i = 0; i < n; i++) {
        m->force_node[m->n_force + i] = nodes[i];
        memcpy(m->force_val + 3 * (m->n_force + i), f, sizeof(double) * 3);
    }
    m->n_force += n;
    return 0;
}

/* Gravity (src/fe/InertiaConstraint.cpp:34-84 with the element mass of
 * src/fe/ElementConstraint.cpp:85-137): the residual gains -M g, with M the
 * consistent mass (rho V sum_g w_g N_i N_j, free-node pairs only) or the
 * lumped one (max(rho V, 4e-12) / nen on each free node of the element).
 * g is the acceleration vector; density[k] belongs to material index k.
 * The mass is built once, at set-up, from the element's own (full) Gauss
 * rule: the reference creates only full-integration elements
 * (src/fe/Constraint.cpp:9-20), so its consistent mass never sees a reduced
 * rule, and under reduced integration the mass keeps the full one. */
int orc_add_gravity(orc_model* m, const double* g, int consistent, const double* density)
{
    if (!m->gvec) m->gvec = calloc(3 * (size_t)(m->n_free > 0 ? m->n_free : 1), sizeof(double));
    double pts[3 * MAXG], w[MAXG], N[MAXN], dN[3 * MAXN];
    const int ngp = gauss(m->nen, 0, pts, w);
    for (int e = 0; e < m->n_elem; e++) {
        const int k = m->elem_mat[e];
        if (k < 0) continue;
        const int* c = m->conn + m->nen * e;
        const double V = m->vol[e], rho = density[k];
        if (consistent) {
            for (int q = 0; q < ngp; q++) {
                shape(m->nen, pts + 3 * q, N, dN);
                double sfree = 0.0;
                for (int j = 0; j < m->nen; j++)
                    if (m->id[c[j]] >= 0) sfree += N[j];
                for (int i = 0; i < m->nen; i++) {
                    const int id = m->id[c[i]];
                    if (id < 0) continue;
                    for (int d = 0; d < 3; d++) m->gvec[3 * id + d] += w[q] * rho * V * N[i] * sfree * g[d];
                }
            }
        } else {
            double mass = V * rho;
            if (mass < 4e-12) mass = 4e-12;
            mass /= m->nen;
            for (int i = 0; i < m->nen; i++) {
                const int id = m->id[c[i]];
                if (id < 0) continue;
                for (int d = 0; d < 3; d++) m->gvec[3 * id + d] += mass * g[d];
            }
        }
    }
    return 0;
}

/* Current nodal positions of element e: X + u for free nodes, X for fixed
 * ones (src/fe/Constraint.cpp:93-101). */
static void elem_pos(const orc_model* m, int e, const double* u, double* Y)
{
    for (int a = 0; a < m->nen; a++) {
        int n = m->conn[m->nen * e + a];
        for (int k = 0; k < 3; k++)
            Y[3 * a + k] = m->X[3 * n + k] + (m->id[n] >= 0 ? u[3 * m->id[n] + k] : 0.0);
    }
}

/* R(u), src/fe/Constraint.cpp:115-126: element internal forces
 * (ElementConstraint.cpp:139-162), then nodal forces (ExternalConstraint.cpp:149-167),
 * then pressure (:928-959), all added into a zeroed vector. */
void orc_residual(orc_model* m, const double* u, double* r)
{
    int nen = m->nen;
    memset(r, 0, sizeof(double) * 3 * m->n_free);
    double Y[3 * MAXN], re[3 * MAXN];
    for (int e = 0; e < m->n_elem; e++) {
        if (m->elem_mat[e] < 0)
            continue;
        const orc_mat* mat = &m->mats[m->elem_mat[e]];
        elem_pos(m, e, u, Y);
        memset(re, 0, sizeof(re));
        for (int g = 0; g < m->ngp; g++) {
            double J[9], F[9], P[9];
            jacobi(nen, Y, m->gdN[g], J);
            mul3(J, m->J0inv + 9 * (m->ngp * e + g), F);
            piola(mat->type, mat->C, F, P);
            double wv = m->vol[e] * m->gw[g];
            const double* T = m->T + 3 * nen * (m->ngp * e + g);
            for (int i = 0; i < 3; i++)
                for (int a = 0; a < nen; a++)
                    re[3 * a + i] += wv * (P[3 * i] * T[a] + P[3 * i + 1] * T[nen + a] + P[3 * i + 2] * T[2 * nen + a]);
        }
        for (int a = 0; a < nen; a++) {
            int id = m->id[m->conn[nen * e + a]];
            if (id >= 0)
                for (int k = 0; k < 3; k++)
                    r[3 * id + k] += re[3 * a + k];
        }
    }
    for (int i = 0; i < m->n_force; i++) {
        int id = m->id[m->force_node[i]];
        if (id >= 0)
            for (int k = 0; k < 3; k++)
                r[3 * id + k] -= m->force_val[3 * i + k];
    }
    for (int f = 0; f < m->n_faces; f++) {
        const orc_face* F = &m->faces[f];
        elem_pos(m, F->elem, u, Y);
        double cA[9][3], cn[9];
        for (int g = 0; g < F->ngp; g++) {
            double J[9], Fg[9], Fi[9];
            jacobi(nen, Y, F->dN[g], J);
            mul3(J, F->J0inv[g], Fg);
            inv3(Fg, Fi);
            double d = det3(Fg);
            /* det(F) F^{-T} A0 */
            for (int i = 0; i < 3; i++)
                cA[g][i] = d * (Fi[i] * F->A0[0] + Fi[3 + i] * F->A0[1] + Fi[6 + i] * F->A0[2]);
            cn[g] = sqrt(cA[g][0] * cA[g][0] + cA[g][1] * cA[g][1] + cA[g][2] * cA[g][2]);
        }
        const int* ec = m->conn + nen * F->elem;
        for (int a = 0; a < nen; a++) {
            double v[3] = { 0, 0, 0 };
            if (F->directed) {
                double area = 0.0;
                for (int g = 0; g < F->ngp; g++)
                    area += F->w[g] * F->N[g][a] * cn[g];
                for (int k = 0; k < 3; k++)
                    v[k] = F->dvalue[k] * area;
            } else {
                for (int g = 0; g < F->ngp; g++)
                    for (int k = 0; k < 3; k++)
                        v[k] += F->w[g] * F->N[g][a] * cA[g][k];
                for (int k = 0; k < 3; k++)
                    v[k] *= F->value;
            }
            int id = m->id[ec[a]];
            if (id >= 0)
                for (int k = 0; k < 3; k++)
                    r[3 * id + k] -= v[k];
        }
    }
    /* the inertia constraint is appended last (src/fe/Constraint.cpp:87-90) */
    if (m->gvec)
        for (int i = 0; i < 3 * m->n_free; i++) r[i] -= m->gvec[i];
}

/* Scalar approximate Jacobian, ElementConstraint.cpp:164-205:
 * L_jk = sum_e V_e kappa_e sum_g w_g (T_g^T T_g)_jk over free node pairs. */
static void add_L_entries(orc_model* m, void (*put)(void*, int, int, double), void* ctx)
{
    int nen = m->nen;
    for (int e = 0; e < m->n_elem; e++) {
        if (m->elem_mat[e] < 0)
            continue;
        double ks = m->vol[e] * m->mats[m->elem_mat[e]].kappa;
        const int* c = m->conn + nen * e;
        for (int g = 0; g < m->ngp; g++) {
            const double* T = m->T + 3 * nen * (m->ngp * e + g);
            double w = ks * m->gw[g];
            for (int j = 0; j < nen; j++) {
                int ij = m->id[c[j]];
                if (ij < 0)
                    continue;
                for (int k = 0; k < nen; k++) {
                    int ik = m->id[c[k]];
                    if (ik < 0)
                        continue;
                    double s = T[j] * T[k] + T[nen + j] * T[nen + k] + T[2 * nen + j] * T[2 * nen + k];
                    put(ctx, ij, ik, w * s);
                }
            }
        }
    }
}

typedef struct {
    double* L;
    int n;
} dense_ctx;

static void put_dense(void* c, int i, int j, double v)
{
    dense_ctx* d = c;
    d->L[(size_t)i * d->n + j] += v;
}

void orc_approx_jacobian_dense(orc_model* m, double* L)
{
    memset(L, 0, sizeof(double) * (size_t)m->n_free * m->n_free);
    dense_ctx c = { L, m->n_free };
    add_L_entries(m, put_dense, &c);
}

/* ------------------------------------------------------------------ skyline Cholesky
 * The reference factors L (x) I3 with Eigen SimplicialLLT + AMD
 * (src/simulation/nlsolver/LBFGS.h:65-81); any exact LL^T of the same matrix
 * applies the same H0 up to rounding, so the restatement uses a reverse
 * Cuthill-McKee ordering and an envelope (skyline) factor of the scalar L. */
typedef struct {
    int n;
    int* perm;   /* new -> old */
    int* iperm;  /* old -> new */
    int* first;  /* first column of row i (new numbering) */
    long* rowp;  /* start of row i in val */
    double* val;
} skyline;

typedef struct {
    skyline* s;
} sky_ctx;

static void put_sky(void* c, int i, int j, double v)
{
    skyline* s = ((sky_ctx*)c)->s;
    int a = s->iperm[i], b = s->iperm[j];
    if (b > a)
        return; /* lower triangle only (symmetric) */
    s->val[s->rowp[a] + (b - s->first[a])] += v;
}

static void sky_free(skyline* s)
{
    if (!s)
        return;
    free(s->perm);
    free(s->iperm);
    free(s->first);
    free(s->rowp);
    free(s->val);
    free(s);
}

static skyline* sky_build(orc_model* m)
{
    int n = m->n_free, nen = m->nen;
    /* node graph of free nodes */
    int* deg = calloc(n + 1, sizeof(int));
    /* adjacency via sorted unique lists per node: gather element neighbours */
    int* ptr = calloc(n + 1, sizeof(int));
    for (int e = 0; e < m->n_elem; e++) {
        if (m->elem_mat[e] < 0)
            continue;
        for (int a = 0; a < nen; a++) {
            int ia = m->id[m->conn[nen * e + a]];
            if (ia >= 0)
                ptr[ia + 1] += nen;
        }
    }
    for (int i = 0; i < n; i++)
        ptr[i + 1] += ptr[i];
    int* adj = malloc(sizeof(int) * (ptr[n] > 0 ? ptr[n] : 1));
    int* fill = calloc(n, sizeof(int));
    for (int e = 0; e < m->n_elem; e++) {
        if (m->elem_mat[e] < 0)
            continue;
        for (int a = 0; a < nen; a++) {
            int ia = m->id[m->conn[nen * e + a]];
            if (ia < 0)
                continue;
            for (int b = 0; b < nen; b++) {
                int ib = m->id[m->conn[nen * e + b]];
                adj[ptr[ia] + fill[ia]++] = ib; /* -1 for fixed, skipped below */
            }
        }
    }
    /* dedupe each list (mark array) */
    int* mark = malloc(sizeof(int) * n);
    for (int i = 0; i < n; i++)
        mark[i] = -1;
    int* nptr = calloc(n + 1, sizeof(int));
    int* nadj = malloc(sizeof(int) * (ptr[n] > 0 ? ptr[n] : 1));
    int q = 0;
    for (int i = 0; i < n; i++) {
        nptr[i] = q;
        for (int k = ptr[i]; k < ptr[i] + fill[i]; k++) {
            int j = adj[k];
            if (j >= 0 && j != i && mark[j] != i) {
                mark[j] = i;
                nadj[q++] = j;
            }
        }
        deg[i] = q - nptr[i];
    }
    nptr[n] = q;
    free(adj);
    free(fill);
    free(ptr);
    /* reverse Cuthill-McKee from a minimum-degree start, per component */
    skyline* s = calloc(1, sizeof(skyline));
    s->n = n;
    s->perm = malloc(sizeof(int) * (n > 0 ? n : 1));
    s->iperm = malloc(sizeof(int) * (n > 0 ? n : 1));
    char* seen = calloc(n > 0 ? n : 1, 1);
    int head = 0, tail = 0;
    while (tail < n) {
        int start = -1;
        for (int i = 0; i < n; i++)
            if (!seen[i] && (start < 0 || deg[i] < deg[start]))
                start = i;
        seen[start] = 1;
        s->perm[tail++] = start;
        while (head < tail) {
            int v = s->perm[head++];
            int b0 = tail;
            for (int k = nptr[v]; k < nptr[v + 1]; k++) {
                int w = nadj[k];
                if (!seen[w]) {
                    seen[w] = 1;
                    s->perm[tail++] = w;
                }
            }
            /* neighbours in increasing degree (insertion sort) */
            for (int a = b0 + 1; a < tail; a++) {
                int x = s->perm[a], bb = a - 1;
                while (bb >= b0 && deg[s->perm[bb]] > deg[x]) {
                    s->perm[bb + 1] = s->perm[bb];
                    bb--;
                }
                s->perm[bb + 1] = x;
            }
        }
    }
    for (int i = 0; i < n / 2; i++) {
        int t = s->perm[i];
        s->perm[i] = s->perm[n - 1 - i];
        s->perm[n - 1 - i] = t;
    }
    for (int i = 0; i < n; i++)
        s->iperm[s->perm[i]] = i;
    s->first = malloc(sizeof(int) * (n > 0 ? n : 1));
    s->rowp = malloc(sizeof(long) * (n + 1));
    for (int i = 0; i < n; i++) {
        int f = i, o = s->perm[i];
        for (int k = nptr[o]; k < nptr[o + 1]; k++) {
            int j = s->iperm[nadj[k]];
            if (j < f)
                f = j;
        }
        s->first[i] = f;
    }
    s->rowp[0] = 0;
    for (int i = 0; i < n; i++)
        s->rowp[i + 1] = s->rowp[i] + (i - s->first[i] + 1);
    s->val = calloc(s->rowp[n] > 0 ? s->rowp[n] : 1, sizeof(double));
    free(seen);
    free(mark);
    free(nptr);
    free(nadj);
    free(deg);
    sky_ctx c = { s };
    add_L_entries(m, put_sky, &c);
    return s;
}

/* In-place row-oriented envelope Cholesky; returns 0 if not positive definite. */
static int sky_factor(skyline* s)
{
    for (int i = 0; i < s->n; i++) {
        double* Li = s->val + s->rowp[i];
        int fi = s->first[i];
        for (int j = fi; j <= i; j++) {
            double* Lj = s->val + s->rowp[j];
            int fj = s->first[j];
            int k0 = fi > fj ? fi : fj;
            double sum = Li[j - fi];
            for (int k = k0; k < j; k++)
                sum -= Li[k - fi] * Lj[k - fj];
            if (j < i) {
                Li[j - fi] = sum / Lj[j - fj];
            } else {
                if (!(sum > 0.0))
                    return 0;
                Li[i - fi] = sqrt(sum);
            }
        }
    }
    return 1;
}

/* v (interleaved 3 components, old numbering) <- L^{-T} L^{-1} v per component */
static void sky_solve(const skyline* s, double* v, double* w)
{
    int n = s->n;
    for (int c = 0; c < 3; c++) {
        for (int i = 0; i < n; i++)
            w[i] = v[3 * s->perm[i] + c];
        for (int i = 0; i < n; i++) {
            const double* Li = s->val + s->rowp[i];
            int fi = s->first[i];
            double sum = w[i];
            for (int k = fi; k < i; k++)
                sum -= Li[k - fi] * w[k];
            w[i] = sum / Li[i - fi];
        }
        for (int i = n - 1; i >= 0; i--) {
            const double* Li = s->val + s->rowp[i];
            int fi = s->first[i];
            w[i] /= Li[i - fi];
            for (int k = fi; k < i; k++)
                w[k] -= Li[k - fi] * w[i];
        }
        for (int i = 0; i < n; i++)
            v[3 * s->perm[i] + c] = w[i];
    }
}

/* ------------------------------------------------------------------ L-BFGS
 * src/simulation/nlsolver/LBFGS.h:96-174, LBFGSMat.h:59-131, LineSearchFEA.h:37-68. */
static double dot(const double* a, const double* b, int n)
{
    double s = 0.0;
    for (int i = 0; i < n; i++)
        s += a[i] * b[i];
    return s;
}

static double inf_norm(const double* a, int n)
{
    double s = 0.0;
    for (int i = 0; i < n; i++)
        if (fabs(a[i]) > s)
            s = fabs(a[i]);
    return s;
}

/* H0 v = (L (x) I3)^{-1} v; returns 0 if L is not positive definite. */
int orc_precond_apply(orc_model* m, double* v)
{
    skyline* sky = sky_build(m);
    int ok = sky->n > 0 && sky_factor(sky);
    if (ok) {
        double* work = malloc(sizeof(double) * (m->n_free + 1));
        sky_solve(sky, v, work);
        free(work);
    }
    sky_free(sky);
    return ok;
}

/* The solve's convergence record (the reference's benchmark vector,
 * src/simulation/nlsolver/LBFGS.h:107-147): record 0 after the initial
 * residual, record i after iteration i's line search; 5 doubles each
 * (0, ||r||_2, ||r||_inf, step of the last trial, residual evaluations). */
void orc_set_trace(orc_model* m, double* buf, int cap)
{
    m->trace = buf;
    m->trace_cap = buf ? cap : 0;
    m->trace_n = 0;
}

int orc_trace_count(const orc_model* m) { return m->trace_n; }

static void trace_record(orc_model* m, const double* r, int n, double step, int evals)
{
    if (m->trace && m->trace_n < m->trace_cap) {
        double* rec = m->trace + 5 * (size_t)m->trace_n;
        rec[0] = 0.0;
        rec[1] = sqrt(dot(r, r, n));
        rec[2] = inf_norm(r, n);
        rec[3] = step;
        rec[4] = evals;
    }
    m->trace_n++;
}

int orc_solve(orc_model* m, const orc_params* p, double* x, orc_info* info)
{
    int n = 3 * m->n_free, mm = p->m;
    double *r = malloc(sizeof(double) * n), *xp = malloc(sizeof(double) * n), *rp = malloc(sizeof(double) * n);
    double *d = malloc(sizeof(double) * n), *S = malloc(sizeof(double) * n * mm), *Yh = malloc(sizeof(double) * n * mm);
    double *ys = malloc(sizeof(double) * mm), *alpha = malloc(sizeof(double) * mm);
    double* work = malloc(sizeof(double) * (m->n_free + 1));
    skyline* sky = NULL;
    int evals = 0, ok = 0, k = 1, ncorr = 0, ptr = mm;
    double theta = 1.0;
    memset(info, 0, sizeof(*info));

    m->trace_n = 0;
    orc_residual(m, x, r);
    evals++;
    trace_record(m, r, n, 0.0, 1);
    double gnorm = inf_norm(r, n);
    if (gnorm <= p->epsilon || gnorm <= p->epsilon * sqrt(dot(x, x, n))) {
        k = 1;
        goto done;
    }
    if (p->use_precond) {
        sky = sky_build(m);
        ok = sky->n > 0 && sky_factor(sky);
        if (!ok) {
            sky_free(sky);
            sky = NULL;
        }
    }
    for (int i = 0; i < n; i++)
        d[i] = -r[i];
    if (ok)
        sky_solve(sky, d, work);
    for (;;) {
        memcpy(xp, x, sizeof(double) * n);
        memcpy(rp, r, sizeof(double) * n);
        /* residual-projection line search */
        double dg0 = dot(r, d, n), step = 1.0, tried = 1.0;
        int trials = 0;
        for (int it = 0; it < p->max_linesearch; it++) {
            for (int i = 0; i < n; i++)
                x[i] = xp[i] + step * d[i];
            orc_residual(m, x, r);
            evals++;
            trials++;
            tried = step;
            double dg = dot(r, d, n);
            if (fabs(dg) <= fabs(dg0))
                break;
            step *= dg * dg0 > 0 ? 1.5 : 0.5;
        }
        trace_record(m, r, n, tried, trials);
        gnorm = inf_norm(r, n);
        if (gnorm <= p->epsilon || gnorm <= p->epsilon * inf_norm(x, n))
            break;
        if (p->max_iterations != 0 && k >= p->max_iterations)
            break;
        /* add_correction */
        int loc = ptr % mm;
        double* s = S + (size_t)n * loc;
        double* y = Yh + (size_t)n * loc;
        for (int i = 0; i < n; i++) {
            s[i] = x[i] - xp[i];
            y[i] = r[i] - rp[i];
        }
        ys[loc] = dot(s, y, n);
        theta = dot(y, y, n) / ys[loc];
        if (ncorr < mm)
            ncorr++;
        ptr = loc + 1;
        /* d = -H r, two-loop recursion */
        for (int i = 0; i < n; i++)
            d[i] = -r[i];
        int j = ptr % mm;
        for (int i = 0; i < ncorr; i++) {
            j = (j + mm - 1) % mm;
            alpha[j] = dot(S + (size_t)n * j, d, n) / ys[j];
            for (int t = 0; t < n; t++)
                d[t] -= alpha[j] * Yh[(size_t)n * j + t];
        }
        if (ok)
            sky_solve(sky, d, work);
        else
            for (int t = 0; t < n; t++)
                d[t] /= theta;
        for (int i = 0; i < ncorr; i++) {
            double beta = dot(Yh + (size_t)n * j, d, n) / ys[j];
            for (int t = 0; t < n; t++)
                d[t] += (alpha[j] - beta) * S[(size_t)n * j + t];
            j = (j + 1) % mm;
        }
        k++;
    }
done:
    info->niter = k;
    info->r_evals = evals;
    info->precond_ok = ok;
    info->u_inf = inf_norm(x, n);
    info->r_inf = inf_norm(r, n);
    sky_free(sky);
    free(r);
    free(xp);
    free(rp);
    free(d);
    free(S);
    free(Yh);
    free(ys);
    free(alpha);
    free(work);
    return 0;
}

void orc_destroy(orc_model* m)
{
    if (!m)
        return;
    free(m->X);
    free(m->conn);
    free(m->id);
    free(m->elem_mat);
    free(m->mats);
    free(m->J0inv);
    free(m->T);
    free(m->vol);
    free(m->faces);
    free(m->force_node);
    free(m->force_val);
    free(m->gvec);
    free(m->inc_ptr);
    free(m->inc);
    free(m);
}
