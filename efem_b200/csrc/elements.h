// Element library on the host: shape functions, Gauss rules and pressure-face
// integration points of the reference's four element families, used to build
// the constant tables the CUDA kernels read.
//
//   C3D4  src/fe/element/TetrahedraElement.cpp:15-33     N = (xi, eta, zeta, 1-xi-eta-zeta)
//   C3D10 src/fe/element/TetrahedraElement.cpp:62-122    node 0 <-> 1-xi-eta-zeta
//   C3D8  src/fe/element/HexahedraElement.cpp:15-58      corners (-,-,-),(+,-,-),...
//   C3D20 src/fe/element/HexahedraElement.cpp:147-238    corner 0 at (1,-1,1), serendipity
//   Gauss rules (weights normalised to sum 1): src/fe/element/IntegralElement.inl:3-223
#pragma once
#include <vector>

namespace efem {

constexpr int MAX_NEN = 20;
constexpr int MAX_NGP = 27;
constexpr int MAX_FGP = 9;

// element kinds, one per node count
enum ElemKind { K_TET4 = 0, K_TET10 = 1, K_HEX8 = 2, K_HEX20 = 3 };

inline int kind_of_nen(int nen)
{
    return nen == 4 ? K_TET4 : nen == 10 ? K_TET10 : nen == 8 ? K_HEX8 : nen == 20 ? K_HEX20 : -1;
}
inline int nen_of_kind(int k)
{
    static const int n[4] = { 4, 10, 8, 20 };
    return n[k];
}

// N[a] and dN[a][3] at local point p
void shape_functions(int kind, const double* p, double* N, double* dN);

// Gauss rule; returns the number of points.
// reduced: C3D4R/C3D10R 1 point, C3D8R 1 point, C3D20R 2x2x2
// (src/fe/element/IntegralElement.h:76-157).
int gauss_rule(int kind, bool reduced, double* pts, double* w);

// Pressure-face integration points in the parent element's local frame,
// chosen by which element corners the face does not hold
// (src/fe/ExternalConstraint.cpp:290-827).  face_nn is the number of distinct
// nodes listed for the face (3, 6, 4 or 8); elem_has(i) tells whether element
// node i belongs to the face.  Returns the number of points (0 if no rule
// matches) and sets *ref_node to the element node A0 is oriented towards.
int face_rule(int face_nn, bool (*elem_has)(const void*, int), const void* ctx, double* pts, double* w,
    int* ref_node);

}  // namespace efem
