#include "elements.h"

#include <cmath>
#include <cstring>

namespace efem {

namespace {
// C3D8 corner signs, src/fe/element/HexahedraElement.cpp:19-26
const double kHex8[8][3] = { { -1, -1, -1 }, { 1, -1, -1 }, { 1, 1, -1 }, { -1, 1, -1 },
    { -1, -1, 1 }, { 1, -1, 1 }, { 1, 1, 1 }, { -1, 1, 1 } };
// C3D20 corner coordinates in the reference's local frame (the corner factor
// of each N_a in src/fe/element/HexahedraElement.cpp:151-158)
const double kHex20[8][3] = { { 1, -1, 1 }, { 1, 1, 1 }, { 1, 1, -1 }, { 1, -1, -1 },
    { -1, -1, 1 }, { -1, 1, 1 }, { -1, 1, -1 }, { -1, -1, -1 } };
const int kHexEdge[12][2] = { { 0, 1 }, { 1, 2 }, { 2, 3 }, { 3, 0 }, { 4, 5 }, { 5, 6 }, { 6, 7 },
    { 7, 4 }, { 0, 4 }, { 1, 5 }, { 2, 6 }, { 3, 7 } };
}  // namespace

void shape_functions(int kind, const double* p, double* N, double* dN)
{
    const double x = p[0], y = p[1], z = p[2];
    switch (kind) {
    case K_TET4: {
        N[0] = x;
        N[1] = y;
        N[2] = z;
        N[3] = 1.0 - x - y - z;
        const double g[12] = { 1, 0, 0, 0, 1, 0, 0, 0, 1, -1, -1, -1 };
        std::memcpy(dN, g, sizeof(g));
        break;
    }
    case K_TET10: {
        const double L = 1.0 - x - y - z;
        const double n[10] = { L * (2 * L - 1), x * (2 * x - 1), y * (2 * y - 1), z * (2 * z - 1), 4 * L * x,
            4 * x * y, 4 * y * L, 4 * z * L, 4 * x * z, 4 * y * z };
        const double g[30] = { 1 - 4 * L, 1 - 4 * L, 1 - 4 * L, 4 * x - 1, 0, 0, 0, 4 * y - 1, 0, 0, 0,
            4 * z - 1, 4 * (L - x), -4 * x, -4 * x, 4 * y, 4 * x, 0, -4 * y, 4 * (L - y), -4 * y, -4 * z,
            -4 * z, 4 * (L - z), 4 * z, 0, 4 * x, 0, 4 * z, 4 * y };
        std::memcpy(N, n, sizeof(n));
        std::memcpy(dN, g, sizeof(g));
        break;
    }
    case K_HEX8:
        for (int a = 0; a < 8; a++) {
            const double sx = kHex8[a][0], sy = kHex8[a][1], sz = kHex8[a][2];
            const double A = 1 + sx * x, B = 1 + sy * y, C = 1 + sz * z;
            N[a] = 0.125 * A * B * C;
            dN[3 * a] = 0.125 * sx * B * C;
            dN[3 * a + 1] = 0.125 * A * sy * C;
            dN[3 * a + 2] = 0.125 * A * B * sz;
        }
        break;
    case K_HEX20:
        for (int a = 0; a < 8; a++) {
            const double sx = kHex20[a][0], sy = kHex20[a][1], sz = kHex20[a][2];
            const double A = 1 + sx * x, B = 1 + sy * y, C = 1 + sz * z;
            N[a] = 0.125 * A * B * C * (sx * x + sy * y + sz * z - 2);
            dN[3 * a] = 0.125 * sx * B * C * (2 * sx * x + sy * y + sz * z - 1);
            dN[3 * a + 1] = 0.125 * sy * A * C * (sx * x + 2 * sy * y + sz * z - 1);
            dN[3 * a + 2] = 0.125 * sz * A * B * (sx * x + sy * y + 2 * sz * z - 1);
        }
        for (int e = 0; e < 12; e++) {
            const int a = 8 + e;
            double c[3];
            for (int k = 0; k < 3; k++) c[k] = 0.5 * (kHex20[kHexEdge[e][0]][k] + kHex20[kHexEdge[e][1]][k]);
            const double A = 1 + c[0] * x, B = 1 + c[1] * y, C = 1 + c[2] * z;
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
        break;
    }
}

int gauss_rule(int kind, bool reduced, double* pts, double* w)
{
    enum { TET1, TET4, HEX1, HEX8, HEX27 } rule;
    if (kind == K_TET4)
        rule = TET1;
    else if (kind == K_TET10)
        rule = reduced ? TET1 : TET4;
    else if (kind == K_HEX8)
        rule = reduced ? HEX1 : HEX8;
    else
        rule = reduced ? HEX8 : HEX27;
    switch (rule) {
    case TET1:
        pts[0] = pts[1] = pts[2] = 0.25;
        w[0] = 1.0;
        return 1;
    case TET4: {
        // the reference's 8-digit constants, IntegralElement.inl:41-47
        const double a = 0.58541020, b = 0.13819660;
        const double t[4][3] = { { a, b, b }, { b, a, b }, { b, b, a }, { b, b, b } };
        for (int g = 0; g < 4; g++) {
            for (int k = 0; k < 3; k++) pts[3 * g + k] = t[g][k];
            w[g] = 0.25;
        }
        return 4;
    }
    case HEX1:
        pts[0] = pts[1] = pts[2] = 0.0;
        w[0] = 1.0;
        return 1;
    case HEX8: {
        const double a = 1.0 / std::sqrt(3.0);
        for (int g = 0; g < 8; g++) {
            for (int k = 0; k < 3; k++) pts[3 * g + k] = a * kHex8[g][k];
            w[g] = 0.125;
        }
        return 8;
    }
    case HEX27: {
        const double c = std::sqrt(3.0 / 5.0);
        const double q[3] = { -c, 0.0, c }, qw[3] = { 5.0, 8.0, 5.0 };
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
    return 0;
}

int face_rule(int face_nn, bool (*elem_has)(const void*, int), const void* ctx, double* pts, double* w,
    int* ref_node)
{
    if (face_nn == 3 || face_nn == 6) {
        // the first element corner (0..3) missing from the face fixes the rule
        int miss = -1;
        for (int k = 0; k < 4; k++)
            if (!elem_has(ctx, k)) {
                miss = k;
                break;
            }
        if (miss < 0) return 0;
        *ref_node = miss;
        if (face_nn == 3) {
            // centroid; ExternalConstraint.cpp:292-337
            for (int k = 0; k < 3; k++) pts[k] = 1.0 / 3.0;
            if (miss < 3) pts[miss] = 0.0;
            w[0] = 1.0;
            return 1;
        }
        // three-point rule; ExternalConstraint.cpp:338-409
        for (int g = 0; g < 3; g++) {
            w[g] = 1.0 / 3.0;
            double* p = pts + 3 * g;
            if (miss == 0) {
                for (int k = 0; k < 3; k++) p[k] = (k == g) ? 2.0 / 3.0 : 1.0 / 6.0;
            } else {
                const int zero = miss - 1;
                int o[2], q = 0;
                for (int k = 0; k < 3; k++)
                    if (k != zero) o[q++] = k;
                p[zero] = 0.0;
                p[o[0]] = g == 0 ? 2.0 / 3.0 : 1.0 / 6.0;
                p[o[1]] = g == 1 ? 2.0 / 3.0 : 1.0 / 6.0;
            }
        }
        return 3;
    }
    if (face_nn == 4 || face_nn == 8) {
        // a hexahedron face is named by two corners it does not hold;
        // ExternalConstraint.cpp:410-564 (4 nodes), :565-816 (8 nodes)
        static const int pairs[6][2] = { { 0, 2 }, { 0, 5 }, { 0, 7 }, { 6, 3 }, { 6, 1 }, { 6, 4 } };
        // (fixed local axis, its value) per pair, C3D8 frame and C3D20 frame
        static const int ax8[6][2] = { { 2, 1 }, { 1, 1 }, { 0, 1 }, { 1, -1 }, { 0, -1 }, { 2, -1 } };
        static const int ax20[6][2] = { { 0, -1 }, { 2, -1 }, { 1, 1 }, { 2, 1 }, { 1, -1 }, { 0, 1 } };
        int p = -1;
        for (int k = 0; k < 6; k++)
            if (!elem_has(ctx, pairs[k][0]) && !elem_has(ctx, pairs[k][1])) {
                p = k;
                break;
            }
        if (p < 0) return 0;
        *ref_node = pairs[p][0];
        const int(*ax)[2] = face_nn == 4 ? ax8 : ax20;
        const int fixed = ax[p][0];
        const double val = ax[p][1];
        const int o0 = fixed == 0 ? 1 : 0, o1 = fixed == 2 ? 1 : 2;
        if (face_nn == 4) {
            const double a = std::sqrt(1.0 / 3.0);
            const double pat[4][2] = { { -a, -a }, { a, -a }, { a, a }, { -a, a } };
            for (int g = 0; g < 4; g++) {
                pts[3 * g + fixed] = val;
                pts[3 * g + o0] = pat[g][0];
                pts[3 * g + o1] = pat[g][1];
                w[g] = 0.25;
            }
            return 4;
        }
        const double c = std::sqrt(0.6);
        const double q[3] = { -c, 0.0, c }, qw[3] = { 5.0, 8.0, 5.0 };
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                const int g = 3 * i + j;
                pts[3 * g + fixed] = val;
                pts[3 * g + o0] = q[i];
                pts[3 * g + o1] = q[j];
                w[g] = 0.25 * qw[i] * qw[j] / 81.0;
            }
        return 9;
    }
    return 0;
}

}  // namespace efem
