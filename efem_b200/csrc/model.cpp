// Model set-up (host) and the C ABI entry points.
//
// Set-up mirrors the reference's Constraint construction
// (src/fe/Constraint.cpp:22-91): element integration data
// (src/fe/element/IntegralElement.cpp:3-19), materials
// (src/fe/ElementConstraint.cpp:11-67), fixed nodes and DOF numbering
// (src/fe/ExternalConstraint.cpp:50-82, src/fe/Constraint.cpp:61-72), nodal
// forces (:91-167) and pressure faces (:184-827).  Host set-up needs no GPU;
// device buffers are created on the first call that computes.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>

#include "efem_internal.h"

namespace efem {

namespace {
thread_local std::string g_error;

void inv3(const double* a, double* o)
{
    const double d = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6])
        + a[2] * (a[3] * a[7] - a[4] * a[6]);
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

// J0 = X . dN for element nodal coordinates Y (nen x 3)
void jacobi(int nen, const double* Y, const double* dN, double* J)
{
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) {
            double s = 0;
            for (int a = 0; a < nen; a++) s += Y[3 * a + i] * dN[3 * a + k];
            J[3 * i + k] = s;
        }
}

// Element volume from the corner nodes: tets |det|/6, hexahedra by the
// divergence theorem over the corner faces split as a-b-c + a-c-d.  For
// straight-edged elements with planar faces this is the exact volume, which
// is what the reference's VTK triangulated-surface volume returns
// (src/model/Element.h:72-89).
double corner_volume(int nen, const double* Y)
{
    if (nen == 4 || nen == 10) {
        double a[3], b[3], c[3];
        for (int k = 0; k < 3; k++) {
            a[k] = Y[3 + k] - Y[k];
            b[k] = Y[6 + k] - Y[k];
            c[k] = Y[9 + k] - Y[k];
        }
        return std::fabs(a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0])
                   + a[2] * (b[0] * c[1] - b[1] * c[0]))
            / 6.0;
    }
    static const int F[6][4] = { { 0, 3, 2, 1 }, { 4, 5, 6, 7 }, { 0, 1, 5, 4 }, { 1, 2, 6, 5 }, { 2, 3, 7, 6 }, { 3, 0, 4, 7 } };
    auto triple = [](const double* a, const double* b, const double* c) {
        return a[0] * (b[1] * c[2] - b[2] * c[1]) + a[1] * (b[2] * c[0] - b[0] * c[2]) + a[2] * (b[0] * c[1] - b[1] * c[0]);
    };
    double v6 = 0;
    for (int f = 0; f < 6; f++) {
        const double *a = Y + 3 * F[f][0], *b = Y + 3 * F[f][1], *c = Y + 3 * F[f][2], *d = Y + 3 * F[f][3];
        v6 += triple(a, b, c) + triple(a, c, d);
    }
    return std::fabs(v6) / 6.0;
}

double elasticity_coeff(const HostMaterial& m)
{
    // the reference's preconditioner scale ("t=2.0" fit), NeoHookean.cpp:41,
    // MooneyRivlin.cpp:48, Yeoh.cpp:47
    if (m.type == EFEM_MOONEY_RIVLIN) return 3.818 * m.C01 + 2.94001 * m.C10 + 2.0 / m.D1;
    if (m.type == EFEM_YEOH) return 2.94001 * m.C10 + 3.51194 * m.C20 + 3.3154 * m.C30 + 2.0 / m.D1;
    return 2.94001 * m.C10 + 2.0 / m.D1;
}

// External load vector: the nodal forces plus, under gravity, M g as the
// reference's inertia constraint adds it (src/fe/InertiaConstraint.cpp:34-50
// with the element mass of src/fe/ElementConstraint.cpp:85-137):
//   consistent  M_ab = rho V_e sum_q w_q N_a(q) N_b(q) over free node pairs,
//               so row a of M g is rho V_e sum_q w_q N_a(q) sum_{b free} N_b(q) g;
//   lumped      max(rho V_e, 4e-12) / nen on each free node.
// The consistent mass always uses the element's full Gauss rule: the reference
// builds it from the full-integration element it creates
// (src/fe/Constraint.cpp:9-20), whatever rule the residual uses.
void external_load(const Model& m, std::vector<double>& f)
{
    f = m.h_fnodal;
    if (!m.has_gravity) return;
    const double* g = m.gravity;
    const bool consistent = m.opts.consistent_inertia != 0;
    for (auto& hb : m.in_blocks) {
        const int kind = kind_of_nen(hb.nen), nen = hb.nen;
        double pts[3 * MAX_NGP], w[MAX_NGP], dN[3 * MAX_NEN];
        std::vector<double> N(static_cast<size_t>(MAX_NGP) * MAX_NEN);
        const int ngp = gauss_rule(kind, false, pts, w);
        for (int q = 0; q < ngp; q++) shape_functions(kind, pts + 3 * q, N.data() + static_cast<size_t>(q) * MAX_NEN, dN);
        double Y[3 * MAX_NEN];
        int d[MAX_NEN];
        for (size_t e = 0; e < hb.mat_id.size(); e++) {
            const int* c = hb.conn.data() + e * nen;
            for (int a = 0; a < nen; a++) {
                std::memcpy(Y + 3 * a, m.X.data() + 3 * static_cast<size_t>(c[a]), sizeof(double) * 3);
                d[a] = m.dnode_of_node[c[a]];
            }
            const double V = corner_volume(nen, Y), rho = m.materials_used[hb.mat_id[e]].density;
            if (consistent) {
                for (int q = 0; q < ngp; q++) {
                    const double* Nq = N.data() + static_cast<size_t>(q) * MAX_NEN;
                    double sfree = 0.0;
                    for (int b = 0; b < nen; b++)
                        if (d[b] < m.n_free) sfree += Nq[b];
                    for (int a = 0; a < nen; a++) {
                        if (d[a] >= m.n_free) continue;
                        const double s = w[q] * rho * V * Nq[a] * sfree;
                        for (int k = 0; k < 3; k++) f[3 * static_cast<size_t>(d[a]) + k] += s * g[k];
                    }
                }
            } else {
                const double mass = std::max(V * rho, 4e-12) / nen;
                for (int a = 0; a < nen; a++)
                    if (d[a] < m.n_free)
                        for (int k = 0; k < 3; k++) f[3 * static_cast<size_t>(d[a]) + k] += mass * g[k];
            }
        }
    }
}

struct FaceHost {
    int kind, table_key, load, ngp;
    std::vector<int> enodes;  // parent element's nodes (original ids)
    double A0[3];
    double J0inv[MAX_FGP][9];
    double pts[3 * MAX_FGP], w[MAX_FGP];
};

struct FaceCtx {
    const std::vector<int>* face;
    const int* enodes;
};
bool face_has_elem_node(const void* c, int i)
{
    const FaceCtx* f = static_cast<const FaceCtx*>(c);
    return std::find(f->face->begin(), f->face->end(), f->enodes[i]) != f->face->end();
}

}  // namespace

void set_error(const std::string& msg) { g_error = msg; }
std::mutex& capture_mutex()
{
    static std::mutex mu;
    return mu;
}
const std::string& get_error() { return g_error; }

Model::~Model()
{
    batch_forget(this);
    if (device >= 0) cudaSetDevice(device);
    free_solver(*this);
    free_adjoint(*this);
    free_precond(*this);
    for (auto& b : blocks) {
        dev_free(b.egroup);
        dev_free(b.conn);
        dev_free(b.mat);
        dev_free(b.vol);
        dev_free(b.vol_f);
        dev_free(b.J0inv);
        dev_free(b.J0inv_f);
        dev_free(b.dN);
        dev_free(b.dN_f);
        dev_free(b.gw);
        dev_free(b.gw_f);
    }
    for (auto& f : faces) {
        dev_free(f.conn);
        dev_free(f.table);
        dev_free(f.A0);
        dev_free(f.J0inv);
        dev_free(f.J0inv_f);
        dev_free(f.load);
        dev_free(f.load_idx);
        dev_free(f.t_ngp);
        dev_free(f.t_w);
        dev_free(f.t_N);
        dev_free(f.t_dN);
        dev_free(f.t_w_f);
        dev_free(f.t_N_f);
        dev_free(f.t_dN_f);
    }
    dev_free(d_mats);
    dev_free(d_mats_f);
    dev_free(d_fext);
    dev_free(d_u);
    dev_free(d_r);
    free_gather(*this);
    if (stream && own_stream) cudaStreamDestroy(stream);
}

// Host set-up shared by both creation paths.
efem_status build_model(ModelInput& in, Model& m)
{
    m.opts = in.opts;
    m.device = -1;
    m.n_nodes = static_cast<int>(in.X.size() / 3);
    m.X = in.X;
    if (in.cell_ptr.empty()) {  // array input: the blocks in the order given
        in.cell_ptr.assign(1, 0);
        for (auto& hb : in.blocks)
            for (size_t e = 0; e < hb.mat_id.size(); e++) {
                in.cell_nodes.insert(in.cell_nodes.end(), hb.conn.begin() + e * hb.nen, hb.conn.begin() + (e + 1) * hb.nen);
                in.cell_ptr.push_back(static_cast<int>(in.cell_nodes.size()));
            }
    }
    m.cell_ptr = in.cell_ptr;
    m.cell_nodes = in.cell_nodes;
    if (m.n_nodes <= 0) {
        set_error("model has no nodes");
        return EFEM_ERR_MESH;
    }
    m.in_loads = in.loads;
    // fixed nodes and DOF numbering
    std::vector<char> fixed(m.n_nodes, 0);
    for (auto& L : in.loads)
        if (L.type == EFEM_LOAD_FIX)
            for (int v : L.nodes) {
                if (v < 0 || v >= m.n_nodes) {
                    set_error("fixed node out of range");
                    return EFEM_ERR_ARG;
                }
                fixed[v] = 1;
            }
    m.dnode_of_node.assign(m.n_nodes, -1);
    m.node_of_dnode.clear();
    for (int i = 0; i < m.n_nodes; i++)
        if (!fixed[i]) {
            m.dnode_of_node[i] = static_cast<int>(m.node_of_dnode.size());
            m.node_of_dnode.push_back(i);
        }
    m.n_free = static_cast<int>(m.node_of_dnode.size());
    for (int i = 0; i < m.n_nodes; i++)
        if (fixed[i]) {
            m.dnode_of_node[i] = static_cast<int>(m.node_of_dnode.size());
            m.node_of_dnode.push_back(i);
        }

    // materials: the first definition of an id is used
    m.materials_used.clear();
    m.kappa.clear();
    std::map<int, int> slot_of_id;
    for (auto& hm : in.materials) {
        if (slot_of_id.count(hm.id)) continue;
        slot_of_id[hm.id] = static_cast<int>(m.materials_used.size());
        m.materials_used.push_back(hm);
        m.kappa.push_back(elasticity_coeff(hm));
    }
    // element blocks without the elements whose material is undefined
    // (src/fe/ElementConstraint.cpp:22-27), in node-count order
    m.in_blocks.clear();
    m.n_elements = 0;
    m.n_skipped = 0;
    std::vector<std::pair<int, const int*>> all_elems;  // (nen, nodes) for the face lookup
    for (auto& hb : in.blocks) {
        if (kind_of_nen(hb.nen) < 0) {
            set_error("unsupported element node count " + std::to_string(hb.nen));
            return EFEM_ERR_MESH;
        }
        const int n = static_cast<int>(hb.mat_id.size());
        if (static_cast<int>(hb.conn.size()) != n * hb.nen) {
            set_error("element block connectivity has the wrong size");
            return EFEM_ERR_ARG;
        }
        for (int v : hb.conn)
            if (v < 0 || v >= m.n_nodes) {
                set_error("element node out of range");
                return EFEM_ERR_MESH;
            }
        HostBlock kept;
        kept.nen = hb.nen;
        for (int e = 0; e < n; e++) {
            all_elems.emplace_back(hb.nen, hb.conn.data() + static_cast<size_t>(e) * hb.nen);
            auto it = slot_of_id.find(hb.mat_id[e]);
            if (it == slot_of_id.end()) {
                m.n_skipped++;
                continue;
            }
            kept.conn.insert(kept.conn.end(), hb.conn.begin() + static_cast<size_t>(e) * hb.nen,
                hb.conn.begin() + static_cast<size_t>(e + 1) * hb.nen);
            kept.mat_id.push_back(it->second);  // now a slot index
        }
        m.n_elements += static_cast<int>(kept.mat_id.size());
        if (!kept.mat_id.empty()) m.in_blocks.push_back(std::move(kept));
    }
    if (m.n_elements == 0) {
        set_error("model has no element with a defined material");
        return EFEM_ERR_CONFIG;
    }

    // nodal forces: r starts from -f_ext (ExternalConstraint.cpp:149-167)
    std::vector<double> fext(3 * static_cast<size_t>(m.n_free), 0.0);
    m.n_force_nodes = 0;
    for (auto& L : in.loads)
        if (L.type == EFEM_LOAD_FORCE)
            for (int v : L.nodes) {
                if (v < 0 || v >= m.n_nodes) {
                    set_error("force node out of range");
                    return EFEM_ERR_ARG;
                }
                m.n_force_nodes++;
                const int d = m.dnode_of_node[v];
                if (d < m.n_free)
                    for (int c = 0; c < 3; c++) fext[3 * d + c] += L.value[c];
            }

    // pressure faces
    std::vector<std::vector<int>> incident(m.n_nodes);
    for (int e = 0; e < static_cast<int>(all_elems.size()); e++)
        for (int a = 0; a < all_elems[e].first; a++) incident[all_elems[e].second[a]].push_back(e);
    std::vector<FaceHost> fh;
    std::vector<double> loadvals;  // 4 per load: directed flag, value or vector
    for (auto& L : in.loads) {
        if (L.type != EFEM_LOAD_PRESSURE && L.type != EFEM_LOAD_DPRESSURE) continue;
        const int li = static_cast<int>(loadvals.size() / 4);
        if (L.type == EFEM_LOAD_PRESSURE)
            loadvals.insert(loadvals.end(), { 0.0, L.value[0], 0.0, 0.0 });
        else
            loadvals.insert(loadvals.end(), { 1.0, L.value[0], L.value[1], L.value[2] });
        if (L.face_ptr.empty()) continue;
        for (size_t f = 0; f + 1 < L.face_ptr.size(); f++) {
            std::vector<int> face;
            for (int k = L.face_ptr[f]; k < L.face_ptr[f + 1]; k++) {
                const int v = L.nodes[k];
                if (v < 0 || v >= m.n_nodes) {
                    set_error("pressure face node out of range");
                    return EFEM_ERR_ARG;
                }
                if (std::find(face.begin(), face.end(), v) == face.end()) face.push_back(v);
            }
            if (face.empty()) continue;
            // the unique element holding every face node (ExternalConstraint.cpp:255-287)
            int parent = -1, count = 0;
            for (int e : incident[face[0]]) {
                const int nen = all_elems[e].first;
                const int* en = all_elems[e].second;
                bool all = true;
                for (size_t i = 1; i < face.size() && all; i++) all = std::find(en, en + nen, face[i]) != en + nen;
                if (all && e != parent) {
                    parent = e;
                    count++;
                }
            }
            if (count != 1) {
                set_error("pressure face " + std::to_string(f + 1) + " lies on " + std::to_string(count)
                    + " elements (exactly one expected)");
                return EFEM_ERR_FACE;
            }
            const int nen = all_elems[parent].first;
            const int* en = all_elems[parent].second;
            const int kind = kind_of_nen(nen);
            FaceCtx ctx { &face, en };
            double pts[3 * MAX_FGP], w[MAX_FGP];
            int ref = -1;
            const int nn = static_cast<int>(face.size());
            const int ngp = face_rule(nn, face_has_elem_node, &ctx, pts, w, &ref);
            if (ngp == 0) {
                set_error("pressure face " + std::to_string(f + 1) + " with " + std::to_string(nn)
                    + " nodes matches no face rule of its element");
                return EFEM_ERR_FACE;
            }
            FaceHost F {};
            F.ngp = ngp;
            std::memcpy(F.pts, pts, sizeof(pts));
            std::memcpy(F.w, w, sizeof(w));
            F.kind = kind;
            F.load = li;
            F.enodes.assign(en, en + nen);
            // branch id: which corner(s) are missing -> table key
            int branch = 0;
            if (nn == 3 || nn == 6) branch = ref;
            else {
                static const int pairs[6][2] = { { 0, 2 }, { 0, 5 }, { 0, 7 }, { 6, 3 }, { 6, 1 }, { 6, 4 } };
                for (int k = 0; k < 6; k++)
                    if (!face_has_elem_node(&ctx, pairs[k][0]) && !face_has_elem_node(&ctx, pairs[k][1])) {
                        branch = k;
                        break;
                    }
            }
            F.table_key = nn * 16 + branch;
            // A0, oriented towards the element node not on the face
            const double* X = m.X.data();
            auto area = [&](int p0, int p1, int p2, double* A) {
                double u[3], v[3];
                for (int k = 0; k < 3; k++) {
                    u[k] = X[3 * p2 + k] - X[3 * p0 + k];
                    v[k] = X[3 * p1 + k] - X[3 * p0 + k];
                }
                A[0] = 0.5 * (u[1] * v[2] - u[2] * v[1]);
                A[1] = 0.5 * (u[2] * v[0] - u[0] * v[2]);
                A[2] = 0.5 * (u[0] * v[1] - u[1] * v[0]);
            };
            auto orient = [&](double* A) {
                const double* r = X + 3 * en[ref];
                const double* p0 = X + 3 * face[0];
                if ((r[0] - p0[0]) * A[0] + (r[1] - p0[1]) * A[1] + (r[2] - p0[2]) * A[2] < 0)
                    for (int k = 0; k < 3; k++) A[k] = -A[k];
            };
            if (nn == 3 || nn == 6) {
                area(face[0], face[1], face[2], F.A0);
                orient(F.A0);
            } else {
                double A1[3], A2[3];
                area(face[0], face[1], face[2], A1);
                area(face[3], face[2], face[0], A2);  // 1/2 (p0 - p3) x (p2 - p3)
                orient(A1);
                orient(A2);
                for (int k = 0; k < 3; k++) F.A0[k] = A1[k] + A2[k];
            }
            // J0^{-1} at each face point from the reference coordinates
            double Y[3 * MAX_NEN];
            for (int a = 0; a < nen; a++) std::memcpy(Y + 3 * a, X + 3 * en[a], sizeof(double) * 3);
            for (int g = 0; g < MAX_FGP; g++)
                for (int k = 0; k < 9; k++) F.J0inv[g][k] = 0.0;
            for (int g = 0; g < ngp; g++) {
                double N[MAX_NEN], dN[3 * MAX_NEN], J0[9];
                shape_functions(kind, pts + 3 * g, N, dN);
                jacobi(nen, Y, dN, J0);
                inv3(J0, F.J0inv[g]);
            }
            fh.push_back(std::move(F));
        }
    }
    m.n_faces = static_cast<int>(fh.size());

    // group faces by parent element kind and build their tables; a table
    // holds weights, N and dN/dxi at the face points of one face rule
    m.faces.clear();
    for (int kind = 0; kind < 4; kind++) {
        std::vector<const FaceHost*> mine;
        for (auto& F : fh)
            if (F.kind == kind) mine.push_back(&F);
        if (mine.empty()) continue;
        DevFaces df;
        df.kind = kind;
        df.nen = nen_of_kind(kind);
        df.n = static_cast<int>(mine.size());
        df.h_conn.assign(static_cast<size_t>(df.nen) * df.n, 0);
        std::map<int, int> table_of_key;
        for (int f = 0; f < df.n; f++) {
            const FaceHost& F = *mine[f];
            for (int a = 0; a < df.nen; a++) df.h_conn[static_cast<size_t>(a) * df.n + f] = m.dnode_of_node[F.enodes[a]];
            auto it = table_of_key.find(F.table_key);
            int t;
            if (it == table_of_key.end()) {
                t = static_cast<int>(table_of_key.size());
                table_of_key[F.table_key] = t;
                df.h_ngp.push_back(F.ngp);
                for (int g = 0; g < MAX_FGP; g++) {
                    double N[MAX_NEN] = { 0 }, dN[3 * MAX_NEN] = { 0 };
                    if (g < F.ngp) shape_functions(kind, F.pts + 3 * g, N, dN);
                    df.h_w.push_back(g < F.ngp ? F.w[g] : 0.0);
                    df.h_N.insert(df.h_N.end(), N, N + df.nen);
                    df.h_dN.insert(df.h_dN.end(), dN, dN + 3 * df.nen);
                }
            } else {
                t = it->second;
            }
            df.h_table.push_back(t);
            df.h_A0.insert(df.h_A0.end(), F.A0, F.A0 + 3);
            for (int g = 0; g < MAX_FGP; g++) df.h_J0inv.insert(df.h_J0inv.end(), F.J0inv[g], F.J0inv[g] + 9);
            df.h_load.insert(df.h_load.end(), loadvals.begin() + 4 * F.load, loadvals.begin() + 4 * F.load + 4);
            df.h_load_idx.push_back(F.load);
        }
        df.n_tables = static_cast<int>(table_of_key.size());
        m.faces.push_back(std::move(df));
    }
    m.h_fnodal = std::move(fext);
    m.has_gravity = false;
    for (int k = 0; k < 3; k++) m.gravity[k] = 0.0;
    for (auto& L : in.loads)
        if (L.type == EFEM_LOAD_GRAVITY) {
            m.has_gravity = true;
            for (int k = 0; k < 3; k++) m.gravity[k] += L.value[k];
        }
    external_load(m, m.h_fext);
    m.n_pressure_loads = static_cast<int>(loadvals.size() / 4);
    return build_blocks(m);
}

}  // namespace efem

namespace efem {

// Per-block integration data for the selected rule: dN/dxi and weights at the
// Gauss points, and per element V_e and J0^{-1} at every point
// (IntegralElement::initial, src/fe/element/IntegralElement.cpp:3-19).
efem_status build_blocks(Model& m)
{
    m.epoch++;
    free_gather(m);
    const bool reduced = m.opts.integration == 1;
    for (auto& b : m.blocks) {
        dev_free(b.conn);
        dev_free(b.mat);
        dev_free(b.vol);
        dev_free(b.vol_f);
        dev_free(b.J0inv);
        dev_free(b.J0inv_f);
        dev_free(b.dN);
        dev_free(b.dN_f);
        dev_free(b.gw);
        dev_free(b.gw_f);
    }
    m.blocks.clear();
    for (auto& hb : m.in_blocks) {
        DevBlock b;
        b.nen = hb.nen;
        b.kind = kind_of_nen(hb.nen);
        b.n = static_cast<int>(hb.mat_id.size());
        double pts[3 * MAX_NGP], w[MAX_NGP];
        b.ngp = gauss_rule(b.kind, reduced, pts, w);
        b.h_gw.assign(w, w + b.ngp);
        b.h_dN.resize(static_cast<size_t>(b.ngp) * b.nen * 3);
        for (int g = 0; g < b.ngp; g++) {
            double N[MAX_NEN];
            shape_functions(b.kind, pts + 3 * g, N, b.h_dN.data() + static_cast<size_t>(g) * b.nen * 3);
        }
        b.h_conn.resize(hb.conn.size());
        for (size_t i = 0; i < hb.conn.size(); i++) b.h_conn[i] = m.dnode_of_node[hb.conn[i]];
        b.h_mat = hb.mat_id;
        // one law for the whole block: the element kernel compiles only its code
        b.mat_type = -1;
        for (size_t e = 0; e < hb.mat_id.size(); e++) {
            const int t = m.materials_used[hb.mat_id[e]].type;
            if (e == 0) b.mat_type = t;
            else if (t != b.mat_type) {
                b.mat_type = -1;
                break;
            }
        }
        b.h_vol.resize(b.n);
        b.h_J0inv.resize(static_cast<size_t>(b.n) * b.ngp * 9);
        double Y[3 * MAX_NEN];
        for (int e = 0; e < b.n; e++) {
            for (int a = 0; a < b.nen; a++)
                std::memcpy(Y + 3 * a, m.X.data() + 3 * static_cast<size_t>(hb.conn[static_cast<size_t>(e) * b.nen + a]),
                    sizeof(double) * 3);
            b.h_vol[e] = corner_volume(b.nen, Y);
            for (int g = 0; g < b.ngp; g++) {
                double J0[9];
                jacobi(b.nen, Y, b.h_dN.data() + static_cast<size_t>(g) * b.nen * 3, J0);
                inv3(J0, b.h_J0inv.data() + (static_cast<size_t>(e) * b.ngp + g) * 9);
            }
        }
        m.blocks.push_back(std::move(b));
    }
    m.built_integration = m.opts.integration;
    if (m.on_device) return ensure_device(m);
    return EFEM_OK;
}

namespace {
template <typename T>
std::vector<float> to_f32(const std::vector<T>& v)
{
    return std::vector<float>(v.begin(), v.end());
}
}  // namespace

efem_status ensure_device(Model& m)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_error("no CUDA device is visible; this library has no CPU path");
        return EFEM_ERR_NO_DEVICE;
    }
    if (m.device < 0) {
        int d = m.opts.device;
        if (d < 0) EFEM_CUDA(cudaGetDevice(&d));
        m.device = d;
    }
    EFEM_CUDA(cudaSetDevice(m.device));
    if (!m.stream) {
        EFEM_CUDA(cudaStreamCreateWithFlags(&m.stream, cudaStreamNonBlocking));
        m.own_stream = true;
    }
    efem_status s;
#define UP(ptr, vec)                          \
    if (!(ptr)) {                             \
        s = dev_upload(&(ptr), (vec));        \
        if (s != EFEM_OK) return s;           \
    }
    for (auto& b : m.blocks) {
        std::vector<int> soa(b.h_conn.size());
        for (int e = 0; e < b.n; e++)
            for (int a = 0; a < b.nen; a++)
                soa[static_cast<size_t>(a) * b.n + e] = b.h_conn[static_cast<size_t>(e) * b.nen + a];
        UP(b.conn, soa);
        UP(b.mat, b.h_mat);
        UP(b.vol, b.h_vol);
        UP(b.vol_f, to_f32(b.h_vol));
        UP(b.J0inv, b.h_J0inv);
        UP(b.J0inv_f, to_f32(b.h_J0inv));
        UP(b.dN, b.h_dN);
        UP(b.dN_f, to_f32(b.h_dN));
        UP(b.gw, b.h_gw);
        UP(b.gw_f, to_f32(b.h_gw));
    }
    for (auto& f : m.faces) {
        UP(f.conn, f.h_conn);
        UP(f.table, f.h_table);
        UP(f.A0, f.h_A0);
        UP(f.J0inv, f.h_J0inv);
        UP(f.J0inv_f, to_f32(f.h_J0inv));
        UP(f.load, f.h_load);
        UP(f.load_idx, f.h_load_idx);
        UP(f.t_ngp, f.h_ngp);
        UP(f.t_w, f.h_w);
        UP(f.t_N, f.h_N);
        UP(f.t_dN, f.h_dN);
        UP(f.t_w_f, to_f32(f.h_w));
        UP(f.t_N_f, to_f32(f.h_N));
        UP(f.t_dN_f, to_f32(f.h_dN));
    }
    if (!m.d_mats) {
        std::vector<MatParams<double>> md;
        std::vector<MatParams<float>> mf;
        for (auto& hm : m.materials_used) {
            md.push_back({ hm.type, hm.C10, hm.C01, hm.C20, hm.C30, hm.D1 });
            mf.push_back({ hm.type, (float)hm.C10, (float)hm.C01, (float)hm.C20, (float)hm.C30, (float)hm.D1 });
        }
        UP(m.d_mats, md);
        UP(m.d_mats_f, mf);
    }
    if (!m.d_fext) {
        std::vector<double> fx = m.h_fext;
        if (fx.empty()) fx.assign(1, 0.0);
        UP(m.d_fext, fx);
    }
    if (!m.d_u) {
        s = dev_alloc(&m.d_u, 3 * static_cast<size_t>(std::max(m.n_free, 1)));
        if (s != EFEM_OK) return s;
        s = dev_alloc(&m.d_r, 3 * static_cast<size_t>(std::max(m.n_free, 1)));
        if (s != EFEM_OK) return s;
    }
#undef UP
    m.on_device = true;
    if (m.opts.deterministic && !m.d_contrib && (s = build_gather(m)) != EFEM_OK) return s;
    if (m.tuned_threads != element_tune_key(m)) {
        // element kernels are tuned before any graph captures them (a retune
        // invalidates captured graphs through the epoch)
        if ((s = tune_element_blocks(m)) != EFEM_OK) return s;
        m.epoch++;
    }
    return EFEM_OK;
}

// Host assembly of the scalar approximate Jacobian,
// L_jk = sum_e V_e kappa_e sum_g w_g (T_g^T T_g)_jk over free node pairs, with
// T_g = J0^{-T} (dN/dxi)^T (ElementConstraint.cpp:164-205).  CSR over free
// nodes, both triangles, columns sorted.
void assemble_L_csr(const Model& m, std::vector<int>& rowptr, std::vector<int>& col, std::vector<double>& val)
{
    const int n = m.n_free;
    // pattern: node adjacency through elements
    std::vector<std::vector<int>> adj(n);
    for (auto& b : m.blocks)
        for (int e = 0; e < b.n; e++) {
            const int* c = b.h_conn.data() + static_cast<size_t>(e) * b.nen;
            for (int a = 0; a < b.nen; a++) {
                if (c[a] >= n) continue;
                for (int q = 0; q < b.nen; q++)
                    if (c[q] < n) adj[c[a]].push_back(c[q]);
            }
        }
    rowptr.assign(n + 1, 0);
    for (int i = 0; i < n; i++) {
        auto& v = adj[i];
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        rowptr[i + 1] = rowptr[i] + static_cast<int>(v.size());
    }
    col.resize(rowptr[n]);
    val.assign(rowptr[n], 0.0);
    for (int i = 0; i < n; i++) std::copy(adj[i].begin(), adj[i].end(), col.begin() + rowptr[i]);
    std::vector<std::vector<int>>().swap(adj);
    auto at = [&](int i, int j) -> double& {
        auto it = std::lower_bound(col.begin() + rowptr[i], col.begin() + rowptr[i + 1], j);
        return val[it - col.begin()];
    };
    double T[3 * MAX_NEN];
    for (auto& b : m.blocks)
        for (int e = 0; e < b.n; e++) {
            const int* c = b.h_conn.data() + static_cast<size_t>(e) * b.nen;
            const double ks = b.h_vol[e] * m.kappa[b.h_mat[e]];
            int loc[MAX_NEN];
            for (int a = 0; a < b.nen; a++) loc[a] = c[a];
            for (int g = 0; g < b.ngp; g++) {
                const double* Ji = b.h_J0inv.data() + (static_cast<size_t>(e) * b.ngp + g) * 9;
                const double* dN = b.h_dN.data() + static_cast<size_t>(g) * b.nen * 3;
                for (int k = 0; k < 3; k++)
                    for (int a = 0; a < b.nen; a++)
                        T[k * b.nen + a] = Ji[k] * dN[3 * a] + Ji[3 + k] * dN[3 * a + 1] + Ji[6 + k] * dN[3 * a + 2];
                const double w = ks * b.h_gw[g];
                for (int j = 0; j < b.nen; j++) {
                    if (loc[j] >= n) continue;
                    for (int q = 0; q < b.nen; q++) {
                        if (loc[q] >= n) continue;
                        const double s = T[j] * T[q] + T[b.nen + j] * T[b.nen + q] + T[2 * b.nen + j] * T[2 * b.nen + q];
                        at(loc[j], loc[q]) += w * s;
                    }
                }
            }
        }
}

}  // namespace efem

// ===================================================================== C ABI
using efem::Model;

namespace {
efem_status guard(void* h, Model** out)
{
    if (!h) {
        efem::set_error("null model handle");
        return EFEM_ERR_ARG;
    }
    *out = static_cast<Model*>(h);
    return EFEM_OK;
}

// With device_ptrs, a vector argument must be memory this model's GPU can
// address: a device allocation on the model's device, managed memory, or
// mapped pinned host memory.  Anything else (pageable host memory, another
// GPU's buffer) is refused here rather than read by a kernel.
efem_status dev_vec(const Model& m, const void* p, const char* what)
{
    cudaPointerAttributes a {};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        efem::set_error(std::string(what) + ": not a CUDA pointer (device_ptrs is set)");
        return EFEM_ERR_ARG;
    }
    const bool ok = a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == m.device)
        || (a.type == cudaMemoryTypeHost && a.devicePointer != nullptr);
    if (!ok) {
        efem::set_error(std::string(what) + (a.type == cudaMemoryTypeDevice
            ? ": device memory of another GPU (device_ptrs is set)"
            : ": host memory the GPU cannot address (device_ptrs is set; pass device memory)"));
        return EFEM_ERR_ARG;
    }
    return EFEM_OK;
}

// copy a vector argument in (device pointer or host pointer) to a device buffer
efem_status vec_in(Model& m, const double* src, double** dst, double* staging)
{
    if (m.opts.device_ptrs) {
        efem_status s = dev_vec(m, src, "input vector");
        if (s != EFEM_OK) return s;
        *dst = const_cast<double*>(src);
        return EFEM_OK;
    }
    EFEM_CUDA(cudaMemcpyAsync(staging, src, sizeof(double) * 3 * m.n_free, cudaMemcpyHostToDevice, m.stream));
    *dst = staging;
    return EFEM_OK;
}
}  // namespace

namespace efem {

// algorithmic traffic and work of one residual evaluation with sz-byte
// geometric factors: every input read once (connectivity, material index,
// V_e, J0^{-1}, u, f_ext), r written once; flops = 2 per FMA (u.dN, H, P(F),
// S, and the nodal reduction); the pressure faces' part only when faces is set
void residual_work(const Model& m, int sz, long long* bytes, double* flops, bool faces)
{
    long long b = 3LL * 8 * m.n_free * 3;
    double f = 0;
    for (auto& blk : m.blocks) {
        b += static_cast<long long>(blk.n) * (4LL * blk.nen + 4 + sz + 9LL * sz * blk.ngp);
        double cmat = 0;
        for (int e = 0; e < blk.n; e++) {
            const int t = m.materials_used[blk.h_mat[e]].type;
            cmat += t == EFEM_MOONEY_RIVLIN ? 510.0 : t == EFEM_YEOH ? 270.0 : 260.0;
        }
        f += static_cast<double>(blk.ngp) * (36.0 * blk.nen * blk.n + cmat);
    }
    for (auto& fc : m.faces) {
        if (!faces) break;
        b += static_cast<long long>(fc.n) * (4LL * fc.nen + 4 + 24 + 32 + 9LL * sz * MAX_FGP);
        f += static_cast<double>(fc.n) * 9.0 * (24.0 * fc.nen + 120.0);
    }
    *bytes = b;
    *flops = f;
}

}  // namespace efem

extern "C" {

efem_status efem_default_options(efem_options* o)
{
    if (!o) return EFEM_ERR_ARG;
    std::memset(o, 0, sizeof(*o));
    o->precision = EFEM_FP64;
    o->integration = 0;
    o->nl_solver = 0;
    o->m = 6;
    o->max_iterations = 0;
    o->max_linesearch = 20;
    o->residual_criterion = 1e-6;
    o->dx_criterion = 1e-8;
    o->device_ptrs = 0;
    o->deterministic = 0;
    o->device = -1;
    o->host_loop = 0;
    o->adjoint_tolerance = 1e-8;
    o->adjoint_max_iterations = 2000;
    o->elem_threads = 0;
    o->consistent_inertia = 0;
    o->trace = 0;
    o->solve_subtree_levels = -1;
    o->line_search = 0;
    return EFEM_OK;
}

efem_status efem_model_create_from_json(const char* cfg_path, void** model)
{
    if (!cfg_path || !model) {
        efem::set_error("null argument");
        return EFEM_ERR_ARG;
    }
    *model = nullptr;
    try {
        efem::ModelInput in;
        efem_status s = efem::read_json_config(cfg_path, in);
        if (s != EFEM_OK) return s;
        auto m = std::make_unique<Model>();
        s = efem::build_model(in, *m);
        if (s != EFEM_OK) return s;
        *model = m.release();
        return EFEM_OK;
    } catch (const std::exception& e) {
        efem::set_error(std::string("set-up failed: ") + e.what());
        return EFEM_ERR_CONFIG;
    }
}

efem_status efem_model_create(const efem_mesh_desc* mesh, const efem_material* materials, int n_materials,
    const efem_load_desc* loads, int n_loads, const efem_options* options, void** model)
{
    if (!mesh || !model || (n_materials > 0 && !materials) || (n_loads > 0 && !loads) || !mesh->X || mesh->n_nodes <= 0) {
        efem::set_error("null or empty argument");
        return EFEM_ERR_ARG;
    }
    *model = nullptr;
    try {
        efem::ModelInput in;
        if (options)
            in.opts = *options;
        else
            efem_default_options(&in.opts);
        in.X.assign(mesh->X, mesh->X + 3 * static_cast<size_t>(mesh->n_nodes));
        for (int b = 0; b < mesh->n_blocks; b++) {
            const efem_element_block& eb = mesh->blocks[b];
            if (eb.n_elem < 0 || (eb.n_elem > 0 && !eb.conn)) {
                efem::set_error("bad element block");
                return EFEM_ERR_ARG;
            }
            efem::HostBlock hb;
            hb.nen = eb.nen;
            hb.conn.assign(eb.conn, eb.conn + static_cast<size_t>(eb.n_elem) * eb.nen);
            hb.mat_id.assign(eb.n_elem, -1);
            if (eb.material_id) hb.mat_id.assign(eb.material_id, eb.material_id + eb.n_elem);
            in.blocks.push_back(std::move(hb));
        }
        for (int i = 0; i < n_materials; i++) {
            const efem_material& mt = materials[i];
            in.materials.push_back({ mt.type, mt.id, mt.C10, mt.C01, mt.C20, mt.C30, mt.D1, mt.density });
        }
        for (int i = 0; i < n_loads; i++) {
            const efem_load_desc& ld = loads[i];
            efem::HostLoad L;
            L.type = ld.type;
            std::memcpy(L.value, ld.value, sizeof(L.value));
            if (ld.type == EFEM_LOAD_FIX || ld.type == EFEM_LOAD_FORCE) {
                if (ld.n > 0 && !ld.nodes) return EFEM_ERR_ARG;
                L.nodes.assign(ld.nodes, ld.nodes + std::max(ld.n, 0));
            } else if (ld.type == EFEM_LOAD_PRESSURE || ld.type == EFEM_LOAD_DPRESSURE) {
                if (ld.n > 0 && (!ld.nodes || !ld.face_ptr)) return EFEM_ERR_ARG;
                const double mag = ld.type == EFEM_LOAD_PRESSURE
                    ? ld.value[0]
                    : std::sqrt(ld.value[0] * ld.value[0] + ld.value[1] * ld.value[1] + ld.value[2] * ld.value[2]);
                if (!(mag > 0)) continue;  // ignored like the reference (ExternalConstraint.cpp:195-197)
                L.face_ptr.assign(ld.face_ptr, ld.face_ptr + std::max(ld.n, 0) + 1);
                L.nodes.assign(ld.nodes, ld.nodes + (ld.n > 0 ? ld.face_ptr[ld.n] : 0));
            } else if (ld.type != EFEM_LOAD_GRAVITY) {
                efem::set_error("unknown load type");
                return EFEM_ERR_ARG;
            }
            in.loads.push_back(std::move(L));
        }
        auto m = std::make_unique<Model>();
        efem_status s = efem::build_model(in, *m);
        if (s != EFEM_OK) return s;
        *model = m.release();
        return EFEM_OK;
    } catch (const std::exception& e) {
        efem::set_error(std::string("set-up failed: ") + e.what());
        return EFEM_ERR_ARG;
    }
}

efem_status efem_model_destroy(void* model)
{
    delete static_cast<Model*>(model);
    return EFEM_OK;
}

efem_status efem_get_options(void* model, efem_options* o)
{
    Model* m;
    efem_status s = guard(model, &m);
    if (s != EFEM_OK) return s;
    if (!o) return EFEM_ERR_ARG;
    *o = m->opts;
    return EFEM_OK;
}

efem_status efem_set_options(void* model, const efem_options* o)
{
    Model* m;
    efem_status s = guard(model, &m);
    if (s != EFEM_OK) return s;
    if (!o || o->m <= 0 || o->max_linesearch <= 0 || o->max_iterations < 0 || o->residual_criterion < 0
        || (o->precision != EFEM_FP64 && o->precision != EFEM_MIXED) || (o->integration != 0 && o->integration != 1)
        || o->trace < 0 || (o->line_search != 0 && o->line_search != 1) || o->wait_limit < 0
        || (o->wait_test != 0 && o->wait_test != 1)) {
        efem::set_error("invalid options (NLSolverParam::check_param rules)");
        return EFEM_ERR_ARG;
    }
    const bool reintegrate = o->integration != m->opts.integration;
    const bool new_history = o->m != m->opts.m;
    const bool new_mass = m->has_gravity && (o->consistent_inertia != 0) != (m->opts.consistent_inertia != 0);
    const bool new_schedule = o->solve_subtree_levels != m->opts.solve_subtree_levels;
    const bool new_waits = o->wait_limit != m->opts.wait_limit || o->wait_test != m->opts.wait_test;
    const int dev = m->device;
    m->opts = *o;
    if (dev >= 0) m->device = dev;  // the device is fixed once buffers exist
    if (m->on_device) cudaSetDevice(m->device);
    if (new_mass) {
        // same device buffer, new values: captured graphs keep pointing at it
        efem::external_load(*m, m->h_fext);
        if (m->d_fext && m->n_free > 0) {
            EFEM_CUDA(cudaMemcpy(m->d_fext, m->h_fext.data(), sizeof(double) * m->h_fext.size(), cudaMemcpyHostToDevice));
        }
    }
    if (reintegrate) {
        efem::free_precond(*m);
        s = efem::build_blocks(*m);
        if (s != EFEM_OK) return s;
    }
    if (new_history) efem::free_solver(*m);
    if (new_schedule && !reintegrate) efem::free_precond(*m);  // the solve schedule is rebuilt at the next factorisation
    else if (new_waits && !reintegrate) efem::precond_drop_graphs(*m);  // captured solves hold the old wait limits
    return EFEM_OK;
}

efem_status efem_get_model_info(void* model, efem_model_info* info)
{
    Model* m;
    efem_status s = guard(model, &m);
    if (s != EFEM_OK) return s;
    if (!info) return EFEM_ERR_ARG;
    std::memset(info, 0, sizeof(*info));
    info->n_nodes = m->n_nodes;
    info->n_free_nodes = m->n_free;
    info->n_dof = 3 * m->n_free;
    info->n_elements = m->n_elements;
    info->n_elements_skipped = m->n_skipped;
    info->n_faces = m->n_faces;
    info->n_force_nodes = m->n_force_nodes;
    info->n_blocks = static_cast<int>(m->blocks.size());
    long long bytes = 0;
    double flops = 0;
    efem::residual_work(*m, m->opts.precision == EFEM_MIXED ? 4 : 8, &bytes, &flops, true);
    info->residual_bytes = bytes;
    info->residual_flops = flops;
    info->n_params = efem::n_params(*m);
    info->elem_threads_fp64 = m->blocks.empty() ? 0 : m->blocks[0].threads[0];
    info->elem_threads_fp32 = m->blocks.empty() ? 0 : m->blocks[0].threads[1];
    efem::precond_info(*m, info);
    return EFEM_OK;
}

efem_status efem_dof_map(void* model, int* node_of_dof)
{
    Model* m;
    efem_status s = guard(model, &m);
    if (s != EFEM_OK) return s;
    if (!node_of_dof) return EFEM_ERR_ARG;
    std::copy(m->node_of_dnode.begin(), m->node_of_dnode.begin() + m->n_free, node_of_dof);
    return EFEM_OK;
}

efem_status efem_external_load(void* model, double* f)
{
    Model* m;
    efem_status s = guard(model, &m);
    if (s != EFEM_OK) return s;
    if (!f) return EFEM_ERR_ARG;
    std::copy(m->h_fext.begin(), m->h_fext.end(), f);
    return EFEM_OK;
}

efem_status efem_residual(void* model, const double* u, double* r)
{
    Model* m;
    efem_status s = guard(model, &m);
    if (s != EFEM_OK) return s;
    if (!u || !r) return EFEM_ERR_ARG;
    s = efem::ensure_device(*m);
    if (s != EFEM_OK) return s;
    if (m->opts.device_ptrs && (s = dev_vec(*m, r, "r")) != EFEM_OK) return s;
    double *du, *dr = m->opts.device_ptrs ? r : m->d_r;
    s = vec_in(*m, u, &du, m->d_u);
    if (s != EFEM_OK) return s;
    s = efem::launch_residual(*m, du, dr);
    if (s != EFEM_OK) return s;
    if (!m->opts.device_ptrs)
        EFEM_CUDA(cudaMemcpyAsync(r, dr, sizeof(double) * 3 * m->n_free, cudaMemcpyDeviceToHost, m->stream));
    EFEM_CUDA(cudaStreamSynchronize(m->stream));
    return EFEM_OK;
}

static efem_status hvp_call(void* model, const double* u, const double* v, double* out, bool transpose)
{
    Model* m;
    efem_status s = guard(model, &m);
    if (s != EFEM_OK) return s;
    if (!u || !v || !out) return EFEM_ERR_ARG;
    if ((s = efem::ensure_device(*m)) != EFEM_OK) return s;
    double *du, *dv, *io = nullptr;
    if ((s = efem::adjoint_io(*m, &io)) != EFEM_OK) return s;
    if (m->opts.device_ptrs && (s = dev_vec(*m, out, "output vector")) != EFEM_OK) return s;
    double* dout = m->opts.device_ptrs ? out : io;
    if ((s = vec_in(*m, u, &du, m->d_u)) != EFEM_OK) return s;
    if ((s = vec_in(*m, v, &dv, m->d_r)) != EFEM_OK) return s;
    if ((s = efem::hvp(*m, du, dv, dout, transpose)) != EFEM_OK) return s;
    if (!m->opts.device_ptrs)
        EFEM_CUDA(cudaMemcpyAsync(out, dout, sizeof(double) * 3 * m->n_free, cudaMemcpyDeviceToHost, m->stream));
    EFEM_CUDA(cudaStreamSynchronize(m->stream));
    return EFEM_OK;
}

efem_status efem_hvp(void* model, const double* u, const double* v, double* Kv)
{
    return hvp_call(model, u, v, Kv, false);
}

efem_status efem_hvp_transpose(void* model, const double* u, const double* w, double* KTw)
{
    return hvp_call(model, u, w, KTw, true);
}

efem_status efem_residual_param_derivative(void* model, const double* u, int k, double* dR)
{
    Model* m;
    efem_status s = guard(model, &m);
    if (s != EFEM_OK) return s;
    if (!u || !dR) return EFEM_ERR_ARG;
    if ((s = efem::ensure_device(*m)) != EFEM_OK) return s;
    double *du, *io = nullptr;
    if ((s = efem::adjoint_io(*m, &io)) != EFEM_OK) return s;
    if (m->opts.device_ptrs && (s = dev_vec(*m, dR, "dR")) != EFEM_OK) return s;
    double* dout = m->opts.device_ptrs ? dR : io;
    if ((s = vec_in(*m, u, &du, m->d_u)) != EFEM_OK) return s;
    if ((s = efem::residual_param_derivative(*m, du, k, dout)) != EFEM_OK) return s;
    if (!m->opts.device_ptrs)
        EFEM_CUDA(cudaMemcpyAsync(dR, dout, sizeof(double) * 3 * m->n_free, cudaMemcpyDeviceToHost, m->stream));
    EFEM_CUDA(cudaStreamSynchronize(m->stream));
    return EFEM_OK;
}

efem_status efem_adjoint(void* model, const double* u, const double* dJdu, double* dJdtheta, double* lambda,
    efem_adjoint_info* info)
{
    Model* m;
    efem_status s = guard(model, &m);
    if (s != EFEM_OK) return s;
    if (!u || !dJdu || !dJdtheta) return EFEM_ERR_ARG;
    if ((s = efem::ensure_device(*m)) != EFEM_OK) return s;
    efem_adjoint_info local;
    if (!info) info = &local;
    double *du, *dg, *io = nullptr;
    if ((s = efem::adjoint_io(*m, &io)) != EFEM_OK) return s;
    if ((s = vec_in(*m, u, &du, m->d_u)) != EFEM_OK) return s;
    if ((s = vec_in(*m, dJdu, &dg, m->d_r)) != EFEM_OK) return s;
    if (lambda && m->opts.device_ptrs && (s = dev_vec(*m, lambda, "lambda")) != EFEM_OK) return s;
    double* dl = lambda ? (m->opts.device_ptrs ? lambda : io) : nullptr;
    if ((s = efem::adjoint(*m, du, dg, dJdtheta, dl, info)) != EFEM_OK) return s;
    if (lambda && !m->opts.device_ptrs)
        EFEM_CUDA(cudaMemcpyAsync(lambda, dl, sizeof(double) * 3 * m->n_free, cudaMemcpyDeviceToHost, m->stream));
    EFEM_CUDA(cudaStreamSynchronize(m->stream));
    return EFEM_OK;
}

efem_status efem_write_vtk(void* model, const double* u, const char* path)
{
    Model* m;
    efem_status s = guard(model, &m);
    if (s != EFEM_OK) return s;
    if (!path) return EFEM_ERR_ARG;
    std::vector<double> uh;
    if (u) {
        uh.resize(3 * static_cast<size_t>(m->n_free));
        if (m->opts.device_ptrs) {
            if ((s = efem::ensure_device(*m)) != EFEM_OK) return s;
            if ((s = dev_vec(*m, u, "u")) != EFEM_OK) return s;
            EFEM_CUDA(cudaMemcpyAsync(uh.data(), u, sizeof(double) * uh.size(), cudaMemcpyDeviceToHost, m->stream));
            EFEM_CUDA(cudaStreamSynchronize(m->stream));
        } else {
            std::copy(u, u + uh.size(), uh.begin());
        }
    }
    std::FILE* f = std::fopen(path, "w");
    if (!f) {
        efem::set_error(std::string("cannot write ") + path);
        return EFEM_ERR_ARG;
    }
    // legacy ASCII unstructured grid, the content of Model::saveVTK (src/model/Model.cpp:50-117):
    // node positions X + dx (fixed nodes stay at X), every element with its VTK cell type
    std::fprintf(f, "# vtk DataFile Version 3.0\nvtk output\nASCII\nDATASET UNSTRUCTURED_GRID\nPOINTS %d double\n",
        m->n_nodes);
    for (int n = 0; n < m->n_nodes; n++) {
        double p[3] = { m->X[3 * n], m->X[3 * n + 1], m->X[3 * n + 2] };
        const int d = m->dnode_of_node[n];
        if (u && d < m->n_free)
            for (int c = 0; c < 3; c++) p[c] += uh[3 * static_cast<size_t>(d) + c];
        std::fprintf(f, "%.17g %.17g %.17g\n", p[0], p[1], p[2]);
    }
    const int nc = static_cast<int>(m->cell_ptr.size()) - 1;
    std::fprintf(f, "CELLS %d %d\n", nc, nc + static_cast<int>(m->cell_nodes.size()));
    for (int e = 0; e < nc; e++) {
        std::fprintf(f, "%d", m->cell_ptr[e + 1] - m->cell_ptr[e]);
        for (int k = m->cell_ptr[e]; k < m->cell_ptr[e + 1]; k++) std::fprintf(f, " %d", m->cell_nodes[k]);
        std::fprintf(f, "\n");
    }
    std::fprintf(f, "CELL_TYPES %d\n", nc);
    for (int e = 0; e < nc; e++) {
        const int nen = m->cell_ptr[e + 1] - m->cell_ptr[e];
        // VTK_TETRA, VTK_QUADRATIC_TETRA, VTK_HEXAHEDRON, VTK_QUADRATIC_HEXAHEDRON
        std::fprintf(f, "%d\n", nen == 4 ? 10 : nen == 10 ? 24 : nen == 8 ? 12 : 25);
    }
    const bool ok = std::fclose(f) == 0;
    if (!ok) {
        efem::set_error(std::string("cannot write ") + path);
        return EFEM_ERR_ARG;
    }
    return EFEM_OK;
}

efem_status efem_strain_energy(void* model, const double* u, double* energy)
{
    Model* m;
    efem_status s = guard(model, &m);
    if (s != EFEM_OK) return s;
    if (!u || !energy) return EFEM_ERR_ARG;
    if ((s = efem::ensure_device(*m)) != EFEM_OK) return s;
    double* du;
    if ((s = vec_in(*m, u, &du, m->d_u)) != EFEM_OK) return s;
    return efem::strain_energy_sum(*m, du, energy);
}

efem_status efem_approx_jacobian_csr(void* model, long long* nnz, int* rowptr, int* colidx, double* vals)
{
    Model* m;
    efem_status s = guard(model, &m);
    if (s != EFEM_OK) return s;
    if (!nnz) return EFEM_ERR_ARG;
    std::vector<int> rp, ci;
    std::vector<double> v;
    efem::assemble_L_csr(*m, rp, ci, v);
    *nnz = static_cast<long long>(v.size());
    if (!vals) return EFEM_OK;
    if (!rowptr || !colidx) return EFEM_ERR_ARG;
    std::copy(rp.begin(), rp.end(), rowptr);
    std::copy(ci.begin(), ci.end(), colidx);
    std::copy(v.begin(), v.end(), vals);
    return EFEM_OK;
}

efem_status efem_precond_apply(void* model, double* v)
{
    Model* m;
    efem_status s = guard(model, &m);
    if (s != EFEM_OK) return s;
    if (!v) return EFEM_ERR_ARG;
    s = efem::ensure_device(*m);
    if (s != EFEM_OK) return s;
    int ok = 0;
    double ms = 0;
    s = efem::precond_setup(*m, false, &ok, &ms);
    if (s != EFEM_OK) return s;
    if (!ok) {
        efem::set_error("approximate Jacobian is not positive definite");
        return EFEM_ERR_NAN;
    }
    double* dv = v;
    if (m->opts.device_ptrs && (s = dev_vec(*m, v, "v")) != EFEM_OK) return s;
    if (!m->opts.device_ptrs) {
        dv = m->d_r;
        EFEM_CUDA(cudaMemcpyAsync(dv, v, sizeof(double) * 3 * m->n_free, cudaMemcpyHostToDevice, m->stream));
    }
    s = efem::precond_apply(*m, dv);
    if (s != EFEM_OK) return s;
    if (!m->opts.device_ptrs)
        EFEM_CUDA(cudaMemcpyAsync(v, dv, sizeof(double) * 3 * m->n_free, cudaMemcpyDeviceToHost, m->stream));
    return efem::precond_check(*m);
}

efem_status efem_solve(void* model, double* u_inout, efem_solve_info* info)
{
    Model* m;
    efem_status s = guard(model, &m);
    if (s != EFEM_OK) return s;
    if (!u_inout) return EFEM_ERR_ARG;
    s = efem::ensure_device(*m);
    if (s != EFEM_OK) return s;
    efem_solve_info tmp;
    if (!info) info = &tmp;
    std::memset(info, 0, sizeof(*info));
    double* du = u_inout;
    if (m->opts.device_ptrs && (s = dev_vec(*m, u_inout, "u")) != EFEM_OK) return s;
    if (!m->opts.device_ptrs) {
        du = m->d_u;
        EFEM_CUDA(cudaMemcpyAsync(du, u_inout, sizeof(double) * 3 * m->n_free, cudaMemcpyHostToDevice, m->stream));
    }
    s = efem::run_solve(*m, du, info);
    if (s != EFEM_OK && s != EFEM_ERR_NAN) return s;
    if (!m->opts.device_ptrs) {
        EFEM_CUDA(cudaMemcpyAsync(u_inout, du, sizeof(double) * 3 * m->n_free, cudaMemcpyDeviceToHost, m->stream));
        EFEM_CUDA(cudaStreamSynchronize(m->stream));
    }
    return s;
}

efem_status efem_solve_trace(void* model, double* out, int capacity, int* n_records)
{
    Model* m;
    efem_status s = guard(model, &m);
    if (s != EFEM_OK) return s;
    if (m->on_device) cudaSetDevice(m->device);
    return efem::solve_trace(*m, out, capacity, n_records);
}

efem_status efem_batch_solve(void** models, int n, double* const* u, efem_solve_info* infos, int max_threads)
{
    if (n < 0 || (n > 0 && (!models || !u))) {
        efem::set_error("null models or solution arrays");
        return EFEM_ERR_ARG;
    }
    if (n == 0) return EFEM_OK;
    // One union model for the whole batch when the members can share one
    // (batch.cu); otherwise the solves run side by side from a thread pool.
    {
        std::vector<Model*> ms(n);
        bool all = true;
        for (int i = 0; i < n; i++) {
            ms[i] = static_cast<Model*>(models[i]);
            all = all && ms[i] && u[i];
        }
        if (all) {
            const efem_status s = efem::batch_union_solve(ms.data(), n, u, infos);
            if (s != EFEM_ERR_UNSUPPORTED) return s;
        }
    }
    int nt = max_threads > 0 ? max_threads : static_cast<int>(std::thread::hardware_concurrency());
    nt = std::max(1, std::min(nt, n));
    // largest models first, so that no large solve starts last and runs alone
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    auto size_of = [&](int i) { return models[i] ? static_cast<const Model*>(models[i])->n_free : 0; };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return size_of(a) > size_of(b); });
    std::atomic<int> next(0);
    std::vector<efem_status> st(n, EFEM_OK);
    std::vector<std::string> err(n);
    auto worker = [&]() {
        efem::t_batch = nt;
        for (;;) {
            const int q = next.fetch_add(1);
            if (q >= n) return;
            const int i = order[q];
            efem_solve_info local;
            st[i] = efem_solve(models[i], u[i], infos ? &infos[i] : &local);
            if (st[i] != EFEM_OK) err[i] = efem::get_error();
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back(worker);
    worker();
    efem::t_batch = 0;
    for (auto& t : pool) t.join();
    for (int i = 0; i < n; i++)
        if (st[i] != EFEM_OK) {
            efem::set_error("model " + std::to_string(i) + ": " + err[i]);
            return st[i];
        }
    return EFEM_OK;
}

efem_status efem_set_stream(void* model, void* cuda_stream)
{
    Model* m;
    efem_status s = guard(model, &m);
    if (s != EFEM_OK) return s;
    s = efem::ensure_device(*m);
    if (s != EFEM_OK) return s;
    EFEM_CUDA(cudaStreamSynchronize(m->stream));
    if (m->own_stream) cudaStreamDestroy(m->stream);
    if (cuda_stream) {
        m->stream = static_cast<cudaStream_t>(cuda_stream);
        m->own_stream = false;
    } else {
        EFEM_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
        m->own_stream = true;
    }
    return EFEM_OK;
}

efem_status efem_last_error(char* buf, size_t len)
{
    if (!buf || len == 0) return EFEM_ERR_ARG;
    const std::string& e = efem::get_error();
    const size_t n = std::min(len - 1, e.size());
    std::memcpy(buf, e.data(), n);
    buf[n] = 0;
    return EFEM_OK;
}

const char* efem_version(void) { return "efem-b200 0.1 (sm_100a)"; }

}  // extern "C"
