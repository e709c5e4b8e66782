// Reader of the reference's input files into a ModelInput.
//
//   config JSON          src/io/Config.cpp:6-82 (analysis / output keys),
//                        src/model/Model.cpp:7-39 (model[] bodies, pose, id),
//                        src/fe/ElementConstraint.cpp:39-67 (material[]),
//                        src/fe/ExternalConstraint.cpp:13-247 (constraint[])
//   mesh text file       src/io/MeshParser.h:22-100, src/model/Body.cpp:49-90
//   constraint files     src/io/IO.cpp:67-96
//   pose transforms      src/math/Math.cpp:37-108
// Paths are relative to the config file's directory (src/io/IO.cpp:36-40).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

#include "efem_internal.h"
#include "json.h"

namespace efem {

namespace {

std::string trim(const std::string& s)
{
    size_t b = 0, e = s.size();
    while (b < e && std::isspace(static_cast<unsigned char>(s[b]))) b++;
    while (e > b && std::isspace(static_cast<unsigned char>(s[e - 1]))) e--;
    return s.substr(b, e - b);
}

// split on any of ',' ' ' with runs of separators merged
std::vector<std::string> split_tokens(const std::string& s)
{
    std::vector<std::string> out;
    std::string cur;
    bool sep = false;
    for (char c : s) {
        if (c == ',' || c == ' ') {
            if (!sep) {
                out.push_back(cur);
                cur.clear();
            }
            sep = true;
        } else {
            cur.push_back(c);
            sep = false;
        }
    }
    out.push_back(cur);
    return out;
}

bool parse_int(const std::string& t, int* v)
{
    if (t.empty()) return false;
    char* e = nullptr;
    long x = std::strtol(t.c_str(), &e, 10);
    if (e == t.c_str()) return false;
    *v = static_cast<int>(x);
    return true;
}

// IO::readFile: trimmed non-empty lines without '#' or '!'
efem_status read_lines(const std::string& path, std::vector<std::string>& lines)
{
    std::ifstream f(path);
    if (!f) {
        set_error("data file " + path + " not found");
        return EFEM_ERR_MESH;
    }
    std::string ln;
    while (std::getline(f, ln)) {
        ln = trim(ln);
        if (!ln.empty() && ln.find('#') == std::string::npos && ln.find('!') == std::string::npos)
            lines.push_back(ln);
    }
    return EFEM_OK;
}

struct Body {
    int id = -1;
    std::vector<double> X;
    std::vector<int> nen;
    std::vector<std::vector<int>> elems;  // 0-based local node ids
    std::vector<int> mat;
};

efem_status read_mesh(const std::string& path, Body& b)
{
    std::ifstream f(path);
    if (!f) {
        set_error("mesh file " + path + " not found");
        return EFEM_ERR_MESH;
    }
    std::vector<std::string> lines;
    std::string ln;
    while (std::getline(f, ln)) {
        ln = trim(ln);
        if (ln.empty() || ln.rfind("##", 0) == 0 || ln.rfind("!!", 0) == 0) continue;
        lines.push_back(ln);
    }
    size_t i = 0;
    while (i < lines.size()) {
        if (lines[i].rfind("#node", 0) == 0) {
            i++;
            while (i < lines.size() && lines[i][0] != '#') {
                std::istringstream is(lines[i]);
                double v[3] = { 0, 0, 0 };
                for (int k = 0; k < 3; k++)
                    if (!(is >> v[k])) {
                        set_error("bad node line in " + path + ": " + lines[i]);
                        return EFEM_ERR_MESH;
                    }
                b.X.insert(b.X.end(), v, v + 3);
                i++;
            }
            continue;
        }
        if (lines[i].rfind("#element", 0) == 0) {
            i++;
            while (i < lines.size() && lines[i][0] != '#') {
                std::vector<int> tok;
                for (auto& t : split_tokens(lines[i])) {
                    int v;
                    if (!parse_int(t, &v)) {
                        set_error("bad element line in " + path + ": " + lines[i]);
                        return EFEM_ERR_MESH;
                    }
                    tok.push_back(v);
                }
                // node count by token count, optional trailing material id (Body.cpp:52-88)
                const int n = static_cast<int>(tok.size());
                const int nen = n <= 5 ? 4 : n <= 9 ? 8 : n <= 11 ? 10 : n <= 21 ? 20 : -1;
                if (nen < 0 || n < nen) {
                    set_error("unsupported element line in " + path + ": " + lines[i]);
                    return EFEM_ERR_MESH;
                }
                std::vector<int> e(nen);
                for (int a = 0; a < nen; a++) e[a] = tok[a] - 1;
                b.elems.push_back(e);
                b.nen.push_back(nen);
                b.mat.push_back(n > nen ? tok[nen] : -1);
                i++;
            }
            continue;
        }
        i++;
    }
    const int nn = static_cast<int>(b.X.size() / 3);
    for (auto& e : b.elems)
        for (int v : e)
            if (v < 0 || v >= nn) {
                set_error("element references node " + std::to_string(v + 1) + " of " + std::to_string(nn) + " in " + path);
                return EFEM_ERR_MESH;
            }
    return EFEM_OK;
}

// 4x4 homogeneous pose, src/math/Math.cpp:37-99 (keys of one pose object are
// visited in sorted order, as the reference's std::map-backed JSON does)
void pose_matrix(const Json& pose, double M[16])
{
    auto mul = [](const double A[16], const double B[16], double C[16]) {
        double T[16];
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) {
                double s = 0;
                for (int k = 0; k < 4; k++) s += A[4 * i + k] * B[4 * k + j];
                T[4 * i + j] = s;
            }
        std::memcpy(C, T, sizeof(T));
    };
    const double pi = 3.14159265358979323846;
    for (int k = 0; k < 16; k++) M[k] = (k % 5 == 0) ? 1.0 : 0.0;
    for (auto& item : pose.arr) {
        if (!item.is_object()) continue;
        std::vector<std::pair<std::string, const Json*>> kv;
        for (auto& p : item.obj) kv.emplace_back(p.first, &p.second);
        std::sort(kv.begin(), kv.end(), [](auto& a, auto& b) { return a.first < b.first; });
        for (auto& p : kv) {
            std::vector<double> v;
            for (auto& x : p.second->arr) v.push_back(x.num);
            double T[16] = { 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1 };
            if (p.first == "r" && v.size() == 3) {
                const double tx = pi * v[0] / 180.0, ty = pi * v[1] / 180.0, tz = pi * v[2] / 180.0;
                double Rx[16] = { 1, 0, 0, 0, 0, std::cos(tx), -std::sin(tx), 0, 0, std::sin(tx), std::cos(tx), 0, 0, 0, 0, 1 };
                double Ry[16] = { std::cos(ty), 0, std::sin(ty), 0, 0, 1, 0, 0, -std::sin(ty), 0, std::cos(ty), 0, 0, 0, 0, 1 };
                double Rz[16] = { std::cos(tz), -std::sin(tz), 0, 0, std::sin(tz), std::cos(tz), 0, 0, 0, 0, 1, 0, 0, 0, 0, 1 };
                mul(Ry, Rx, T);
                mul(Rz, T, T);
            } else if (p.first == "r" && v.size() == 4) {
                // axis-angle; the reference divides the angle by 180.8 (Math.cpp:69)
                double u = v[0], vv = v[1], w = v[2];
                const double t = pi * v[3] / 180.8, l = std::sqrt(u * u + vv * vv + w * w);
                u /= l;
                vv /= l;
                w /= l;
                const double c = std::cos(t), s = std::sin(t);
                double R[16] = { u * u + (1 - u * u) * c, u * vv * (1 - c) - w * s, u * w * (1 - c) + vv * s, 0,
                    u * vv * (1 - c) + w * s, vv * vv + (1 - vv * vv) * c, vv * w * (1 - c) - u * s, 0,
                    u * w * (1 - c) - vv * s, vv * w * (1 - c) + u * s, w * w + (1 - w * w) * c, 0, 0, 0, 0, 1 };
                std::memcpy(T, R, sizeof(R));
            } else if (p.first == "s" && v.size() >= 3) {
                T[0] = v[0];
                T[5] = v[1];
                T[10] = v[2];
            } else if (p.first == "t" && v.size() >= 3) {
                T[3] = v[0];
                T[7] = v[1];
                T[11] = v[2];
            } else {
                continue;
            }
            mul(T, M, M);
        }
    }
}

std::vector<int> model_ids_of(const Json& c)
{
    std::vector<int> ids;
    const Json* m = c.find("model_id");
    if (m && m->is_array())
        for (auto& x : m->arr) ids.push_back(static_cast<int>(x.num));
    else if (m && m->is_number())
        ids.push_back(static_cast<int>(m->num));
    if (ids.empty()) ids.push_back(-1);
    return ids;
}

}  // namespace

efem_status read_json_config(const char* path, ModelInput& in)
{
    std::string p(path ? path : "");
    const std::string wd = p.substr(0, p.find_last_of('/') + 1);
    std::ifstream f(p);
    if (!f) {
        set_error("config file " + p + " not found");
        return EFEM_ERR_CONFIG;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    Json cfg;
    try {
        cfg = JsonParser(text).parse();
    } catch (const std::exception& e) {
        set_error(std::string("config ") + p + ": " + e.what());
        return EFEM_ERR_CONFIG;
    }
    if (!cfg.is_object()) {
        set_error("config root is not an object");
        return EFEM_ERR_CONFIG;
    }
    efem_default_options(&in.opts);

    // analysis keys, src/io/Config.cpp:25-81 (+ library extensions)
    if (const Json* a = cfg.find("analysis"); a && a->is_object()) {
        if (const Json* s = a->find("nl_solver"); s && s->is_string()) {
            if (s->str == "lbfgs_ah") in.opts.nl_solver = 0;
            else if (s->str == "lbfgs") in.opts.nl_solver = 1;
        }
        // "max_optim_iters" is the key the reference's README and samples use;
        // the reference itself only reads "max_solver_iters"
        if (const Json* s = a->find("max_optim_iters"); s && s->is_number()) in.opts.max_iterations = (int)s->num;
        if (const Json* s = a->find("max_solver_iters"); s && s->is_number()) in.opts.max_iterations = (int)s->num;
        if (const Json* s = a->find("max_line_search"); s && s->is_number()) in.opts.max_linesearch = (int)s->num;
        if (const Json* s = a->find("dx_criterion"); s && s->is_number()) in.opts.dx_criterion = s->num;
        if (const Json* s = a->find("residual_criterion"); s && s->is_number()) in.opts.residual_criterion = s->num;
        if (const Json* s = a->find("integration"); s && s->is_string()) in.opts.integration = s->str == "reduced" ? 1 : 0;
        if (const Json* s = a->find("precision"); s && s->is_string()) in.opts.precision = s->str == "mixed" ? EFEM_MIXED : EFEM_FP64;
        // gravity as a load of 9.8 along one signed axis (src/io/Config.cpp:45-65,
        // src/fe/InertiaConstraint.cpp:64-84); other strings leave it off
        if (const Json* s = a->find("gravity"); s && s->is_string()) {
            static const char* axes[6] = { "x", "-x", "y", "-y", "z", "-z" };
            for (int k = 0; k < 6; k++)
                if (s->str == axes[k]) {
                    HostLoad L;
                    L.type = EFEM_LOAD_GRAVITY;
                    L.value[k / 2] = (k % 2) ? -9.8 : 9.8;
                    in.loads.push_back(std::move(L));
                }
        }
        if (const Json* s = a->find("consistent_inertia"); s && s->is_bool()) in.opts.consistent_inertia = s->b ? 1 : 0;
        if (const Json* s = a->find("line_search"); s && s->is_string()) in.opts.line_search = s->str == "armijo" ? 1 : 0;
    }

    // bodies, src/model/Model.cpp:14-37
    std::vector<Body> bodies;
    if (const Json* ms = cfg.find("model"); ms && ms->is_array()) {
        for (auto& mj : ms->arr) {
            const Json* t = mj.find("type");
            const Json* mf = mj.find("mesh_file");
            if (!t || !t->is_string() || !mf || !mf->is_string()) continue;
            Body b;
            b.id = static_cast<int>(mj.number_or("id", -1));
            efem_status s = read_mesh(wd + mf->str, b);
            if (s != EFEM_OK) return s;
            if (const Json* pose = mj.find("pose"); pose && pose->is_array()) {
                double M[16];
                pose_matrix(*pose, M);
                for (size_t n = 0; n < b.X.size() / 3; n++) {
                    double x = b.X[3 * n], y = b.X[3 * n + 1], z = b.X[3 * n + 2];
                    for (int i = 0; i < 3; i++) b.X[3 * n + i] = M[4 * i] * x + M[4 * i + 1] * y + M[4 * i + 2] * z + M[4 * i + 3];
                }
            }
            bodies.push_back(std::move(b));
        }
    }
    if (bodies.empty()) {
        set_error("config has no model[] body with a mesh_file");
        return EFEM_ERR_CONFIG;
    }
    // global node numbering: bodies concatenated in order (src/fe/Constraint.cpp:26-40)
    std::map<int, int> body_of_id;  // last body with an id wins (m_body_map[id] = body)
    std::vector<int> offset(bodies.size());
    int total = 0;
    for (size_t k = 0; k < bodies.size(); k++) {
        offset[k] = total;
        total += static_cast<int>(bodies[k].X.size() / 3);
        body_of_id[bodies[k].id] = static_cast<int>(k);
        in.X.insert(in.X.end(), bodies[k].X.begin(), bodies[k].X.end());
    }
    // every element in body then file order (the order of the reference's output mesh)
    in.cell_ptr.assign(1, 0);
    for (size_t k = 0; k < bodies.size(); k++)
        for (size_t e = 0; e < bodies[k].elems.size(); e++) {
            for (int v : bodies[k].elems[e]) in.cell_nodes.push_back(v + offset[k]);
            in.cell_ptr.push_back(static_cast<int>(in.cell_nodes.size()));
        }
    // element blocks by node count, in body then file order
    for (int nen : { 4, 8, 10, 20 }) {
        HostBlock hb;
        hb.nen = nen;
        for (size_t k = 0; k < bodies.size(); k++)
            for (size_t e = 0; e < bodies[k].elems.size(); e++) {
                if (bodies[k].nen[e] != nen) continue;
                for (int v : bodies[k].elems[e]) hb.conn.push_back(v + offset[k]);
                hb.mat_id.push_back(bodies[k].mat[e]);
            }
        if (!hb.mat_id.empty()) in.blocks.push_back(std::move(hb));
    }

    // materials, src/fe/ElementConstraint.cpp:39-67
    if (const Json* ms = cfg.find("material"); ms && ms->is_array()) {
        for (auto& mj : ms->arr) {
            const Json* t = mj.find("type");
            if (!t || !t->is_string()) continue;
            HostMaterial hm {};
            if (t->str == "neo_hookean") hm.type = EFEM_NEO_HOOKEAN;
            else if (t->str == "mo_riv") hm.type = EFEM_MOONEY_RIVLIN;
            else if (t->str == "yeoh") hm.type = EFEM_YEOH;
            else continue;
            hm.id = static_cast<int>(mj.number_or("id", -1));
            hm.density = mj.number_or("density", 0.0);
            hm.C10 = mj.number_or("C10", 0.0);
            hm.C01 = hm.type == EFEM_MOONEY_RIVLIN ? mj.number_or("C01", 0.0) : 0.0;
            hm.C20 = hm.type == EFEM_YEOH ? mj.number_or("C20", 0.0) : 0.0;
            hm.C30 = hm.type == EFEM_YEOH ? mj.number_or("C30", 0.0) : 0.0;
            hm.D1 = mj.number_or("D1", 0.0);
            in.materials.push_back(hm);
        }
    }

    // constraints, src/fe/ExternalConstraint.cpp:13-247
    if (const Json* cs = cfg.find("constraint"); cs && cs->is_array()) {
        for (auto& cj : cs->arr) {
            const Json* t = cj.find("type");
            if (!t || !t->is_string()) continue;
            const std::string type = t->str;
            if (type != "fix" && type != "force" && type != "pressure") continue;
            std::vector<std::string> lines;
            if (const Json* fn = cj.find("constraint_file"); fn && fn->is_string() && !fn->str.empty()) {
                efem_status s = read_lines(wd + fn->str, lines);
                if (s != EFEM_OK) return s;
            }
            std::vector<int> ids = model_ids_of(cj);
            for (int mid : ids) {
                auto it = body_of_id.find(mid);
                if (it == body_of_id.end()) {
                    set_error("constraint refers to model_id " + std::to_string(mid) + " that no body has");
                    return EFEM_ERR_CONFIG;
                }
                const int k = it->second, off = offset[k];
                const int nb = static_cast<int>(bodies[k].X.size() / 3);
                HostLoad L;
                auto node = [&](const std::string& tok, int* out) -> bool {
                    int v;
                    if (!parse_int(tok, &v) || v < 1 || v > nb) {
                        set_error("constraint node '" + tok + "' out of range");
                        return false;
                    }
                    *out = v - 1 + off;
                    return true;
                };
                if (type == "fix" || type == "force") {
                    L.type = type == "fix" ? EFEM_LOAD_FIX : EFEM_LOAD_FORCE;
                    for (auto& ln : lines)
                        for (auto& tok : split_tokens(ln)) {
                            int v;
                            if (!node(tok, &v)) return EFEM_ERR_MESH;
                            L.nodes.push_back(v);
                        }
                    if (type == "force") {
                        const Json* v = cj.find("value");
                        if (v && v->is_array() && v->arr.size() >= 3)
                            for (int c = 0; c < 3; c++) L.value[c] = v->arr[c].num;
                    }
                } else {
                    const Json* v = cj.find("value");
                    if (v && v->is_number()) {
                        if (!(v->num > 0)) continue;  // ignored (ExternalConstraint.cpp:195-197)
                        L.type = EFEM_LOAD_PRESSURE;
                        L.value[0] = v->num;
                    } else if (v && v->is_array() && v->arr.size() >= 3) {
                        for (int c = 0; c < 3; c++) L.value[c] = v->arr[c].num;
                        if (!(std::sqrt(L.value[0] * L.value[0] + L.value[1] * L.value[1] + L.value[2] * L.value[2]) > 0)) continue;
                        L.type = EFEM_LOAD_DPRESSURE;
                    } else {
                        continue;
                    }
                    L.face_ptr.push_back(0);
                    for (auto& ln : lines) {
                        std::vector<int> face;
                        for (auto& tok : split_tokens(ln)) {
                            int vv;
                            if (!node(tok, &vv)) return EFEM_ERR_MESH;
                            if (std::find(face.begin(), face.end(), vv) == face.end()) face.push_back(vv);
                        }
                        L.nodes.insert(L.nodes.end(), face.begin(), face.end());
                        L.face_ptr.push_back(static_cast<int>(L.nodes.size()));
                    }
                }
                in.loads.push_back(std::move(L));
            }
        }
    }
    return EFEM_OK;
}

}  // namespace efem
