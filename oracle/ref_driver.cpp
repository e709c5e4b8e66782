// Test infrastructure only -- never part of the product path.
//
// Command-line driver around the UNMODIFIED reference sources (compiled in
// place by oracle/Makefile against the shims in oracle/shim/).  It exposes the
// reference's own public entry points so the C restatement (efem_oracle.c)
// and the CUDA path can be pinned against the reference itself:
//
//   efem_ref residual <cfg.json> <u.f64|zero> <r_out.f64> [--reduced]
//       Constraint::assignDx + Constraint::getResidual   (src/fe/Constraint.cpp:93-126)
//   efem_ref jacobi   <cfg.json> <trip_out.bin> [--reduced]
//       Constraint::getJacobi triplets                    (src/fe/Constraint.cpp:128-138)
//   efem_ref solve    <cfg.json> <u_out.f64> [--reduced] [--max-iters N] [--trace <r2_out.f64>]
//       LBFGSSolver<SoftObjective>::solve from x = 0      (src/simulation/Integrator.cpp:22-42,
//                                                          src/simulation/nlsolver/LBFGS.h:96-174)
//   efem_ref info     <cfg.json> <dofmap_out.i32>
//       free-DOF numbering: node -> id (-1 fixed)         (src/fe/Constraint.cpp:61-72)
//   efem_ref bench    <cfg.json> <iters_per_step> <warmup_steps> <steps>
//       the same solve driven step by step through the reference's own
//       components (SoftObjective, LBFGSMat, LineSearchFEA, SimplicialLLT),
//       timing the one-time approximate-Jacobian factorisation and then each
//       step of <iters_per_step> L-BFGS iterations separately
//   efem_ref piola    <neo_hookean|mo_riv|yeoh> C10 C01 C20 C30 D1 <F.f64> <P_out.f64>
//       Material::getFirstPiola on a batch of column-major 3x3 F
//                                                         (src/material/*.cpp)
//
// --reduced swaps every element's integration rule for the reduced-integration
// class of the same element (TetElement3D4R / TetElement3D10R / HexElement3D8R /
// HexElement3D20R, src/fe/element/IntegralElement.h:76-157), which the
// reference defines but never selects (src/fe/Constraint.cpp:9-20).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "Eigen/Core"
#include "Eigen/Dense"
#include "Eigen/Sparse"
#include "Eigen/SparseCholesky"
#include "nlohmann/json.hpp"
#include "spdlog/sinks/basic_file_sink.h"
#include "spdlog/spdlog.h"

// The reduced-integration swap replaces a member the reference keeps private
// (ElementConstraint::m_integral_element) and walks Constraint::m_constraints;
// this driver is the only translation unit that sees them as public.
#define private public
#define protected public
#include "fe/Constraint.h"
#include "fe/ElementConstraint.h"
#include "fe/ExternalConstraint.h"
#include "fe/element/IntegralElement.h"
#include "io/Config.h"
#include "material/Material.h"
#include "model/Model.h"
#include "simulation/Integrator.h"
#include "simulation/nlsolver/LBFGS.h"
#undef private
#undef protected

using namespace EFEM;

static std::vector<double> read_f64(const std::string& path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        fprintf(stderr, "cannot open %s\n", path.c_str());
        exit(2);
    }
    f.seekg(0, std::ios::end);
    size_t n = f.tellg() / sizeof(double);
    f.seekg(0);
    std::vector<double> v(n);
    f.read(reinterpret_cast<char*>(v.data()), n * sizeof(double));
    return v;
}

static void write_raw(const std::string& path, const void* p, size_t bytes)
{
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(p), bytes);
}

struct Problem {
    std::shared_ptr<Config> config;
    std::shared_ptr<Model> model;
    std::shared_ptr<Constraint> constraint;
};

static void swap_to_reduced(Constraint& c)
{
    for (auto& con : c.m_constraints) {
        auto ec = std::dynamic_pointer_cast<ElementConstraint>(con);
        if (!ec)
            continue;
        auto el = ec->m_element;
        std::shared_ptr<IntegralElement> r;
        switch (el->nodes.size()) {
        case 4: r = std::make_shared<TetElement3D4R>(el); break;
        case 8: r = std::make_shared<HexElement3D8R>(el); break;
        case 10: r = std::make_shared<TetElement3D10R>(el); break;
        case 20: r = std::make_shared<HexElement3D20R>(el); break;
        }
        ec->m_integral_element = r;
    }
}

static Problem load(const std::string& cfg, bool reduced)
{
    Problem p;
    p.config = std::make_shared<Config>(cfg);
    if (!p.config->io()->configJson()) {
        fprintf(stderr, "config not loaded: %s\n", cfg.c_str());
        exit(3);
    }
    p.model = std::make_shared<Model>(p.config);
    p.constraint = std::make_shared<Constraint>(p.config, p.model);
    if (reduced)
        swap_to_reduced(*p.constraint);
    return p;
}

static int cmd_piola(int argc, char** argv)
{
    if (argc < 10)
        return 1;
    std::string type = argv[2];
    double C10 = atof(argv[3]), C01 = atof(argv[4]), C20 = atof(argv[5]), C30 = atof(argv[6]), D1 = atof(argv[7]);
    Json j = { { "C10", C10 }, { "C01", C01 }, { "C20", C20 }, { "C30", C30 }, { "D1", D1 } };
    std::shared_ptr<Material> m;
    if (type == "neo_hookean")
        m = std::make_shared<NeoHookean>();
    else if (type == "mo_riv")
        m = std::make_shared<MooneyRivlin>();
    else
        m = std::make_shared<Yeoh>();
    m->initFromJson(j);
    std::vector<double> F = read_f64(argv[8]);
    std::vector<double> P(F.size());
    for (size_t k = 0; k + 9 <= F.size(); k += 9) {
        Eigen::Matrix3d Fm = Eigen::Map<Eigen::Matrix3d>(F.data() + k);
        Eigen::Matrix3d Pm = m->getFirstPiola(Fm);
        Eigen::Map<Eigen::Matrix3d>(P.data() + k) = Pm;
    }
    write_raw(argv[9], P.data(), P.size() * sizeof(double));
    printf("{\"elasticity_coeff\": %.17g}\n", m->elasticity_coeff);
    return 0;
}

// LBFGSSolver::solve (src/simulation/nlsolver/LBFGS.h:96-174) with its loop
// cut into timed steps; every call below is the reference's own code.
static int cmd_bench(Problem& p, int ipstep, int warm, int steps)
{
    using clk = std::chrono::steady_clock;
    auto ac = p.config->analysisConfig();
    NLSolverParam param;
    param.epsilon = ac->residual_criterion;
    param.epsilon_rel = ac->residual_criterion;
    param.max_linesearch = ac->max_line_search;
    param.config = p.config;
    SoftObjective obj;
    obj.constraint = p.constraint;
    obj.dimens = p.constraint->getDimens();
    const int n = obj.dimens;
    Eigen::VectorXd x = Eigen::VectorXd::Zero(n), xp(n), r(n), rp(n), d(n);
    LBFGSMat bfgs;
    bfgs.reset(n, param.m);
    obj.residual(x, r);
    auto t0 = clk::now();
    Eigen::SparseMatrix<double> K;
    obj.jacobi(x, K);
    auto llt = std::make_shared<Eigen::SimplicialLLT<Eigen::SparseMatrix<double>, Eigen::Upper>>();
    llt->analyzePattern(K);
    llt->factorize(K);
    const bool ok = llt->info() == Eigen::Success;
    if (!ok) llt.reset();
    bfgs.setApproxJacobiSolverPtr(llt);
    d = ok ? Eigen::VectorXd(-llt->solve(r)) : Eigen::VectorXd(-r);
    auto t1 = clk::now();
    int k = 1, converged_at = 0;
    std::vector<double> st;
    for (int step = 0; step < warm + steps && !converged_at; step++) {
        auto a = clk::now();
        int done = 0;
        for (int it = 0; it < ipstep; it++) {
            double s1 = 1.0;
            xp = x;
            rp = r;
            LineSearchFEA::LineSearch(obj, x, r, s1, d, xp, param);
            done++;
            const double g = r.lpNorm<Eigen::Infinity>();
            if (g <= param.epsilon || g <= param.epsilon_rel * x.lpNorm<Eigen::Infinity>()) {
                converged_at = k;
                break;
            }
            bfgs.add_correction(x - xp, r - rp);
            bfgs.apply_Hv(r, -1.0, d);
            k++;
        }
        auto b = clk::now();
        if (step >= warm) st.push_back(std::chrono::duration<double>(b - a).count() / done * ipstep);
    }
    printf("{\"n_dof\": %d, \"factor_ok\": %d, \"factor_s\": %.6f, \"iters_per_step\": %d, \"converged_at\": %d, "
           "\"r_evals\": %d, \"step_s\": [",
        n, ok ? 1 : 0, std::chrono::duration<double>(t1 - t0).count(), ipstep, converged_at, obj.r_evalutes);
    for (size_t i = 0; i < st.size(); i++) printf("%s%.6f", i ? ", " : "", st[i]);
    printf("]}\n");
    return 0;
}

int main(int argc, char** argv)
{
    if (argc < 2) {
        fprintf(stderr, "usage: efem_ref residual|jacobi|solve|info|piola ...\n");
        return 1;
    }
    std::string cmd = argv[1];
    if (cmd == "piola")
        return cmd_piola(argc, argv);
    if (argc < 4)
        return 1;
    bool reduced = false;
    int max_iters = -1;
    const char* trace_path = nullptr;
    for (int i = 4; i < argc; i++) {
        if (!strcmp(argv[i], "--reduced"))
            reduced = true;
        if (!strcmp(argv[i], "--max-iters") && i + 1 < argc)
            max_iters = atoi(argv[i + 1]);
        if (!strcmp(argv[i], "--trace") && i + 1 < argc)
            trace_path = argv[i + 1];
    }
    std::string cfg = argv[2];
    auto t0 = std::chrono::steady_clock::now();
    Problem p = load(cfg, reduced);
    auto t1 = std::chrono::steady_clock::now();
    int n = p.constraint->getDimens();

    if (cmd == "bench") {
        if (argc < 6) return 1;
        return cmd_bench(p, atoi(argv[3]), atoi(argv[4]), atoi(argv[5]));
    }
    if (cmd == "info") {
        std::vector<int> ids;
        for (auto& body : p.model->getBodies())
            for (auto& node : body->getNodes())
                ids.push_back(std::static_pointer_cast<ConstraintNodeInfo>(node->extra_info["constraint_info"])->id);
        write_raw(argv[3], ids.data(), ids.size() * sizeof(int));
        printf("{\"n_dof\": %d, \"n_nodes\": %zu}\n", n, ids.size());
        return 0;
    }
    if (cmd == "residual") {
        if (argc < 5)
            return 1;
        Eigen::VectorXd u = Eigen::VectorXd::Zero(n);
        if (strcmp(argv[3], "zero")) {
            std::vector<double> uv = read_f64(argv[3]);
            if ((int)uv.size() != n) {
                fprintf(stderr, "u has %zu values, model has %d dofs\n", uv.size(), n);
                return 4;
            }
            u = Eigen::Map<Eigen::VectorXd>(uv.data(), n);
        }
        Eigen::VectorXd r;
        p.constraint->assignDx(u);
        p.constraint->getResidual(r);
        write_raw(argv[4], r.data(), n * sizeof(double));
        printf("{\"n_dof\": %d}\n", n);
        return 0;
    }
    if (cmd == "jacobi") {
        std::vector<SparseMatrixTriplet> trip;
        Eigen::VectorXd u = Eigen::VectorXd::Zero(n);
        p.constraint->assignDx(u);
        p.constraint->getJacobi(trip);
        std::ofstream f(argv[3], std::ios::binary);
        long long cnt = trip.size();
        f.write(reinterpret_cast<const char*>(&cnt), sizeof(cnt));
        for (auto& t : trip) {
            int rc[2] = { (int)t.row(), (int)t.col() };
            double v = t.value();
            f.write(reinterpret_cast<const char*>(rc), sizeof(rc));
            f.write(reinterpret_cast<const char*>(&v), sizeof(v));
        }
        printf("{\"n_dof\": %d, \"n_triplets\": %lld}\n", n, cnt);
        return 0;
    }
    if (cmd == "solve") {
        // Integrator::Integrator (src/simulation/Integrator.cpp:6-20) maps the
        // config onto the solver parameters exactly like this.
        NLSolverParam param;
        auto ac = p.config->analysisConfig();
        param.epsilon = ac->residual_criterion;
        param.epsilon_rel = ac->residual_criterion;
        param.max_iterations = max_iters >= 0 ? max_iters : ac->max_solver_iters;
        param.max_linesearch = ac->max_line_search;
        param.config = p.config;
        // --trace: the reference's own benchmark record (LBFGS.h:107-147),
        // ||r||_2 after the initial residual and after every line search
        param.benchmark = trace_path != nullptr;
        SoftObjective obj;
        obj.constraint = p.constraint;
        obj.dimens = n;
        LBFGSSolver<SoftObjective> solver(param);
        Eigen::VectorXd x = Eigen::VectorXd::Zero(n);
        auto t2 = std::chrono::steady_clock::now();
        int niter = solver.solve(obj, x);
        auto t3 = std::chrono::steady_clock::now();
        write_raw(argv[3], x.data(), n * sizeof(double));
        if (trace_path)
            write_raw(trace_path, solver.m_f_benchmark.data(), solver.m_f_benchmark.size() * sizeof(double));
        double rinf = obj.nl_residual.size() ? obj.nl_residual.lpNorm<Eigen::Infinity>() : 0.0;
        // precond_ok: the approximate-Jacobian factorisation succeeded
        // (LBFGSSolver::updateApproxJacobi, LBFGS.h:65-81); 0 = the H0 = I/theta fallback ran
        printf("{\"n_dof\": %d, \"niter\": %d, \"r_evals\": %d, \"j_evals\": %d, \"precond_ok\": %d, "
               "\"u_inf\": %.17g, \"r_inf\": %.17g, \"setup_s\": %.6f, \"solve_s\": %.6f}\n",
            n, niter, obj.r_evalutes, obj.j_evalutes, solver.m_jacobi_available ? 1 : 0, x.lpNorm<Eigen::Infinity>(), rinf,
            std::chrono::duration<double>(t1 - t0).count(), std::chrono::duration<double>(t3 - t2).count());
        return 0;
    }
    fprintf(stderr, "unknown command %s\n", cmd.c_str());
    return 1;
}
