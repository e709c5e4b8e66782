// efem_gpu -f cfg.json: the reference's command line (src/main/main.cpp,
// src/simulation/Simulator.cpp:6-41) on the GPU library.  Same config file;
// same log line after the solve (src/simulation/Integrator.cpp:36-40); with
// output.save_frame the undeformed and deformed meshes are written as legacy
// VTK files under <config dir>/results/<date>/<date-time-ms>-{undeformed,deformed}.vtk
// like Model::saveVTK (src/model/Model.cpp:50-117).  --benchmark prints the
// solve's convergence record as LBFGSSolver::printBenchmark does
// (src/simulation/nlsolver/LBFGS.h:176-189): per record the residual norm
// scaled to (f_i - f_last) / (f_0 - f_last) and the seconds since the solve
// started, at most 9000 lines.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/efem_gpu.h"
#include "../csrc/json.h"

namespace {

void info(const std::string& msg)
{
    std::printf("[info] %s\n", msg.c_str());
    std::fflush(stdout);
}

int fail(const char* what)
{
    char buf[1024];
    efem_last_error(buf, sizeof buf);
    std::fprintf(stderr, "[error] %s: %s\n", what, buf);
    return 1;
}

std::string stamp(std::string* day)
{
    using namespace std::chrono;
    const auto now = system_clock::now();
    const std::time_t t = system_clock::to_time_t(now);
    std::tm tm {};
    localtime_r(&t, &tm);
    char d[32], s[64];
    std::strftime(d, sizeof d, "%Y-%m-%d", &tm);
    std::strftime(s, sizeof s, "%Y-%m-%d-%H-%M-%S", &tm);
    const long ms = static_cast<long>(duration_cast<milliseconds>(now.time_since_epoch()).count() % 1000);
    char out[96];
    std::snprintf(out, sizeof out, "%s-%03ld", s, ms);
    *day = d;
    return out;
}

int save_vtk(void* model, const double* u, const std::string& workdir, const char* name)
{
    std::string day;
    const std::string st = stamp(&day);
    const std::filesystem::path dir = std::filesystem::path(workdir) / "results" / day;
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    const std::string path = (dir / (st + "-" + name + ".vtk")).string();
    if (efem_write_vtk(model, u, path.c_str()) != EFEM_OK) return fail("writing VTK");
    return 0;
}

}  // namespace

int main(int argc, char** argv)
{
    std::string cfg;
    int device = -1;
    bool benchmark = false;
    for (int i = 1; i < argc; i++) {
        if (!std::strcmp(argv[i], "-f") && i + 1 < argc) {
            cfg = argv[++i];
        } else if (!std::strcmp(argv[i], "--device") && i + 1 < argc) {
            device = std::atoi(argv[++i]);
        } else if (!std::strcmp(argv[i], "--benchmark")) {
            benchmark = true;
        } else if (!std::strcmp(argv[i], "-h") || !std::strcmp(argv[i], "--help")) {
            std::printf("Efficient FEM on the GPU\nUsage: %s -f <config.json> [--device N] [--benchmark]\n", argv[0]);
            return 0;
        } else {
            std::fprintf(stderr, "unknown argument %s\n", argv[i]);
            return 2;
        }
    }
    if (cfg.empty()) {
        std::fprintf(stderr, "Usage: %s -f <config.json> [--device N]\n", argv[0]);
        return 2;
    }
    info("config_file=" + cfg);
    bool save_frame = false, show_log = true;
    {
        std::ifstream f(cfg);
        std::stringstream ss;
        ss << f.rdbuf();
        try {
            const efem::Json j = efem::JsonParser(ss.str()).parse();
            if (const efem::Json* o = j.find("output")) {
                if (const efem::Json* s = o->find("save_frame"); s && s->is_bool()) save_frame = s->b;
                if (const efem::Json* s = o->find("show_log"); s && s->is_bool()) show_log = s->b;
            }
        } catch (const std::exception&) {
            // the library reports unreadable configs below
        }
    }
    const std::string workdir = std::filesystem::path(cfg).parent_path().string();
    void* model = nullptr;
    if (efem_model_create_from_json(cfg.c_str(), &model) != EFEM_OK) return fail("reading the config");
    constexpr int kBenchmarkRows = 9000;
    if (device >= 0 || benchmark) {
        efem_options o;
        efem_get_options(model, &o);
        if (device >= 0) o.device = device;
        if (benchmark) o.trace = kBenchmarkRows;
        efem_set_options(model, &o);
    }
    if (show_log) info("Simulator initialed");
    if (save_frame && save_vtk(model, nullptr, workdir, "undeformed")) return 1;
    efem_model_info mi;
    efem_get_model_info(model, &mi);
    std::vector<double> u(static_cast<size_t>(mi.n_dof), 0.0);
    if (show_log) info("Simulator started");
    const auto t0 = std::chrono::steady_clock::now();
    efem_solve_info si;
    const efem_status st = efem_solve(model, u.data(), &si);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (st == EFEM_ERR_NAN) {
        std::fprintf(stderr, "[error] LBFGS solver error!\n");
    } else if (st != EFEM_OK) {
        return fail("solve");
    } else if (show_log) {
        char line[512];
        std::snprintf(line, sizeof line, "dx=%.17g, residual=%.17g, niter=%d, r_evalutes=%d, j_evalutes=%d", si.u_inf,
            si.r_inf, si.niter, si.n_residual_evals, si.n_jacobian_evals);
        info(line);
    }
    if (benchmark) {
        int n = 0;
        efem_solve_trace(model, nullptr, 0, &n);
        n = std::min(n, kBenchmarkRows);
        std::vector<double> rec(static_cast<size_t>(n) * 5);
        if (n > 0) efem_solve_trace(model, rec.data(), n, &n);
        n = std::min(n, kBenchmarkRows);
        if (n == 0) {
            info("no benchmark!");
        } else {
            const double last = rec[5 * static_cast<size_t>(n - 1) + 1], span = rec[1] - last;
            for (int i = 0; i < n; i++) {
                char line[128];
                std::snprintf(line, sizeof line, "benchmark[%d]: f=%.17g, time=%.9gs", i,
                    (rec[5 * static_cast<size_t>(i) + 1] - last) / span, rec[5 * static_cast<size_t>(i)]);
                info(line);
            }
        }
    }
    if (show_log) {
        char line[128];
        std::snprintf(line, sizeof line, "Simulator step end, use %gs", secs);
        info(line);
    }
    if (save_frame && save_vtk(model, u.data(), workdir, "deformed")) return 1;
    efem_model_destroy(model);
    return st == EFEM_OK ? 0 : 1;
}
