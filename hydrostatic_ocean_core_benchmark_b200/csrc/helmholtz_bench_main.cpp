// helmholtz_bench_b200 <case.nml> [solver]
//
// Standalone variable-coefficient Helmholtz bench over the C ABI, with the
// command line, inputs and outputs of the reference's bench
// (libs/cuda/src/helmholtz_bench.cu:263-500):
//   - case.nml (&helmholtz: nx, ny, dx, dy, coef, rtol, max_iter, n_repeat,
//     n_warmup, datadir, optional solver and outfile), written by the
//     reference's tools/write_helmholtz_case.py;
//   - datadir/{ku,kv,mask,rhs}.bin fp64 [ny][nx], optional eta_ref.bin;
//   - n_warmup untimed solves, then n_repeat timed solves: median, MAD and min
//     of the wall time of one solve with the data on the device;
//   - metrics JSON (outfile, else datadir/metrics_b200_<solver>.json) and the
//     line "solver=... iters=... wall=... l2_vs_ref=...".
// "residual" is the true relative residual ||rhs - A x|| / ||rhs|| of the
// returned solution, formed in fp64 on the host with the operator of
// libs/core/solvers_var.py:47-53.
// Besides the reference's four solvers, solver "pcg_refined" (no reference
// counterpart) runs the FP32-inner, FP64-refined solver; its JSON then says
// "precision": "fp32+fp64-refined".

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "ocean_b200.h"

namespace {

struct Case {
    int nx = 128, ny = 128, max_iter = 20000, n_repeat = 5, n_warmup = 1;
    double dx = 1.0, dy = 1.0, coef = 1.0, rtol = 1e-10;
    std::string datadir = ".", solver = "pcg_jacobi", outfile;
};

std::string trim(std::string s) {
    const char* ws = " \t\r\n'\"";
    s.erase(0, s.find_first_not_of(ws));
    const size_t e = s.find_last_not_of(ws);
    s.erase(e == std::string::npos ? 0 : e + 1);
    return s;
}

bool read_case(const char* path, Case& c) {
    FILE* f = std::fopen(path, "r");
    if (!f) return false;
    char line[4096];
    while (std::fgets(line, sizeof line, f)) {
        std::string s(line);
        const size_t eq = s.find('=');
        if (eq == std::string::npos) continue;
        const std::string key = trim(s.substr(0, eq));
        std::string val = trim(s.substr(eq + 1));
        if (!val.empty() && val.back() == ',') val = trim(val.substr(0, val.size() - 1));
        if (key != "datadir" && key != "solver" && key != "outfile")  // Fortran d exponents
            for (char& ch : val)
                if (ch == 'd' || ch == 'D') ch = 'e';
        if (key == "nx") c.nx = std::atoi(val.c_str());
        else if (key == "ny") c.ny = std::atoi(val.c_str());
        else if (key == "dx") c.dx = std::strtod(val.c_str(), nullptr);
        else if (key == "dy") c.dy = std::strtod(val.c_str(), nullptr);
        else if (key == "coef") c.coef = std::strtod(val.c_str(), nullptr);
        else if (key == "rtol") c.rtol = std::strtod(val.c_str(), nullptr);
        else if (key == "max_iter") c.max_iter = std::atoi(val.c_str());
        else if (key == "n_repeat") c.n_repeat = std::atoi(val.c_str());
        else if (key == "n_warmup") c.n_warmup = std::atoi(val.c_str());
        else if (key == "datadir") c.datadir = val;
        else if (key == "solver") c.solver = val;
        else if (key == "outfile") c.outfile = val;
    }
    std::fclose(f);
    return true;
}

bool read_bin(const std::string& path, std::vector<double>& a, size_t n) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    a.resize(n);
    const size_t got = std::fread(a.data(), sizeof(double), n, f);
    std::fclose(f);
    return got == n;
}

double median_of(std::vector<double> v) {
    std::sort(v.begin(), v.end());
    const size_t m = v.size();
    return m % 2 ? v[m / 2] : 0.5 * (v[m / 2 - 1] + v[m / 2]);
}

// ||b - A x|| / ||b|| with A x = (xm - coef lap) m + xm (1 - m), xm = x m, on the
// periodic index layout (VarOperator.apply)
double relative_residual(const Case& c, const std::vector<double>& ku, const std::vector<double>& kv,
                         const std::vector<double>& m, const std::vector<double>& b,
                         const std::vector<double>& x) {
    const int nx = c.nx, ny = c.ny;
    const double dx2 = c.dx * c.dx, dy2 = c.dy * c.dy;
    double num = 0.0, den = 0.0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const int e = j * nx + i;
            const int ie = j * nx + (i + 1) % nx, iw = j * nx + (i + nx - 1) % nx;
            const int jn = ((j + 1) % ny) * nx + i, js = ((j + ny - 1) % ny) * nx + i;
            const double xm = x[e] * m[e];
            const double fx = ku[e] * (x[ie] * m[ie] - xm), fxw = ku[iw] * (xm - x[iw] * m[iw]);
            const double fy = kv[e] * (x[jn] * m[jn] - xm), fys = kv[js] * (xm - x[js] * m[js]);
            const double lap = (fx - fxw) / dx2 + (fy - fys) / dy2;
            const double ax = (xm - c.coef * lap) * m[e] + xm * (1.0 - m[e]);
            const double r = b[e] * m[e] - ax;
            num += r * r;
            den += b[e] * m[e] * b[e] * m[e];
        }
    return std::sqrt(num) / (den > 0.0 ? std::sqrt(den) : 1.0);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::printf("usage: %s <case.nml> [solver]\n", argv[0]);
        return 1;
    }
    Case cs;
    if (!read_case(argv[1], cs)) {
        std::fprintf(stderr, "FATAL: cannot open %s\n", argv[1]);
        return 1;
    }
    if (argc >= 3) cs.solver = argv[2];
    int kind = -1;
    if (cs.solver == "pcg_jacobi") kind = OC_SOLVER_PCG_JACOBI;
    else if (cs.solver == "pcg_rbgs") kind = OC_SOLVER_PCG_RBGS;
    else if (cs.solver == "rbgs") kind = OC_SOLVER_RBGS;
    else if (cs.solver == "multigrid") kind = OC_SOLVER_MULTIGRID;
    else if (cs.solver == "pcg_refined") kind = OC_SOLVER_PCG_REFINED;  // FP32 inner, FP64 refinement
    if (kind < 0) {
        std::fprintf(stderr, "FATAL: unknown solver %s\n", cs.solver.c_str());
        return 1;
    }
    const size_t n = (size_t)cs.nx * cs.ny;
    std::vector<double> ku, kv, msk, rhs, ref;
    if (!read_bin(cs.datadir + "/ku.bin", ku, n) || !read_bin(cs.datadir + "/kv.bin", kv, n) ||
        !read_bin(cs.datadir + "/mask.bin", msk, n) || !read_bin(cs.datadir + "/rhs.bin", rhs, n)) {
        std::fprintf(stderr, "FATAL: missing input binaries in %s\n", cs.datadir.c_str());
        return 1;
    }
    const bool have_ref = read_bin(cs.datadir + "/eta_ref.bin", ref, n);

    oc_helm_config cfg{};
    cfg.nx = cs.nx;
    cfg.ny = cs.ny;
    cfg.dx = cs.dx;
    cfg.dy = cs.dy;
    cfg.coef = cs.coef;
    cfg.solver = kind;
    cfg.rtol = cs.rtol;
    cfg.max_iter = cs.max_iter;
    cfg.device = 0;
    oc_helm* h = nullptr;
    int rc = oc_helm_create(&cfg, ku.data(), kv.data(), msk.data(), &h);
    if (rc) {
        std::fprintf(stderr, "FATAL: oc_helm_create failed (%d)\n", rc);
        return 1;
    }
    double *d_rhs = nullptr, *d_x = nullptr;
    if (cudaMalloc(&d_rhs, n * sizeof(double)) != cudaSuccess || cudaMalloc(&d_x, n * sizeof(double)) != cudaSuccess) {
        std::fprintf(stderr, "FATAL: cudaMalloc failed\n");
        return 1;
    }
    cudaMemcpy(d_rhs, rhs.data(), n * sizeof(double), cudaMemcpyHostToDevice);
    int32_t iters = 0, conv = 0;
    auto run = [&]() {
        const int r = oc_helm_solve(h, d_rhs, d_x, 1, &iters, &conv, nullptr);
        if (r) {
            std::fprintf(stderr, "FATAL: oc_helm_solve failed (%d): %s\n", r, oc_helm_last_error(h));
            std::exit(1);
        }
    };
    for (int w = 0; w < cs.n_warmup; ++w) run();
    std::vector<double> samples;
    for (int r = 0; r < cs.n_repeat; ++r) {
        const auto t0 = std::chrono::steady_clock::now();
        run();
        const auto t1 = std::chrono::steady_clock::now();
        samples.push_back(std::chrono::duration<double>(t1 - t0).count());
    }
    const double wall = median_of(samples);
    const double wall_min = *std::min_element(samples.begin(), samples.end());
    std::vector<double> dev;
    for (double s : samples) dev.push_back(std::fabs(s - wall));
    const double wall_mad = median_of(dev);

    std::vector<double> x(n);
    cudaMemcpy(x.data(), d_x, n * sizeof(double), cudaMemcpyDeviceToHost);
    const double residual = relative_residual(cs, ku, kv, msk, rhs, x);
    double err = -1.0;
    if (have_ref) {
        double num = 0.0, den = 0.0;
        for (size_t t = 0; t < n; ++t) {
            const double d = x[t] - ref[t];
            num += d * d;
            den += ref[t] * ref[t];
        }
        err = std::sqrt(num) / (den > 0.0 ? std::sqrt(den) : 1.0);
    }
    const std::string out = cs.outfile.empty() ? cs.datadir + "/metrics_b200_" + cs.solver + ".json" : cs.outfile;
    FILE* f = std::fopen(out.c_str(), "w");
    if (!f) {
        std::fprintf(stderr, "FATAL: cannot write %s\n", out.c_str());
        return 1;
    }
    std::fprintf(f,
                 "{\n  \"backend\": \"cuda_b200\",\n  \"precision\": \"%s\",\n  \"solver\": \"%s\",\n"
                 "  \"nx\": %d,\n  \"ny\": %d,\n  \"iterations\": %d,\n  \"converged\": %s,\n"
                 "  \"wall_s\": %.16e,\n  \"wall_mad_s\": %.16e,\n  \"wall_min_s\": %.16e,\n"
                 "  \"residual\": %.16e,\n  \"l2_rel_vs_reference\": %.16e,\n  \"n_repeat\": %d\n}\n",
                 kind == OC_SOLVER_PCG_REFINED ? "fp32+fp64-refined" : "fp64", cs.solver.c_str(), cs.nx, cs.ny, iters, conv ? "true" : "false", wall, wall_mad, wall_min,
                 residual, err, cs.n_repeat);
    std::fclose(f);
    std::printf("solver=%12s iters=%8d wall=%12.5e l2_vs_ref=%12.5e\n", cs.solver.c_str(), iters, wall, err);
    cudaFree(d_rhs);
    cudaFree(d_x);
    oc_helm_destroy(h);
    return 0;
}
