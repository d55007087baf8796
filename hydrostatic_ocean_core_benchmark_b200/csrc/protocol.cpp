// The backend file protocol of the reference's compiled v0.5 binaries, as a
// library call (oc_run_namelist) over the C ABI.
//
//   <prefix>.nml + <prefix>_domain.bin + <prefix>_init.bin
//       -> <out_prefix>_state3d5.bin + <out_prefix>_metrics.json
//
// The namelist is read as the format the reference's bundle writer emits
// (tools/toml2nml.py:27-34, 188-268); missing keys take the defaults of the
// reference binary's RunConfig (libs/cuda/src/config.hpp:18-50) and V05Config
// (cfd_exp3d5_cuda.cu:72-86); the run loop, divergence guard, timing (median and
// MAD of wall time) and output layout follow cfd_exp3d5_cuda.cu:1104-1237.
// Options the step cannot run are refused with "FATAL: ..." and a non-zero
// status, never silently changed.

#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iterator>
#include <map>
#include <string>
#include <vector>

#include "ocean_b200.h"

namespace {

// A Fortran namelist file as the reference's v0.5 bundle writer emits it
// (tools/toml2nml.py:188-268): `&group` opens a group and `/` closes it; inside,
// `name = value` items are separated by newlines or commas; character values
// are quoted ('...' or "...", a doubled quote standing for itself); reals carry
// a Fortran exponent letter d/D (tools/toml2nml.py:27-34) or e/E; logicals are
// .true./.false. (or T/F); `!` outside quotes starts a comment. Names are
// case-insensitive. Values are kept as their raw text until asked for.
class Namelist {
  public:
    bool load(const std::string& path) {
        std::ifstream in(path, std::ios::binary);
        if (!in) return false;
        const std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
        scan(text);
        return true;
    }
    double num(const char* name, double dflt) const {
        const std::string* raw = find(name);
        double v;
        return (raw && fortran_real(*raw, v)) ? v : dflt;
    }
    std::string str(const char* name, const std::string& dflt) const {
        const std::string* raw = find(name);
        return raw ? *raw : dflt;
    }
    bool logical(const char* name, bool dflt) const {
        const std::string* raw = find(name);
        if (!raw || raw->empty()) return dflt;
        size_t p = (*raw)[0] == '.' ? 1 : 0;
        if (p >= raw->size()) return dflt;
        const char c = (char)std::tolower((unsigned char)(*raw)[p]);
        return c == 't' ? true : c == 'f' ? false : dflt;
    }

  private:
    std::map<std::string, std::string> items_;

    const std::string* find(const char* name) const {
        const auto it = items_.find(lower(name));
        return it == items_.end() ? nullptr : &it->second;
    }
    static std::string lower(std::string s) {
        for (char& c : s) c = (char)std::tolower((unsigned char)c);
        return s;
    }
    static bool name_char(char c) { return std::isalnum((unsigned char)c) || c == '_' || c == '%'; }

    // one pass over the characters: outside a group everything is ignored; in a
    // group, read a name, an '=' and one value (quoted or up to a separator)
    void scan(const std::string& t) {
        const size_t n = t.size();
        size_t i = 0;
        bool in_group = false;
        auto skip_comment = [&]() {
            while (i < n && t[i] != '\n') ++i;
        };
        while (i < n) {
            const char c = t[i];
            if (c == '!') {
                skip_comment();
                continue;
            }
            if (!in_group) {
                if (c == '&' || c == '$') {  // group name follows; the name itself is not needed
                    in_group = true;
                    ++i;
                    while (i < n && name_char(t[i])) ++i;
                } else {
                    ++i;
                }
                continue;
            }
            if (std::isspace((unsigned char)c) || c == ',') {
                ++i;
                continue;
            }
            if (c == '/' || c == '&' || c == '$') {  // end of the group (`/`, `&end`, `$end`)
                in_group = false;
                ++i;
                while (i < n && name_char(t[i])) ++i;
                continue;
            }
            // an item: name = value
            const size_t n0 = i;
            while (i < n && name_char(t[i])) ++i;
            std::string name = lower(t.substr(n0, i - n0));
            while (i < n && (t[i] == ' ' || t[i] == '\t')) ++i;
            if (name.empty() || i >= n || t[i] != '=') {  // not an item: drop the rest of the line
                skip_comment();
                continue;
            }
            ++i;
            while (i < n && (t[i] == ' ' || t[i] == '\t')) ++i;
            std::string value;
            if (i < n && (t[i] == '\'' || t[i] == '"')) {
                const char q = t[i++];
                while (i < n) {
                    if (t[i] == q) {
                        if (i + 1 < n && t[i + 1] == q) {  // doubled quote
                            value += q;
                            i += 2;
                            continue;
                        }
                        ++i;
                        break;
                    }
                    value += t[i++];
                }
            } else {
                const size_t v0 = i;
                while (i < n && !std::isspace((unsigned char)t[i]) && t[i] != ',' && t[i] != '/' && t[i] != '!') ++i;
                value = t.substr(v0, i - v0);
            }
            items_[name] = value;
        }
    }

    // a Fortran real or integer literal: the exponent letter d/D/q/Q after the
    // mantissa is read as e; anything left unparsed makes the literal invalid
    static bool fortran_real(const std::string& raw, double& out) {
        std::string s;
        s.reserve(raw.size());
        bool mantissa = false;
        for (char c : raw) {
            if (mantissa && (c == 'd' || c == 'D' || c == 'q' || c == 'Q')) c = 'e';
            if (std::isdigit((unsigned char)c) || c == '.') mantissa = true;
            s += c;
        }
        if (s.empty()) return false;
        char* end = nullptr;
        out = std::strtod(s.c_str(), &end);
        return end && *end == '\0';
    }
};

int fatal(const std::string& msg) {
    std::fprintf(stderr, "FATAL: %s\n", msg.c_str());
    return 1;
}

bool read_doubles(FILE* f, std::vector<double>& dst, size_t n) {
    dst.resize(n);
    return std::fread(dst.data(), sizeof(double), n, f) == n;
}

double median_of(std::vector<double> x) {
    if (x.empty()) return 0.0;
    std::sort(x.begin(), x.end());
    const size_t n = x.size();
    return n % 2 ? x[n / 2] : 0.5 * (x[n / 2 - 1] + x[n / 2]);
}

std::string jnum(double x) {
    if (!std::isfinite(x)) return "null";
    char b[64];
    std::snprintf(b, sizeof b, "%.16e", x);
    return b;
}

int pick(const std::string& v, std::initializer_list<const char*> names, int& out) {
    int i = 0;
    for (const char* n : names) {
        if (v == n) {
            out = i;
            return 0;
        }
        ++i;
    }
    return 1;
}

}  // namespace

extern "C" int oc_run_namelist(const char* nml_path) {
    if (!nml_path) return fatal("usage: ocean3d5_b200 <namelist>");
    Namelist n;
    if (!n.load(nml_path)) return fatal(std::string("cannot open namelist ") + nml_path);
    oc_config c{};
    c.nx = (int)n.num("nx", 100);
    c.ny = (int)n.num("ny", 100);
    c.nz = (int)n.num("nz", 1);
    c.lx = n.num("lx", 1.0e7);
    c.ly = n.num("ly", 1.0e7);
    c.g = n.num("g", 9.80616);
    c.f0 = n.num("f0", 1.0e-4);
    c.h0 = n.num("h0", 1000.0);
    c.n2 = n.num("n2", 0.0);
    c.nu = n.num("nu", 0.0);
    c.kappa = n.num("kappa", 0.0);
    c.rho0 = n.num("rho0", 1025.0);
    c.tau_x = n.num("tau_x", 0.0);
    c.tau_y = n.num("tau_y", 0.0);
    c.bottom_drag = n.num("bottom_drag", 0.0);
    const std::string scheme = n.str("scheme_name", "theta");
    if (pick(scheme, {"fb", "theta", "split_explicit"}, c.scheme))
        return fatal("unknown scheme " + scheme + " (expected fb|theta|split_explicit)");
    c.theta = n.num("theta", 0.5);
    c.theta_cor = n.num("theta_cor", 0.5);
    c.theta_v = n.num("theta_v", 0.5);
    c.n_picard = (int)n.num("n_picard", 2);
    c.n_split = (int)n.num("n_split", 0);
    if (pick(n.str("barotropic_average", "none"), {"none", "mean"}, c.barotropic_average))
        return fatal("barotropic_average must be none|mean");
    const std::string solver = n.str("solver_kind", "pcg_jacobi");
    if (c.scheme == OC_SCHEME_THETA && pick(solver, {"pcg_jacobi", "pcg_rbgs", "rbgs", "multigrid"}, c.solver))
        return fatal("unknown variable-coefficient solver " + solver);
    c.rtol = n.num("rtol", 1.0e-12);
    c.max_iter = (int)n.num("max_iter", 2000);
    c.dt = n.num("dt", 0.0);
    const int n_steps = (int)n.num("n_steps", 0);
    const int n_repeat = (int)n.num("n_repeat", 5);
    const int n_warmup = (int)n.num("n_warmup", 1);
    if (c.scheme == OC_SCHEME_THETA && !(c.theta > 0.0 && c.theta <= 1.0))
        return fatal("theta must lie in (0,1]");
    if (c.n_picard < 1 || n_steps < 1 || c.dt <= 0.0)
        return fatal("dt, n_steps and n_picard must come from the driver");
    const std::string out_prefix = n.str("out_prefix", "output/cuda_run");
    if (n.str("vcoord", "zlevel") != "zlevel") return fatal("vcoord=zlevel only");
    if (pick(n.str("bc_x", "periodic"), {"periodic", "closed"}, c.bc_x) ||
        pick(n.str("bc_y", "periodic"), {"periodic", "closed"}, c.bc_y))
        return fatal("periodic|closed boundaries only");
    if (pick(n.str("face_rule", "min"), {"min", "mean", "harmonic"}, c.face_rule))
        return fatal("face_rule must be min|mean|harmonic");
    c.min_partial = n.num("min_partial", 0.1);
    const std::string eos = n.str("eos", "linear");
    if (pick(eos, {"linear", "seos", "teos10"}, c.eos)) return fatal("eos must be linear|seos|teos10");
    if (pick(n.str("pgf", "remove"), {"remove", "keep"}, c.pgf)) return fatal("pgf must be remove|keep");
    c.pgf_correction = n.logical("pgf_correction", true) ? 1 : 0;
    const std::string adv = n.str("advection", "none");
    if (pick(adv, {"none", "centered2", "upwind1", "up3", "up3_tvd"}, c.advection))
        return fatal("unknown advection " + adv);
    const std::string tracers = n.str("tracers", "buoyancy");
    if (pick(tracers, {"buoyancy", "TS"}, c.tracers)) return fatal("tracers must be buoyancy|TS");
    c.alpha_t = n.num("alpha_t", 2.0e-4);
    c.beta_s = n.num("beta_s", 7.4e-4);
    c.t0 = n.num("t0", 10.0);
    c.s0 = n.num("s0", 35.0);
    c.cp = n.num("cp", 3990.0);
    c.a_h = n.num("a_h", 0.0);
    c.k_h = n.num("k_h", 0.0);
    c.q_heat = n.num("q_heat", 0.0);
    c.q_salt = n.num("q_salt", 0.0);
    if (pick(n.str("closure", "none"), {"none", "tke"}, c.closure)) return fatal("closure must be none|tke");
    if (pick(n.str("mxl", "integral"), {"integral", "recursive"}, c.mxl))
        return fatal("mxl must be integral|recursive");
    c.c_k = n.num("c_k", 0.1);
    c.c_eps = n.num("c_eps", 0.7);
    c.pr_t = n.num("pr_t", 1.0);
    c.z_0 = n.num("z_0", 0.1);
    c.e_min = n.num("e_min", 1.0e-6);
    c.l_min = n.num("l_min", 0.01);
    c.e_bb = n.num("e_bb", 3.75);
    c.n2_min = n.num("n2_min", 1.0e-8);
    c.device = 0;
    const bool ts = c.tracers == OC_TRACERS_TS;
    const size_t n2 = (size_t)c.nx * c.ny, n3 = n2 * c.nz;

    // bundle files
    std::vector<double> H, mask, e0, u0, v0, b0, T0, S0, dzr, tx, ty;
    {
        const std::string df = n.str("domain_file", "");
        FILE* f = std::fopen(df.c_str(), "rb");
        if (!f) return fatal("cannot read " + df);
        const bool ok = read_doubles(f, H, n2) && read_doubles(f, mask, n2);
        std::fclose(f);
        if (!ok) return fatal(df + " is shorter than 2*nx*ny doubles");
    }
    {
        const std::string inf = n.str("init_file", "");
        FILE* f = std::fopen(inf.c_str(), "rb");
        if (!f) return fatal("cannot read " + inf);
        bool ok = read_doubles(f, e0, n2) && read_doubles(f, u0, n3) && read_doubles(f, v0, n3) &&
                  read_doubles(f, b0, n3);
        if (ok && ts) ok = read_doubles(f, T0, n3) && read_doubles(f, S0, n3);
        std::fclose(f);
        if (!ok) return fatal(inf + " is shorter than the state it must hold");
    }
    const std::string lf = n.str("levels_file", "");
    if (!lf.empty()) {
        FILE* f = std::fopen(lf.c_str(), "rb");
        if (!f) return fatal("cannot read " + lf);
        const bool ok = read_doubles(f, dzr, (size_t)c.nz);
        std::fclose(f);
        if (!ok) return fatal(lf + " is shorter than nz doubles");
    }
    const std::string ff = n.str("forcing_file", "");
    if (!ff.empty()) {
        FILE* f = std::fopen(ff.c_str(), "rb");
        if (!f) return fatal("cannot read " + ff);
        const bool ok = read_doubles(f, tx, n2) && read_doubles(f, ty, n2);
        std::fclose(f);
        if (!ok) return fatal(ff + " is shorter than 2*nx*ny doubles");
    }

    oc_handle* h = nullptr;
    int rc = oc_create(&c, &h);
    if (rc) return fatal("invalid configuration");
    rc = oc_set_domain(h, H.data(), mask.data(), dzr.empty() ? nullptr : dzr.data());
    if (!rc && !tx.empty()) rc = oc_set_forcing(h, tx.data(), ty.data());
    if (rc) {
        const int r = fatal(oc_last_error(h));
        oc_destroy(h);
        return r;
    }
    oc_state_view init{};
    init.eta = e0.data();
    init.u = u0.data();
    init.v = v0.data();
    init.b = b0.data();
    init.T = ts ? T0.data() : nullptr;
    init.S = ts ? S0.data() : nullptr;
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, 0);
    auto diverged = [&]() -> bool {
        oc_stats st{};
        oc_get_stats(h, &st);
        return st.diverged != 0;
    };
    std::printf("ocean3d5_b200: case=%s nx=%d ny=%d nz=%d scheme=%s solver=%s eos=%s dt=%12.5E steps=%d gpu=%s\n",
                n.str("case_name", "").c_str(), c.nx, c.ny, c.nz, scheme.c_str(), solver.c_str(), eos.c_str(),
                c.dt, n_steps, prop.name);
    bool run_diverged = false;
    for (int rep = 0; rep < n_warmup && !run_diverged; ++rep) {
        if ((rc = oc_reset_mixing(h)) || (rc = oc_set_state(h, &init, 0))) break;
        for (int s = 0; s < n_steps;) {
            // chunks of up to ten steps, replayed as CUDA graphs, ending where the
            // reference checks for divergence (every tenth step)
            const int chunk = std::min(10 - s % 10, n_steps - s);
            if ((rc = oc_step_graph(h, chunk, nullptr))) break;
            s += chunk;
            if (s % 10 == 0 && diverged()) {
                run_diverged = true;
                break;
            }
        }
        if (rc) break;
    }
    std::vector<double> samples;
    long long iters_total = 0, failures = 0, tridiag = 0, rebuilds = 0, subs_total = 0;
    int n_split = 0;
    long long device_bytes = 0;
    for (int rep = 0; rep < n_repeat && !rc; ++rep) {
        if ((rc = oc_reset_mixing(h)) || (rc = oc_set_state(h, &init, 0))) break;
        oc_reset_stats(h);
        cudaDeviceSynchronize();
        const auto t0 = std::chrono::steady_clock::now();
        for (int s = 0; s < n_steps;) {
            // chunks of up to ten steps, replayed as CUDA graphs, ending where the
            // reference checks for divergence (every tenth step)
            const int chunk = std::min(10 - s % 10, n_steps - s);
            if ((rc = oc_step_graph(h, chunk, nullptr))) break;
            s += chunk;
            if (s % 10 == 0 && diverged()) {
                run_diverged = true;
                break;
            }
        }
        cudaDeviceSynchronize();
        const auto t1 = std::chrono::steady_clock::now();
        if (rc) break;
        samples.push_back(std::chrono::duration<double>(t1 - t0).count());
        oc_stats st{};
        rc = oc_get_stats(h, &st);
        iters_total += st.solver_iterations;
        failures += st.solver_failures;
        tridiag += st.tridiagonal_solves;
        rebuilds += st.solver_rebuilds;
        subs_total += st.barotropic_substeps;
        n_split = st.n_split;
        device_bytes = st.device_bytes;
        if (run_diverged) {
            std::printf("  DIVERGED (|eta| > 1e6 or NaN) - run stopped early\n");
            break;
        }
    }
    if (rc) {
        const int r = fatal(oc_last_error(h));
        oc_destroy(h);
        return r;
    }
    const int n_done = (int)samples.size();
    const long long iters = iters_total / std::max(1, n_done);
    const long long subs = subs_total / std::max(1, n_done);
    const double t_med = median_of(samples);
    std::vector<double> dev;
    for (double x : samples) dev.push_back(std::fabs(x - t_med));
    const double t_mad = median_of(dev);
    std::printf("  wall median=%12.5E s  mad=%12.5E s  solver_iters/run=%lld  substeps/run=%lld\n", t_med, t_mad,
                iters, subs);
    std::vector<double> hu(n3), hv(n3), hb(n3), hT(ts ? n3 : 0), hS(ts ? n3 : 0), he(n2);
    oc_state_view out{};
    out.eta = he.data();
    out.u = hu.data();
    out.v = hv.data();
    out.b = hb.data();
    out.T = ts ? hT.data() : nullptr;
    out.S = ts ? hS.data() : nullptr;
    if ((rc = oc_get_state(h, &out, 0))) {
        const int r = fatal(oc_last_error(h));
        oc_destroy(h);
        return r;
    }
    oc_destroy(h);
    const std::string bin = out_prefix + "_state3d5.bin";
    if (FILE* f = std::fopen(bin.c_str(), "wb")) {
        std::fwrite(he.data(), sizeof(double), n2, f);
        std::fwrite(hu.data(), sizeof(double), n3, f);
        std::fwrite(hv.data(), sizeof(double), n3, f);
        std::fwrite(hb.data(), sizeof(double), n3, f);
        if (ts) {
            std::fwrite(hT.data(), sizeof(double), n3, f);
            std::fwrite(hS.data(), sizeof(double), n3, f);
        }
        std::fclose(f);
    } else {
        return fatal("cannot write " + bin);
    }
    const std::string mj = out_prefix + "_metrics.json";
    if (FILE* f = std::fopen(mj.c_str(), "w")) {
        const double cells = (double)n3;
        std::fprintf(f,
                     "{\n  \"backend\": \"ocean3d5_b200\",\n  \"gpu\": \"%s\",\n  \"nx\": %d,\n  \"ny\": %d,\n"
                     "  \"nz\": %d,\n  \"cells\": %lld,\n  \"n_steps\": %d,\n  \"scheme\": \"%s\",\n"
                     "  \"solver\": \"%s\",\n  \"eos\": \"%s\",\n  \"advection\": \"%s\",\n  \"tracers\": \"%s\",\n"
                     "  \"theta\": %s,\n  \"dt\": %s,\n  \"solver_iterations\": %lld,\n  \"solver_failures\": %lld,\n"
                     "  \"tridiagonal_solves\": %lld,\n  \"solver_rebuilds\": %lld,\n  \"n_split\": %d,\n"
                     "  \"barotropic_substeps\": %lld,\n  \"device_bytes\": %lld,\n  \"bytes_per_cell\": %s,\n"
                     "  \"diverged\": %s,\n  \"wall_s\": %s,\n  \"wall_mad_s\": %s,\n  \"n_repeat\": %d,\n"
                     "  \"omp_num_threads\": 0,\n  \"cell_steps_per_s\": %s\n}\n",
                     prop.name, c.nx, c.ny, c.nz, (long long)n3, n_steps, scheme.c_str(), solver.c_str(), eos.c_str(),
                     adv.c_str(), tracers.c_str(), jnum(c.theta).c_str(), jnum(c.dt).c_str(), iters, failures, tridiag,
                     rebuilds, n_split, subs, device_bytes, jnum(device_bytes / cells).c_str(),
                     run_diverged ? "true" : "false", jnum(t_med).c_str(), jnum(t_mad).c_str(), n_done,
                     jnum(t_med > 0 ? cells * n_steps / t_med : 0.0).c_str());
        std::fclose(f);
    } else {
        return fatal("cannot write " + mj);
    }
    return 0;
}
