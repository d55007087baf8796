// Standalone pieces of the step behind their own entry points, the B200 side of
// the reference's standalone kernel benches:
//   - the variable-coefficient free-surface Helmholtz solver on given face
//     coefficients (reference libs/cuda/src/helmholtz_bench.cu, solving the
//     system that tools/write_helmholtz_case.py writes with
//     libs/core/solvers_var.py HelmholtzVar) -> oc_helm_create / oc_helm_solve;
//   - the three equations of state on flat arrays (reference
//     libs/cuda/src/eos_bench.cu over libs/core/eos.py) -> oc_density.
// The solver is the step's own persistent cooperative HelmSolver, so its
// iteration counts and solutions are those of the step's solves; solver kind
// OC_SOLVER_PCG_REFINED selects the mixed-precision RefinedHelm instead.

#include <cuda_runtime.h>

#include <string>

#include "helm_refined.cuh"
#include "helmholtz.cuh"
#include "ocean_b200.h"
#include "oc_internal.cuh"

struct oc_helm {
    oc::HelmSolver solver;
    oc::RefinedHelm* refined = nullptr;  // set for OC_SOLVER_PCG_REFINED
    double* ku = nullptr;
    double* kv = nullptr;
    double* rhs = nullptr;  // device staging for host right-hand sides
    double* x = nullptr;
    int* status = nullptr;
    int nx = 0, ny = 0, device = 0;
    std::string err;
    ~oc_helm() {
        delete refined;
        for (void* p : {(void*)ku, (void*)kv, (void*)rhs, (void*)x, (void*)status})
            if (p) cudaFree(p);
    }
};

namespace {

int helm_fail(oc_helm* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}

// rho' for linear and S-EOS (eos.py:103-127), full in-situ rho for polyTEOS10-bsq
// (eos.py:68-100): what the reference's EOS bench evaluates per cell
__global__ void k_density(int eos, double rho0, double alpha_t, double beta_s, double t0, double s0,
                          const double* __restrict__ T, const double* __restrict__ S,
                          const double* __restrict__ z, double* __restrict__ rho, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
        const double Tv = T[t], Sv = S[t], zv = z[t];
        rho[t] = eos == OC_EOS_TEOS10 ? oc::rho_teos10(Tv, Sv, zv)
                                      : oc::rho_anomaly_of(eos, rho0, alpha_t, beta_s, t0, s0, Tv, Sv, zv);
    }
}

}  // namespace

extern "C" int oc_helm_create(const oc_helm_config* cfg, const double* ku, const double* kv,
                              const double* mask, oc_helm** out) {
    if (!cfg || !ku || !kv || !mask || !out) return OC_ERR_ARG;
    *out = nullptr;
    if (cfg->nx < 2 || cfg->ny < 2 || !(cfg->dx > 0.0) || !(cfg->dy > 0.0) || !(cfg->coef >= 0.0) ||
        !(cfg->rtol > 0.0) || cfg->max_iter < 1 || cfg->solver < OC_SOLVER_PCG_JACOBI ||
        cfg->solver > OC_SOLVER_PCG_MG)
        return OC_ERR_ARG;
    if (cudaSetDevice(cfg->device) != cudaSuccess) return OC_ERR_CUDA;
    oc_helm* h = new oc_helm();
    h->nx = cfg->nx;
    h->ny = cfg->ny;
    h->device = cfg->device;
    const size_t n = (size_t)cfg->nx * cfg->ny, bytes = n * sizeof(double);
    for (double** p : {&h->ku, &h->kv, &h->rhs, &h->x})
        if (cudaMalloc(p, bytes) != cudaSuccess) {
            delete h;
            return OC_ERR_CUDA;
        }
    if (cudaMalloc(&h->status, sizeof(int)) != cudaSuccess) {
        delete h;
        return OC_ERR_CUDA;
    }
    cudaMemset(h->status, 0, sizeof(int));
    cudaMemcpy(h->ku, ku, bytes, cudaMemcpyHostToDevice);
    cudaMemcpy(h->kv, kv, bytes, cudaMemcpyHostToDevice);
    if (cfg->solver == OC_SOLVER_PCG_REFINED) {
        h->refined = new oc::RefinedHelm();
        const int rc = h->refined->init(cfg->nx, cfg->ny, cfg->dx, cfg->dy, cfg->coef, cfg->rtol, cfg->max_iter,
                                        mask, h->ku, h->kv, h->err);
        if (rc) {
            delete h;
            return rc;
        }
    } else {
        const int rc = h->solver.init(cfg->nx, cfg->ny, cfg->dx, cfg->dy, cfg->coef, cfg->solver, cfg->rtol,
                                      cfg->max_iter, mask, h->ku, h->kv, 1, h->status, h->err);
        if (rc) {
            delete h;
            return rc;
        }
        h->solver.rebuild(0);
    }
    if (cudaDeviceSynchronize() != cudaSuccess) {
        delete h;
        return OC_ERR_CUDA;
    }
    *out = h;
    return OC_OK;
}

extern "C" int oc_helm_solve(oc_helm* h, const double* rhs, double* x, int32_t on_device,
                             int32_t* iterations, int32_t* converged, void* stream) {
    if (!h || !rhs || !x) return OC_ERR_ARG;
    cudaSetDevice(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t bytes = (size_t)h->nx * h->ny * sizeof(double);
    const double* d_rhs = rhs;
    double* d_x = x;
    if (!on_device) {
        if (cudaMemcpyAsync(h->rhs, rhs, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
            return helm_fail(h, OC_ERR_CUDA, "right-hand side upload failed");
        d_rhs = h->rhs;
        d_x = h->x;
    }
    int rc;
    if (h->refined) {
        rc = h->refined->solve(d_rhs, d_x, s, h->err);
    } else {
        cudaMemsetAsync(h->solver.d_log_count(), 0, sizeof(int), s);
        rc = h->solver.solve(d_rhs, d_x, s, h->err);
    }
    if (rc) return rc;
    if (!on_device && cudaMemcpyAsync(x, h->x, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return helm_fail(h, OC_ERR_CUDA, "solution download failed");
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return helm_fail(h, OC_ERR_CUDA, cudaGetErrorString(e));
    if (h->refined) return h->refined->report(iterations, converged, nullptr, nullptr, h->err);
    int st = 0, it = 0, cv = 0;
    cudaMemcpy(&st, h->status, sizeof(int), cudaMemcpyDeviceToHost);
    if (st) return helm_fail(h, st, "a device-side wait ran out its bound");
    cudaMemcpy(&it, h->solver.d_log_iters(), sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(&cv, h->solver.d_log_conv(), sizeof(int), cudaMemcpyDeviceToHost);
    if (iterations) *iterations = it;
    if (converged) *converged = cv;
    return OC_OK;
}

extern "C" int oc_helm_refine_report(oc_helm* h, int32_t* refinement_steps, double* relative_residual) {
    if (!h) return OC_ERR_ARG;
    if (!h->refined) return helm_fail(h, OC_ERR_UNSUPPORTED, "not the refined solver");
    cudaSetDevice(h->device);
    int outer = 0;
    const int rc = h->refined->report(nullptr, nullptr, &outer, relative_residual, h->err);
    if (rc == OC_OK && refinement_steps) *refinement_steps = outer;
    return rc;
}

extern "C" int oc_helm_set_inner_rtol(oc_helm* h, double inner_rtol) {
    if (!h || !(inner_rtol > 0.0) || !(inner_rtol < 1.0)) return OC_ERR_ARG;
    if (!h->refined) return helm_fail(h, OC_ERR_UNSUPPORTED, "not the refined solver");
    h->refined->set_inner_rtol(inner_rtol);
    return OC_OK;
}

extern "C" const char* oc_helm_last_error(oc_helm* h) { return h ? h->err.c_str() : "null handle"; }

extern "C" int oc_helm_destroy(oc_helm* h) {
    if (!h) return OC_ERR_ARG;
    cudaSetDevice(h->device);
    delete h;
    return OC_OK;
}

extern "C" int oc_density(int32_t eos, double rho0, double alpha_t, double beta_s, double t0, double s0,
                          const double* T, const double* S, const double* z, double* rho, int64_t count,
                          void* stream) {
    if (!T || !S || !z || !rho || count < 0 || eos < OC_EOS_LINEAR || eos > OC_EOS_TEOS10) return OC_ERR_ARG;
    if (count == 0) return OC_OK;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int block = 256;
    const int64_t need = (count + block - 1) / block;
    const int64_t cap = (int64_t)(sms > 0 ? sms : 1) * 8;
    const int grid = (int)(need < cap ? need : cap);
    k_density<<<grid, block, 0, (cudaStream_t)stream>>>(eos, rho0, alpha_t, beta_s, t0, s0, T, S, z, rho,
                                                         count);
    return cudaGetLastError() == cudaSuccess ? OC_OK : OC_ERR_CUDA;
}
