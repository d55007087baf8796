// Mixed-precision Helmholtz solver: FP32 inner PCG-Jacobi inside FP64 iterative
// refinement, for the operator A = I - c D[K G[.]] of helmholtz.cuh.
#pragma once

#include <string>
#include <vector>

#include "oc_internal.cuh"

namespace oc {

struct RefineParams {
    int nx, ny, n;
    int max_iter;   // bound on the inner iterations summed over the refinement
    int max_outer;  // bound on the refinement steps
    double coef, dx2, dy2;
    double rtol;        // stop when |b - A x|_2 <= rtol |b|_2, evaluated in FP64
    double inner_rtol;  // an inner solve stops when its residual is inner_rtol times its start
    // FP64 system: face coefficients, mask, right-hand side, solution
    const double *ku, *kv, *mask, *rhs;
    double* x;
    // FP32 operator: ax = c Ku / dx^2, ay = c Kv / dy^2, the diagonal, its inverse
    // (1 on dry cells) and the wet flag
    const float *ax, *ay, *diag, *dinv;
    const unsigned char* wet;
    // FP32 inner work vectors; the search directions of consecutive iterations
    // alternate between p and p2
    float *p, *p2, *Ap, *rr, *z, *d;
    double* part;  // per-CTA partial sums: two slots of two values, 4 * gridDim.x
    unsigned long long* bar_count;
    int* status;
    long long wait_cycles;  // bound of a barrier wait in SM clock cycles
    int* report;     // inner iterations, converged, refinement steps
    double* relres;  // |b - A x|_2 / |b|_2 at exit
    // optional per-solve log (the step's): inner iterations (-1 when a barrier
    // gave up) and converged flag appended at log_count, if below log_cap
    int* log_iters;
    int* log_conv;
    int* log_count;
    int log_cap;
};

class RefinedHelm {
   public:
    ~RefinedHelm();
    // ku, kv device arrays owned by the caller (kept for the FP64 residual), mask a host array;
    // status: a status word of the caller's (the step's), or null for one of its own
    int init(int nx, int ny, double dx, double dy, double coef, double rtol, int max_iter,
             const double* mask_host, const double* ku, const double* kv, std::string& err,
             int* status = nullptr);
    // the FP32 operator again from ku, kv (after the caller changed them), on stream s
    void rebuild(cudaStream_t s);
    // append every solve's inner iterations and converged flag to these device arrays
    void set_log(int* iters, int* conv, int* count, int cap) {
        rp_.log_iters = iters;
        rp_.log_conv = conv;
        rp_.log_count = count;
        rp_.log_cap = cap;
    }
    void set_wait_cycles(long long cycles) { rp_.wait_cycles = cycles; }
    // x = A^-1 rhs on the device; the report is read back by report()
    int solve(const double* rhs, double* x, cudaStream_t s, std::string& err);
    // after a synchronised solve: inner iterations, converged, refinement steps, relative residual
    int report(int* iterations, int* converged, int* outer, double* relres, std::string& err);
    void set_inner_rtol(double r) { rp_.inner_rtol = r; }
    size_t bytes() const { return bytes_; }

   private:
    RefineParams rp_{};
    std::vector<void*> allocs_;
    double cx_ = 0.0, cy_ = 0.0;  // coef / dx^2, coef / dy^2 of the FP32 operator
    int grid_ = 0;
    size_t bytes_ = 0;
    void* dalloc(size_t nbytes);
};

}  // namespace oc
