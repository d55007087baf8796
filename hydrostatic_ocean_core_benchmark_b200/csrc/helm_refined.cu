// Mixed-precision solve of the free-surface Helmholtz system A x = b,
// A = I - c D[K G[.]] (the operator of libs/core/solvers_var.py:22-60).
//
// There is no such solver in the reference. Its FP64 solvers are the parity
// path (helmholtz.cu); this one stores the Krylov vectors and the operator in
// FP32 and keeps FP64 where the answer's accuracy is decided, following
// classical mixed-precision iterative refinement (Wilkinson; Moler 1967; for
// Krylov inner solvers Carson and Higham, SIAM J. Sci. Comput. 40 (2018)):
//
//   x = 0, r = b                                   FP64
//   while |r|_2 > rtol |b|_2:                      FP64 norm
//       solve A d = r by PCG-Jacobi from d = 0     FP32 vectors and operator,
//           to |r - A d| <= inner_rtol |r|         dot products summed in FP64
//       x += d                                     FP64 correction
//       r = b - A x                                FP64 operator
//
// A product of two FP32 numbers is exact in FP64, so every dot product is an
// FP64 sum of exact terms, added in a fixed order (per thread, per warp, per
// CTA, then over the CTAs' partial sums in CTA order), and every CTA forms the
// same global sums and takes the same branches. The whole solve is one
// persistent cooperative launch over the bounded grid barrier of
// grid_barrier.cuh: a barrier that waits past its bound sets OC_ERR_TIMEOUT
// and every CTA leaves. Data written by another CTA in the same launch (the
// search directions, z, the iterate, the partial sums) is read through L2 (ld.cg).
//
// An inner iteration takes two barriers: the pass that forms A p also forms
// the new direction p = z + beta p_old, each thread at its own cell and,
// redundantly, at the four neighbours it needs, from z and the previous
// direction, which lives in the other of two buffers.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "grid_barrier.cuh"
#include "helm_refined.cuh"
#include "ocean_b200.h"

namespace oc {

static constexpr int RT = 512;          // threads per CTA
static constexpr int RW = RT / 32;      // warps per CTA
static constexpr int kMaxOuter = 64;    // refinement steps
static constexpr double kInnerRtol = 1e-3;

struct Nb {
    int ie, iw, jn, js;  // periodic neighbour indices, as the reference's np.roll
};

__device__ __forceinline__ Nb neighbours(int e, int nx, int ny) {
    const int j = e / nx, i = e - j * nx;
    Nb b;
    b.ie = i + 1 == nx ? e - i : e + 1;
    b.iw = i == 0 ? e + nx - 1 : e - 1;
    b.jn = j + 1 == ny ? i : e + nx;
    b.js = j == 0 ? e + (ny - 1) * nx : e - nx;
    return b;
}

// (a, b) summed over the CTA in a fixed order; every thread gets the totals
__device__ __forceinline__ double2 cta_sum2(double a, double b, double* sm) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sm[w] = a;
        sm[RW + w] = b;
    }
    __syncthreads();
    if (w == 0) {
        a = l < RW ? sm[l] : 0.0;
        b = l < RW ? sm[RW + l] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if (l == 0) {
            sm[2 * RW] = a;
            sm[2 * RW + 1] = b;
        }
    }
    __syncthreads();
    const double2 t = make_double2(sm[2 * RW], sm[2 * RW + 1]);
    __syncthreads();
    return t;
}

// this CTA's partial sums into slot `slot` (0 or 1) of the partial-sum array
__device__ __forceinline__ void publish(const RefineParams& R, int slot, double a, double b, double* sm) {
    const double2 t = cta_sum2(a, b, sm);
    if (threadIdx.x == 0) {
        double* part = R.part + 2 * slot * gridDim.x;
        part[blockIdx.x] = t.x;
        part[gridDim.x + blockIdx.x] = t.y;
    }
}

// the global sums of a slot, after the barrier that follows every CTA's publish
__device__ __forceinline__ double2 gather(const RefineParams& R, int slot, double* sm) {
    const double* part = R.part + 2 * slot * gridDim.x;
    double a = 0.0, b = 0.0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += RT) {
        a += __ldcg(part + k);
        b += __ldcg(part + gridDim.x + k);
    }
    return cta_sum2(a, b, sm);
}

// the search direction at cell k: z for the first iteration of an inner solve,
// else z + beta p_old
__device__ __forceinline__ float direction(const RefineParams& R, const float* pold, float beta, bool fresh, int k) {
    const float zk = __ldcg(R.z + k);
    return fresh ? zk : zk + beta * __ldcg(pold + k);
}

// FP32 operator on the search direction: diag p - (neighbour couplings); dry
// cells are the identity, as in the FP64 operator. Returns A p, with p at e in pc.
// The wet test selects after the arithmetic, so no load waits for the flag.
__device__ __forceinline__ float apply32(const RefineParams& R, const float* pold, float beta, bool fresh, int e,
                                         const Nb& b, float& pc) {
    pc = direction(R, pold, beta, fresh, e);
    const float off = R.ax[e] * direction(R, pold, beta, fresh, b.ie) +
                      R.ax[b.iw] * direction(R, pold, beta, fresh, b.iw) +
                      R.ay[e] * direction(R, pold, beta, fresh, b.jn) +
                      R.ay[b.js] * direction(R, pold, beta, fresh, b.js);
    const float full = R.diag[e] * pc - off;
    return R.wet[e] ? full : pc;
}

// FP64 operator on the iterate, term by term as HelmOp.apply: the masked
// iterate, face fluxes K (x_nb - x), their divergence over dx^2 and dy^2, and
// the masked iterate again on dry cells (solvers_var.py:47-53)
__device__ __forceinline__ double apply64(const RefineParams& R, int e, const Nb& b) {
    const double m = R.mask[e];
    const double xc = __ldcg(R.x + e) * m;
    const double xe = __ldcg(R.x + b.ie) * R.mask[b.ie], xw = __ldcg(R.x + b.iw) * R.mask[b.iw];
    const double xn = __ldcg(R.x + b.jn) * R.mask[b.jn], xs = __ldcg(R.x + b.js) * R.mask[b.js];
    const double fe = R.ku[e] * (xe - xc), fw = R.ku[b.iw] * (xc - xw);
    const double fn = R.kv[e] * (xn - xc), fs = R.kv[b.js] * (xc - xs);
    const double lap = (fe - fw) / R.dx2 + (fn - fs) / R.dy2;
    return (xc - R.coef * lap) * m + xc * (1.0 - m);
}

// a new residual r (FP64) starts an inner solve: rr = r in FP32, z = D^-1 rr,
// d = 0 (its first direction is z); returns the terms of |r|^2 and rr.z
__device__ __forceinline__ void start_inner(const RefineParams& R, int e, double r, double& r2, double& rz) {
    const float r32 = (float)r;
    const float z32 = R.dinv[e] * r32;
    R.rr[e] = r32;
    R.z[e] = z32;
    R.d[e] = 0.0f;
    r2 += r * r;
    rz += (double)r32 * (double)z32;
}

__global__ void __launch_bounds__(RT, 1) k_helm_refined(RefineParams R) {
    __shared__ double sm[2 * RW + 2];
    grid_sync_begin(R.status);
    const int n = R.n, nx = R.nx, ny = R.ny;
    const int first = blockIdx.x * RT + threadIdx.x, stride = gridDim.x * RT;

    // b = rhs * mask, x = 0, r = b
    double r2 = 0.0, rz0 = 0.0;
    for (int e = first; e < n; e += stride) {
        R.x[e] = 0.0;
        start_inner(R, e, R.rhs[e] * R.mask[e], r2, rz0);
    }
    publish(R, 1, r2, rz0, sm);
    bool ok = grid_sync(R.bar_count, R.status, gridDim.x, R.wait_cycles);
    double2 s = gather(R, 1, sm);
    const double norm_b = sqrt(s.x), tol = R.rtol * norm_b;
    double res = norm_b, rz = s.y;
    int inner = 0, outer = 0;
    bool conv = false;

    while (ok) {
        if (res <= tol) {
            conv = true;
            break;
        }
        if (inner >= R.max_iter || outer >= R.max_outer) break;
        ++outer;
        const double inner_tol = R.inner_rtol * res;
        bool fresh = true;
        float beta = 0.0f;
        float *pold = R.p2, *pnew = R.p;
        for (;;) {
            // p = z + beta p_old, Ap = A p and p.Ap; two cells (e, e + stride) per
            // turn, their loads ahead of their stores, added in the order of the cells
            double pap = 0.0;
            for (int e = first; e < n; e += 2 * stride) {
                const int e2 = e + stride;
                const bool two = e2 < n;
                float pc, pc2 = 0.0f, ap2 = 0.0f;
                const float ap = apply32(R, pold, beta, fresh, e, neighbours(e, nx, ny), pc);
                if (two) ap2 = apply32(R, pold, beta, fresh, e2, neighbours(e2, nx, ny), pc2);
                pnew[e] = pc;
                R.Ap[e] = ap;
                pap += (double)pc * (double)ap;
                if (two) {
                    pnew[e2] = pc2;
                    R.Ap[e2] = ap2;
                    pap += (double)pc2 * (double)ap2;
                }
            }
            publish(R, 0, pap, 0.0, sm);
            ok = grid_sync(R.bar_count, R.status, gridDim.x, R.wait_cycles);
            if (!ok) break;
            s = gather(R, 0, sm);
            if (!(s.x > 0.0)) break;  // p = 0: the FP32 residual vanished
            const float alpha = (float)(rz / s.x);
            // d += alpha p, rr -= alpha Ap, z = D^-1 rr, with |rr|^2 and rr.z; two
            // cells per turn as above
            double rr2 = 0.0, rzn = 0.0;
            for (int e = first; e < n; e += 2 * stride) {
                const int e2 = e + stride;
                const bool two = e2 < n;
                const float d1 = R.d[e] + alpha * pnew[e];
                const float r1 = R.rr[e] - alpha * R.Ap[e];
                const float z1 = R.dinv[e] * r1;
                float d2 = 0.0f, r2v = 0.0f, z2 = 0.0f;
                if (two) {
                    d2 = R.d[e2] + alpha * pnew[e2];
                    r2v = R.rr[e2] - alpha * R.Ap[e2];
                    z2 = R.dinv[e2] * r2v;
                }
                R.d[e] = d1;
                R.rr[e] = r1;
                R.z[e] = z1;
                rr2 += (double)r1 * (double)r1;
                rzn += (double)r1 * (double)z1;
                if (two) {
                    R.d[e2] = d2;
                    R.rr[e2] = r2v;
                    R.z[e2] = z2;
                    rr2 += (double)r2v * (double)r2v;
                    rzn += (double)r2v * (double)z2;
                }
            }
            publish(R, 1, rr2, rzn, sm);
            ok = grid_sync(R.bar_count, R.status, gridDim.x, R.wait_cycles);
            if (!ok) break;
            s = gather(R, 1, sm);
            ++inner;
            if (sqrt(s.x) <= inner_tol || inner >= R.max_iter) break;
            beta = (float)(s.y / rz);
            rz = s.y;
            fresh = false;
            float* t = pold;
            pold = pnew;
            pnew = t;
        }
        if (!ok) break;
        // the correction, in FP64
        for (int e = first; e < n; e += stride) R.x[e] += (double)R.d[e];
        ok = grid_sync(R.bar_count, R.status, gridDim.x, R.wait_cycles);
        if (!ok) break;
        // r = b - A x in FP64 starts the next inner solve
        r2 = 0.0;
        rz0 = 0.0;
        for (int e = first; e < n; e += stride)
            start_inner(R, e, R.rhs[e] * R.mask[e] - apply64(R, e, neighbours(e, nx, ny)), r2, rz0);
        publish(R, 1, r2, rz0, sm);
        ok = grid_sync(R.bar_count, R.status, gridDim.x, R.wait_cycles);
        if (!ok) break;
        s = gather(R, 1, sm);
        res = sqrt(s.x);
        rz = s.y;
    }
    grid_sync_end(R.bar_count, blockIdx.x == 0);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        R.report[0] = inner;
        R.report[1] = conv ? 1 : 0;
        R.report[2] = outer;
        *R.relres = norm_b > 0.0 ? res / norm_b : 0.0;
        if (R.log_count) {
            const int idx = *R.log_count;
            if (idx < R.log_cap) {
                R.log_iters[idx] = ok ? inner : -1;
                R.log_conv[idx] = (ok && conv) ? 1 : 0;
            }
            *R.log_count = idx + 1;
        }
    }
}

// FP32 operator of the fine grid from the FP64 coefficients, with the diagonal
// and its inverse as HelmOp builds them (solvers_var.py:30-36)
__global__ void k_refine_setup(RefineParams R, double cx, double cy, float* ax, float* ay, float* diag,
                               float* dinv, unsigned char* wet) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= R.n) return;
    const Nb b = neighbours(e, R.nx, R.ny);
    const double d = 1.0 + cx * (R.ku[e] + R.ku[b.iw]) + cy * (R.kv[e] + R.kv[b.js]);
    const bool w = R.mask[e] > 0.0;
    ax[e] = (float)(cx * R.ku[e]);
    ay[e] = (float)(cy * R.kv[e]);
    diag[e] = (float)d;
    dinv[e] = w ? (float)(1.0 / d) : 1.0f;
    wet[e] = w ? 1 : 0;
}

// ------------------------------------------------------------------ host side
RefinedHelm::~RefinedHelm() {
    for (void* p : allocs_) cudaFree(p);
}

void* RefinedHelm::dalloc(size_t nbytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, nbytes) != cudaSuccess) return nullptr;
    allocs_.push_back(p);
    bytes_ += nbytes;
    return p;
}

int RefinedHelm::init(int nx, int ny, double dx, double dy, double coef, double rtol, int max_iter,
                      const double* mask_host, const double* ku, const double* kv, std::string& err,
                      int* status) {
    if (nx < 2 || ny < 2 || (long long)nx * ny > (1LL << 30) || !(dx > 0.0) || !(dy > 0.0) || !(coef >= 0.0) ||
        !(rtol > 0.0) || max_iter < 1 || !mask_host || !ku || !kv) {
        err = "invalid refined-solver configuration";
        return OC_ERR_ARG;
    }
    const int n = nx * ny;
    int dev = 0, sms = 0, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_helm_refined, RT, 0) != cudaSuccess || occ < 1 ||
        sms < 1) {
        err = "refined solver kernel does not fit on an SM";
        return OC_ERR_CUDA;
    }
    // one CTA per SM at most, and no CTA without cells
    grid_ = std::max(1, std::min(sms, (n + RT - 1) / RT));
    RefineParams& R = rp_;
    R.nx = nx;
    R.ny = ny;
    R.n = n;
    R.max_iter = max_iter;
    R.max_outer = kMaxOuter;
    R.coef = coef;
    R.dx2 = dx * dx;
    R.dy2 = dy * dy;
    R.rtol = rtol;
    R.inner_rtol = kInnerRtol;
    R.ku = ku;
    R.kv = kv;
    const size_t n8 = (size_t)n * sizeof(double), n4 = (size_t)n * sizeof(float);
    double* mask = (double*)dalloc(n8);
    float* ax = (float*)dalloc(n4);
    float* ay = (float*)dalloc(n4);
    float* diag = (float*)dalloc(n4);
    float* dinv = (float*)dalloc(n4);
    unsigned char* wet = (unsigned char*)dalloc((size_t)n);
    R.p = (float*)dalloc(n4);
    R.p2 = (float*)dalloc(n4);
    R.Ap = (float*)dalloc(n4);
    R.rr = (float*)dalloc(n4);
    R.z = (float*)dalloc(n4);
    R.d = (float*)dalloc(n4);
    R.part = (double*)dalloc(4 * (size_t)grid_ * sizeof(double));
    R.bar_count = (unsigned long long*)dalloc(sizeof(unsigned long long));
    R.status = status ? status : (int*)dalloc(sizeof(int));
    R.wait_cycles = kBarrierCycles;
    R.report = (int*)dalloc(3 * sizeof(int));
    R.relres = (double*)dalloc(sizeof(double));
    if (!mask || !ax || !ay || !diag || !dinv || !wet || !R.p || !R.p2 || !R.Ap || !R.rr || !R.z || !R.d || !R.part ||
        !R.bar_count || !R.status || !R.report || !R.relres) {
        err = "refined solver: device allocation failed";
        return OC_ERR_CUDA;
    }
    cudaMemcpy(mask, mask_host, n8, cudaMemcpyHostToDevice);
    cudaMemset(R.bar_count, 0, sizeof(unsigned long long));
    if (!status) cudaMemset(R.status, 0, sizeof(int));
    cudaMemset(R.report, 0, 3 * sizeof(int));
    cudaMemset(R.relres, 0, sizeof(double));  // a report before the first solve reads zeros
    R.mask = mask;
    R.ax = ax;
    R.ay = ay;
    R.diag = diag;
    R.dinv = dinv;
    R.wet = wet;
    cx_ = coef * (1.0 / (dx * dx));
    cy_ = coef * (1.0 / (dy * dy));
    k_refine_setup<<<(n + 255) / 256, 256>>>(R, cx_, cy_, ax, ay, diag, dinv, wet);
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        err = std::string("refined solver setup: ") + cudaGetErrorString(e);
        return OC_ERR_CUDA;
    }
    return OC_OK;
}

void RefinedHelm::rebuild(cudaStream_t s) {
    const RefineParams& R = rp_;
    k_refine_setup<<<(R.n + 255) / 256, 256, 0, s>>>(R, cx_, cy_, const_cast<float*>(R.ax), const_cast<float*>(R.ay),
                                                     const_cast<float*>(R.diag), const_cast<float*>(R.dinv),
                                                     const_cast<unsigned char*>(R.wet));
}

int RefinedHelm::solve(const double* rhs, double* x, cudaStream_t s, std::string& err) {
    if (!rhs || !x) return OC_ERR_ARG;
    RefineParams R = rp_;
    R.rhs = rhs;
    R.x = x;
    // a cooperative launch through the extensible launch API, which stream
    // capture records into a graph (the step replays its solves in graphs)
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid_);
    cfg.blockDim = dim3(RT);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_helm_refined, R);
    if (e != cudaSuccess) {
        err = std::string("refined Helmholtz solve launch: ") + cudaGetErrorString(e);
        return OC_ERR_CUDA;
    }
    return OC_OK;
}

int RefinedHelm::report(int* iterations, int* converged, int* outer, double* relres, std::string& err) {
    int st = 0, rep[3] = {0, 0, 0};
    double rel = 0.0;
    if (cudaMemcpy(&st, rp_.status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(rep, rp_.report, sizeof(rep), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&rel, rp_.relres, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) {
        err = "refined solver: report read failed";
        return OC_ERR_CUDA;
    }
    if (st) {
        err = "refined solver: a grid barrier ran out its bound";
        return st;
    }
    if (iterations) *iterations = rep[0];
    if (converged) *converged = rep[1];
    if (outer) *outer = rep[2];
    if (relres) *relres = rel;
    return OC_OK;
}

}  // namespace oc
