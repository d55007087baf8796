// Variable-coefficient Helmholtz solver (reference libs/core/solvers_var.py:22-197).
//
// One persistent cooperative kernel runs a whole solve: no host round trip per
// iteration (the reference CUDA backend copies every dot product to the host,
// cfd_exp3d5_cuda.cu:346-352). The stopping test and the CG scalars are
// bit-identical to the reference because every global sum reproduces NumPy's
// pairwise summation: the vector is cut into the same <=128-element leaves,
// each leaf is summed with NumPy's eight interleaved accumulators (eight
// lanes, combined ((0+1)+(2+3))+((4+5)+(6+7)) by shuffles), and the leaf sums
// are folded by the same binary tree. Every CTA folds the tree itself, so all
// CTAs hold the same scalar and take the same branch without another barrier.
//
// Grid-wide barriers are bounded spins: after ~1 s without progress a CTA sets
// OC_ERR_TIMEOUT in the status word and every CTA leaves the solve.
//
// Multigrid levels up to 64x64 cells run inside CTA 0 with block barriers.

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "ocean_b200.h"
#include "helmholtz.cuh"

namespace oc {

static constexpr long long kBarrierCycles = 2000000000LL;
static constexpr int kCoarseCells = 4096;

// ------------------------------------------------------------------ barrier
__device__ __forceinline__ bool grid_sync(const HelmParams& H) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = H.bar_gen;
        const unsigned g0 = *gen;
        __threadfence();
        const unsigned arrived = atomicAdd(H.bar_count, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(H.bar_count, 0u);
            __threadfence();
            atomicAdd(H.bar_gen, 1u);
        } else {
            const long long t0 = clock64();
            while (*gen == g0) {
                if (clock64() - t0 > kBarrierCycles) {
                    atomicExch(H.status, OC_ERR_TIMEOUT);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *((volatile int*)H.status) == 0;
}

// ------------------------------------------------------------------ level operators
struct Cell {
    int e, ie, iw, jn, js;  // flat index and its four neighbours (periodic)
};

__device__ __forceinline__ Cell cell_of(const HLevel& L, int e) {
    const int j = e / L.nx, i = e - j * L.nx;
    Cell c;
    c.e = e;
    c.ie = j * L.nx + (i + 1 == L.nx ? 0 : i + 1);
    c.iw = j * L.nx + (i == 0 ? L.nx - 1 : i - 1);
    c.jn = (j + 1 == L.ny ? 0 : j + 1) * L.nx + i;
    c.js = (j == 0 ? L.ny - 1 : j - 1) * L.nx + i;
    return c;
}

// (A x)[e] with x read through L2 (other CTAs write it): VarOperator.apply
// (solvers_var.py:47-53)
__device__ __forceinline__ double apply_at(const HLevel& L, double coef, const double* x, const Cell& c) {
    const double m = L.mask[c.e];
    const double xm = __ldcg(x + c.e) * m;
    const double xe = __ldcg(x + c.ie) * L.mask[c.ie];
    const double xw = __ldcg(x + c.iw) * L.mask[c.iw];
    const double xn = __ldcg(x + c.jn) * L.mask[c.jn];
    const double xs = __ldcg(x + c.js) * L.mask[c.js];
    const double fx = L.Ku[c.e] * (xe - xm);
    const double fxw = L.Ku[c.iw] * (xm - xw);
    const double fy = L.Kv[c.e] * (xn - xm);
    const double fys = L.Kv[c.js] * (xm - xs);
    const double lap = (fx - fxw) / L.dx2 + (fy - fys) / L.dy2;
    return (xm - coef * lap) * m + xm * (1.0 - m);
}

// Gauss-Seidel value of cell e from the neighbours' current x (solvers_var.py:55-69)
__device__ __forceinline__ double gs_at(const HLevel& L, const double* x, const double* b, const Cell& c) {
    const double nb = L.cx * (L.Ku[c.e] * __ldcg(x + c.ie) + L.Ku[c.iw] * __ldcg(x + c.iw)) +
                      L.cy * (L.Kv[c.e] * __ldcg(x + c.jn) + L.Kv[c.js] * __ldcg(x + c.js));
    return L.inv_diag[c.e] * (__ldcg(b + c.e) + nb);
}

// the same after the coarse correction x + prolong(xc) * mask of the neighbours
__device__ __forceinline__ double corrected(const HLevel& L, const HLevel& C, const double* x, int e) {
    const int j = e / L.nx, i = e - j * L.nx;
    const double ec = __ldcg(C.x + (j >> 1) * C.nx + (i >> 1));
    return __ldcg(x + e) + ec * L.mask[e];
}

__device__ __forceinline__ double gs_at_prolonged(const HLevel& L, const HLevel& C, const double* x,
                                                  const double* b, const Cell& c) {
    const double nb = L.cx * (L.Ku[c.e] * corrected(L, C, x, c.ie) + L.Ku[c.iw] * corrected(L, C, x, c.iw)) +
                      L.cy * (L.Kv[c.e] * corrected(L, C, x, c.jn) + L.Kv[c.js] * corrected(L, C, x, c.js));
    return L.inv_diag[c.e] * (__ldcg(b + c.e) + nb);
}

__device__ __forceinline__ bool is_colour(const HLevel& L, int e, int colour) {
    const int j = e / L.nx, i = e - j * L.nx;
    return ((i + j) & 1) == colour;
}

// ------------------------------------------------------------------ phases
// Work distribution: `first`/`stride` index the threads taking part (the whole
// grid, or one CTA for the coarse levels).
struct Team {
    int first, stride;
};

__device__ __forceinline__ Team grid_team() {
    Team t;
    t.first = blockIdx.x * blockDim.x + threadIdx.x;
    t.stride = gridDim.x * blockDim.x;
    return t;
}

__device__ __forceinline__ Team block_team() {
    Team t;
    t.first = threadIdx.x;
    t.stride = blockDim.x;
    return t;
}

// one colour of a Gauss-Seidel sweep; the cell mask multiply of the sweep end
// is folded into each assignment (identical for wet cells, 0 for dry ones)
__device__ void colour_phase(const HLevel& L, double* x, const double* b, int colour, Team t) {
    for (int e = t.first; e < L.n; e += t.stride) {
        if (!is_colour(L, e, colour)) continue;
        const Cell c = cell_of(L, e);
        x[e] = gs_at(L, x, b, c) * L.mask[e];
    }
}

__device__ void colour_phase_prolonged(const HLevel& L, const HLevel& C, double* x, const double* b,
                                       int colour, Team t) {
    for (int e = t.first; e < L.n; e += t.stride) {
        if (!is_colour(L, e, colour)) continue;
        const Cell c = cell_of(L, e);
        x[e] = gs_at_prolonged(L, C, x, b, c) * L.mask[e];
    }
}

// coarse rhs = restrict((b - A x) mask), coarse x = 0 (solvers_var.py:143-147)
__device__ void restrict_phase(const HLevel& L, const HLevel& C, double coef, Team t) {
    for (int ec = t.first; ec < C.n; ec += t.stride) {
        const int J = ec / C.nx, I = ec - J * C.nx;
        const int e00 = (2 * J) * L.nx + 2 * I, e01 = e00 + 1;
        const int e10 = e00 + L.nx, e11 = e10 + 1;
        const double r00 = (__ldcg(L.b + e00) - apply_at(L, coef, L.x, cell_of(L, e00))) * L.mask[e00];
        const double r01 = (__ldcg(L.b + e01) - apply_at(L, coef, L.x, cell_of(L, e01))) * L.mask[e01];
        const double r10 = (__ldcg(L.b + e10) - apply_at(L, coef, L.x, cell_of(L, e10))) * L.mask[e10];
        const double r11 = (__ldcg(L.b + e11) - apply_at(L, coef, L.x, cell_of(L, e11))) * L.mask[e11];
        C.b[ec] = 0.25 * (r00 + r01 + r10 + r11);
        C.x[ec] = 0.0;
    }
}

// ------------------------------------------------------------------ pairwise sums
// Calls f(e) exactly once per element of level 0, grouped by NumPy's leaves;
// f returns the two values to accumulate. Writes the per-leaf sums.
template <class F>
__device__ void leaf_phase(const HelmParams& H, F f, double* outA, double* outB) {
    const int lane = threadIdx.x & 31;
    const int lane8 = lane & 7;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int base = warp * 4; base < H.n_leaves; base += nwarps * 4) {
        const int L = base + (lane >> 3);
        const bool act = L < H.n_leaves;
        int s = 0, len = 0;
        if (act) {
            s = H.leaf_start[L];
            len = H.leaf_start[L + 1] - s;
        }
        const int m = len >= 8 ? len - (len % 8) : 0;
        double ra = 0.0, rb = 0.0;
        if (act && len >= 8) {
            double2 v = f(s + lane8);
            ra = v.x;
            rb = v.y;
            for (int t = 8 + lane8; t < m; t += 8) {
                v = f(s + t);
                ra = ra + v.x;
                rb = rb + v.y;
            }
        }
        ra = ra + __shfl_xor_sync(0xffffffffu, ra, 1);
        rb = rb + __shfl_xor_sync(0xffffffffu, rb, 1);
        ra = ra + __shfl_xor_sync(0xffffffffu, ra, 2);
        rb = rb + __shfl_xor_sync(0xffffffffu, rb, 2);
        ra = ra + __shfl_xor_sync(0xffffffffu, ra, 4);
        rb = rb + __shfl_xor_sync(0xffffffffu, rb, 4);
        if (act && lane8 == 0) {
            double a = len >= 8 ? ra : 0.0;
            double bsum = len >= 8 ? rb : 0.0;
            for (int t = m; t < len; ++t) {
                const double2 v = f(s + t);
                a = a + v.x;
                bsum = bsum + v.y;
            }
            outA[L] = a;
            if (outB) outB[L] = bsum;
        }
    }
}

// fold the leaf sums by NumPy's tree, in every CTA (the result is the same
// everywhere); sm holds n_leaves doubles
__device__ double tree_fold(const HelmParams& H, const double* leaf, double* sm) {
    for (int t = threadIdx.x; t < H.n_leaves; t += blockDim.x) sm[t] = __ldcg(leaf + t);
    __syncthreads();
    for (int h = 0; h < H.n_heights; ++h) {
        for (int t = H.height_start[h] + threadIdx.x; t < H.height_start[h + 1]; t += blockDim.x) {
            const int2 op = H.ops[t];
            sm[op.x] = sm[op.x] + sm[op.y];
        }
        __syncthreads();
    }
    const double r = sm[0];
    __syncthreads();
    return r;
}

// ------------------------------------------------------------------ multigrid V-cycle
// smoothing sweeps of one level: forward = red then black, reverse = black then red
__device__ void smooth(const HLevel& L, int sweeps, bool reverse, bool grid, const HelmParams& H,
                       bool& ok) {
    for (int s = 0; s < sweeps && ok; ++s) {
        for (int h = 0; h < 2 && ok; ++h) {
            const int colour = reverse ? 1 - h : h;
            colour_phase(L, L.x, L.b, colour, grid ? grid_team() : block_team());
            if (grid)
                ok = grid_sync(H);
            else
                __syncthreads();
        }
    }
}

// post-smoothing of level l after the coarse correction: the first (black)
// half-sweep reads the prolonged neighbours (solvers_var.py:148-150)
__device__ void post_smooth(const HelmParams& H, int l, bool grid, bool& ok) {
    const HLevel& L = H.lv[l];
    const HLevel& C = H.lv[l + 1];
    colour_phase_prolonged(L, C, L.x, L.b, 1, grid ? grid_team() : block_team());
    if (grid)
        ok = grid_sync(H);
    else
        __syncthreads();
    if (!ok) return;
    colour_phase(L, L.x, L.b, 0, grid ? grid_team() : block_team());
    if (grid)
        ok = grid_sync(H);
    else
        __syncthreads();
    if (!ok) return;
    smooth(L, 1, true, grid, H, ok);
}

__device__ void vcycle(const HelmParams& H, bool& ok) {
    const int nl = H.n_levels;
    const int cf = H.coarse_from;  // levels >= cf run in CTA 0
    // descend over the grid-wide levels
    for (int l = 0; l < nl - 1 && l < cf && ok; ++l) {
        smooth(H.lv[l], 2, false, true, H, ok);
        if (!ok) return;
        restrict_phase(H.lv[l], H.lv[l + 1], H.coef, grid_team());
        ok = grid_sync(H);
    }
    if (!ok) return;
    if (cf < nl) {
        if (blockIdx.x == 0) {
            bool bok = true;
            for (int l = cf; l < nl - 1; ++l) {
                smooth(H.lv[l], 2, false, false, H, bok);
                restrict_phase(H.lv[l], H.lv[l + 1], H.coef, block_team());
                __syncthreads();
            }
            smooth(H.lv[nl - 1], 2, false, false, H, bok);
            smooth(H.lv[nl - 1], 2, true, false, H, bok);
            for (int l = nl - 2; l >= cf; --l) post_smooth(H, l, false, bok);
        }
        ok = grid_sync(H);
        if (!ok) return;
    } else {
        // coarsest level on the whole grid
        smooth(H.lv[nl - 1], 2, false, true, H, ok);
        if (!ok) return;
        smooth(H.lv[nl - 1], 2, true, true, H, ok);
        if (!ok) return;
    }
    for (int l = (cf < nl - 1 ? cf : nl - 1) - 1; l >= 0 && ok; --l) post_smooth(H, l, true, ok);
}

// ------------------------------------------------------------------ the solve kernel
__global__ void __launch_bounds__(512) k_helm_solve(HelmParams H) {
    extern __shared__ double sm[];
    const HLevel& L0 = H.lv[0];
    const double* rhs = H.rhs;
    double* x = L0.x;
    double* b0 = L0.b;
    bool ok = true;
    int iters = 0, conv = 1;

    // norm of the masked right-hand side (solvers_var.py:163-168)
    leaf_phase(H,
               [&](int e) {
                   const double r = rhs[e] * L0.mask[e];
                   b0[e] = r;
                   if (H.kind <= HK_PCG_RBGS) H.r[e] = r;
                   x[e] = 0.0;
                   return make_double2(r * r, 0.0);
               },
               H.leafA, nullptr);
    ok = grid_sync(H);
    const double norm_b = ok ? sqrt(tree_fold(H, H.leafA, sm)) : 0.0;
    if (!ok || norm_b == 0.0) goto done;
    {
        const double tol = H.rtol * norm_b;
        if (H.kind == HK_RBGS || H.kind == HK_MULTIGRID) {
            // stationary iteration with the true residual (solvers_var.py:170-179)
            conv = 0;
            for (int it = 1; it <= H.max_iter && ok; ++it) {
                if (H.kind == HK_MULTIGRID) {
                    vcycle(H, ok);
                } else {
                    colour_phase(L0, x, b0, 0, grid_team());
                    ok = grid_sync(H);
                    if (!ok) break;
                    colour_phase(L0, x, b0, 1, grid_team());
                    ok = grid_sync(H);
                }
                if (!ok) break;
                leaf_phase(H,
                           [&](int e) {
                               const double d = __ldcg(b0 + e) - apply_at(L0, H.coef, x, cell_of(L0, e));
                               return make_double2(d * d, 0.0);
                           },
                           H.leafA, nullptr);
                ok = grid_sync(H);
                if (!ok) break;
                iters = it;
                const double res = sqrt(tree_fold(H, H.leafA, sm));
                if (res <= tol) {
                    conv = 1;
                    break;
                }
            }
        } else {
            // preconditioned CG (solvers_var.py:181-197)
            double* r = H.r;
            double* z = H.z;
            double* p = H.p;
            double* Ap = H.Ap;
            const bool jac = H.kind == HK_PCG_JACOBI;
            // z = M^-1 r
            auto precondition = [&](bool& okp) {
                if (jac) return;
                for (int e = grid_team().first; e < L0.n; e += grid_team().stride) z[e] = 0.0;
                okp = grid_sync(H);
                if (!okp) return;
                for (int h = 0; h < 4 && okp; ++h) {
                    const int colour = (h == 0 || h == 3) ? 0 : 1;
                    colour_phase(L0, z, r, colour, grid_team());
                    okp = grid_sync(H);
                }
            };
            precondition(ok);
            if (!ok) goto done;
            leaf_phase(H,
                       [&](int e) {
                           const double re = __ldcg(r + e);
                           const double ze = jac ? L0.inv_diag[e] * re : __ldcg(z + e);
                           if (jac) z[e] = ze;
                           p[e] = ze;
                           return make_double2(re * ze, 0.0);
                       },
                       H.leafA, nullptr);
            ok = grid_sync(H);
            if (!ok) goto done;
            double rz = tree_fold(H, H.leafA, sm);
            conv = 0;
            for (int it = 1; it <= H.max_iter; ++it) {
                leaf_phase(H,
                           [&](int e) {
                               const double a = apply_at(L0, H.coef, p, cell_of(L0, e));
                               Ap[e] = a;
                               return make_double2(__ldcg(p + e) * a, 0.0);
                           },
                           H.leafA, nullptr);
                ok = grid_sync(H);
                if (!ok) break;
                const double alpha = rz / tree_fold(H, H.leafA, sm);
                leaf_phase(H,
                           [&](int e) {
                               const double pe = __ldcg(p + e);
                               const double ae = __ldcg(Ap + e);
                               const double xe = __ldcg(x + e) + alpha * pe;
                               const double re = __ldcg(r + e) - alpha * ae;
                               x[e] = xe;
                               r[e] = re;
                               double ze = 0.0;
                               if (jac) {
                                   ze = L0.inv_diag[e] * re;
                                   z[e] = ze;
                               }
                               return make_double2(re * re, re * ze);
                           },
                           H.leafA, H.leafB);
                ok = grid_sync(H);
                if (!ok) break;
                iters = it;
                const double res = sqrt(tree_fold(H, H.leafA, sm));
                if (res <= tol) {
                    conv = 1;
                    break;
                }
                if (!jac) {
                    precondition(ok);
                    if (!ok) break;
                    leaf_phase(H,
                               [&](int e) {
                                   const double re = __ldcg(r + e);
                                   return make_double2(re * __ldcg(z + e), 0.0);
                               },
                               H.leafB, nullptr);
                    ok = grid_sync(H);
                    if (!ok) break;
                }
                const double rz_new = tree_fold(H, H.leafB, sm);
                const double beta = rz_new / rz;
                for (int e = grid_team().first; e < L0.n; e += grid_team().stride)
                    p[e] = __ldcg(z + e) + beta * __ldcg(p + e);
                ok = grid_sync(H);
                if (!ok) break;
                rz = rz_new;
            }
        }
    }
done:
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const int idx = *H.log_count;
        if (idx < H.log_cap) {
            H.log_iters[idx] = ok ? iters : -1;
            H.log_conv[idx] = ok ? conv : 0;
        }
        *H.log_count = idx + 1;
    }
}

// ------------------------------------------------------------------ level rebuild
// coarse face coefficients (solvers_var.py:118-123) and inverse diagonal
// (solvers_var.py:39-45) of level `L` from the finer level `F`
__global__ void k_helm_level(HLevel F, HLevel L, int coarse) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= L.n) return;
    const int J = e / L.nx, I = e - J * L.nx;
    const int Iw = I == 0 ? L.nx - 1 : I - 1, Js = J == 0 ? L.ny - 1 : J - 1;
    double ku, kuw, kv, kvs;
    if (coarse) {
        auto cku = [&](int jj, int ii) {
            return 0.5 * (F.Ku[(2 * jj) * F.nx + 2 * ii + 1] + F.Ku[(2 * jj + 1) * F.nx + 2 * ii + 1]);
        };
        auto ckv = [&](int jj, int ii) {
            return 0.5 * (F.Kv[(2 * jj + 1) * F.nx + 2 * ii] + F.Kv[(2 * jj + 1) * F.nx + 2 * ii + 1]);
        };
        ku = cku(J, I);
        kuw = cku(J, Iw);
        kv = ckv(J, I);
        kvs = ckv(Js, I);
        L.Ku[e] = ku;
        L.Kv[e] = kv;
    } else {
        ku = L.Ku[e];
        kuw = L.Ku[J * L.nx + Iw];
        kv = L.Kv[e];
        kvs = L.Kv[Js * L.nx + I];
    }
    const double d = 1.0 + L.cx * (ku + kuw) + L.cy * (kv + kvs);
    L.inv_diag[e] = 1.0 / (L.mask[e] > 0.0 ? d : 1.0);
}

// ------------------------------------------------------------------ host side
// NumPy's pairwise summation tree of n contiguous elements
// (numpy/core/src/umath/loops_utils.h.src, pairwise_sum: leaves of <= 128
// elements, split at n/2 rounded down to a multiple of 8)
struct PwNode {
    int lo, height;
};

static PwNode pairwise_build(long start, long n, std::vector<int>& leaves,
                             std::vector<std::vector<int2>>& by_height) {
    if (n <= 128) {
        leaves.push_back((int)start);
        return {(int)leaves.size() - 1, 0};
    }
    long h = n / 2;
    h -= h % 8;
    const PwNode a = pairwise_build(start, h, leaves, by_height);
    const PwNode b = pairwise_build(start + h, n - h, leaves, by_height);
    const int height = std::max(a.height, b.height) + 1;
    if ((int)by_height.size() < height) by_height.resize(height);
    by_height[height - 1].push_back(make_int2(a.lo, b.lo));
    return {a.lo, height};
}

void* HelmSolver::dalloc(size_t nbytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, nbytes) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, nbytes);
    allocs_.push_back(p);
    bytes_ += nbytes;
    return p;
}

HelmSolver::~HelmSolver() {
    for (void* p : allocs_) cudaFree(p);
}

int HelmSolver::init(int nx, int ny, double lx, double ly, double coef, int kind, double rtol,
                     int max_iter, const double* mask_host, double* Ku, double* Kv, int log_cap,
                     int* status, std::string& err) {
    HelmParams& H = hp_;
    H.kind = kind;
    H.coef = coef;
    H.rtol = rtol;
    H.max_iter = max_iter;
    H.status = status;
    // level geometry and masks
    std::vector<std::vector<double>> masks;
    masks.push_back(std::vector<double>(mask_host, mask_host + (size_t)nx * ny));
    int lnx = nx, lny = ny;
    std::vector<std::pair<int, int>> dims{{nx, ny}};
    if (kind == HK_MULTIGRID) {
        while (lnx % 2 == 0 && lny % 2 == 0 && lnx / 2 >= 8 && lny / 2 >= 8 &&
               (int)dims.size() < OC_MAX_LEVELS) {
            const int cnx = lnx / 2, cny = lny / 2;
            const std::vector<double>& fm = masks.back();
            std::vector<double> cm((size_t)cnx * cny);
            for (int J = 0; J < cny; ++J)
                for (int I = 0; I < cnx; ++I) {
                    const double a = fm[(size_t)(2 * J) * lnx + 2 * I], b = fm[(size_t)(2 * J) * lnx + 2 * I + 1];
                    const double c = fm[(size_t)(2 * J + 1) * lnx + 2 * I], d = fm[(size_t)(2 * J + 1) * lnx + 2 * I + 1];
                    cm[(size_t)J * cnx + I] = std::max(std::max(std::max(a, b), c), d);
                }
            masks.push_back(cm);
            dims.push_back({cnx, cny});
            lnx = cnx;
            lny = cny;
        }
    }
    H.n_levels = (int)dims.size();
    H.coarse_from = H.n_levels;
    for (int l = 0; l < H.n_levels; ++l) {
        HLevel& L = H.lv[l];
        L.nx = dims[l].first;
        L.ny = dims[l].second;
        L.n = L.nx * L.ny;
        const double dx = lx / L.nx, dy = ly / L.ny;
        L.dx2 = std::pow(dx, 2.0);
        L.dy2 = std::pow(dy, 2.0);
        L.cx = coef * (1.0 / std::pow(dx, 2.0));
        L.cy = coef * (1.0 / std::pow(dy, 2.0));
        double* m = (double*)dalloc(sizeof(double) * L.n);
        if (!m) {
            err = "cudaMalloc failed (Helmholtz levels)";
            return OC_ERR_CUDA;
        }
        cudaMemcpy(m, masks[l].data(), sizeof(double) * L.n, cudaMemcpyHostToDevice);
        L.mask = m;
        L.inv_diag = (double*)dalloc(sizeof(double) * L.n);
        L.b = (double*)dalloc(sizeof(double) * L.n);
        if (l == 0) {
            L.Ku = Ku;
            L.Kv = Kv;
            L.x = nullptr;  // set per solve
        } else {
            L.Ku = (double*)dalloc(sizeof(double) * L.n);
            L.Kv = (double*)dalloc(sizeof(double) * L.n);
            L.x = (double*)dalloc(sizeof(double) * L.n);
        }
        if (!L.inv_diag || !L.b || (l > 0 && (!L.Ku || !L.Kv || !L.x))) {
            err = "cudaMalloc failed (Helmholtz levels)";
            return OC_ERR_CUDA;
        }
        if (l > 0 && L.n <= kCoarseCells && H.coarse_from == H.n_levels) H.coarse_from = l;
    }
    const size_t n = (size_t)nx * ny;
    H.r = (double*)dalloc(sizeof(double) * n);
    H.z = (double*)dalloc(sizeof(double) * n);
    H.p = (double*)dalloc(sizeof(double) * n);
    H.Ap = (double*)dalloc(sizeof(double) * n);
    // pairwise plan
    std::vector<int> leaves;
    std::vector<std::vector<int2>> by_height;
    pairwise_build(0, (long)n, leaves, by_height);
    leaves.push_back((int)n);
    std::vector<int> hstart{0};
    std::vector<int2> ops;
    for (auto& v : by_height) {
        ops.insert(ops.end(), v.begin(), v.end());
        hstart.push_back((int)ops.size());
    }
    H.n_leaves = (int)leaves.size() - 1;
    H.n_heights = (int)by_height.size();
    int* d_leaves = (int*)dalloc(sizeof(int) * leaves.size());
    int* d_hstart = (int*)dalloc(sizeof(int) * hstart.size());
    int2* d_ops = (int2*)dalloc(sizeof(int2) * std::max<size_t>(1, ops.size()));
    H.leafA = (double*)dalloc(sizeof(double) * H.n_leaves);
    H.leafB = (double*)dalloc(sizeof(double) * H.n_leaves);
    unsigned* bar = (unsigned*)dalloc(sizeof(unsigned) * 2);
    H.log_cap = log_cap;
    H.log_iters = (int*)dalloc(sizeof(int) * log_cap);
    H.log_conv = (int*)dalloc(sizeof(int) * log_cap);
    H.log_count = (int*)dalloc(sizeof(int));
    if (!H.r || !H.z || !H.p || !H.Ap || !d_leaves || !d_hstart || !d_ops || !H.leafA || !H.leafB ||
        !bar || !H.log_iters || !H.log_conv || !H.log_count) {
        err = "cudaMalloc failed (Helmholtz work)";
        return OC_ERR_CUDA;
    }
    cudaMemcpy(d_leaves, leaves.data(), sizeof(int) * leaves.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(d_hstart, hstart.data(), sizeof(int) * hstart.size(), cudaMemcpyHostToDevice);
    if (!ops.empty()) cudaMemcpy(d_ops, ops.data(), sizeof(int2) * ops.size(), cudaMemcpyHostToDevice);
    H.leaf_start = d_leaves;
    H.height_start = d_hstart;
    H.ops = d_ops;
    H.bar_count = bar;
    H.bar_gen = bar + 1;
    // co-resident grid for the cooperative launch
    int dev = 0, sms = 0, coop = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop) {
        err = "device does not support cooperative launches";
        return OC_ERR_UNSUPPORTED;
    }
    smem_ = sizeof(double) * (size_t)H.n_leaves;
    if (smem_ > 200 * 1024) {
        err = "Helmholtz grid too large for the single-pass reduction tree";
        return OC_ERR_UNSUPPORTED;
    }
    if (smem_ > 48 * 1024)
        cudaFuncSetAttribute(k_helm_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_helm_solve, block_, smem_);
    if (per_sm < 1) {
        err = "Helmholtz solve kernel cannot be resident";
        return OC_ERR_CUDA;
    }
    grid_ = sms * std::min(per_sm, 2);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = std::string("Helmholtz init: ") + cudaGetErrorString(e);
        return OC_ERR_CUDA;
    }
    return OC_OK;
}

int HelmSolver::grow_log(int cap, cudaStream_t s, std::string& err) {
    if (cap <= hp_.log_cap) return OC_OK;
    int* it = nullptr;
    int* cv = nullptr;
    if (cudaMalloc(&it, sizeof(int) * cap) != cudaSuccess || cudaMalloc(&cv, sizeof(int) * cap) != cudaSuccess) {
        err = "cudaMalloc failed (solve log)";
        return OC_ERR_CUDA;
    }
    cudaMemcpyAsync(it, hp_.log_iters, sizeof(int) * hp_.log_cap, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(cv, hp_.log_conv, sizeof(int) * hp_.log_cap, cudaMemcpyDeviceToDevice, s);
    cudaStreamSynchronize(s);
    for (auto& p : allocs_) {
        if (p == hp_.log_iters || p == hp_.log_conv) {
            cudaFree(p);
            p = (p == hp_.log_iters) ? (void*)it : (void*)cv;
        }
    }
    bytes_ += sizeof(int) * 2 * (size_t)(cap - hp_.log_cap);
    hp_.log_iters = it;
    hp_.log_conv = cv;
    hp_.log_cap = cap;
    return OC_OK;
}

void HelmSolver::rebuild(cudaStream_t s) {
    for (int l = 0; l < hp_.n_levels; ++l) {
        const HLevel& L = hp_.lv[l];
        const HLevel& F = hp_.lv[l > 0 ? l - 1 : 0];
        k_helm_level<<<(L.n + 255) / 256, 256, 0, s>>>(F, L, l > 0 ? 1 : 0);
    }
}

int HelmSolver::solve(const double* rhs, double* x, cudaStream_t s, std::string& err) {
    HelmParams H = hp_;
    H.rhs = rhs;
    H.lv[0].x = x;
    void* args[] = {&H};
    const cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_helm_solve, dim3(grid_),
                                                      dim3(block_), args, smem_, s);
    if (e != cudaSuccess) {
        err = std::string("Helmholtz solve launch: ") + cudaGetErrorString(e);
        return OC_ERR_CUDA;
    }
    return OC_OK;
}

}  // namespace oc
