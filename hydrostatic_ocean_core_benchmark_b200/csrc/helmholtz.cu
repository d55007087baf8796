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
// Multigrid fine levels run as shared-memory tiles with a redundant halo (two
// grid barriers per level and V-cycle); levels of at most 32x32 cells run
// inside CTA 0's shared memory.

#include <cooperative_groups.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <cmath>
#include <string>
#include <vector>

#include "ocean_b200.h"
#include "grid_barrier.cuh"
#include "helmholtz.cuh"

namespace oc {

static constexpr int kCoarseCells = 1024;
// fine-level tiles: interior TX x TY cells plus a halo of HALO cells, enough
// for four red-black half-sweeps and one residual on a shrinking region
static constexpr int HALO = 5;
template <int TX_, int TY_>
struct TileShape {
    static constexpr int TX = TX_, TY = TY_;
    static constexpr int RW = TX + 2 * HALO, RH = TY + 2 * HALO, RN = RW * RH;
};
using Tile32 = TileShape<32, 32>;
using Tile3216 = TileShape<32, 16>;
using Tile16 = TileShape<16, 16>;
using Tile8 = TileShape<8, 8>;
using TileWide = TileShape<128, 16>;  // level 0 of large grids: one tile per CTA, one NumPy leaf per row
// per-level tile shape codes (HLevel::shape)
enum { SHAPE_32 = 0, SHAPE_3216 = 1, SHAPE_16 = 2, SHAPE_8 = 3, SHAPE_WIDE = 4 };

// ------------------------------------------------------------------ the solve's CTAs
// A solve runs on the CTAs of its launch, or, in a batched launch that solves
// several systems at once, on one system's share of them: s_grid.cta is the
// CTA's index among the solve's CTAs and s_grid.ncta their number. Every
// work-distribution loop and the barrier use these instead of the launch's grid.
struct SolveGrid {
    int cta, ncta;
};
static __shared__ SolveGrid s_grid;

// ------------------------------------------------------------------ barrier
// the bounded grid barrier of grid_barrier.cuh on the solver's counter and status
__device__ __forceinline__ void grid_sync_begin(const HelmParams& H) { grid_sync_begin(H.status); }

__device__ __forceinline__ bool grid_sync(const HelmParams& H) {
    return grid_sync(H.bar_count, H.status, (unsigned)s_grid.ncta, H.wait_cycles);
}

// ------------------------------------------------------------------ asynchronous copies
// cp.async into shared memory without a register round trip, so a thread's
// copies are all in flight at once. The 8-byte form goes through L1, which is not
// coherent with other SMs' writes, so it serves only arrays that stay constant
// during the solve (the level coefficients); b and x, which other CTAs of the
// launch write, are read through L2 (__ldcg).
__device__ __forceinline__ void cpa_ca8(double* sdst, const double* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cpa_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
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
    t.first = s_grid.cta * blockDim.x + threadIdx.x;
    t.stride = s_grid.ncta * blockDim.x;
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

// ------------------------------------------------------------------ pairwise sums
// element e of a warp's leaf values held as r[e / 32] on lane e mod 32, on every
// lane; e / 32 must be the same on all lanes (the source register is the caller's)
__device__ __forceinline__ double leaf_pick(const double* r, int e) {
    const int q = e >> 5;
    const double x = q == 0 ? r[0] : (q == 1 ? r[1] : (q == 2 ? r[2] : r[3]));
    return __shfl_sync(0xffffffffu, x, e & 31);
}

// NumPy's pairwise sum of one leaf (len <= 128 values) that a warp holds as
// va[q] = element lane + 32 q. The eight interleaved accumulators of NumPy's
// unrolled loop are formed in their sequential order by lanes j = 0..7
// (element 8t + j sits on lane (8t + j) mod 32 in register t / 32, the same
// register on every lane for a given t), folded as
// ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7)), and the len mod 8 remaining elements are
// added one by one. Every lane returns the sum.
__device__ __forceinline__ double leaf_sum_warp(const double* va, int len) {
    const int lane8 = threadIdx.x & 7;
    const int m = len >= 8 ? len - (len % 8) : 0;
    double ra = 0.0;
    if (len >= 8) {
        ra = leaf_pick(va, lane8);
        for (int t = 8; t < m; t += 8) ra = ra + leaf_pick(va, t + lane8);
    }
    ra = ra + __shfl_xor_sync(0xffffffffu, ra, 1);
    ra = ra + __shfl_xor_sync(0xffffffffu, ra, 2);
    ra = ra + __shfl_xor_sync(0xffffffffu, ra, 4);
    double a = len >= 8 ? __shfl_sync(0xffffffffu, ra, 0) : 0.0;
    for (int t = m; t < len; ++t) a = a + leaf_pick(va, t);
    return a;
}

// Calls f(e) exactly once per element of level 0, grouped by NumPy's leaves;
// f returns the two values to accumulate. Writes the per-leaf sums. One warp
// per leaf, consecutive leaves on different CTAs; lane l evaluates f for leaf
// elements l, l+32, l+64, l+96 with independent loads.
template <class F>
__device__ void leaf_phase(const HelmParams& H, F f, double* outA, double* outB) {
    const int lane = threadIdx.x & 31;
    const int nwarps = s_grid.ncta * (blockDim.x >> 5);
    const int my = (threadIdx.x >> 5) * s_grid.ncta + s_grid.cta;  // leaf L runs on CTA L mod grid
    for (int L = my; L < H.n_leaves; L += nwarps) {
        const int s = H.leaf_start[L];
        const int len = H.leaf_start[L + 1] - s;
        double va[4], vb[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int e = lane + 32 * q;
            double2 v = make_double2(0.0, 0.0);
            if (e < len) v = f(s + e);
            va[q] = v.x;
            vb[q] = v.y;
        }
        const double a = leaf_sum_warp(va, len);
        const double bsum = outB ? leaf_sum_warp(vb, len) : 0.0;
        if (lane == 0) {
            outA[L] = a;
            if (outB) outB[L] = bsum;
        }
    }
}

// the fold's plan (ops, then the height offsets): a shared-memory copy made at
// the start of the solve when it fits, else the global arrays
struct FoldPlan {
    const int2* ops;
    const int* height_start;
};

// fold the leaf sums by NumPy's tree, in every CTA (the result is the same
// everywhere); sm holds n_leaves doubles
__device__ double tree_fold(const HelmParams& H, const FoldPlan& F, const double* leaf, double* sm) {
    for (int t = threadIdx.x; t < H.n_leaves; t += blockDim.x) sm[t] = __ldcg(leaf + t);
    __syncthreads();
    for (int h = 0; h < H.n_heights; ++h) {
        for (int t = F.height_start[h] + threadIdx.x; t < F.height_start[h + 1]; t += blockDim.x) {
            const int2 op = F.ops[t];
            sm[op.x] = sm[op.x] + sm[op.y];
        }
        __syncthreads();
    }
    const double r = sm[0];
    __syncthreads();
    return r;
}

// The same fold for grids whose leaf sums do not fit one CTA's shared memory
// (H.big_fold): the tree is cut below the nodes of at most a block's worth of
// leaves. Each block subtree is folded by one CTA and its root written to
// `broot`; after a grid barrier every CTA folds the top of the tree over the
// block roots. Every addition is the one of the whole-tree fold, in the same
// order, so the result is bit-identical; it costs one more grid barrier. Each
// leaf buffer has its own root buffer, so folds that follow one another without
// a barrier never overwrite roots another CTA is still reading.
__device__ double fold_blocks(const HelmParams& H, const double* leaf, double* broot, double* sm, bool& ok) {
    for (int j = s_grid.cta; j < H.n_blocks; j += s_grid.ncta) {
        const int4 B = H.blocks[j];  // first leaf, leaves, offset of its height starts, heights
        for (int t = threadIdx.x; t < B.y; t += blockDim.x) sm[t] = __ldcg(leaf + B.x + t);
        __syncthreads();
        for (int h = 0; h < B.w; ++h) {
            for (int t = H.bh_start[B.z + h] + threadIdx.x; t < H.bh_start[B.z + h + 1]; t += blockDim.x) {
                const int2 op = H.bops[t];
                sm[op.x] = sm[op.x] + sm[op.y];
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) broot[j] = sm[0];
        __syncthreads();
    }
    ok = grid_sync(H);
    if (!ok) return 0.0;
    for (int t = threadIdx.x; t < H.n_blocks; t += blockDim.x) sm[t] = __ldcg(broot + t);
    __syncthreads();
    for (int h = 0; h < H.top_heights; ++h) {
        for (int t = H.top_hstart[h] + threadIdx.x; t < H.top_hstart[h + 1]; t += blockDim.x) {
            const int2 op = H.top_ops[t];
            sm[op.x] = sm[op.x] + sm[op.y];
        }
        __syncthreads();
    }
    const double r = sm[0];
    __syncthreads();
    return r;
}

// The same fold when NumPy's tree over the leaves is perfect (2^m leaves, node
// (i, i + 2^h) at height h; H.perfect_lanes = P > 0): each lane folds P
// consecutive leaves in registers, the lanes of a warp fold their subtrees by
// shuffles, and warp 0 folds the warps' subtrees. Every addition is the tree's
// (left + right), so the result is bit-identical to tree_fold's, with two CTA
// barriers instead of one per height.
template <int P>
__device__ __forceinline__ double lane_tree(const double* v) {
    if constexpr (P == 1)
        return v[0];
    else
        return lane_tree<P / 2>(v) + lane_tree<P / 2>(v + P / 2);
}

template <int P>
__device__ double perfect_fold(int n, const double* leaf, double* sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwa = n / (32 * P);  // warps in use: a power of two, at most the CTA's
    if (warp < nwa) {
        double v[P];
        const double* src = leaf + warp * 32 * P + lane * P;
#pragma unroll
        for (int q = 0; q < P; ++q) v[q] = __ldcg(src + q);
        double x = lane_tree<P>(v);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double y = __shfl_down_sync(0xffffffffu, x, o);
            if ((lane & (2 * o - 1)) == 0) x = x + y;
        }
        if (lane == 0) sm[warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
        double x = lane < nwa ? sm[lane] : 0.0;
        for (int o = 1; o < nwa; o <<= 1) {
            const double y = __shfl_down_sync(0xffffffffu, x, o);
            if ((lane & (2 * o - 1)) == 0) x = x + y;
        }
        __syncwarp();
        if (lane == 0) sm[0] = x;
    }
    __syncthreads();
    const double r = sm[0];
    __syncthreads();
    return r;
}

// the sum of one of the leaf buffers (leafA, leafB or leafC) in NumPy's order
__device__ __forceinline__ double fold_sum(const HelmParams& H, const FoldPlan& F, const double* leaf, double* sm,
                                           bool& ok) {
    switch (H.perfect_lanes) {
        case 1: return perfect_fold<1>(H.n_leaves, leaf, sm);
        case 2: return perfect_fold<2>(H.n_leaves, leaf, sm);
        case 4: return perfect_fold<4>(H.n_leaves, leaf, sm);
        case 8: return perfect_fold<8>(H.n_leaves, leaf, sm);
        case 16: return perfect_fold<16>(H.n_leaves, leaf, sm);
        default: break;
    }
    if (!H.big_fold) return tree_fold(H, F, leaf, sm);
    double* broot = leaf == H.leafA ? H.broot : (leaf == H.leafB ? H.broot + H.n_blocks : H.broot + 2 * H.n_blocks);
    return fold_blocks(H, leaf, broot, sm, ok);
}

// ------------------------------------------------------------------ tiled multigrid
// A fine level is processed tile by tile in shared memory. The down phase loads
// x, b and the coefficients of a tile plus a HALO-wide ring, runs the two
// pre-smoothing sweeps (four red-black half-sweeps) on a region that shrinks by
// one cell per half-sweep, and forms the restricted residual of the interior;
// the up phase adds the prolonged coarse correction and runs the two reverse
// post-smoothing sweeps the same way. Every value in the valid region is the
// one the whole-grid sweep produces (same inputs, same operations), so the
// result is identical to sweeping the level with a grid barrier between
// half-sweeps, with two barriers per level instead of nine.
__device__ __forceinline__ int wrap_any(int i, int n) {
    if (i >= 0 && i < n) return i;
    if (i < 0 && i + n >= 0) return i + n;
    if (i >= n && i - n < n) return i - n;
    const int r = i % n;
    return r < 0 ? r + n : r;
}

struct TileRefs {
    double *x, *b, *ku, *kv, *id, *m;
};

template <class S>
__device__ __forceinline__ TileRefs tile_refs(double* base) {
    TileRefs t;
    t.x = base;
    t.b = base + S::RN;
    t.ku = base + 2 * S::RN;
    t.kv = base + 3 * S::RN;
    t.id = base + 4 * S::RN;
    t.m = base + 5 * S::RN;
    return t;
}

// load a tile region of level L whose interior starts at (i0, j0); x from xin
// (or zero), plus the coarse correction e * mask when C is given
// (with `coef` false the coefficients ku, kv, id, m are already in place).
// A thread gathers CH of its cells at a time into registers and only then
// writes them to shared memory: the tile arrays reach here as plain pointers,
// so the compiler may not move a later cell's global loads above an earlier
// cell's stores, and cell by cell the loads of a thread would run one L2 round
// trip after another.
template <class S, int CH, bool COEF>
__device__ __forceinline__ void tile_load_chunks(const HLevel& L, int i0, int j0, const double* xin,
                                                 const HLevel* C, TileRefs t) {
    const int nt = blockDim.x;
    for (int base = threadIdx.x; base < S::RN; base += CH * nt) {
        double xv[CH], bv[CH];
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            const int r = base + q * nt;
            xv[q] = bv[q] = 0.0;
            if (r < S::RN) {
                const int rj = r / S::RW, ri = r - rj * S::RW;
                const int gi = wrap_any(i0 - HALO + ri, L.nx), gj = wrap_any(j0 - HALO + rj, L.ny);
                const int g = gj * L.nx + gi;
                if (COEF) {
                    // the coefficients, constant during the solve: asynchronous copies
                    cpa_ca8(t.ku + r, L.Ku + g);
                    cpa_ca8(t.kv + r, L.Kv + g);
                    cpa_ca8(t.id + r, L.inv_diag + g);
                    cpa_ca8(t.m + r, L.mask + g);
                }
                double x = xin ? __ldcg(xin + g) : 0.0;
                if (C) x = x + __ldcg(C->x + (gj >> 1) * C->nx + (gi >> 1)) * (COEF ? L.mask[g] : t.m[r]);
                xv[q] = x;
                bv[q] = __ldcg(L.b + g);
            }
        }
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            const int r = base + q * nt;
            if (r < S::RN) {
                t.x[r] = xv[q];
                t.b[r] = bv[q];
            }
        }
    }
    if (COEF) cpa_wait_all();
}

template <class S>
__device__ void tile_load(const HLevel& L, int i0, int j0, const double* xin, const HLevel* C,
                          TileRefs t, bool coef = true) {
    if (coef)
        tile_load_chunks<S, 2, true>(L, i0, j0, xin, C, t);
    else
        tile_load_chunks<S, 4, false>(L, i0, j0, xin, C, t);
    __syncthreads();
}

// Level 0's coefficients stay in shared memory for a whole solve when every
// level-0 tile has a CTA of its own (H.persist0): the first RN x 4 doubles hold
// the CTA's tile's ku, kv, id and m, and the tile phases of level 0 load only x
// and b. Everything else works above them.
template <class S>
__device__ __forceinline__ TileRefs tile_refs_persist(double* persist, double* work) {
    TileRefs t;
    t.ku = persist;
    t.kv = persist + S::RN;
    t.id = persist + 2 * S::RN;
    t.m = persist + 3 * S::RN;
    t.x = work;
    t.b = work + S::RN;
    return t;
}

// With a CTA of its own for every level-0 tile, the tiles go to the last CTAs
// (tile = CTA - (CTAs - tiles)), so CTA 0, which runs the coarse levels, keeps
// its persistent region for their coefficients (H.coarse_persist).
__device__ __forceinline__ int level0_tile_of_cta(int tiles) { return s_grid.cta - (s_grid.ncta - tiles); }

__device__ void persist_level0(const HelmParams& H, double* persist) {
    using S = TileWide;
    const HLevel& L = H.lv[0];
    const int tx = (L.nx + S::TX - 1) / S::TX;
    const int tile = level0_tile_of_cta(tx * ((L.ny + S::TY - 1) / S::TY));
    if (tile < 0) return;
    const int i0 = (tile % tx) * S::TX, j0 = (tile / tx) * S::TY;
    for (int r = threadIdx.x; r < S::RN; r += blockDim.x) {
        const int rj = r / S::RW, ri = r - rj * S::RW;
        const int g = wrap_any(j0 - HALO + rj, L.ny) * L.nx + wrap_any(i0 - HALO + ri, L.nx);
        persist[r] = L.Ku[g];
        persist[S::RN + r] = L.Kv[g];
        persist[2 * S::RN + r] = L.inv_diag[g];
        persist[3 * S::RN + r] = L.mask[g];
    }
    __syncthreads();
}

// one red-black half-sweep of colour `colour` on the region ring >= SHRINK. On
// even-sized levels the colour of a region cell follows from its region
// coordinates (a wrap by an even size keeps the parity), so only the cells of
// that colour are visited; odd-sized levels test each cell.
template <class S, int SHRINK>
__device__ void tile_half_sweep_t(const HLevel& L, int i0, int j0, TileRefs t, int colour) {
    constexpr int RW = S::RW, RH = S::RH;
    constexpr int ROWS = RH - 2 * SHRINK, COLS = RW - 2 * SHRINK;
    constexpr int HALF = (COLS + 1) / 2;
    const bool even = ((L.nx | L.ny) & 1) == 0;
    if (even) {
        for (int q = threadIdx.x; q < ROWS * HALF; q += blockDim.x) {
            const int rj = SHRINK + q / HALF;
            const int ri = SHRINK + ((colour - i0 - j0 - rj - SHRINK) & 1) + 2 * (q % HALF);
            if (ri >= RW - SHRINK) continue;
            const int r = rj * RW + ri;
            const double nb = L.cx * (t.ku[r] * t.x[r + 1] + t.ku[r - 1] * t.x[r - 1]) +
                              L.cy * (t.kv[r] * t.x[r + RW] + t.kv[r - RW] * t.x[r - RW]);
            t.x[r] = t.id[r] * (t.b[r] + nb) * t.m[r];
        }
    } else {
        for (int r = threadIdx.x; r < S::RN; r += blockDim.x) {
            const int rj = r / RW, ri = r - rj * RW;
            if (ri < SHRINK || ri >= RW - SHRINK || rj < SHRINK || rj >= RH - SHRINK) continue;
            const int gi = wrap_any(i0 - HALO + ri, L.nx), gj = wrap_any(j0 - HALO + rj, L.ny);
            if (((gi + gj) & 1) != colour) continue;
            const double nb = L.cx * (t.ku[r] * t.x[r + 1] + t.ku[r - 1] * t.x[r - 1]) +
                              L.cy * (t.kv[r] * t.x[r + RW] + t.kv[r - RW] * t.x[r - RW]);
            t.x[r] = t.id[r] * (t.b[r] + nb) * t.m[r];
        }
    }
    __syncthreads();
}

// four half-sweeps with colours c0, 1 - c0, c0, 1 - c0 on a region shrinking by one ring each
template <class S>
__device__ __forceinline__ void tile_four_half_sweeps(const HLevel& L, int i0, int j0, TileRefs t, int c0) {
    tile_half_sweep_t<S, 1>(L, i0, j0, t, c0);
    tile_half_sweep_t<S, 2>(L, i0, j0, t, 1 - c0);
    tile_half_sweep_t<S, 3>(L, i0, j0, t, c0);
    tile_half_sweep_t<S, 4>(L, i0, j0, t, 1 - c0);
}

// (b - A x) * mask at region cell r (VarOperator.apply, solvers_var.py:47-53)
template <class S>
__device__ __forceinline__ double tile_residual(const HLevel& L, double coef, TileRefs t, int r) {
    constexpr int RW = S::RW;
    const double m = t.m[r];
    const double xm = t.x[r] * m;
    const double xe = t.x[r + 1] * t.m[r + 1];
    const double xw = t.x[r - 1] * t.m[r - 1];
    const double xn = t.x[r + RW] * t.m[r + RW];
    const double xs = t.x[r - RW] * t.m[r - RW];
    const double fx = t.ku[r] * (xe - xm);
    const double fxw = t.ku[r - 1] * (xm - xw);
    const double fy = t.kv[r] * (xn - xm);
    const double fys = t.kv[r - RW] * (xm - xs);
    const double lap = (fx - fxw) / L.dx2 + (fy - fys) / L.dy2;
    const double ax = (xm - coef * lap) * m + xm * (1.0 - m);
    return (t.b[r] - ax) * m;
}

template <class S>
__device__ void tile_store_x(const HLevel& L, int i0, int j0, TileRefs t, double* xout) {
    for (int r = threadIdx.x; r < S::TX * S::TY; r += blockDim.x) {
        const int cj = r / S::TX, ci = r - cj * S::TX;
        const int gi = i0 + ci, gj = j0 + cj;
        if (gi >= L.nx || gj >= L.ny) continue;
        xout[gj * L.nx + gi] = t.x[(cj + HALO) * S::RW + ci + HALO];
    }
}

// down phase of level l: pre-smoothing, restricted residual into level l+1
// (solvers_var.py:141-147); x of level l+1 starts at zero implicitly
template <class S>
__device__ void mg_down(const HelmParams& H, int l, const double* xin, double* xout, double* smem,
                        double* persist = nullptr) {
    const HLevel& L = H.lv[l];
    const HLevel& C = H.lv[l + 1];
    const int tx = (L.nx + S::TX - 1) / S::TX, ty = (L.ny + S::TY - 1) / S::TY;
    const bool keep = persist != nullptr;
    TileRefs t = keep ? tile_refs_persist<S>(persist, smem) : tile_refs<S>(smem);
    for (int tile = keep ? level0_tile_of_cta(tx * ty) : s_grid.cta; tile < tx * ty; tile += s_grid.ncta) {
        if (tile < 0) continue;  // CTA-uniform: this CTA holds no persistent tile
        const int i0 = (tile % tx) * S::TX, j0 = (tile / tx) * S::TY;
        tile_load<S>(L, i0, j0, xin, nullptr, t, !keep);
        tile_four_half_sweeps<S>(L, i0, j0, t, 0);
        constexpr int NC = (S::TX / 2) * (S::TY / 2);  // coarse cells of the tile
        if constexpr (4 * NC <= 1024 && (4 * NC) % 32 == 0 && S::TX != TileWide::TX) {
            // four lanes per coarse cell, one child residual each, summed by the
            // first of them in the order a + b + c + d (the loop bound is a
            // multiple of 32, so whole warps take part in the shuffles)
            for (int q = threadIdx.x; q < 4 * NC; q += blockDim.x) {
                const int r = q >> 2, child = q & 3;
                const int cj = r / (S::TX / 2), ci = r - cj * (S::TX / 2);
                const int I = i0 / 2 + ci, J = j0 / 2 + cj;
                const int rr = (HALO + 2 * cj + (child >> 1)) * S::RW + HALO + 2 * ci + (child & 1);
                const double val = tile_residual<S>(L, H.coef, t, rr);
                const double b = __shfl_down_sync(0xffffffffu, val, 1);
                const double c = __shfl_down_sync(0xffffffffu, val, 2);
                const double d = __shfl_down_sync(0xffffffffu, val, 3);
                if (child == 0 && I < C.nx && J < C.ny) C.b[J * C.nx + I] = 0.25 * (val + b + c + d);
            }
        } else {
            for (int r = threadIdx.x; r < NC; r += blockDim.x) {
                const int cj = r / (S::TX / 2), ci = r - cj * (S::TX / 2);
                const int I = i0 / 2 + ci, J = j0 / 2 + cj;
                if (I >= C.nx || J >= C.ny) continue;
                const int r00 = (HALO + 2 * cj) * S::RW + HALO + 2 * ci;
                const double a = tile_residual<S>(L, H.coef, t, r00);
                const double b = tile_residual<S>(L, H.coef, t, r00 + 1);
                const double c = tile_residual<S>(L, H.coef, t, r00 + S::RW);
                const double d = tile_residual<S>(L, H.coef, t, r00 + S::RW + 1);
                C.b[J * C.nx + I] = 0.25 * (a + b + c + d);
            }
        }
        tile_store_x<S>(L, i0, j0, t, xout);
        __syncthreads();
    }
}

// up phase of level l: x + prolong(x_coarse) * mask, then the two reverse sweeps
// (solvers_var.py:148-150). With `leaves`, level 0's tiles are one NumPy leaf
// per interior row (128 cells starting at a multiple of 128): after the sweeps
// every interior cell and its four neighbours hold the new x, so each warp forms
// the squared residual (b - A x)^2 of one row and its leaf sum in NumPy's order
// -- the per-cycle residual norm without another pass over the grid.
template <class S>
__device__ void mg_up(const HelmParams& H, int l, const double* xin, const HLevel& C, double* xout,
                      double* smem, double* leaves, double* persist = nullptr) {
    const HLevel& L = H.lv[l];
    const int tx = (L.nx + S::TX - 1) / S::TX, ty = (L.ny + S::TY - 1) / S::TY;
    const bool keep = persist != nullptr;
    TileRefs t = keep ? tile_refs_persist<S>(persist, smem) : tile_refs<S>(smem);
    for (int tile = keep ? level0_tile_of_cta(tx * ty) : s_grid.cta; tile < tx * ty; tile += s_grid.ncta) {
        if (tile < 0) continue;  // CTA-uniform: this CTA holds no persistent tile
        const int i0 = (tile % tx) * S::TX, j0 = (tile / tx) * S::TY;
        tile_load<S>(L, i0, j0, xin, &C, t, !keep);
        tile_four_half_sweeps<S>(L, i0, j0, t, 1);
        tile_store_x<S>(L, i0, j0, t, xout);
        if constexpr (S::TX == 128) {
            if (leaves) {
                const int lane = threadIdx.x & 31;
                for (int cj = threadIdx.x >> 5; cj < S::TY; cj += blockDim.x >> 5) {
                    if (j0 + cj >= L.ny) continue;  // warp-uniform
                    double va[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const double d = tile_residual<S>(L, H.coef, t, (cj + HALO) * S::RW + HALO + lane + 32 * q);
                        va[q] = d * d;
                    }
                    const double a = leaf_sum_warp(va, 128);
                    if (lane == 0) leaves[((j0 + cj) * L.nx + i0) / 128] = a;
                }
            }
        }
        __syncthreads();
    }
}

// ---- coarse levels: all of them inside CTA 0, in shared memory
struct CoarseRefs {
    double *x, *b, *ku, *kv, *id, *m;
};

// the coarse levels' arrays take 6 x (sum of their cells) doubles; the restriction
// scratch (one value per cell of the first coarse level) follows them
__device__ __forceinline__ double* coarse_scratch(const HelmParams& H, double* base) {
    int tot = 0;
    for (int q = H.coarse_from; q < H.n_levels; ++q) tot += H.lv[q].n;
    return base + 6 * tot;
}

// coef: where ku, kv, id and m live when they persist for the solve (CTA 0's
// persistent region), else null (they follow x and b in `base`)
__device__ __forceinline__ CoarseRefs coarse_refs(const HelmParams& H, double* base, int l,
                                                  double* coef = nullptr) {
    int off = 0, tot = 0;
    for (int q = H.coarse_from; q < H.n_levels; ++q) {
        if (q < l) off += H.lv[q].n;
        tot += H.lv[q].n;
    }
    double* cb = coef ? coef : base + 2 * tot;
    CoarseRefs c;
    c.x = base + off;
    c.b = base + tot + off;
    c.ku = cb + off;
    c.kv = cb + tot + off;
    c.id = cb + 2 * tot + off;
    c.m = cb + 3 * tot + off;
    return c;
}

// the coarse levels' coefficients into `coef` (asynchronous copies; the caller
// waits for them before its next CTA barrier)
__device__ void coarse_coef_load(const HelmParams& H, double* coef, double* base) {
    for (int l = H.coarse_from; l < H.n_levels; ++l) {
        const HLevel& L = H.lv[l];
        CoarseRefs s = coarse_refs(H, base, l, coef);
        for (int e = threadIdx.x; e < L.n; e += blockDim.x) {
            cpa_ca8(s.ku + e, L.Ku + e);
            cpa_ca8(s.kv + e, L.Kv + e);
            cpa_ca8(s.id + e, L.inv_diag + e);
            cpa_ca8(s.m + e, L.mask + e);
        }
    }
}

// Gauss-Seidel update of coarse cell (i, j) = e; with C, the neighbours carry
// the coarse correction x + prolong(e) * mask (the first reverse half-sweep)
__device__ __forceinline__ void coarse_cell_update(const HLevel& L, CoarseRefs s, int i, int j, int e,
                                                   const CoarseRefs* C, const HLevel* LC) {
    const int nx = L.nx;
    const int i_e = i + 1 == nx ? 0 : i + 1, i_w = i == 0 ? nx - 1 : i - 1;
    const int j_n = j + 1 == L.ny ? 0 : j + 1, j_s = j == 0 ? L.ny - 1 : j - 1;
    const int ie = j * nx + i_e, iw = j * nx + i_w, jn = j_n * nx + i, js = j_s * nx + i;
    double xe = s.x[ie], xw = s.x[iw], xn = s.x[jn], xs = s.x[js];
    if (C) {
        const int cnx = LC->nx;
        xe = xe + C->x[(j >> 1) * cnx + (i_e >> 1)] * s.m[ie];
        xw = xw + C->x[(j >> 1) * cnx + (i_w >> 1)] * s.m[iw];
        xn = xn + C->x[(j_n >> 1) * cnx + (i >> 1)] * s.m[jn];
        xs = xs + C->x[(j_s >> 1) * cnx + (i >> 1)] * s.m[js];
    }
    const double nb = L.cx * (s.ku[e] * xe + s.ku[iw] * xw) + L.cy * (s.kv[e] * xn + s.kv[js] * xs);
    s.x[e] = s.id[e] * (s.b[e] + nb) * s.m[e];
}

// one colour of a coarse-level sweep by the CTA. On even-sized levels only the
// cells of that colour are visited (cell q of the colour: row q / (nx/2), column
// 2 (q mod nx/2) + the row's parity offset); odd-sized levels test each cell.
__device__ void coarse_half_sweep(const HLevel& L, CoarseRefs s, int colour, const CoarseRefs* C,
                                  const HLevel* LC) {
    const int nx = L.nx;
    if (((nx | L.ny) & 1) == 0) {
        const int hx = nx >> 1, nh = L.n >> 1;
        for (int q = threadIdx.x; q < nh; q += blockDim.x) {
            const int j = q / hx;
            const int i = 2 * (q - j * hx) + ((j + colour) & 1);
            coarse_cell_update(L, s, i, j, j * nx + i, C, LC);
        }
    } else {
        for (int e = threadIdx.x; e < L.n; e += blockDim.x) {
            const int j = e / nx, i = e - j * nx;
            if (((i + j) & 1) != colour) continue;
            coarse_cell_update(L, s, i, j, e, C, LC);
        }
    }
    __syncthreads();
}

__device__ double coarse_residual(const HLevel& L, double coef, CoarseRefs s, int e) {
    const int j = e / L.nx, i = e - j * L.nx;
    const int ie = j * L.nx + (i + 1 == L.nx ? 0 : i + 1), iw = j * L.nx + (i == 0 ? L.nx - 1 : i - 1);
    const int jn = (j + 1 == L.ny ? 0 : j + 1) * L.nx + i, js = (j == 0 ? L.ny - 1 : j - 1) * L.nx + i;
    const double m = s.m[e];
    const double xm = s.x[e] * m, xe = s.x[ie] * s.m[ie], xw = s.x[iw] * s.m[iw];
    const double xn = s.x[jn] * s.m[jn], xs = s.x[js] * s.m[js];
    const double fx = s.ku[e] * (xe - xm), fxw = s.ku[iw] * (xm - xw);
    const double fy = s.kv[e] * (xn - xm), fys = s.kv[js] * (xm - xs);
    const double lap = (fx - fxw) / L.dx2 + (fy - fys) / L.dy2;
    const double ax = (xm - coef * lap) * m + xm * (1.0 - m);
    return (s.b[e] - ax) * m;
}

// the V-cycle below and including level cf, by CTA 0 alone; reads level cf's b
// (and x when cf is the finest level) from global memory, writes level cf's x
// coef: the coarse coefficients kept for the whole solve (coarse_coef_load at its
// start), or null to load them here
__device__ void mg_coarse(const HelmParams& H, double* smem, const double* xin_cf, double* xout_cf,
                          double* coef = nullptr) {
    const int cf = H.coarse_from, nl = H.n_levels;
    // the level coefficients (constant during the solve) by asynchronous copies, all
    // in flight at once; level cf's b and x (written by this launch) through L2
    if (!coef) coarse_coef_load(H, nullptr, smem);
    {
        const HLevel& L = H.lv[cf];
        CoarseRefs s = coarse_refs(H, smem, cf, coef);
        for (int e = threadIdx.x; e < L.n; e += blockDim.x) {
            const double bv = __ldcg(L.b + e);
            const double xv = xin_cf ? __ldcg(xin_cf + e) : 0.0;
            s.b[e] = bv;
            s.x[e] = xv;
        }
    }
    cpa_wait_all();
    __syncthreads();
    for (int l = cf; l < nl; ++l) {
        const HLevel& L = H.lv[l];
        CoarseRefs s = coarse_refs(H, smem, l, coef);
        for (int h = 0; h < 4; ++h) coarse_half_sweep(L, s, h & 1, nullptr, nullptr);
        if (l + 1 < nl) {
            // the residual of every cell of level l (a coarser level exists only
            // below an even-sized one, so they are exactly the 2x2 children),
            // then the children's mean per coarse cell
            const HLevel& C = H.lv[l + 1];
            CoarseRefs c = coarse_refs(H, smem, l + 1, coef);
            double* res = coarse_scratch(H, smem);
            for (int f = threadIdx.x; f < L.n; f += blockDim.x) res[f] = coarse_residual(L, H.coef, s, f);
            __syncthreads();
            for (int e = threadIdx.x; e < C.n; e += blockDim.x) {
                const int J = e / C.nx, I = e - J * C.nx;
                const int f00 = (2 * J) * L.nx + 2 * I;
                c.b[e] = 0.25 * (res[f00] + res[f00 + 1] + res[f00 + L.nx] + res[f00 + L.nx + 1]);
                c.x[e] = 0.0;
            }
            __syncthreads();
        }
    }
    {  // the coarsest level: its reverse sweeps follow the forward ones directly
        const HLevel& L = H.lv[nl - 1];
        CoarseRefs s = coarse_refs(H, smem, nl - 1, coef);
        for (int h = 0; h < 4; ++h) coarse_half_sweep(L, s, 1 - (h & 1), nullptr, nullptr);
    }
    for (int l = nl - 2; l >= cf; --l) {
        const HLevel& L = H.lv[l];
        CoarseRefs s = coarse_refs(H, smem, l, coef);
        CoarseRefs c = coarse_refs(H, smem, l + 1, coef);
        coarse_half_sweep(L, s, 1, &c, &H.lv[l + 1]);
        coarse_half_sweep(L, s, 0, nullptr, nullptr);
        coarse_half_sweep(L, s, 1, nullptr, nullptr);
        coarse_half_sweep(L, s, 0, nullptr, nullptr);
    }
    const HLevel& L = H.lv[cf];
    CoarseRefs s = coarse_refs(H, smem, cf, coef);
    for (int e = threadIdx.x; e < L.n; e += blockDim.x) xout_cf[e] = s.x[e];
    __syncthreads();
}

// smoothing only (the coarsest level when it is too large for CTA 0): two
// forward or two reverse sweeps
__device__ void mg_smooth(const HelmParams& H, int l, const double* xin, double* xout, bool reverse,
                          double* smem) {
    const HLevel& L = H.lv[l];
    const int tx = (L.nx + Tile32::TX - 1) / Tile32::TX, ty = (L.ny + Tile32::TY - 1) / Tile32::TY;
    TileRefs t = tile_refs<Tile32>(smem);
    for (int tile = s_grid.cta; tile < tx * ty; tile += s_grid.ncta) {
        const int i0 = (tile % tx) * Tile32::TX, j0 = (tile / tx) * Tile32::TY;
        tile_load<Tile32>(L, i0, j0, xin, nullptr, t);
        tile_four_half_sweeps<Tile32>(L, i0, j0, t, reverse ? 1 : 0);
        tile_store_x<Tile32>(L, i0, j0, t, xout);
        __syncthreads();
    }
}

// one V(2,2) cycle on x0 (level 0's current x); returns the buffer holding the
// new x (x0 or level 0's second buffer). Levels below coarse_from have a grid
// down and up phase; the rest run in CTA 0, or, when every level is too large
// for it, the coarsest level is smoothed on the grid.
__device__ double* vcycle_tiled(const HelmParams& H, double* x0, double* x0b, double* smem, double* persist,
                                bool& ok) {
    const int cf = H.coarse_from, nl = H.n_levels;
    // CTA 0 keeps the coarse coefficients in its persistent region when it holds no level-0 tile
    double* ccoef = (H.coarse_persist && s_grid.cta == 0) ? persist : nullptr;
    if (cf == 0) {
        if (s_grid.cta == 0) mg_coarse(H, smem, x0, x0b);
        ok = grid_sync(H);
        return x0b;
    }
    const int ndown = cf < nl ? cf : nl - 1;
    for (int l = 0; l < ndown && ok; ++l) {
        const double* xin = l == 0 ? x0 : nullptr;
        double* xout = l == 0 ? x0b : H.lv[l].x;
        switch (H.lv[l].shape) {
            case SHAPE_WIDE: mg_down<TileWide>(H, l, xin, xout, smem, l == 0 ? persist : nullptr); break;
            case SHAPE_3216: mg_down<Tile3216>(H, l, xin, xout, smem); break;
            case SHAPE_16: mg_down<Tile16>(H, l, xin, xout, smem); break;
            case SHAPE_8: mg_down<Tile8>(H, l, xin, xout, smem); break;
            default: mg_down<Tile32>(H, l, xin, xout, smem); break;
        }
        ok = grid_sync(H);
    }
    if (!ok) return x0;
    if (cf < nl) {
        if (s_grid.cta == 0) mg_coarse(H, smem, nullptr, H.lv[cf].x2, ccoef);
        ok = grid_sync(H);
    } else {
        const int l = nl - 1;
        double* xa = (l == 0) ? x0b : H.lv[l].x;
        double* xb = (l == 0) ? x0 : H.lv[l].x2;
        mg_smooth(H, l, l == 0 ? x0 : nullptr, xa, false, smem);
        ok = grid_sync(H);
        if (!ok) return x0;
        mg_smooth(H, l, xa, xb, true, smem);
        ok = grid_sync(H);
        if (l == 0) return x0;
    }
    // ascend: level l reads its down-phase result and level l+1's final x (in x2)
    for (int l = ndown - 1; l >= 0 && ok; --l) {
        const double* xin = (l == 0) ? x0b : H.lv[l].x;
        double* xout = (l == 0) ? x0 : H.lv[l].x2;
        HLevel C = H.lv[l + 1];
        C.x = H.lv[l + 1].x2;
        switch (H.lv[l].shape) {
            case SHAPE_WIDE:
                mg_up<TileWide>(H, l, xin, C, xout, smem, H.fused_res ? H.leafA : nullptr, l == 0 ? persist : nullptr);
                break;
            case SHAPE_3216: mg_up<Tile3216>(H, l, xin, C, xout, smem, nullptr); break;
            case SHAPE_16: mg_up<Tile16>(H, l, xin, C, xout, smem, nullptr); break;
            case SHAPE_8: mg_up<Tile8>(H, l, xin, C, xout, smem, nullptr); break;
            default: mg_up<Tile32>(H, l, xin, C, xout, smem, nullptr); break;
        }
        ok = grid_sync(H);
    }
    return x0;
}

// ------------------------------------------------------------------ the solve kernel
// A whole solve on the CTAs s_grid names (set by the kernel, followed by a CTA
// barrier, before the call).
__device__ __forceinline__ void helm_solve_body(const HelmParams& H, double* smem_all) {
    // with H.persist0 the first 4 RN doubles hold level 0's coefficient tile for the
    // whole solve; every other use of shared memory works above them
    double* persist = H.persist0 ? smem_all : nullptr;
    double* const ops_base = smem_all + (H.persist0 ? 4 * TileWide::RN : 0);
    double* sm = ops_base + H.ops_smem;
    FoldPlan fold{H.ops, H.height_start};
    if (H.ops_smem) {
        int2* so = reinterpret_cast<int2*>(ops_base);
        int* sh = reinterpret_cast<int*>(so + H.n_ops);
        for (int t = threadIdx.x; t < H.n_ops; t += blockDim.x) so[t] = H.ops[t];
        for (int t = threadIdx.x; t <= H.n_heights; t += blockDim.x) sh[t] = H.height_start[t];
        fold = FoldPlan{so, sh};  // first read after the barrier that ends the first leaf phase
    }
    const HLevel& L0 = H.lv[0];
    const double* rhs = H.rhs;
    double* x = L0.x;
    double* b0 = L0.b;
    bool ok = true;
    int iters = 0, conv = 1;
    grid_sync_begin(H);

    // norm of the masked right-hand side (solvers_var.py:163-168)
    leaf_phase(H,
               [&](int e) {
                   const double r = rhs[e] * L0.mask[e];
                   b0[e] = r;
                   // the CG residual of the starting iterate: b, or b - A x with a warm start
                   if (H.kind <= HK_PCG_RBGS || H.kind == HK_PCG_MG)
                       H.r[e] = H.warm ? r - apply_at(L0, H.coef, x, cell_of(L0, e)) : r;
                   if (!H.warm) x[e] = 0.0;
                   return make_double2(r * r, 0.0);
               },
               H.leafA, nullptr);
    ok = grid_sync(H);
    const double norm_b = ok ? sqrt(fold_sum(H, fold, H.leafA, sm, ok)) : 0.0;
    if (persist) persist_level0(H, persist);  // the coefficients are fixed during the solve
    if (H.coarse_persist && s_grid.cta == 0) {
        coarse_coef_load(H, persist, sm);
        cpa_wait_all();
        __syncthreads();
    }
    if (!ok || norm_b == 0.0) goto done;
    {
        const double tol = H.rtol * norm_b;
        if (H.kind == HK_RBGS || H.kind == HK_MULTIGRID) {
            // stationary iteration with the true residual (solvers_var.py:170-179)
            conv = 0;
            double* xc = x;  // the level-0 buffer holding the current iterate
            for (int it = 1; it <= H.max_iter && ok; ++it) {
                if (H.kind == HK_MULTIGRID) {
                    xc = vcycle_tiled(H, xc, xc == H.lv[0].x ? H.lv[0].x2 : H.lv[0].x, sm, persist, ok);
                } else {
                    colour_phase(L0, x, b0, 0, grid_team());
                    ok = grid_sync(H);
                    if (!ok) break;
                    colour_phase(L0, x, b0, 1, grid_team());
                    ok = grid_sync(H);
                }
                if (!ok) break;
                // the true residual's leaf sums: formed by the last up phase when
                // level 0's tiles are NumPy's leaves, else by a pass of their own
                if (!(H.kind == HK_MULTIGRID && H.fused_res)) {
                    const double* xr = xc;
                    leaf_phase(H,
                               [&](int e) {
                                   const double d = __ldcg(b0 + e) - apply_at(L0, H.coef, xr, cell_of(L0, e));
                                   return make_double2(d * d, 0.0);
                               },
                               H.leafA, nullptr);
                    ok = grid_sync(H);
                    if (!ok) break;
                }
                iters = it;
                const double res = sqrt(fold_sum(H, fold, H.leafA, sm, ok));
                if (!ok) break;
                if (res <= tol) {
                    conv = 1;
                    break;
                }
            }
            if (ok && xc != x) {
                for (int e = grid_team().first; e < L0.n; e += grid_team().stride) x[e] = __ldcg(xc + e);
            }
        } else {
            // preconditioned CG (solvers_var.py:181-197). A fold reads its leaf
            // sums after a grid barrier, and a leaf phase that follows a fold with
            // no barrier between them writes a different buffer: a CTA that leaves
            // its fold early must not overwrite sums another CTA is still reading.
            // <r,z> at the start: leafB (leafA holds |b|); <p,Ap>: leafC; <r,r>
            // and <r,z> of the update: leafA and leafB, read last before the
            // barrier that ends the previous iteration.
            double* r = H.r;
            double* z = H.z;
            double* p = H.p;
            double* Ap = H.Ap;
            const bool jac = H.kind == HK_PCG_JACOBI;
            // z = M^-1 r
            auto precondition = [&](bool& okp) {
                if (jac) return;
                if (H.kind == HK_PCG_MG) {
                    // one V(2,2) cycle on level 0's rhs r from a zero iterate (symmetric:
                    // red-black pre-smoothing, black-red post-smoothing)
                    for (int e = grid_team().first; e < L0.n; e += grid_team().stride) {
                        b0[e] = __ldcg(r + e);
                        z[e] = 0.0;
                    }
                    okp = grid_sync(H);
                    if (!okp) return;
                    double* zr = vcycle_tiled(H, z, L0.x2, sm, persist, okp);
                    if (!okp || zr == z) return;
                    for (int e = grid_team().first; e < L0.n; e += grid_team().stride) z[e] = __ldcg(zr + e);
                    okp = grid_sync(H);
                    return;
                }
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
                       H.leafB, nullptr);
            ok = grid_sync(H);
            if (!ok) goto done;
            double rz = fold_sum(H, fold, H.leafB, sm, ok);
            if (!ok) goto done;
            conv = 0;
            for (int it = 1; it <= H.max_iter; ++it) {
                leaf_phase(H,
                           [&](int e) {
                               const double a = apply_at(L0, H.coef, p, cell_of(L0, e));
                               Ap[e] = a;
                               return make_double2(__ldcg(p + e) * a, 0.0);
                           },
                           H.leafC, nullptr);
                ok = grid_sync(H);
                if (!ok) break;
                const double alpha = rz / fold_sum(H, fold, H.leafC, sm, ok);
                if (!ok) break;
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
                const double res = sqrt(fold_sum(H, fold, H.leafA, sm, ok));
                if (!ok) break;
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
                const double rz_new = fold_sum(H, fold, H.leafB, sm, ok);
                if (!ok) break;
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
    grid_sync_end(H.bar_count, s_grid.cta == 0);
    if (s_grid.cta == 0 && threadIdx.x == 0) {
        const int idx = *H.log_count;
        if (idx < H.log_cap) {
            H.log_iters[idx] = ok ? iters : -1;
            H.log_conv[idx] = ok ? conv : 0;
        }
        *H.log_count = idx + 1;
    }
}

// The parameters are read through a reference throughout the solve: a copy in
// shared memory, made once per CTA (a reference to the kernel parameter itself
// would give every thread a copy of its own in local memory).
__global__ void __launch_bounds__(512) k_helm_solve(HelmParams H) {
    extern __shared__ double smem_all[];
    __shared__ HelmParams sH;
    if (threadIdx.x == 0) s_grid = SolveGrid{(int)blockIdx.x, (int)gridDim.x};
    const int* src = reinterpret_cast<const int*>(&H);
    int* dst = reinterpret_cast<int*>(&sH);
    for (int t = threadIdx.x; t < (int)(sizeof(HelmParams) / sizeof(int)); t += blockDim.x) dst[t] = src[t];
    __syncthreads();
    helm_solve_body(sH, smem_all);
}

// Several systems in one cooperative launch: system m runs on CTAs
// [cta_start[m], cta_start[m + 1]) with its own parameters (copied into shared
// memory), its own barrier counter, status word and solve log; the systems
// never wait on one another.
__global__ void __launch_bounds__(512) k_helm_solve_batched(const HelmParams* __restrict__ systems,
                                                            const int* __restrict__ cta_start, int n) {
    extern __shared__ double smem_all[];
    __shared__ HelmParams sH;
    __shared__ int s_m;
    if (threadIdx.x == 0) {
        int m = 0;
        while (m + 1 < n && (int)blockIdx.x >= cta_start[m + 1]) ++m;
        s_m = m;
        s_grid = SolveGrid{(int)blockIdx.x - cta_start[m], cta_start[m + 1] - cta_start[m]};
    }
    __syncthreads();
    const int* src = reinterpret_cast<const int*>(systems + s_m);
    int* dst = reinterpret_cast<int*>(&sH);
    for (int t = threadIdx.x; t < (int)(sizeof(HelmParams) / sizeof(int)); t += blockDim.x) dst[t] = src[t];
    __syncthreads();
    helm_solve_body(sH, smem_all);
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

// P > 0 when the tree over the leaves is perfect -- 2^m leaves, the nodes of
// height h (0: pairs of leaves) exactly (i, i + 2^h) for i a multiple of 2^(h+1)
// -- with at least 32 leaves: the leaves per lane of perfect_fold for `warps`
// warps (at most 16); 0 otherwise
static int perfect_lanes(int n, const std::vector<std::vector<int2>>& by_height, int warps) {
    if (n < 32 || (n & (n - 1)) != 0) return 0;
    int m = 0;
    while ((1 << m) < n) ++m;
    if ((int)by_height.size() != m) return 0;
    for (int h = 0; h < m; ++h) {
        std::vector<int2> ops = by_height[h];
        const int step = 1 << (h + 1);
        if ((int)ops.size() != n / step) return 0;
        std::sort(ops.begin(), ops.end(), [](int2 a, int2 b) { return a.x < b.x; });
        for (int q = 0; q < (int)ops.size(); ++q)
            if (ops[q].x != q * step || ops[q].y != q * step + (1 << h)) return 0;
    }
    const int P = std::max(1, n / (32 * warps));
    return P <= 16 ? P : 0;
}

// leaves of NumPy's pairwise tree over n contiguous elements
static long pairwise_leaves(long n) {
    if (n <= 128) return 1;
    long h = n / 2;
    h -= h % 8;
    return pairwise_leaves(h) + pairwise_leaves(n - h);
}

// The two-level form of the same tree: nodes of at most `block_leaves` leaves
// become blocks, each with its own plan (leaf indices relative to its first
// leaf; `hstart` gets heights + 1 offsets into `bops` per block), and the nodes
// above them form the top plan over the block indices. `leaves` receives every
// leaf in order, as pairwise_build gives them.
struct TwoLevelPlan {
    std::vector<int> leaves;
    std::vector<int4> blocks;
    std::vector<int2> bops;
    std::vector<int> bh_start;
    std::vector<std::vector<int2>> top_by_height;
};

static PwNode pairwise_build_two_level(long start, long n, long block_leaves, TwoLevelPlan& T) {
    if (pairwise_leaves(n) <= block_leaves) {
        std::vector<int> lv;
        std::vector<std::vector<int2>> byh;
        pairwise_build(start, n, lv, byh);
        const int4 b = make_int4((int)T.leaves.size(), (int)lv.size(), (int)T.bh_start.size(), (int)byh.size());
        T.leaves.insert(T.leaves.end(), lv.begin(), lv.end());
        for (const auto& ops : byh) {
            T.bh_start.push_back((int)T.bops.size());
            T.bops.insert(T.bops.end(), ops.begin(), ops.end());
        }
        T.bh_start.push_back((int)T.bops.size());
        T.blocks.push_back(b);
        return {(int)T.blocks.size() - 1, 0};
    }
    long h = n / 2;
    h -= h % 8;
    const PwNode a = pairwise_build_two_level(start, h, block_leaves, T);
    const PwNode b = pairwise_build_two_level(start + h, n - h, block_leaves, T);
    const int height = std::max(a.height, b.height) + 1;
    if ((int)T.top_by_height.size() < height) T.top_by_height.resize(height);
    T.top_by_height[height - 1].push_back(make_int2(a.lo, b.lo));
    return {a.lo, height};
}

// leaf sums beyond which the fold runs in two levels (their doubles would not
// fit one CTA's shared memory beside the rest), and the leaves of one block
static constexpr long kFoldOneLevelLeaves = 16384;
static constexpr long kFoldBlockLeaves = 8192;

void* HelmSolver::dalloc(size_t nbytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, nbytes) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, nbytes);
    allocs_.push_back(p);
    bytes_ += nbytes;
    return p;
}

HelmSolver::~HelmSolver() {
    delete refined_;
    for (void* p : allocs_) cudaFree(p);
}

int HelmSolver::init(int nx, int ny, double dx0, double dy0, double coef, int kind, double rtol,
                     int max_iter, const double* mask_host, double* Ku, double* Kv, int log_cap,
                     int* status, std::string& err) {
    HelmParams& H = hp_;
    // the refined solver keeps this solver's log, counters and level-0 arrays
    // (built as for PCG-Jacobi) and runs its solves itself
    const bool refined = kind == HK_REFINED;
    if (refined) kind = HK_PCG_JACOBI;
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
    const bool mg_levels = kind == HK_MULTIGRID || kind == HK_PCG_MG;
    if (mg_levels) {
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
        // coarse level l spans the same length with nx / 2^l cells: Lx / (nx / 2^l)
        // is exactly (Lx / nx) * 2^l, the reference's CGrid spacing of that level
        const double dx = std::ldexp(dx0, l), dy = std::ldexp(dy0, l);
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
        L.x2 = (double*)dalloc(sizeof(double) * L.n);
        if (l == 0) {
            L.Ku = Ku;
            L.Kv = Kv;
            L.x = nullptr;  // set per solve
        } else {
            L.Ku = (double*)dalloc(sizeof(double) * L.n);
            L.Kv = (double*)dalloc(sizeof(double) * L.n);
            L.x = (double*)dalloc(sizeof(double) * L.n);
        }
        if (!L.inv_diag || !L.b || !L.x2 || (l > 0 && (!L.Ku || !L.Kv || !L.x))) {
            err = "cudaMalloc failed (Helmholtz levels)";
            return OC_ERR_CUDA;
        }
        if (L.n <= kCoarseCells && H.coarse_from == H.n_levels) H.coarse_from = l;
    }
    const size_t n = (size_t)nx * ny;
    H.r = (double*)dalloc(sizeof(double) * n);
    H.z = (double*)dalloc(sizeof(double) * n);
    H.p = (double*)dalloc(sizeof(double) * n);
    H.Ap = (double*)dalloc(sizeof(double) * n);
    // pairwise plan (two-level for grids whose leaf sums exceed shared memory)
    std::vector<int> leaves;
    std::vector<std::vector<int2>> by_height;
    TwoLevelPlan two;
    H.big_fold = pairwise_leaves((long)n) > kFoldOneLevelLeaves ? 1 : 0;
    if (H.big_fold) {
        pairwise_build_two_level(0, (long)n, kFoldBlockLeaves, two);
        leaves = two.leaves;
    } else {
        pairwise_build(0, (long)n, leaves, by_height);
    }
    leaves.push_back((int)n);
    std::vector<int> hstart{0};
    std::vector<int2> ops;
    for (auto& v : by_height) {
        ops.insert(ops.end(), v.begin(), v.end());
        hstart.push_back((int)ops.size());
    }
    H.n_leaves = (int)leaves.size() - 1;
    H.n_heights = (int)by_height.size();
    H.perfect_lanes = H.big_fold ? 0 : perfect_lanes(H.n_leaves, by_height, block_ / 32);
    int* d_leaves = (int*)dalloc(sizeof(int) * leaves.size());
    int* d_hstart = (int*)dalloc(sizeof(int) * hstart.size());
    int2* d_ops = (int2*)dalloc(sizeof(int2) * std::max<size_t>(1, ops.size()));
    H.leafA = (double*)dalloc(sizeof(double) * H.n_leaves);
    H.leafB = (double*)dalloc(sizeof(double) * H.n_leaves);
    H.leafC = (double*)dalloc(sizeof(double) * H.n_leaves);
    unsigned long long* bar = (unsigned long long*)dalloc(sizeof(unsigned long long));
    H.log_cap = log_cap;
    H.log_iters = (int*)dalloc(sizeof(int) * log_cap);
    H.log_conv = (int*)dalloc(sizeof(int) * log_cap);
    H.log_count = (int*)dalloc(sizeof(int));
    if (!H.r || !H.z || !H.p || !H.Ap || !d_leaves || !d_hstart || !d_ops || !H.leafA || !H.leafB || !H.leafC ||
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
    H.n_ops = (int)ops.size();
    H.bar_count = bar;
    H.wait_cycles = kBarrierCycles;
    size_t fold_doubles = (size_t)H.n_leaves;  // shared memory the fold needs
    if (H.big_fold) {
        H.n_blocks = (int)two.blocks.size();
        std::vector<int> top_hstart{0};
        std::vector<int2> top_ops;
        for (auto& v : two.top_by_height) {
            top_ops.insert(top_ops.end(), v.begin(), v.end());
            top_hstart.push_back((int)top_ops.size());
        }
        H.top_heights = (int)two.top_by_height.size();
        int4* d_blocks = (int4*)dalloc(sizeof(int4) * two.blocks.size());
        int2* d_bops = (int2*)dalloc(sizeof(int2) * std::max<size_t>(1, two.bops.size()));
        int* d_bh = (int*)dalloc(sizeof(int) * two.bh_start.size());
        int2* d_top = (int2*)dalloc(sizeof(int2) * std::max<size_t>(1, top_ops.size()));
        int* d_top_h = (int*)dalloc(sizeof(int) * top_hstart.size());
        H.broot = (double*)dalloc(sizeof(double) * 3 * (size_t)H.n_blocks);
        if (!d_blocks || !d_bops || !d_bh || !d_top || !d_top_h || !H.broot) {
            err = "cudaMalloc failed (Helmholtz reduction plan)";
            return OC_ERR_CUDA;
        }
        cudaMemcpy(d_blocks, two.blocks.data(), sizeof(int4) * two.blocks.size(), cudaMemcpyHostToDevice);
        if (!two.bops.empty())
            cudaMemcpy(d_bops, two.bops.data(), sizeof(int2) * two.bops.size(), cudaMemcpyHostToDevice);
        cudaMemcpy(d_bh, two.bh_start.data(), sizeof(int) * two.bh_start.size(), cudaMemcpyHostToDevice);
        if (!top_ops.empty())
            cudaMemcpy(d_top, top_ops.data(), sizeof(int2) * top_ops.size(), cudaMemcpyHostToDevice);
        cudaMemcpy(d_top_h, top_hstart.data(), sizeof(int) * top_hstart.size(), cudaMemcpyHostToDevice);
        H.blocks = d_blocks;
        H.bops = d_bops;
        H.bh_start = d_bh;
        H.top_ops = d_top;
        H.top_hstart = d_top_h;
        fold_doubles = (size_t)H.n_blocks;
        for (const int4& b : two.blocks) fold_doubles = std::max(fold_doubles, (size_t)b.y);
    }
    // co-resident grid for the cooperative launch
    int dev = 0, sms = 0, coop = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop) {
        err = "device does not support cooperative launches";
        return OC_ERR_UNSUPPORTED;
    }
    size_t coarse_cells = 0;
    for (int l = H.coarse_from; l < H.n_levels; ++l) coarse_cells += (size_t)H.lv[l].n;
    // Level 0 of a grid whose 32 x 32 tiles need more than one round over the SMs
    // runs 128 x 16 tiles instead. When NumPy's leaves are then exactly the tiles'
    // 128-cell rows, the last up phase forms the residual's leaf sums itself.
    const bool grid_levels = mg_levels && H.n_levels >= 2 && H.coarse_from >= 1;
    const long long tiles32 = (long long)((nx + 31) / 32) * ((ny + 31) / 32);
    H.wide0 = (grid_levels && nx % TileWide::TX == 0 && tiles32 > sms) ? 1 : 0;
    // every other grid level takes the smallest tile whose count fits one round
    // over the SMs: the phases are latency-bound, so less work per CTA is faster
    // as long as no CTA takes a second tile
    for (int l = 0; l < H.n_levels; ++l) {
        HLevel& L = H.lv[l];
        L.shape = SHAPE_32;
        if (!mg_levels) continue;
        if (l == 0 && H.wide0) {
            L.shape = SHAPE_WIDE;
            continue;
        }
        auto count = [&](int tx, int ty) { return (long long)((L.nx + tx - 1) / tx) * ((L.ny + ty - 1) / ty); };
        if (count(8, 8) <= sms) L.shape = SHAPE_8;
        else if (count(16, 16) <= sms) L.shape = SHAPE_16;
        else if (count(32, 16) <= sms) L.shape = SHAPE_3216;
    }
    // level 0's coefficients persist in shared memory when each wide tile has its own CTA
    const long long wide_tiles = (long long)((nx + TileWide::TX - 1) / TileWide::TX) * ((ny + TileWide::TY - 1) / TileWide::TY);
    H.persist0 = (H.wide0 && wide_tiles <= sms) ? 1 : 0;
    bool aligned = H.n_leaves > 0;
    for (int q = 0; q < H.n_leaves && aligned; ++q)
        aligned = leaves[q] == 128 * q && leaves[q + 1] - leaves[q] == 128;
    H.fused_res = (kind == HK_MULTIGRID && H.wide0 && aligned) ? 1 : 0;
    // shared memory: the persistent tile (if any), then the largest of the tree
    // fold, the grid levels' tiles and the coarse levels of CTA 0
    size_t tile_work = 0;
    const int n_grid = H.coarse_from < H.n_levels ? H.coarse_from : H.n_levels;
    auto rn_of = [](int shape) {
        switch (shape) {
            case SHAPE_WIDE: return TileWide::RN;
            case SHAPE_3216: return Tile3216::RN;
            case SHAPE_16: return Tile16::RN;
            case SHAPE_8: return Tile8::RN;
            default: return Tile32::RN;
        }
    };
    if (mg_levels) {
        for (int l = 0; l < n_grid; ++l)
            tile_work = std::max<size_t>(tile_work, (l == 0 && H.persist0 ? 2 : 6) * (size_t)rn_of(H.lv[l].shape));
        if (H.coarse_from >= H.n_levels) tile_work = std::max<size_t>(tile_work, 6 * (size_t)Tile32::RN);
    }
    const size_t coarse_work = 6 * coarse_cells + (H.coarse_from < H.n_levels ? (size_t)H.lv[H.coarse_from].n : 0);
    const size_t mg_work = mg_levels ? std::max<size_t>(tile_work, coarse_work) : 0;
    // in a batched launch a system has fewer CTAs than tiles: no persistent level-0
    // tile (its six arrays are loaded per tile instead) and no shared copy of the plan
    size_t tile_work_b = 0;
    if (mg_levels) {
        for (int l = 0; l < n_grid; ++l) tile_work_b = std::max<size_t>(tile_work_b, 6 * (size_t)rn_of(H.lv[l].shape));
        if (H.coarse_from >= H.n_levels) tile_work_b = std::max<size_t>(tile_work_b, 6 * (size_t)Tile32::RN);
    }
    const size_t mg_work_b = mg_levels ? std::max<size_t>(tile_work_b, coarse_work) : 0;
    smem_batched_ = sizeof(double) * std::max<size_t>(fold_doubles, mg_work_b);
    // the tree fold and the V-cycle never run at the same time: one region serves both
    smem_ = sizeof(double) * ((H.persist0 ? 4 * (size_t)TileWide::RN : 0) + std::max<size_t>(fold_doubles, mg_work));
    int smem_optin = 0;
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, k_helm_solve);  // static shared memory (the barrier's word) comes first
    // the fold's plan joins shared memory when it fits beside the rest
    const size_t plan_doubles = (sizeof(int2) * ops.size() + sizeof(int) * hstart.size() + sizeof(double) - 1) / sizeof(double);
    H.ops_smem = 0;
    if (!H.big_fold && smem_ + sizeof(double) * plan_doubles + fa.sharedSizeBytes <= (size_t)smem_optin) {
        H.ops_smem = (int)plan_doubles;
        smem_ += sizeof(double) * plan_doubles;
    }
    if (smem_ + fa.sharedSizeBytes > (size_t)smem_optin) {
        err = "Helmholtz grid too large for the single-pass reduction tree";
        return OC_ERR_UNSUPPORTED;
    }
    if (smem_ > 48 * 1024) {
        // the allowance belongs to the kernel on this device, not to this solver:
        // it only ever grows, so the solvers of other grids keep launching
        static std::mutex mu;
        static std::map<int, size_t> allowance;
        std::lock_guard<std::mutex> lock(mu);
        size_t& a = allowance[dev];
        if (smem_ > a) {
            cudaFuncSetAttribute(k_helm_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_);
            a = smem_;
        }
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_helm_solve, block_, smem_);
    if (per_sm < 1) {
        err = "Helmholtz solve kernel cannot be resident";
        return OC_ERR_CUDA;
    }
    grid_ = sms * std::min(per_sm, 2);
    // CTA 0 holds no level-0 tile when there are more CTAs than tiles: its
    // persistent region then keeps the coarse levels' four coefficient arrays
    {
        size_t ccells = 0;
        for (int l = H.coarse_from; l < H.n_levels; ++l) ccells += (size_t)H.lv[l].n;
        const int tiles0 = ((nx + TileWide::TX - 1) / TileWide::TX) * ((ny + TileWide::TY - 1) / TileWide::TY);
        H.coarse_persist = (H.persist0 && mg_levels && H.coarse_from > 0 && H.coarse_from < H.n_levels &&
                            grid_ > tiles0 && ccells <= (size_t)TileWide::RN) ? 1 : 0;
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = std::string("Helmholtz init: ") + cudaGetErrorString(e);
        return OC_ERR_CUDA;
    }
    if (refined) {
        refined_ = new RefinedHelm();
        const int rc = refined_->init(nx, ny, dx0, dy0, coef, rtol, max_iter, mask_host, Ku, Kv, err, status);
        if (rc) return rc;
        refined_->set_log(H.log_iters, H.log_conv, H.log_count, H.log_cap);
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
    if (refined_) refined_->set_log(hp_.log_iters, hp_.log_conv, hp_.log_count, hp_.log_cap);
    return OC_OK;
}

void HelmSolver::rebuild(cudaStream_t s) {
    if (refined_) {
        refined_->rebuild(s);
        return;
    }
    for (int l = 0; l < hp_.n_levels; ++l) {
        const HLevel& L = hp_.lv[l];
        const HLevel& F = hp_.lv[l > 0 ? l - 1 : 0];
        k_helm_level<<<(L.n + 255) / 256, 256, 0, s>>>(F, L, l > 0 ? 1 : 0);
    }
}

HelmParams HelmSolver::batched_params(const double* rhs, double* x) const {
    HelmParams H = hp_;
    H.rhs = rhs;
    H.lv[0].x = x;
    H.persist0 = 0;
    H.coarse_persist = 0;
    H.warm = warm_ ? 1 : 0;
    H.ops_smem = 0;
    return H;
}

int helm_batch_plan(HelmSolver* const* solvers, const double* const* rhs, double* const* x, int n, HelmBatch& b,
                    std::string& err) {
    helm_batch_free(b);
    if (n < 1) {
        err = "a batched solve needs at least one system";
        return OC_ERR_ARG;
    }
    size_t smem = 0;
    double total = 0.0;
    std::vector<HelmParams> hp(n);
    for (int m = 0; m < n; ++m) {
        if (!solvers[m]->batchable()) {
            err = "batched Helmholtz solve: the refined solver has no batched form";
            return OC_ERR_UNSUPPORTED;
        }
        hp[m] = solvers[m]->batched_params(rhs[m], x[m]);
        smem = std::max(smem, solvers[m]->batched_smem());
        total += solvers[m]->work_weight();
    }
    int dev = 0, sms = 0, smem_optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, k_helm_solve_batched);
    if (smem + fa.sharedSizeBytes > (size_t)smem_optin) {
        err = "batched Helmholtz solve: a system needs more shared memory than a CTA has";
        return OC_ERR_UNSUPPORTED;
    }
    if (smem > 48 * 1024) {
        static std::mutex mu;
        static std::map<int, size_t> allowance;
        std::lock_guard<std::mutex> lock(mu);
        size_t& a = allowance[dev];
        if (smem > a) {
            cudaFuncSetAttribute(k_helm_solve_batched, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            a = smem;
        }
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_helm_solve_batched, 512, smem);
    if (per_sm < 1) {
        err = "batched Helmholtz solve kernel cannot be resident";
        return OC_ERR_CUDA;
    }
    const int grid = sms * std::min(per_sm, 2);
    if (n > grid) {
        err = "more systems than co-resident CTAs";
        return OC_ERR_UNSUPPORTED;
    }
    // CTAs in proportion to the cells, at least one each, the remainder to the largest shares
    std::vector<int> share(n, 1);
    int left = grid - n;
    std::vector<double> want(n);
    for (int m = 0; m < n; ++m) want[m] = (grid - n) * solvers[m]->work_weight() / total;
    for (int m = 0; m < n; ++m) {
        const int add = std::min(left, (int)want[m]);
        share[m] += add;
        left -= add;
        want[m] -= add;
    }
    while (left > 0) {
        int best = 0;
        for (int m = 1; m < n; ++m)
            if (want[m] > want[best]) best = m;
        share[best] += 1;
        want[best] -= 1.0;
        --left;
    }
    b.cta_start.assign(n + 1, 0);
    for (int m = 0; m < n; ++m) b.cta_start[m + 1] = b.cta_start[m] + share[m];
    if (cudaMalloc(&b.d_params, sizeof(HelmParams) * n) != cudaSuccess ||
        cudaMalloc(&b.d_cta_start, sizeof(int) * (n + 1)) != cudaSuccess) {
        helm_batch_free(b);
        err = "cudaMalloc failed (batched solve plan)";
        return OC_ERR_CUDA;
    }
    cudaMemcpy(b.d_params, hp.data(), sizeof(HelmParams) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(b.d_cta_start, b.cta_start.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice);
    b.n = n;
    b.grid = b.cta_start[n];
    b.smem = smem;
    return OC_OK;
}

int helm_batch_grid() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return std::max(1, sms);
}

int helm_batch_launch(const HelmBatch& b, cudaStream_t s, std::string& err) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(b.grid);
    cfg.blockDim = dim3(512);
    cfg.dynamicSmemBytes = b.smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_helm_solve_batched, (const HelmParams*)b.d_params,
                                             (const int*)b.d_cta_start, b.n);
    if (e != cudaSuccess) {
        err = std::string("batched Helmholtz solve launch: ") + cudaGetErrorString(e);
        return OC_ERR_CUDA;
    }
    return OC_OK;
}

void helm_batch_free(HelmBatch& b) {
    if (b.d_params) cudaFree(b.d_params);
    if (b.d_cta_start) cudaFree(b.d_cta_start);
    b = HelmBatch{};
}

int HelmSolver::solve(const double* rhs, double* x, cudaStream_t s, std::string& err) {
    if (refined_) return refined_->solve(rhs, x, s, err);
    HelmParams H = hp_;
    H.rhs = rhs;
    H.lv[0].x = x;
    H.warm = warm_ ? 1 : 0;
    // a cooperative launch (every CTA resident, for the grid barriers) through
    // the extensible launch API, which stream capture records into a graph
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid_);
    cfg.blockDim = dim3(block_);
    cfg.dynamicSmemBytes = smem_;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_helm_solve, H);
    if (e != cudaSuccess) {
        err = std::string("Helmholtz solve launch: ") + cudaGetErrorString(e);
        return OC_ERR_CUDA;
    }
    return OC_OK;
}

}  // namespace oc
