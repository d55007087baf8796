// Variable-coefficient free-surface Helmholtz solver, A = I - c D[K G[.]].
#pragma once

#include <algorithm>
#include <vector>

#include "helm_refined.cuh"
#include "oc_internal.cuh"

namespace oc {

// HK_PCG_MG (no reference counterpart): CG preconditioned by one symmetric
// V(2,2) cycle of the multigrid hierarchy; the mixed-precision step's solver
// HK_REFINED (no reference counterpart): FP32 inner PCG-Jacobi inside FP64
// refinement (RefinedHelm), for the mixed-precision step
enum { HK_PCG_JACOBI = 0, HK_PCG_RBGS = 1, HK_RBGS = 2, HK_MULTIGRID = 3, HK_REFINED = 4, HK_PCG_MG = 5 };

struct HLevel {
    int nx, ny, n;
    int shape;        // tile shape of the level's grid phases
    double dx2, dy2;  // dx**2, dy**2 of the level
    double cx, cy;    // coef * (1 / dx**2)
    const double* mask;
    double* Ku;
    double* Kv;
    double* inv_diag;
    double* x;   // current solution of the level (level 0: the caller's output)
    double* x2;  // second buffer: the smoothing phases read one and write the other
    double* b;
};

struct HelmParams {
    int n_levels, kind, max_iter, coarse_from;
    int warm;       // the solve starts from the x it is given (else from zero)
    int wide0;      // level 0 runs 128 x 16 tiles
    int fused_res;  // ... whose rows are NumPy's leaves: the up phase forms the residual sums
    int persist0;   // ... one per CTA: their coefficients stay in shared memory for the solve
    int coarse_persist;  // CTA 0 (no level-0 tile) keeps the coarse levels' coefficients in its region
    double coef, rtol;
    HLevel lv[OC_MAX_LEVELS];
    double *r, *z, *p, *Ap;  // level-0 work vectors
    const double* rhs;
    // NumPy pairwise-summation plan of the level-0 vectors
    int n_leaves;
    const int* leaf_start;    // n_leaves + 1
    int n_heights;
    const int* height_start;  // n_heights + 1 offsets into ops
    const int2* ops;          // (lo, mid): value[lo] += value[mid]
    int n_ops;
    int ops_smem;             // doubles of shared memory holding a copy of ops and height_start (0: none)
    int perfect_lanes;        // > 0: the tree is perfect, folded with this many leaves per lane (perfect_fold)
    double* leafA;
    double* leafB;
    double* leafC;
    // two-level fold when the leaf sums exceed shared memory (big_fold): block
    // subtrees (first leaf, leaves, offset into bh_start, heights) with their ops
    // relative to the block's first leaf, then the top of the tree over the roots
    int big_fold, n_blocks, top_heights;
    const int4* blocks;
    const int2* bops;
    const int* bh_start;
    const int2* top_ops;
    const int* top_hstart;
    double* broot;  // 3 x n_blocks: one root buffer per leaf buffer
    // grid barrier and status
    unsigned long long* bar_count;  // grid barrier arrivals (only grows)
    int* status;
    long long wait_cycles;          // bound of a barrier wait in SM clock cycles
    // per-solve log
    int* log_iters;
    int* log_conv;
    int* log_count;
    int log_cap;
};

class HelmSolver {
   public:
    ~HelmSolver();
    // Ku/Kv are device arrays of the fine level owned by the caller, mask a host
    // array; dx, dy the fine-level spacing.
    int init(int nx, int ny, double dx, double dy, double coef, int kind, double rtol, int max_iter,
             const double* mask_host, double* Ku, double* Kv, int log_cap, int* status,
             std::string& err);
    // recompute coarse coefficients and inverse diagonals after Ku/Kv changed
    void rebuild(cudaStream_t s);
    // x = A^-1 rhs on the device, iteration count appended to the log
    int solve(const double* rhs, double* x, cudaStream_t s, std::string& err);
    // warm start: the solve starts from the x it is given instead of zero (the
    // reference starts from zero; the mixed-precision step warm-starts)
    void set_warm_start(bool w) { warm_ = w; }
    int n_levels() const { return hp_.n_levels; }
    int log_capacity() const { return hp_.log_cap; }
    int* d_log_iters() const { return hp_.log_iters; }
    int* d_log_conv() const { return hp_.log_conv; }
    int* d_log_count() const { return hp_.log_count; }
    int grow_log(int cap, cudaStream_t s, std::string& err);
    // bound of the solve's barrier waits in SM clock cycles (default ~1 s)
    void set_wait_cycles(long long cycles) {
        hp_.wait_cycles = cycles;
        if (refined_) refined_->set_wait_cycles(cycles);
    }
    // false for the refined solver, which has no batched form
    bool batchable() const { return refined_ == nullptr; }
    // CTAs a solve of this grid keeps busy: about one per 2048 cells (a 128 x 16
    // tile of level 0), at least one, at most the solve's own grid
    int preferred_ctas() const {
        const long long want = ((long long)hp_.lv[0].n + 2047) / 2048;
        return (int)std::max(1LL, std::min<long long>(want, grid_ > 0 ? grid_ : want));
    }
    // this solver's system for a batched launch (helm_batch_*): the parameters
    // of x = A^-1 rhs without the one-CTA-per-tile assumptions, and the dynamic
    // shared memory it needs
    HelmParams batched_params(const double* rhs, double* x) const;
    size_t batched_smem() const { return smem_batched_; }
    double work_weight() const { return (double)hp_.lv[0].n; }
    size_t bytes() const { return bytes_ + (refined_ ? refined_->bytes() : 0); }

   private:
    HelmParams hp_{};
    RefinedHelm* refined_ = nullptr;  // kind HK_REFINED: the solves go here
    bool warm_ = false;
    std::vector<void*> allocs_;
    int grid_ = 0, block_ = 512;
    size_t smem_ = 0, smem_batched_ = 0;
    size_t bytes_ = 0;
    void* dalloc(size_t nbytes);
};

// Several solvers' systems solved by one cooperative launch (k_helm_solve_batched):
// system m on its own share of the CTAs, proportional to its cells. The plan's
// device arrays hold the systems' parameters, so a recorded launch replays them.
struct HelmBatch {
    int n = 0, grid = 0;
    size_t smem = 0;
    HelmParams* d_params = nullptr;
    int* d_cta_start = nullptr;
    std::vector<int> cta_start;
};
int helm_batch_plan(HelmSolver* const* solvers, const double* const* rhs, double* const* x, int n, HelmBatch& b,
                    std::string& err);
int helm_batch_launch(const HelmBatch& b, cudaStream_t s, std::string& err);
// CTAs of one batched launch at the least (one per SM of the current device)
int helm_batch_grid();
void helm_batch_free(HelmBatch& b);

}  // namespace oc
