// The handle of the C ABI (include/ocean_b200.h), shared by the fp64
// orchestration (capi.cu) and the mixed-precision path (mixed.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "helmholtz.cuh"
#include "oc_internal.cuh"
#include "ocean_b200.h"

namespace oc {
struct AdjointWork;
struct BatchRecorder;
}

using oc::HelmSolver;
using oc::KP;
using oc::KPT;

struct oc_handle {
    oc_config cfg{};
    std::string err;
    bool has_domain = false, has_state = false;
    KP P{};
    int nx = 0, ny = 0, nz = 0;
    size_t n2 = 0, n3 = 0, n3i = 0;
    double h_max = 0.0;
    int n_split = 0;
    // host geometry (for oc_get_field and the stress fields)
    std::vector<double> H, mask, mask_u, mask_v, dzr, dz3, mask3, mask3u, mask3v, dz3u, dz3v, zc;
    std::vector<double> taux_c, tauy_c;
    bool stress_field = false;
    // device memory
    std::vector<void*> allocs;
    size_t bytes = 0;
    double *d_H = nullptr, *d_mask = nullptr, *d_mask_u = nullptr, *d_mask_v = nullptr;
    double *d_tau_u = nullptr, *d_tau_v = nullptr, *d_ustar2 = nullptr;
    double *U[2] = {}, *V[2] = {}, *B[2] = {}, *Tt[2] = {}, *Ss[2] = {}, *ETA[2] = {};
    int cur = 0;
    // the handle's own state buffers while caller-owned ones are bound
    // (oc_bind_state): ETA, U, V, B, Tt, Ss for both parities, then e, km, kh
    bool bound = false;
    int bound_base = 0;  // the parity that was current when the buffers were bound
    double* own_state[15] = {};
    double *e = nullptr, *km = nullptr, *kh = nullptr, *q = nullptr, *w = nullptr;
    double *phi = nullptr, *pgx = nullptr, *pgy = nullptr, *avpv = nullptr, *avpu = nullptr;
    double *dzu = nullptr, *dzv = nullptr, *stu = nullptr, *stv = nullptr;
    double *ghu = nullptr, *ghv = nullptr, *uit = nullptr, *vit = nullptr;
    double *Ku = nullptr, *Kv = nullptr, *gx2 = nullptr, *gy2 = nullptr, *Uold = nullptr,
           *Vold = nullptr, *div_old = nullptr, *Ug = nullptr, *Vg = nullptr, *rhs2 = nullptr;
    double *bt[12] = {};  // split-explicit 2D work
    double* d_part = nullptr;
    int* d_status = nullptr;
    HelmSolver* solver = nullptr;
    // host counters (model3d_v05.py:89-94)
    long long steps = 0, tridiag = 0, rebuilds = 0, substeps = 0, solves = 0, launches = 0;
    cudaStream_t last_stream = nullptr;
    // optional per-kernel event timing
    bool profiling = false;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<std::pair<int, size_t>> ev_marks;  // (kernel class, index of the start event)
    std::vector<std::string> prof_names;
    std::vector<long long> prof_launches;
    std::vector<double> prof_ms;
    // CUDA graphs of two steps (one period of the ping-pong buffers), one per
    // starting buffer, and the counter increments one launch stands for
    struct Counters {
        long long steps, tridiag, rebuilds, substeps, solves, launches;
    };
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    // second stream for the old-state kernels that do not depend on the closure
    cudaStream_t aux = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    Counters graph_delta[2] = {};
    cudaStream_t capture_stream = nullptr;
    long long graph_version = 0;  // bumped whenever recorded graphs go stale
    // while an ensemble records its graph: every Helmholtz solve of every member
    // waits on this event and records it, so the cooperative solves run one at a
    // time and never compete for the SMs
    cudaEvent_t solve_chain = nullptr;
    // ---- mixed-precision path (precision = OC_PRECISION_MIXED): the 3D fields
    // of the state and of the step in FP32; b, phi, eta and every 2D field stay
    // fp64 in the buffers above. The fp64 3D buffers above are then not allocated.
    bool mixed = false;
    KPT<float> P32{};
    float *U32[2] = {}, *V32[2] = {}, *T32[2] = {}, *S32[2] = {};
    float *e32 = nullptr, *km32 = nullptr, *kh32 = nullptr, *q32 = nullptr, *w32 = nullptr;
    float *pgx32 = nullptr, *pgy32 = nullptr, *avpv32 = nullptr, *avpu32 = nullptr;
    float *dzu32 = nullptr, *dzv32 = nullptr, *stu32 = nullptr, *stv32 = nullptr;
    float *ghu32 = nullptr, *ghv32 = nullptr, *uit32 = nullptr, *vit32 = nullptr;
    float *H32 = nullptr, *mask32 = nullptr, *mask_u32 = nullptr, *mask_v32 = nullptr;
    float *tau_u32 = nullptr, *tau_v32 = nullptr, *ustar2_32 = nullptr, *dzx32 = nullptr;
    double* stage = nullptr;  // (nz+1) n2 doubles: a state field on its way in or out
    // work of the adjoint step (adjoint.cu), made on its first call
    oc::AdjointWork* adj = nullptr;
    // while an ensemble records with batched solves: where the step's solves are deferred to
    oc::BatchRecorder* batch_rec = nullptr;
};


namespace oc {

// mixed.cu: the mixed-precision path
int mixed_validate(const oc_config* c, std::string& err);
int mixed_alloc(oc_handle* h, const std::vector<int2>& kinfo, const std::vector<double2>& dzx);
int mixed_upload_stress(oc_handle* h);
int mixed_build_coefficients(oc_handle* h, cudaStream_t s);
int mixed_set_state(oc_handle* h, const oc_state_view* s, int32_t on_device, cudaStream_t st);
int mixed_get_state(oc_handle* h, const oc_state_view* s, int32_t on_device, cudaStream_t st);
int mixed_reset_mixing(oc_handle* h, cudaStream_t s);
int step_once_mixed(oc_handle* h, cudaStream_t s);

// adjoint.cu: the adjoint of the fp64 step
int adjoint_step(oc_handle* h, const oc_state_view* x0, const oc_state_view* x1, const oc_state_view* x1_b,
                 const oc_state_view* x0_b, double* taux_b, double* tauy_b, cudaStream_t s);
int adjoint_eos(oc_handle* h, const double* T, const double* S, const double* b_b, double* T_b, double* S_b,
                cudaStream_t s);
void adjoint_free(oc_handle* h);

// capi.cu: a solve deferred to the ensemble's batched solve while it records
int batch_defer(oc_handle* h, cudaStream_t s, const double* rhs, double* x);

// capi.cu helpers the mixed path shares
int fail(oc_handle* h, int code, const std::string& msg);
int cuda_fail(oc_handle* h, cudaError_t e, const char* where);
int check_launch(oc_handle* h, const char* where);
int ensure_log(oc_handle* h, long long needed, cudaStream_t s);
void prof_harvest(oc_handle* h);
int prof_class(oc_handle* h, const char* name);
double* dalloc(oc_handle* h, size_t n);

// brackets one kernel (or one fixed group of kernels) with events
struct Prof {
    oc_handle* h;
    cudaStream_t s;
    int cls = -1;
    size_t idx = 0;
    Prof(oc_handle* h_, cudaStream_t s_, const char* name, int n_kernels = 1) : h(h_), s(s_) {
        h->launches += n_kernels;
        if (!h->profiling) return;
        cls = prof_class(h, name);
        h->prof_launches[cls] += n_kernels;
        if (h->ev_used + 2 > h->ev_pool.size()) prof_harvest(h);
        if (h->ev_pool.size() < h->ev_used + 2) {
            cudaEvent_t a, b;
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            h->ev_pool.push_back(a);
            h->ev_pool.push_back(b);
        }
        idx = h->ev_used;
        h->ev_used += 2;
        cudaEventRecord(h->ev_pool[idx], s);
    }
    ~Prof() {
        if (cls < 0) return;
        cudaEventRecord(h->ev_pool[idx + 1], s);
        h->ev_marks.push_back({cls, idx});
    }
};

}  // namespace oc
