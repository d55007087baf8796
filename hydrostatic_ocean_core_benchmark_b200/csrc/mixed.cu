// The mixed-precision path of the step (precision = OC_PRECISION_MIXED).
//
// The 3D state (u, v, T, S, e, K_m, K_h) and every 3D stencil, column solve and
// work field of the step are FP32: the kernels of step_kernels.cu built a
// second time for float (OC_MIXED), with contraction. FP64 stays where FP32
// would lose the result:
//   - the buoyancy b, its potential phi and the pressure-gradient arithmetic
//     (the baroclinic pressure force is a small difference of large potentials);
//   - the EOS evaluation (rho - rho0 of a ~1027 kg m-3 density);
//   - the surface elevation eta, its gradients, the depth-integrated transports
//     and divergences, and the Helmholtz system and its solve.
// The step's sequence of kernels is the fp64 path's (capi.cu step_once,
// reference model3d_v05.py:337-415) for the theta and fb schemes. No reference
// counterpart: the reference's precision variants are whole-program FP32 or
// FP32-closure builds (libs/cuda/Makefile:77-113, docs/34_precision_axis.md).

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "capi_internal.cuh"
#include "step_kernels.cuh"

namespace oc {

namespace {

__global__ void k_to_float(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        b[t] = (float)a[t];
}

__global__ void k_to_double(const float* __restrict__ a, double* __restrict__ b, int64_t n) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        b[t] = (double)a[t];
}

__global__ void k_fill_f(float* __restrict__ a, float v, int64_t n) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        a[t] = v;
}

unsigned grid_for(int64_t n) {
    const int64_t blocks = (n + 255) / 256;
    return (unsigned)(blocks < 148 * 16 ? (blocks > 0 ? blocks : 1) : 148 * 16);
}

void to_float(const double* a, float* b, int64_t n, cudaStream_t s) {
    if (n > 0) k_to_float<<<grid_for(n), 256, 0, s>>>(a, b, n);
}

void to_double(const float* a, double* b, int64_t n, cudaStream_t s) {
    if (n > 0) k_to_double<<<grid_for(n), 256, 0, s>>>(a, b, n);
}

void fill_f(float* a, double v, int64_t n, cudaStream_t s) {
    if (n > 0) k_fill_f<<<grid_for(n), 256, 0, s>>>(a, (float)v, n);
}

float* falloc(oc_handle* h, size_t n) {
    void* p = nullptr;
    if (n == 0) n = 1;
    if (cudaMalloc(&p, n * sizeof(float)) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, n * sizeof(float));
    h->allocs.push_back(p);
    h->bytes += n * sizeof(float);
    return (float*)p;
}

// the FP32 parameter block: every scalar of the fp64 one rounded once (the
// scalar products are formed in fp64 first), the fp64 copies kept as they are
void convert_params(const KP& a, KPT<float>& b) {
    b.nx = a.nx, b.ny = a.ny, b.nz = a.nz, b.n2 = a.n2, b.n3 = a.n3, b.n3i = a.n3i;
    b.dx = (float)a.dx, b.dy = (float)a.dy;
    b.eos = a.eos, b.pgf_remove = a.pgf_remove, b.pgf_correction = a.pgf_correction;
    b.advection = a.advection, b.tracers_ts = a.tracers_ts, b.closure_tke = a.closure_tke;
    b.mxl_recursive = a.mxl_recursive, b.scheme = a.scheme;
    b.dt = (float)a.dt, b.g = (float)a.g, b.f0 = (float)a.f0, b.rho0 = (float)a.rho0, b.N2 = (float)a.N2;
    b.nu = (float)a.nu, b.kappa = (float)a.kappa, b.bottom_drag = (float)a.bottom_drag;
    b.a_h = (float)a.a_h, b.k_h = (float)a.k_h;
    b.alpha_t = (float)a.alpha_t, b.beta_s = (float)a.beta_s, b.t0 = (float)a.t0, b.s0 = (float)a.s0;
    b.c_k = (float)a.c_k, b.c_eps = (float)a.c_eps, b.pr_t = (float)a.pr_t, b.z_0 = (float)a.z_0;
    b.e_min = (float)a.e_min, b.l_min = (float)a.l_min, b.e_bb = (float)a.e_bb, b.n2_min = (float)a.n2_min;
    b.theta = (float)a.theta, b.theta_cor = (float)a.theta_cor, b.theta_v = (float)a.theta_v;
    b.thv_dt = (float)a.thv_dt, b.thv_dt_drag = (float)a.thv_dt_drag, b.thv_dt_zero = (float)a.thv_dt_zero;
    b.c1 = (float)a.c1, b.c2 = (float)a.c2, b.c3 = (float)a.c3;
    b.one_m_tc = (float)a.one_m_tc, b.one_m_th = (float)a.one_m_th;
    b.neg_f0 = (float)a.neg_f0, b.neg_g = (float)a.neg_g, b.neg_n2 = (float)a.neg_n2;
    b.flux_t = (float)a.flux_t, b.flux_s = (float)a.flux_s;
    b.one_m_kappa3 = (float)a.one_m_kappa3, b.one_p_kappa3 = (float)a.one_p_kappa3;
    for (int k = 0; k <= OC_MAXNZ; ++k) b.edge[k] = (float)a.edge[k];
    for (int k = 0; k < OC_MAXNZ; ++k) {
        b.dzr[k] = (float)a.dzr[k];
        b.thin[k] = (float)a.thin[k];
        b.dz_nom[k] = (float)a.dz_nom[k];
    }
    b.kinfo = a.kinfo, b.kface = a.kface, b.face_rule = a.face_rule;
    b.mom_kl = a.mom_kl, b.tr_kl = a.tr_kl;
    b.dx64 = a.dx64, b.dy64 = a.dy64;
    b.rho0_64 = a.rho0_64, b.alpha_t64 = a.alpha_t64, b.beta_s64 = a.beta_s64;
    b.t0_64 = a.t0_64, b.s0_64 = a.s0_64, b.neg_g64 = a.neg_g64;
    b.mask_u64 = a.mask_u64, b.mask_v64 = a.mask_v64, b.dzx64 = a.dzx64;
    for (int k = 0; k <= OC_MAXNZ; ++k) b.edge64[k] = a.edge64[k];
    for (int k = 0; k < OC_MAXNZ; ++k) b.dzr64[k] = a.dzr64[k];
}

// one field of a state into its FP32 buffer: device sources convert in place,
// host sources pass through the fp64 staging buffer (same stream, so in order)
int field_in(oc_handle* h, float* dst, const double* src, size_t n, int32_t on_device, cudaStream_t st) {
    if (on_device) {
        to_float(src, dst, (int64_t)n, st);
        return OC_OK;
    }
    const cudaError_t e = cudaMemcpyAsync(h->stage, src, n * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(h, e, "state copy");
    to_float(h->stage, dst, (int64_t)n, st);
    return OC_OK;
}

int field_out(oc_handle* h, double* dst, const float* src, size_t n, int32_t on_device, cudaStream_t st) {
    if (on_device) {
        to_double(src, dst, (int64_t)n, st);
        return OC_OK;
    }
    to_double(src, h->stage, (int64_t)n, st);
    const cudaError_t e = cudaMemcpyAsync(dst, h->stage, n * sizeof(double), cudaMemcpyDeviceToHost, st);
    return e == cudaSuccess ? OC_OK : cuda_fail(h, e, "oc_get_state copy");
}

}  // namespace

int mixed_validate(const oc_config* c, std::string& err) {
    if (c->scheme == OC_SCHEME_SPLIT)
        return err = "the mixed-precision step runs the theta and fb schemes", OC_ERR_UNSUPPORTED;
    if (c->tracers != OC_TRACERS_TS)
        return err = "the mixed-precision step carries T and S (tracers = TS)", OC_ERR_UNSUPPORTED;
    return OC_OK;
}

int mixed_alloc(oc_handle* h, const std::vector<int2>& kinfo, const std::vector<double2>& dzx) {
    (void)kinfo;
    const size_t n2 = h->n2, n3 = h->n3, n3i = h->n3i;
    for (int t = 0; t < 2; ++t) {
        h->U32[t] = falloc(h, n3);
        h->V32[t] = falloc(h, n3);
        h->T32[t] = falloc(h, n3);
        h->S32[t] = falloc(h, n3);
    }
    for (float** p : {&h->e32, &h->km32, &h->kh32, &h->w32}) *p = falloc(h, n3i);
    for (float** p : {&h->q32, &h->pgx32, &h->pgy32, &h->avpv32, &h->avpu32, &h->dzu32, &h->dzv32, &h->stu32,
                      &h->stv32, &h->ghu32, &h->ghv32, &h->uit32, &h->vit32})
        *p = falloc(h, n3);
    for (float** p : {&h->H32, &h->mask32, &h->mask_u32, &h->mask_v32, &h->tau_u32, &h->tau_v32, &h->ustar2_32})
        *p = falloc(h, n2);
    h->dzx32 = falloc(h, 2 * n2);
    h->stage = dalloc(h, n3i);
    for (float* p : {h->U32[1], h->S32[1], h->vit32, h->ustar2_32, h->dzx32})
        if (!p) return fail(h, OC_ERR_CUDA, "device allocation failed (mixed-precision fields)");
    if (!h->stage) return fail(h, OC_ERR_CUDA, "device allocation failed (staging buffer)");
    // static fields in FP32 (masks are 0/1, so exact)
    std::vector<float> tmp(2 * n2);
    auto up = [&](float* dst, const std::vector<double>& src) {
        for (size_t c = 0; c < n2; ++c) tmp[c] = (float)src[c];
        cudaMemcpy(dst, tmp.data(), n2 * sizeof(float), cudaMemcpyHostToDevice);
    };
    up(h->H32, h->H);
    up(h->mask32, h->mask);
    up(h->mask_u32, h->mask_u);
    up(h->mask_v32, h->mask_v);
    for (size_t c = 0; c < n2; ++c) {
        tmp[2 * c] = (float)dzx[c].x;
        tmp[2 * c + 1] = (float)dzx[c].y;
    }
    cudaMemcpy(h->dzx32, tmp.data(), 2 * n2 * sizeof(float), cudaMemcpyHostToDevice);
    KPT<float>& Q = h->P32;
    convert_params(h->P, Q);
    Q.H = h->H32;
    Q.mask = h->mask32;
    Q.mask_u = h->mask_u32;
    Q.mask_v = h->mask_v32;
    Q.tau_u = h->tau_u32;
    Q.tau_v = h->tau_v32;
    Q.ustar2 = h->ustar2_32;
    Q.dzx = reinterpret_cast<const float2*>(h->dzx32);
    fill_f(h->e32, h->cfg.e_min, (int64_t)n3i, 0);
    fill_f(h->km32, h->cfg.nu, (int64_t)n3i, 0);
    fill_f(h->kh32, h->cfg.kappa, (int64_t)n3i, 0);
    return check_launch(h, "mixed-precision set-up");
}

int mixed_upload_stress(oc_handle* h) {
    to_float(h->d_tau_u, h->tau_u32, (int64_t)h->n2, 0);
    to_float(h->d_tau_v, h->tau_v32, (int64_t)h->n2, 0);
    to_float(h->d_ustar2, h->ustar2_32, (int64_t)h->n2, 0);
    const cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? OC_OK : cuda_fail(h, e, "stress upload");
}

int mixed_build_coefficients(oc_handle* h, cudaStream_t s) {
    launch_qsolve(h->P32, h->km32, h->q32, s);
    launch_kukv(h->P32, h->q32, h->Ku, h->Kv, s);
    return check_launch(h, "coefficients");
}

int mixed_reset_mixing(oc_handle* h, cudaStream_t s) {
    fill_f(h->km32, h->cfg.nu, (int64_t)h->n3i, s);
    fill_f(h->kh32, h->cfg.kappa, (int64_t)h->n3i, s);
    return mixed_build_coefficients(h, s);
}

int mixed_set_state(oc_handle* h, const oc_state_view* s, int32_t on_device, cudaStream_t st) {
    const int c = h->cur;
    int rc = OC_OK;
    cudaError_t e = cudaMemcpyAsync(h->ETA[c], s->eta, h->n2 * sizeof(double),
                                    on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(h, e, "state copy");
    if ((rc = field_in(h, h->U32[c], s->u, h->n3, on_device, st))) return rc;
    if ((rc = field_in(h, h->V32[c], s->v, h->n3, on_device, st))) return rc;
    if ((rc = field_in(h, h->T32[c], s->T, h->n3, on_device, st))) return rc;
    if ((rc = field_in(h, h->S32[c], s->S, h->n3, on_device, st))) return rc;
    if (s->b) {
        e = cudaMemcpyAsync(h->B[c], s->b, h->n3 * sizeof(double),
                            on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return cuda_fail(h, e, "state copy");
    } else {
        // b of the FP32 tracers, by the fp64 EOS
        launch_diag_buoyancy(h->P32, h->T32[c], h->S32[c], h->B[c], st);
    }
    if (s->e) {
        if ((rc = field_in(h, h->e32, s->e, h->n3i, on_device, st))) return rc;
    } else {
        fill_f(h->e32, h->cfg.e_min, (int64_t)h->n3i, st);
    }
    if (s->km && (rc = field_in(h, h->km32, s->km, h->n3i, on_device, st))) return rc;
    if (s->kh && (rc = field_in(h, h->kh32, s->kh, h->n3i, on_device, st))) return rc;
    launch_wcol(h->P32, h->U32[c], h->V32[c], h->w32, st);
    if (s->km) {
        launch_qsolve(h->P32, h->km32, h->q32, st);
        launch_kukv(h->P32, h->q32, h->Ku, h->Kv, st);
        if (h->solver) h->solver->rebuild(st);
    }
    return check_launch(h, "oc_set_state");
}

int mixed_get_state(oc_handle* h, const oc_state_view* s, int32_t on_device, cudaStream_t st) {
    const int c = h->cur;
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    int rc = OC_OK;
    if (s->eta) {
        const cudaError_t e = cudaMemcpyAsync(s->eta, h->ETA[c], h->n2 * sizeof(double), kind, st);
        if (e != cudaSuccess) return cuda_fail(h, e, "oc_get_state copy");
    }
    if (s->b) {
        const cudaError_t e = cudaMemcpyAsync(s->b, h->B[c], h->n3 * sizeof(double), kind, st);
        if (e != cudaSuccess) return cuda_fail(h, e, "oc_get_state copy");
    }
    struct {
        double* dst;
        const float* src;
        size_t n;
    } items[] = {{s->u, h->U32[c], h->n3}, {s->v, h->V32[c], h->n3}, {s->T, h->T32[c], h->n3},
                 {s->S, h->S32[c], h->n3}, {s->e, h->e32, h->n3i},   {s->km, h->km32, h->n3i},
                 {s->kh, h->kh32, h->n3i}};
    for (auto& it : items)
        if (it.dst && (rc = field_out(h, it.dst, it.src, it.n, on_device, st))) return rc;
    return check_launch(h, "oc_get_state");
}

// one step of the mixed-precision path: the fp64 path's kernel sequence
// (capi.cu step_once) for the theta and fb schemes, 3D kernels on FP32 fields
int step_once_mixed(oc_handle* h, cudaStream_t s) {
    const oc_config& c = h->cfg;
    const KP& P = h->P;          // 2D kernels: fp64
    const KPT<float>& Q = h->P32;  // 3D kernels: FP32
    const int cur = h->cur, nxt = 1 - cur;
    const float *u = h->U32[cur], *v = h->V32[cur];
    float *un = h->U32[nxt], *vn = h->V32[nxt];
    const double* b = h->B[cur];
    const double* eta = h->ETA[cur];
    double* etan = h->ETA[nxt];
    const bool theta = c.scheme == OC_SCHEME_THETA;
    // old-state kernels that do not depend on the closure, on the second stream
    cudaStream_t a = h->aux;
    cudaEventRecord(h->fork, s);
    cudaStreamWaitEvent(a, h->fork, 0);
    { Prof pr(h, a, "phi"); launch_phi(Q, b, h->phi, a); }
    { Prof pr(h, a, "grad2"); launch_grad2(P, eta, h->gx2, h->gy2, a); }
    if (theta) {
        { Prof pr(h, a, "transport"); launch_transport(Q, u, v, h->Uold, h->Vold, a); }
        { Prof pr(h, a, "div2"); launch_div2(P, h->Uold, h->Vold, h->div_old, a); }
    }
    cudaEventRecord(h->join, a);
    if (c.closure == OC_CLOSURE_TKE) {
        { Prof pr(h, s, "closure"); launch_closure(Q, u, v, b, h->e32, h->km32, h->kh32, h->q32, s); }
        h->tridiag += 2;
        { Prof pr(h, s, "kukv"); launch_kukv(Q, h->q32, h->Ku, h->Kv, s); }
        if (theta) {
            { Prof pr(h, s, "helm_rebuild", h->solver->n_levels()); h->solver->rebuild(s); }
            h->rebuilds += 1;
        }
    }
    cudaStreamWaitEvent(s, h->join, 0);
    {
        Prof pr(h, s, "mom_explicit");
        launch_mom_explicit(Q, u, v, b, h->phi, h->w32, h->km32, h->pgx32, h->pgy32, h->avpv32, h->avpu32,
                            h->dzu32, h->dzv32, h->stu32, h->stv32, s);
    }
    const float *uit = u, *vit = v;
    for (int m = 0; m < c.n_picard; ++m) {
        const bool last = m == c.n_picard - 1;
        float *tu, *tv;
        if (theta) {
            tu = h->ghu32;
            tv = h->ghv32;
        } else if (last) {
            tu = un;
            tv = vn;
        } else {
            tu = (m % 2 == 0) ? h->ghu32 : h->uit32;
            tv = (m % 2 == 0) ? h->ghv32 : h->vit32;
        }
        {
            Prof pr(h, s, "predictor_rhs");
            launch_predictor_rhs(Q, u, v, uit, vit, h->pgx32, h->pgy32, h->avpv32, h->avpu32, h->dzu32, h->dzv32,
                                 h->stu32, h->stv32, h->gx2, h->gy2, tu, tv, s);
        }
        { Prof pr(h, s, "momentum_solve"); launch_momentum_solve(Q, h->km32, tu, tv, h->Ug, h->Vg, s); }
        h->tridiag += 2;
        if (theta) {
            { Prof pr(h, s, "helm_rhs"); launch_helm_rhs(P, eta, h->div_old, h->Ug, h->Vg, h->rhs2, s); }
            int rc = ensure_log(h, h->solves + 1, s);
            if (rc) return rc;
            // the mixed step owes the reference no iteration counts: its multigrid
            // starts from the current eta (first pass) or the first pass's solution
            // (the solver's warm start), under the same stopping test
            if (m == 0) cudaMemcpyAsync(etan, eta, h->n2 * sizeof(double), cudaMemcpyDeviceToDevice, s);
            if (h->batch_rec) {
                // an ensemble recording its batched graph: the solve becomes a pair of
                // placeholder nodes the batched solve is later wired between
                rc = batch_defer(h, s, h->rhs2, etan);
            } else {
                if (h->solve_chain) cudaStreamWaitEvent(s, h->solve_chain, 0);
                {
                    Prof pr(h, s, "helm_solve");
                    rc = h->solver->solve(h->rhs2, etan, s, h->err);
                }
                if (h->solve_chain) cudaEventRecord(h->solve_chain, s);
            }
            if (rc) return rc;
            h->solves += 1;
            float* ou = last ? un : h->uit32;
            float* ov = last ? vn : h->vit32;
            { Prof pr(h, s, "backsub"); launch_backsub(Q, h->ghu32, h->ghv32, h->q32, etan, ou, ov, s); }
            uit = ou;
            vit = ov;
        } else {
            uit = tu;
            vit = tv;
        }
    }
    if (c.scheme == OC_SCHEME_FB) { Prof pr(h, s, "eta_fb"); launch_eta_fb(P, eta, h->Ug, h->Vg, etan, s); }
    { Prof pr(h, s, "wcol"); launch_wcol(Q, un, vn, h->w32, s); }
    {
        // the explicit momentum terms are dead by now: their buffers hold the tracer right-hand sides
        Prof pr(h, s, "tracer_rhs");
        launch_tracer_rhs(Q, h->T32[cur], h->S32[cur], un, vn, h->w32, h->kh32, h->pgx32, h->pgy32, s);
    }
    {
        Prof pr(h, s, "tracer_solve");
        launch_tracer_solve(Q, h->pgx32, h->pgy32, h->kh32, h->T32[nxt], h->S32[nxt], h->B[nxt], s);
    }
    h->tridiag += 2;
    h->cur = nxt;
    h->steps += 1;
    return check_launch(h, "step");
}

}  // namespace oc
