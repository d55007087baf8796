// C ABI of the ocean-core step: handle, geometry, state, step orchestration.
//
// The step follows reference libs/core/model3d_v05.py Stepper3DV05.step
// (lines 337-415; split-explicit 417-463; tracers 466-533) as a fixed
// sequence of fused column kernels plus one persistent Helmholtz solve per
// Picard iteration; state lives in ping-pong buffers so no step ever copies a
// 3D field.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "capi_internal.cuh"
#include "helmholtz.cuh"
#include "oc_internal.cuh"
#include "ocean_b200.h"
#include "step_kernels.cuh"

namespace oc {

__global__ void k_fill(double* a, double v, int64_t n) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) a[t] = v;
}

// the larger of two magnitudes, NaN winning over every number (a NaN surface
// elevation must reach the divergence check, as the reference's isnan test does)
__host__ __device__ inline double nan_max(double a, double b) {
    if (a != a) return a;
    if (b != b) return b;
    return b > a ? b : a;
}

__global__ void k_absmax_partial(const double* a, int64_t n, double* part) {
    __shared__ double sh[256];
    double m = 0.0;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        m = nan_max(m, fabs(a[t]));
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) sh[threadIdx.x] = nan_max(sh[threadIdx.x], sh[threadIdx.x + k]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

static void fill(double* a, double v, int64_t n, cudaStream_t s) {
    if (n > 0) k_fill<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, v, n);
}

}  // namespace oc

using namespace oc;


namespace oc {

// levels one CTA of k_mom_column / k_tracer_rhs marches unless tuned
constexpr int kDefaultLevelsPerCta = 10;

int fail(oc_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}

int cuda_fail(oc_handle* h, cudaError_t e, const char* where) {
    return fail(h, OC_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

double* dalloc(oc_handle* h, size_t n) {
    void* p = nullptr;
    if (n == 0) n = 1;
    if (cudaMalloc(&p, n * sizeof(double)) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, n * sizeof(double));
    h->allocs.push_back(p);
    h->bytes += n * sizeof(double);
    return (double*)p;
}

int check_launch(oc_handle* h, const char* where) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(h, e, where);
    return OC_OK;
}

int validate(const oc_config* c, std::string& err) {
    if (c->nx < 1 || c->ny < 1 || c->nz < 1) return err = "nx, ny, nz must be >= 1", OC_ERR_ARG;
    if (c->nz > OC_MAXNZ) return err = "nz above the supported maximum of 128", OC_ERR_UNSUPPORTED;
    if (!(c->lx > 0.0) || !(c->ly > 0.0)) return err = "lx, ly must be > 0", OC_ERR_ARG;
    if (c->scheme < 0 || c->scheme > 2) return err = "unknown scheme (expected fb|theta|split_explicit)", OC_ERR_ARG;
    if (c->scheme == OC_SCHEME_THETA && !(c->theta > 0.0 && c->theta <= 1.0))
        return err = "theta must lie in (0,1]", OC_ERR_ARG;
    if (c->n_picard < 1) return err = "n_picard must be >= 1", OC_ERR_ARG;
    if (!(c->dt > 0.0)) return err = "dt must be > 0", OC_ERR_ARG;
    if (c->solver < 0 || c->solver > OC_SOLVER_PCG_MG) return err = "unknown Helmholtz solver", OC_ERR_ARG;
    if (c->solver == OC_SOLVER_PCG_REFINED && c->precision != OC_PRECISION_MIXED)
        return err = "the FP32-inner refined solver serves the mixed-precision step only", OC_ERR_ARG;
    if (c->max_iter < 1) return err = "max_iter must be >= 1", OC_ERR_ARG;
    if (c->bc_x < 0 || c->bc_x > 1 || c->bc_y < 0 || c->bc_y > 1)
        return err = "bc must be periodic|closed (open boundaries are not supported)", OC_ERR_UNSUPPORTED;
    if (c->face_rule < 0 || c->face_rule > 2) return err = "face_rule must be min|mean|harmonic", OC_ERR_ARG;
    if (c->eos < 0 || c->eos > 2) return err = "eos must be linear|seos|teos10", OC_ERR_ARG;
    if (c->pgf < 0 || c->pgf > 1) return err = "pgf must be remove|keep", OC_ERR_ARG;
    if (c->advection < 0 || c->advection > 4) return err = "unknown advection scheme", OC_ERR_ARG;
    if (c->tracers < 0 || c->tracers > 1) return err = "tracers must be buoyancy|TS", OC_ERR_ARG;
    if (c->closure < 0 || c->closure > 1) return err = "closure must be none|tke", OC_ERR_ARG;
    if (c->mxl < 0 || c->mxl > 1) return err = "mxl must be integral|recursive", OC_ERR_ARG;
    if (c->barotropic_average < 0 || c->barotropic_average > 1)
        return err = "barotropic_average must be none|mean", OC_ERR_ARG;
    if (c->precision != OC_PRECISION_FP64 && c->precision != OC_PRECISION_MIXED)
        return err = "precision must be fp64 or mixed", OC_ERR_ARG;
    if (c->precision == OC_PRECISION_MIXED) return mixed_validate(c, err);
    return OC_OK;
}

// scalar constants of the step, formed in the reference's operation order
void fill_scalars(oc_handle* h) {
    const oc_config& c = h->cfg;
    KP& P = h->P;
    P.nx = c.nx;
    P.ny = c.ny;
    P.nz = c.nz;
    P.n2 = c.nx * c.ny;
    P.n3 = P.n2 * c.nz;
    P.n3i = P.n2 * (c.nz + 1);
    P.dx = c.lx / c.nx;
    P.dy = c.ly / c.ny;
    P.eos = c.eos;
    P.pgf_remove = c.pgf == OC_PGF_REMOVE;
    P.pgf_correction = c.pgf_correction != 0;
    P.advection = c.advection;
    P.tracers_ts = c.tracers == OC_TRACERS_TS;
    P.closure_tke = c.closure == OC_CLOSURE_TKE;
    P.mxl_recursive = c.mxl == OC_MXL_RECURSIVE;
    P.scheme = c.scheme;
    P.face_rule = c.face_rule;
    P.dt = c.dt;
    P.g = c.g;
    P.f0 = c.f0;
    P.rho0 = c.rho0;
    P.N2 = c.n2;
    P.nu = c.nu;
    P.kappa = c.kappa;
    P.bottom_drag = c.bottom_drag;
    P.a_h = c.a_h;
    P.k_h = c.k_h;
    P.alpha_t = c.alpha_t;
    P.beta_s = c.beta_s;
    P.t0 = c.t0;
    P.s0 = c.s0;
    P.c_k = c.c_k;
    P.c_eps = c.c_eps;
    P.pr_t = c.pr_t;
    P.z_0 = c.z_0;
    P.e_min = c.e_min;
    P.l_min = c.l_min;
    P.e_bb = c.e_bb;
    P.n2_min = c.n2_min;
    const double th = (c.scheme == OC_SCHEME_THETA) ? c.theta : 0.0;
    P.theta = th;
    P.theta_cor = c.theta_cor;
    P.theta_v = c.theta_v;
    P.thv_dt = c.theta_v * c.dt;
    P.thv_dt_drag = (c.theta_v * c.dt) * c.bottom_drag;
    P.thv_dt_zero = (c.theta_v * c.dt) * 0.0;
    P.c1 = (c.g * c.dt) * (1.0 - th);
    P.c2 = (c.g * c.dt) * th;
    P.c3 = (1.0 - c.theta_v) * c.dt;
    P.one_m_tc = 1.0 - c.theta_cor;
    P.one_m_th = 1.0 - th;
    P.neg_f0 = -c.f0;
    P.neg_g = -c.g;
    P.neg_n2 = -c.n2;
    P.flux_t = c.q_heat / (c.rho0 * c.cp);
    P.flux_s = c.q_salt;
    const double kap = 1.0 / 3.0;
    P.one_m_kappa3 = 1.0 - kap;
    P.one_p_kappa3 = 1.0 + kap;
    P.mom_kl = c.nz < kDefaultLevelsPerCta ? c.nz : kDefaultLevelsPerCta;
    P.tr_kl = P.mom_kl;
    // the fp64 copies the kernels read for their fp64 quantities (equal to the
    // fields above on this path; dx64, dy64 and the level table are set with the domain)
    P.rho0_64 = c.rho0;
    P.alpha_t64 = c.alpha_t;
    P.beta_s64 = c.beta_s;
    P.t0_64 = c.t0;
    P.s0_64 = c.s0;
    P.neg_g64 = -c.g;
}

double face_host(int rule, double a, double b) {
    if (rule == 0) return std::min(a, b);
    if (rule == 1) return 0.5 * (a + b);
    const double tot = a + b;
    return tot > 0.0 ? 2.0 * a * b / tot : 0.0;
}

// host geometry, same operations as the device's on-the-fly form
// (reference domain.py:60-154)
void build_host_geometry(oc_handle* h) {
    const int nx = h->nx, ny = h->ny, nz = h->nz;
    const size_t n2 = h->n2, n3 = h->n3;
    const KP& P = h->P;
    h->dz3.assign(n3, 0.0);
    h->mask3.assign(n3, 0.0);
    for (int k = 0; k < nz; ++k)
        for (size_t c = 0; c < n2; ++c) {
            const double rem = h->H[c] - P.edge[k];
            double dz = std::min(std::max(rem, 0.0), P.dzr[k]);
            if (dz > 0.0 && dz < P.thin[k]) dz = 0.0;
            const double m3 = (dz > 0.0 ? 1.0 : 0.0) * h->mask[c];
            h->dz3[k * n2 + c] = dz * m3;
            h->mask3[k * n2 + c] = m3;
        }
    h->mask3u.assign(n3, 0.0);
    h->mask3v.assign(n3, 0.0);
    h->dz3u.assign(n3, 0.0);
    h->dz3v.assign(n3, 0.0);
    h->zc.assign(n3, 0.0);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const size_t c = (size_t)j * nx + i, o = k * n2;
                const size_t ce = (size_t)j * nx + (i + 1) % nx, cn = (size_t)((j + 1) % ny) * nx + i;
                h->mask3u[o + c] = h->mask3[o + c] * h->mask3[o + ce] * h->mask_u[c];
                h->mask3v[o + c] = h->mask3[o + c] * h->mask3[o + cn] * h->mask_v[c];
                h->dz3u[o + c] = h->mask3u[o + c] * face_host(P.face_rule, h->dz3[o + c], h->dz3[o + ce]);
                h->dz3v[o + c] = h->mask3v[o + c] * face_host(P.face_rule, h->dz3[o + c], h->dz3[o + cn]);
            }
    for (size_t c = 0; c < n2; ++c) {
        double above = 0.0;
        for (int k = 0; k < nz; ++k) {
            h->zc[k * n2 + c] = above + 0.5 * h->dz3[k * n2 + c];
            above = (k == 0) ? h->dz3[c] : above + h->dz3[k * n2 + c];
        }
    }
}

// surface stress at the faces and u*^2 (model3d_v05.py:176, 355-356; field form
// reduces to it for a uniform field)
int upload_stress(oc_handle* h) {
    const int nx = h->nx, ny = h->ny;
    const size_t n2 = h->n2;
    const oc_config& c = h->cfg;
    std::vector<double> tu(n2), tv(n2), us(n2);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t k = (size_t)j * nx + i;
            const size_t ke = (size_t)j * nx + (i + 1) % nx, kn = (size_t)((j + 1) % ny) * nx + i;
            if (!h->stress_field) {
                tu[k] = (c.tau_x / c.rho0) * h->mask3u[k];
                tv[k] = (c.tau_y / c.rho0) * h->mask3v[k];
                us[k] = std::hypot(c.tau_x, c.tau_y) / c.rho0;
            } else {
                tu[k] = (0.5 * (h->taux_c[k] + h->taux_c[ke])) / c.rho0 * h->mask3u[k];
                tv[k] = (0.5 * (h->tauy_c[k] + h->tauy_c[kn])) / c.rho0 * h->mask3v[k];
                us[k] = std::hypot(h->taux_c[k], h->tauy_c[k]) / c.rho0;
            }
        }
    cudaMemcpy(h->d_tau_u, tu.data(), n2 * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_tau_v, tv.data(), n2 * sizeof(double), cudaMemcpyHostToDevice);
    const cudaError_t e = cudaMemcpy(h->d_ustar2, us.data(), n2 * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(h, e, "stress upload");
    return h->mixed ? mixed_upload_stress(h) : OC_OK;
}

// q, Ku, Kv and the Helmholtz levels for the current K_m (model3d_v05.py:141-167)
int build_coefficients(oc_handle* h, cudaStream_t s, bool count_rebuild) {
    if (h->mixed) {
        const int rc = mixed_build_coefficients(h, s);
        if (rc) return rc;
        h->tridiag += 1;
        if (h->solver) {
            h->solver->rebuild(s);
            if (count_rebuild) h->rebuilds += 1;
        }
        return check_launch(h, "coefficients");
    }
    launch_qsolve(h->P, h->km, h->q, s);
    h->tridiag += 1;
    launch_kukv(h->P, h->q, h->Ku, h->Kv, s);
    if (h->solver) {
        h->solver->rebuild(s);
        if (count_rebuild) h->rebuilds += 1;
    }
    return check_launch(h, "coefficients");
}

int ensure_log(oc_handle* h, long long needed, cudaStream_t s) {
    if (!h->solver) return OC_OK;
    if (needed <= h->solver->log_capacity()) return OC_OK;
    long long cap = h->solver->log_capacity();
    while (cap < needed) cap *= 2;
    return h->solver->grow_log((int)std::min<long long>(cap, 1 << 30), s, h->err);
}

// ---- per-kernel event timing
void prof_harvest(oc_handle* h) {
    if (h->ev_marks.empty()) return;
    for (const auto& m : h->ev_marks) {
        float ms = 0.0f;
        cudaEventSynchronize(h->ev_pool[m.second + 1]);  // launches on two streams complete out of order
        cudaEventElapsedTime(&ms, h->ev_pool[m.second], h->ev_pool[m.second + 1]);
        h->prof_ms[m.first] += ms;
    }
    h->ev_marks.clear();
    h->ev_used = 0;
}

int prof_class(oc_handle* h, const char* name) {
    for (size_t i = 0; i < h->prof_names.size(); ++i)
        if (h->prof_names[i] == name) return (int)i;
    h->prof_names.push_back(name);
    h->prof_launches.push_back(0);
    h->prof_ms.push_back(0.0);
    return (int)h->prof_names.size() - 1;
}


// one step (model3d_v05.py:337-415)
int step_once(oc_handle* h, cudaStream_t s) {
    if (h->mixed) return step_once_mixed(h, s);
    const oc_config& c = h->cfg;
    const KP& P = h->P;
    const int cur = h->cur, nxt = 1 - cur;
    double *u = h->U[cur], *v = h->V[cur], *b = h->B[cur], *eta = h->ETA[cur];
    double *un = h->U[nxt], *vn = h->V[nxt], *etan = h->ETA[nxt];
    const bool theta = c.scheme == OC_SCHEME_THETA, split = c.scheme == OC_SCHEME_SPLIT;
    // The kernels of the old state that do not depend on the closure (phi, the
    // barotropic gradient, transports and divergence) run on a second stream,
    // beside the closure chain (TKE closure -> Ku/Kv -> multigrid rebuild);
    // both join before the explicit momentum terms. w of the old velocities is
    // already in h->w: the state setters compute it and every step ends by
    // computing it for the velocities it leaves behind.
    cudaStream_t a = h->aux;
    cudaEventRecord(h->fork, s);
    cudaStreamWaitEvent(a, h->fork, 0);
    { Prof pr(h, a, "phi"); launch_phi(P, b, h->phi, a); }
    if (!split) { Prof pr(h, a, "grad2"); launch_grad2(P, eta, h->gx2, h->gy2, a); }
    if (theta) {
        { Prof pr(h, a, "transport"); launch_transport(P, u, v, h->Uold, h->Vold, a); }
        { Prof pr(h, a, "div2"); launch_div2(P, h->Uold, h->Vold, h->div_old, a); }
    }
    if (split) { Prof pr(h, a, "transport"); launch_transport(P, u, v, h->bt[0], h->bt[1], a); }  // U0, V0
    cudaEventRecord(h->join, a);
    if (c.closure == OC_CLOSURE_TKE) {
        { Prof pr(h, s, "closure"); launch_closure(P, u, v, b, h->e, h->km, h->kh, h->q, s); }
        h->tridiag += 2;
        { Prof pr(h, s, "kukv"); launch_kukv(P, h->q, h->Ku, h->Kv, s); }
        if (theta) {
            { Prof pr(h, s, "helm_rebuild", h->solver->n_levels()); h->solver->rebuild(s); }
            h->rebuilds += 1;
        }
    }
    cudaStreamWaitEvent(s, h->join, 0);
    {
        Prof pr(h, s, "mom_explicit");
        launch_mom_explicit(P, u, v, b, h->phi, h->w, h->km, h->pgx, h->pgy, h->avpv, h->avpu, h->dzu,
                            h->dzv, h->stu, h->stv, s);
    }
    const double *uit = u, *vit = v;
    double *last_gu = nullptr, *last_gv = nullptr;
    for (int m = 0; m < c.n_picard; ++m) {
        const bool last = m == c.n_picard - 1;
        double *tu, *tv;
        if (theta) {
            tu = h->ghu;
            tv = h->ghv;
        } else if (last && !split) {
            tu = un;
            tv = vn;
        } else {
            tu = (m % 2 == 0) ? h->ghu : h->uit;
            tv = (m % 2 == 0) ? h->ghv : h->vit;
        }
        {
            Prof pr(h, s, "predictor_rhs");
            launch_predictor_rhs(P, u, v, uit, vit, h->pgx, h->pgy, h->avpv, h->avpu, h->dzu, h->dzv,
                                 h->stu, h->stv, h->gx2, h->gy2, tu, tv, s);
        }
        { Prof pr(h, s, "momentum_solve"); launch_momentum_solve(P, h->km, tu, tv, h->Ug, h->Vg, s); }
        h->tridiag += 2;
        if (theta) {
            { Prof pr(h, s, "helm_rhs"); launch_helm_rhs(P, eta, h->div_old, h->Ug, h->Vg, h->rhs2, s); }
            int rc = ensure_log(h, h->solves + 1, s);  // graphs reserve the log before recording
            if (rc) return rc;
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
            double* ou = last ? un : h->uit;
            double* ov = last ? vn : h->vit;
            { Prof pr(h, s, "backsub"); launch_backsub(P, h->ghu, h->ghv, h->q, etan, ou, ov, s); }
            uit = ou;
            vit = ov;
        } else {
            uit = tu;
            vit = tv;
            last_gu = tu;
            last_gv = tv;
        }
    }
    if (c.scheme == OC_SCHEME_FB) { Prof pr(h, s, "eta_fb"); launch_eta_fb(P, eta, h->Ug, h->Vg, etan, s); }
    if (split) {
        double *U0 = h->bt[0], *V0 = h->bt[1], *fx = h->bt[2], *fy = h->bt[3];
        double *avv = h->bt[4], *avu = h->bt[5], *gxe = h->bt[6], *gye = h->bt[7];
        double* Ub[3] = {h->bt[8], h->bt[10], h->Uold};
        double* Vb[3] = {h->bt[9], h->bt[11], h->Vold};
        double *accu = h->gx2, *accv = h->gy2;
        { Prof pr(h, s, "split_forcing"); launch_split_forcing(P, U0, V0, h->Ug, h->Vg, fx, fy, s); }
        cudaMemcpyAsync(etan, eta, h->n2 * sizeof(double), cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(Ub[0], U0, h->n2 * sizeof(double), cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(Vb[0], V0, h->n2 * sizeof(double), cudaMemcpyDeviceToDevice, s);
        const double ddt = c.dt / h->n_split;
        int ib = 0;
        for (int n = 0; n < h->n_split; ++n) {
            { Prof pr(h, s, "split_sub_avg"); launch_split_sub_avg(P, Ub[ib], Vb[ib], etan, avv, avu, gxe, gye, s); }
            int ii = ib;
            for (int qi = 0; qi < c.n_picard; ++qi) {
                int io = 0;
                while (io == ib || io == ii) ++io;
                Prof pr(h, s, "split_sub_mom");
                launch_split_sub_mom(P, ddt, Ub[ib], Vb[ib], Ub[ii], Vb[ii], avv, avu, gxe, gye, h->Ku,
                                     h->Kv, fx, fy, Ub[io], Vb[io], s);
                ii = io;
            }
            ib = ii;
            { Prof pr(h, s, "split_sub_eta"); launch_split_sub_eta(P, ddt, Ub[ib], Vb[ib], etan, accu, accv, n == 0 ? 1 : 0, s); }
        }
        h->substeps += h->n_split;
        const double *Uf = Ub[ib], *Vf = Vb[ib];
        if (c.barotropic_average == OC_BTAVG_MEAN) {
            { Prof pr(h, s, "split_mean"); launch_split_mean(P, h->n_split, accu, accv, s); }
            Uf = accu;
            Vf = accv;
        }
        { Prof pr(h, s, "split_correct"); launch_split_correct(P, last_gu, last_gv, h->Ug, h->Vg, Uf, Vf, un, vn, s); }
    }
    { Prof pr(h, s, "wcol"); launch_wcol(P, un, vn, h->w, s); }
    {
        // the explicit momentum terms are dead by now: their buffers hold the tracer right-hand sides
        Prof pr(h, s, "tracer_rhs");
        launch_tracer_rhs(P, c.tracers == OC_TRACERS_TS ? h->Tt[cur] : b, h->Ss[cur], un, vn, h->w, h->kh, h->pgx,
                          h->pgy, s);
    }
    {
        Prof pr(h, s, "tracer_solve");
        launch_tracer_solve(P, h->pgx, h->pgy, h->kh, h->Tt[nxt], h->Ss[nxt], h->B[nxt], s);
    }
    h->tridiag += (c.tracers == OC_TRACERS_TS) ? 2 : 1;
    h->cur = nxt;
    h->steps += 1;
    return check_launch(h, "step");
}

void drop_graphs(oc_handle* h) {
    ++h->graph_version;
    for (auto& g : h->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

// Record two steps from the current buffers into a graph. Nothing runs: the
// host state the recording advanced (buffer index, counters) is put back and
// the counters one launch stands for are kept.
int capture_graph(oc_handle* h) {
    if (!h->capture_stream && cudaStreamCreateWithFlags(&h->capture_stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(h, OC_ERR_CUDA, "cudaStreamCreate failed");
    const int cur = h->cur;
    const oc_handle::Counters before{h->steps, h->tridiag, h->rebuilds, h->substeps, h->solves, h->launches};
    const bool prof = h->profiling;
    h->profiling = false;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(h->capture_stream, cudaStreamCaptureModeThreadLocal);
    int rc = e == cudaSuccess ? OC_OK : cuda_fail(h, e, "graph capture begin");
    for (int n = 0; n < 2 && rc == OC_OK; ++n) rc = step_once(h, h->capture_stream);
    e = cudaStreamEndCapture(h->capture_stream, &g);
    h->profiling = prof;
    const oc_handle::Counters after{h->steps, h->tridiag, h->rebuilds, h->substeps, h->solves, h->launches};
    h->cur = cur;
    h->steps = before.steps;
    h->tridiag = before.tridiag;
    h->rebuilds = before.rebuilds;
    h->substeps = before.substeps;
    h->solves = before.solves;
    h->launches = before.launches;
    if (rc == OC_OK && e != cudaSuccess) rc = cuda_fail(h, e, "graph capture (a step call cannot be recorded)");
    if (rc == OC_OK && cudaGraphInstantiate(&h->graph[cur], g, 0) != cudaSuccess)
        rc = fail(h, OC_ERR_CUDA, "graph instantiation failed");
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    if (rc) {
        h->graph[cur] = nullptr;
        return rc;
    }
    h->graph_delta[cur] = {after.steps - before.steps, after.tridiag - before.tridiag, after.rebuilds - before.rebuilds,
                           after.substeps - before.substeps, after.solves - before.solves,
                           after.launches - before.launches};
    return OC_OK;
}

}  // namespace oc

namespace oc {
// the solves of the steps an ensemble records with batched solves: per member,
// in recording order, the placeholder nodes each solve was replaced by
struct BatchRecorder {
    struct Deferred {
        const double* rhs;
        double* x;
        cudaGraphNode_t pre, post;
    };
    std::vector<std::vector<Deferred>> per_member;
    int member = 0;
};

int batch_defer(oc_handle* h, cudaStream_t s, const double* rhs, double* x) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd);
    if (e != cudaSuccess || st != cudaStreamCaptureStatusActive)
        return fail(h, OC_ERR_CUDA, "a deferred solve outside a recording");
    cudaGraphNode_t pre = nullptr, post = nullptr;
    e = cudaGraphAddEmptyNode(&pre, g, deps, nd);
    if (e == cudaSuccess) e = cudaGraphAddEmptyNode(&post, g, &pre, 1);
    if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(s, &post, 1, cudaStreamSetCaptureDependencies);
    if (e != cudaSuccess) return cuda_fail(h, e, "deferred solve");
    BatchRecorder* r = h->batch_rec;
    r->per_member[r->member].push_back({rhs, x, pre, post});
    return OC_OK;
}
}  // namespace oc

extern "C" {

const char* oc_version(void) {
    return "ocean_b200 1.1 (sm_100a; fp64 path bit-identical to the NumPy reference; mixed FP32/FP64 path)";
}

int oc_create(const oc_config* cfg, oc_handle** out) {
    if (!cfg || !out) return OC_ERR_ARG;
    *out = nullptr;
    std::string err;
    const int rc = validate(cfg, err);
    if (rc) {
        std::fprintf(stderr, "oc_create: %s\n", err.c_str());
        return rc;
    }
    cudaError_t e = cudaSetDevice(cfg->device);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "oc_create: cudaSetDevice(%d): %s\n", cfg->device, cudaGetErrorString(e));
        return OC_ERR_CUDA;
    }
    oc_handle* h = new oc_handle();
    h->cfg = *cfg;
    if (cudaStreamCreateWithFlags(&h->aux, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming) != cudaSuccess) {
        std::fprintf(stderr, "oc_create: stream or event creation failed\n");
        delete h;
        return OC_ERR_CUDA;
    }
    h->nx = cfg->nx;
    h->ny = cfg->ny;
    h->nz = cfg->nz;
    h->n2 = (size_t)cfg->nx * cfg->ny;
    h->n3 = h->n2 * cfg->nz;
    h->n3i = h->n2 * (cfg->nz + 1);
    h->mixed = cfg->precision == OC_PRECISION_MIXED;
    fill_scalars(h);
    *out = h;
    return OC_OK;
}

// the domain: masks, partial cells, face thicknesses and the device buffers.
// mask_u_in / mask_v_in, when given, replace the face masks the boundary
// conditions would give (a slab of a larger domain carries the larger domain's).
static int set_domain_impl(oc_handle* h, const double* Hh, const double* maskh, const double* dzrh,
                           const double* mask_u_in, const double* mask_v_in) {
    if (!h || !Hh || !maskh) return fail(h, OC_ERR_ARG, "H and mask are required");
    if (h->has_domain) return fail(h, OC_ERR_STATE, "the domain is already set");
    cudaSetDevice(h->cfg.device);
    const int nx = h->nx, ny = h->ny, nz = h->nz;
    const size_t n2 = h->n2;
    h->H.assign(Hh, Hh + n2);
    h->mask.assign(maskh, maskh + n2);
    bool any_wet = false;
    double hmax = 0.0;
    for (size_t c = 0; c < n2; ++c) {
        if (h->mask[c] > 0.0) {
            if (!(h->H[c] > 0.0)) return fail(h, OC_ERR_ARG, "bathymetry must be positive in every wet cell");
            hmax = any_wet ? std::max(hmax, h->H[c]) : h->H[c];
            any_wet = true;
        }
    }
    if (!any_wet) return fail(h, OC_ERR_ARG, "the domain has no wet cell");
    h->h_max = hmax;
    h->mask_u.assign(n2, 0.0);
    h->mask_v.assign(n2, 0.0);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t c = (size_t)j * nx + i;
            h->mask_u[c] = h->mask[c] * h->mask[(size_t)j * nx + (i + 1) % nx];
            h->mask_v[c] = h->mask[c] * h->mask[(size_t)((j + 1) % ny) * nx + i];
            if (h->cfg.bc_x != OC_BC_PERIODIC && i == nx - 1) h->mask_u[c] = 0.0;
            if (h->cfg.bc_y != OC_BC_PERIODIC && j == ny - 1) h->mask_v[c] = 0.0;
        }
    if (mask_u_in && mask_v_in) {
        for (size_t c = 0; c < n2; ++c) {
            const double mu = mask_u_in[c], mv = mask_v_in[c];
            if ((mu != 0.0 && mu != 1.0) || (mv != 0.0 && mv != 1.0))
                return fail(h, OC_ERR_ARG, "face mask values must be 0 or 1");
            h->mask_u[c] = mu;
            h->mask_v[c] = mv;
        }
    }
    h->dzr.assign(nz, hmax / nz);
    if (dzrh) {
        for (int k = 0; k < nz; ++k) {
            if (!(dzrh[k] > 0.0)) return fail(h, OC_ERR_ARG, "level thicknesses must be > 0");
            h->dzr[k] = dzrh[k];
        }
    }
    KP& P = h->P;
    P.edge[0] = 0.0;
    for (int k = 0; k < nz; ++k) {
        P.edge[k + 1] = (k == 0) ? h->dzr[0] : P.edge[k] + h->dzr[k];
        P.dzr[k] = h->dzr[k];
        P.thin[k] = h->cfg.min_partial * h->dzr[k];
        P.dz_nom[k] = h->cfg.h0 / nz;  // the reference's nominal H/nz (model3d_v05.py:247)
    }
    for (int k = 0; k <= nz; ++k) P.edge64[k] = P.edge[k];
    for (int k = 0; k < nz; ++k) P.dzr64[k] = P.dzr[k];
    P.dx64 = P.dx;
    P.dy64 = P.dy;
    build_host_geometry(h);
    // compact per-column form of the z-level geometry (kfull, kb, two explicit
    // thicknesses), accepted only where it reproduces the formula exactly
    std::vector<int2> kinfo(n2);
    std::vector<double2> dzx(n2);
    std::vector<int2> kface(n2);
    for (size_t c = 0; c < n2; ++c) {
        if (h->mask[c] != 0.0 && h->mask[c] != 1.0) return fail(h, OC_ERR_ARG, "mask values must be 0 or 1");
        int kb = 0;
        while (kb < nz && h->mask3[(size_t)kb * n2 + c] > 0.0) ++kb;
        for (int k = kb; k < nz; ++k)
            if (h->mask3[(size_t)k * n2 + c] > 0.0)
                return fail(h, OC_ERR_UNSUPPORTED, "a column has a dry level above a wet one");
        int kf = 0;
        while (kf < kb && h->dz3[(size_t)kf * n2 + c] == h->dzr[kf]) ++kf;
        if (kb - kf > 2)
            return fail(h, OC_ERR_UNSUPPORTED, "a column has more than two partial levels");
        kinfo[c] = make_int2(kf, kb);
        int ku = 0, kv = 0;
        while (ku < nz && h->mask3u[(size_t)ku * n2 + c] > 0.0) ++ku;
        while (kv < nz && h->mask3v[(size_t)kv * n2 + c] > 0.0) ++kv;
        for (int k = 0; k < nz; ++k)
            if (h->mask3u[(size_t)k * n2 + c] != (k < ku ? 1.0 : 0.0) ||
                h->mask3v[(size_t)k * n2 + c] != (k < kv ? 1.0 : 0.0))
                return fail(h, OC_ERR_UNSUPPORTED, "a face mask is not a contiguous top block of 0/1 levels");
        kface[c] = make_int2(ku, kv);
        dzx[c] = make_double2(kf < kb ? h->dz3[(size_t)kf * n2 + c] : 0.0,
                              kf + 1 < kb ? h->dz3[(size_t)(kf + 1) * n2 + c] : 0.0);
    }
    if (h->cfg.scheme == OC_SCHEME_SPLIT) {
        const double cc = std::sqrt(h->cfg.g * hmax);
        const double dt_baro = 1.0 / (cc * std::sqrt(1.0 / std::pow(P.dx, 2.0) + 1.0 / std::pow(P.dy, 2.0)));
        h->n_split = h->cfg.n_split > 0 ? h->cfg.n_split
                                        : std::max(1, (int)std::ceil(1.2 * h->cfg.dt / dt_baro));
        if (h->cfg.dt / h->n_split > dt_baro)
            return fail(h, OC_ERR_ARG, "n_split leaves a barotropic substep above the gravity-wave limit");
    }
    // device buffers
    const size_t n3 = h->n3, n3i = h->n3i;
    h->d_H = dalloc(h, n2);
    h->d_mask = dalloc(h, n2);
    h->d_mask_u = dalloc(h, n2);
    h->d_mask_v = dalloc(h, n2);
    h->d_tau_u = dalloc(h, n2);
    h->d_tau_v = dalloc(h, n2);
    h->d_ustar2 = dalloc(h, n2);
    double* d_kinfo = dalloc(h, n2);
    double* d_dzx = dalloc(h, 2 * n2);
    double* d_kface = dalloc(h, n2);
    const bool ts = h->cfg.tracers == OC_TRACERS_TS;
    const bool f64 = !h->mixed;  // the mixed path keeps its 3D fields in FP32 buffers (mixed.cu)
    h->bound = false;            // a new domain drops caller-owned state buffers
    for (int t = 0; t < 2; ++t) {
        h->U[t] = f64 ? dalloc(h, n3) : nullptr;
        h->V[t] = f64 ? dalloc(h, n3) : nullptr;
        h->B[t] = dalloc(h, n3);
        h->Tt[t] = (ts && f64) ? dalloc(h, n3) : nullptr;
        h->Ss[t] = (ts && f64) ? dalloc(h, n3) : nullptr;
        h->ETA[t] = dalloc(h, n2);
    }
    h->phi = dalloc(h, n3);
    if (f64) {
        h->e = dalloc(h, n3i);
        h->km = dalloc(h, n3i);
        h->kh = dalloc(h, n3i);
        h->w = dalloc(h, n3i);
        for (double** p : {&h->q, &h->pgx, &h->pgy, &h->avpv, &h->avpu, &h->dzu, &h->dzv, &h->stu, &h->stv,
                           &h->ghu, &h->ghv, &h->uit, &h->vit})
            *p = dalloc(h, n3);
    }
    for (double** p : {&h->Ku, &h->Kv, &h->gx2, &h->gy2, &h->Uold, &h->Vold, &h->div_old, &h->Ug, &h->Vg,
                       &h->rhs2})
        *p = dalloc(h, n2);
    for (int t = 0; t < 12; ++t) h->bt[t] = (h->cfg.scheme == OC_SCHEME_SPLIT) ? dalloc(h, n2) : nullptr;
    h->d_part = dalloc(h, 1024);
    {
        void* st = nullptr;
        if (cudaMalloc(&st, sizeof(int)) != cudaSuccess) return fail(h, OC_ERR_CUDA, "cudaMalloc failed");
        cudaMemset(st, 0, sizeof(int));
        h->allocs.push_back(st);
        h->d_status = (int*)st;
    }
    for (void* p : h->allocs)
        if (!p) return fail(h, OC_ERR_CUDA, "device allocation failed");
    if ((f64 && !h->km) || !h->ETA[1] || !h->rhs2) return fail(h, OC_ERR_CUDA, "device allocation failed");
    cudaMemcpy(h->d_H, h->H.data(), n2 * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_mask, h->mask.data(), n2 * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_mask_u, h->mask_u.data(), n2 * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_mask_v, h->mask_v.data(), n2 * sizeof(double), cudaMemcpyHostToDevice);
    P.H = h->d_H;
    P.mask = h->d_mask;
    P.mask_u = h->d_mask_u;
    P.mask_v = h->d_mask_v;
    P.tau_u = h->d_tau_u;
    P.tau_v = h->d_tau_v;
    P.ustar2 = h->d_ustar2;
    cudaMemcpy(d_kinfo, kinfo.data(), n2 * sizeof(int2), cudaMemcpyHostToDevice);
    cudaMemcpy(d_dzx, dzx.data(), n2 * sizeof(double2), cudaMemcpyHostToDevice);
    P.kinfo = reinterpret_cast<const int2*>(d_kinfo);
    P.dzx = reinterpret_cast<const double2*>(d_dzx);
    cudaMemcpy(d_kface, kface.data(), n2 * sizeof(int2), cudaMemcpyHostToDevice);
    P.kface = reinterpret_cast<const int2*>(d_kface);
    P.dzx64 = P.dzx;
    P.mask_u64 = P.mask_u;
    P.mask_v64 = P.mask_v;
    int rc = OC_OK;
    if (h->mixed && (rc = mixed_alloc(h, kinfo, dzx))) return rc;
    rc = upload_stress(h);
    if (rc) return rc;
    if (f64) {
        fill(h->e, h->cfg.e_min, (int64_t)n3i, 0);
        fill(h->km, h->cfg.nu, (int64_t)n3i, 0);
        fill(h->kh, h->cfg.kappa, (int64_t)n3i, 0);
    }
    if (h->cfg.scheme == OC_SCHEME_THETA) {
        h->solver = new HelmSolver();
        const double coef = h->cfg.g * std::pow(h->cfg.theta, 2.0) * std::pow(h->cfg.dt, 2.0);
        rc = h->solver->init(nx, ny, h->cfg.lx / nx, h->cfg.ly / ny, coef, h->cfg.solver, h->cfg.rtol,
                             h->cfg.max_iter, h->mask.data(), h->Ku, h->Kv, 4096, h->d_status, h->err);
        if (rc) return rc;
        h->solver->set_warm_start(h->mixed);  // the fp64 step starts from zero, as the reference
    }
    rc = build_coefficients(h, 0, false);
    if (rc) return rc;
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(h, e, "oc_set_domain");
    h->has_domain = true;
    return OC_OK;
}

int oc_set_domain(oc_handle* h, const double* Hh, const double* maskh, const double* dzrh) {
    return set_domain_impl(h, Hh, maskh, dzrh, nullptr, nullptr);
}

int oc_set_domain_slab(oc_handle* h, const double* Hh, const double* maskh, const double* dzrh,
                       const double* mask_u, const double* mask_v, double dx, double dy) {
    if (!h) return OC_ERR_ARG;
    if (h->has_domain) return fail(h, OC_ERR_STATE, "the domain is already set");
    if (h->cfg.scheme != OC_SCHEME_FB)
        return fail(h, OC_ERR_UNSUPPORTED,
                    "a slab of a larger domain steps with scheme fb only: theta needs a global elliptic solve "
                    "and split_explicit a halo exchange per substep");
    if (h->mixed) return fail(h, OC_ERR_UNSUPPORTED, "slabs of a larger domain step in fp64 only");
    if (!dzrh || !mask_u || !mask_v)
        return fail(h, OC_ERR_ARG, "a slab needs the larger domain's level table and face masks");
    if (!(dx > 0.0) || !(dy > 0.0) || !std::isfinite(dx) || !std::isfinite(dy))
        return fail(h, OC_ERR_ARG, "dx and dy must be finite and > 0");
    h->P.dx = dx;
    h->P.dy = dy;
    return set_domain_impl(h, Hh, maskh, dzrh, mask_u, mask_v);
}

namespace {

// the fields a slab exchanges with its neighbours, in packing order, with their levels
struct HaloField {
    double* ptr;
    int levels;
};

int halo_fields(oc_handle* h, HaloField* out) {
    const int c = h->cur, nz = h->nz;
    int n = 0;
    out[n++] = {h->ETA[c], 1};
    out[n++] = {h->U[c], nz};
    out[n++] = {h->V[c], nz};
    out[n++] = {h->B[c], nz};
    if (h->cfg.tracers == OC_TRACERS_TS) {
        out[n++] = {h->Tt[c], nz};
        out[n++] = {h->Ss[c], nz};
    }
    if (h->cfg.closure == OC_CLOSURE_TKE) {
        out[n++] = {h->e, nz + 1};
        out[n++] = {h->km, nz + 1};
        out[n++] = {h->kh, nz + 1};
    }
    return n;
}

int rows_check(oc_handle* h, int32_t j0, int32_t nrows, const void* buf) {
    if (!h || !buf) return OC_ERR_ARG;
    if (h->mixed) return fail(h, OC_ERR_UNSUPPORTED, "row exchange serves the fp64 slabs only");
    if (!h->has_state) return fail(h, OC_ERR_STATE, "set the state before exchanging rows");
    if (j0 < 0 || nrows < 1 || (int64_t)j0 + nrows > h->ny) return fail(h, OC_ERR_ARG, "rows outside the domain");
    return OC_OK;
}

// copy rows [j0, j0 + nrows) of every exchanged field between the state and a
// packed device buffer (field after field, level after level, row-major)
int copy_rows(oc_handle* h, int32_t j0, int32_t nrows, double* buf, bool pack, cudaStream_t s) {
    HaloField f[9];
    const int n = halo_fields(h, f);
    const size_t nx = h->nx, row_bytes = nx * nrows * sizeof(double);
    size_t off = 0;
    for (int q = 0; q < n; ++q) {
        double* field = f[q].ptr + (size_t)j0 * nx;
        double* packed = buf + off;
        const cudaError_t e =
            pack ? cudaMemcpy2DAsync(packed, row_bytes, field, h->n2 * sizeof(double), row_bytes, f[q].levels,
                                     cudaMemcpyDeviceToDevice, s)
                 : cudaMemcpy2DAsync(field, h->n2 * sizeof(double), packed, row_bytes, row_bytes, f[q].levels,
                                     cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return cuda_fail(h, e, pack ? "oc_pack_rows" : "oc_unpack_rows");
        off += nx * nrows * f[q].levels;
    }
    return OC_OK;
}

}  // namespace

int oc_halo_values_per_row(oc_handle* h, int64_t* count) {
    if (!h || !count) return OC_ERR_ARG;
    if (h->mixed) return fail(h, OC_ERR_UNSUPPORTED, "row exchange serves the fp64 slabs only");
    if (!h->has_domain) return fail(h, OC_ERR_STATE, "set the domain first");
    HaloField f[9];
    const int n = halo_fields(h, f);
    int64_t levels = 0;
    for (int q = 0; q < n; ++q) levels += f[q].levels;
    *count = levels * h->nx;
    return OC_OK;
}

int oc_pack_rows(oc_handle* h, int32_t j0, int32_t nrows, double* buf, void* stream) {
    int rc = rows_check(h, j0, nrows, buf);
    if (rc) return rc;
    cudaSetDevice(h->cfg.device);
    return copy_rows(h, j0, nrows, buf, true, (cudaStream_t)stream);
}

int oc_unpack_rows(oc_handle* h, int32_t j0, int32_t nrows, const double* buf, void* stream) {
    int rc = rows_check(h, j0, nrows, buf);
    if (rc) return rc;
    cudaSetDevice(h->cfg.device);
    cudaStream_t s = (cudaStream_t)stream;
    rc = copy_rows(h, j0, nrows, const_cast<double*>(buf), false, s);
    if (rc) return rc;
    // w of the velocities now in the state, which a step reads first
    launch_wcol(h->P, h->U[h->cur], h->V[h->cur], h->w, s);
    return check_launch(h, "oc_unpack_rows");
}

int oc_set_tiling(oc_handle* h, int32_t mom_levels, int32_t tracer_levels) {
    if (!h) return OC_ERR_ARG;
    if (mom_levels < 1 || mom_levels > h->nz || tracer_levels < 1 || tracer_levels > h->nz)
        return fail(h, OC_ERR_ARG, "levels per CTA must lie in 1..nz");
    h->P.mom_kl = mom_levels;
    h->P.tr_kl = tracer_levels;
    h->P32.mom_kl = mom_levels;
    h->P32.tr_kl = tracer_levels;
    drop_graphs(h);  // recorded launches carry the old values
    return OC_OK;
}

int oc_autotune(oc_handle* h, int32_t* mom_levels, int32_t* tracer_levels) {
    if (!h) return OC_ERR_ARG;
    if (!h->has_state) return fail(h, OC_ERR_STATE, "set the state before tuning");
    cudaSetDevice(h->cfg.device);
    const int c = h->cur, nz = h->nz;
    std::vector<int> cand;
    for (int kl : {2, 3, 4, 5, 6, 8, 10, 13, 17, 25, nz})
        if (kl >= 1 && kl <= nz && std::find(cand.begin(), cand.end(), kl) == cand.end()) cand.push_back(kl);
    cudaStream_t s = nullptr;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // time one kernel class over the candidates (run(kl) launches it with kl levels
    // per CTA); the outputs are scratch that the next step writes again before reading
    auto best_of = [&](int start, auto run) {
        int best = start;
        float best_ms = 1e30f;
        for (int kl : cand) {
            run(kl);
            float ms = 1e30f;
            for (int r = 0; r < 3; ++r) {
                cudaEventRecord(e0, s);
                run(kl);
                cudaEventRecord(e1, s);
                cudaEventSynchronize(e1);
                float t = 0.0f;
                cudaEventElapsedTime(&t, e0, e1);
                ms = std::min(ms, t);
            }
            if (ms < best_ms) {
                best_ms = ms;
                best = kl;
            }
        }
        return best;
    };
    int mk, tk;
    if (h->mixed) {
        // the FP32 kernels of the mixed path on its FP32 fields (TS tracers)
        const KPT<float>& P = h->P32;
        launch_phi(P, h->B[c], h->phi, s);  // the explicit momentum terms read phi
        mk = best_of(P.mom_kl, [&](int kl) {
            KPT<float> Q = P;
            Q.mom_kl = kl;
            launch_mom_explicit(Q, h->U32[c], h->V32[c], h->B[c], h->phi, h->w32, h->km32, h->pgx32, h->pgy32,
                                h->avpv32, h->avpu32, h->dzu32, h->dzv32, h->stu32, h->stv32, s);
        });
        tk = best_of(P.tr_kl, [&](int kl) {
            KPT<float> Q = P;
            Q.tr_kl = kl;
            launch_tracer_rhs(Q, h->T32[c], h->S32[c], h->U32[c], h->V32[c], h->w32, h->kh32, h->pgx32, h->pgy32,
                              s);
        });
    } else {
        const KP& P = h->P;
        launch_phi(P, h->B[c], h->phi, s);
        mk = best_of(P.mom_kl, [&](int kl) {
            KP Q = P;
            Q.mom_kl = kl;
            launch_mom_explicit(Q, h->U[c], h->V[c], h->B[c], h->phi, h->w, h->km, h->pgx, h->pgy, h->avpv, h->avpu,
                                h->dzu, h->dzv, h->stu, h->stv, s);
        });
        tk = best_of(P.tr_kl, [&](int kl) {
            KP Q = P;
            Q.tr_kl = kl;
            launch_tracer_rhs(Q, h->cfg.tracers == OC_TRACERS_TS ? h->Tt[c] : h->B[c], h->Ss[c], h->U[c], h->V[c],
                              h->w, h->kh, h->pgx, h->pgy, s);
        });
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const int rc = check_launch(h, "oc_autotune");
    if (rc) return rc;
    h->P.mom_kl = mk;
    h->P.tr_kl = tk;
    h->P32.mom_kl = mk;
    h->P32.tr_kl = tk;
    drop_graphs(h);
    if (mom_levels) *mom_levels = mk;
    if (tracer_levels) *tracer_levels = tk;
    return OC_OK;
}

int oc_set_forcing(oc_handle* h, const double* taux_c, const double* tauy_c) {
    if (!h) return OC_ERR_ARG;
    drop_graphs(h);
    if (!h->has_domain) return fail(h, OC_ERR_STATE, "set the domain before the forcing");
    cudaSetDevice(h->cfg.device);
    if (!taux_c && !tauy_c) {
        h->stress_field = false;
    } else {
        h->stress_field = true;
        h->taux_c.assign(h->n2, 0.0);
        h->tauy_c.assign(h->n2, 0.0);
        if (taux_c) h->taux_c.assign(taux_c, taux_c + h->n2);
        if (tauy_c) h->tauy_c.assign(tauy_c, tauy_c + h->n2);
    }
    return upload_stress(h);
}

static int copy_in(double* dst, const double* src, size_t n, int on_device, cudaStream_t s) {
    return cudaMemcpyAsync(dst, src, n * sizeof(double),
                           on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s) == cudaSuccess
               ? 0
               : 1;
}

// enqueue the copies (and the derived fields) of a state on stream st
static int set_state_on(oc_handle* h, const oc_state_view* s, int32_t on_device, cudaStream_t st) {
    if (!h || !s) return OC_ERR_ARG;
    if (!h->has_domain) return fail(h, OC_ERR_STATE, "set the domain before the state");
    if (!s->eta || !s->u || !s->v) return fail(h, OC_ERR_ARG, "eta, u and v are required");
    const bool ts = h->cfg.tracers == OC_TRACERS_TS;
    if (ts && (!s->T || !s->S)) return fail(h, OC_ERR_ARG, "T and S are required with TS tracers");
    if (!ts && !s->b) return fail(h, OC_ERR_ARG, "b is required with buoyancy tracers");
    cudaSetDevice(h->cfg.device);
    if (h->mixed) {
        const int rc = mixed_set_state(h, s, on_device, st);
        if (rc) return rc;
        h->has_state = true;
        return OC_OK;
    }
    const int c = h->cur;
    int bad = 0;
    bad |= copy_in(h->ETA[c], s->eta, h->n2, on_device, st);
    bad |= copy_in(h->U[c], s->u, h->n3, on_device, st);
    bad |= copy_in(h->V[c], s->v, h->n3, on_device, st);
    if (ts) {
        bad |= copy_in(h->Tt[c], s->T, h->n3, on_device, st);
        bad |= copy_in(h->Ss[c], s->S, h->n3, on_device, st);
    }
    if (s->b)
        bad |= copy_in(h->B[c], s->b, h->n3, on_device, st);
    else
        launch_diag_buoyancy(h->P, h->Tt[c], h->Ss[c], h->B[c], st);
    if (s->e)
        bad |= copy_in(h->e, s->e, h->n3i, on_device, st);
    else
        fill(h->e, h->cfg.e_min, (int64_t)h->n3i, st);
    if (s->km) bad |= copy_in(h->km, s->km, h->n3i, on_device, st);
    if (s->kh) bad |= copy_in(h->kh, s->kh, h->n3i, on_device, st);
    if (bad) return fail(h, OC_ERR_CUDA, "state copy failed");
    // w of the new velocities (vertical_var.py:109-121), which a step reads first
    launch_wcol(h->P, h->U[c], h->V[c], h->w, st);
    if (s->km) {
        // coefficients of the given viscosity (model3d_v05.py:141-167)
        launch_qsolve(h->P, h->km, h->q, st);
        launch_kukv(h->P, h->q, h->Ku, h->Kv, st);
        if (h->solver) h->solver->rebuild(st);
    }
    h->has_state = true;
    return OC_OK;
}

int oc_set_state(oc_handle* h, const oc_state_view* s, int32_t on_device) {
    const int rc = set_state_on(h, s, on_device, 0);
    if (rc) return rc;
    const cudaError_t e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) return cuda_fail(h, e, "oc_set_state");
    return OC_OK;
}

int oc_set_state_async(oc_handle* h, const oc_state_view* s, int32_t on_device, void* stream) {
    return set_state_on(h, s, on_device, (cudaStream_t)stream);
}

// the handle's state pointers in one array: ETA, U, V, B, Tt, Ss of parity 0,
// the same of parity 1, then e, km, kh
static void state_slots(oc_handle* h, double** slot[15]) {
    double** per[6] = {h->ETA, h->U, h->V, h->B, h->Tt, h->Ss};
    for (int p = 0; p < 2; ++p)
        for (int f = 0; f < 6; ++f) slot[6 * p + f] = &per[f][p];
    slot[12] = &h->e;
    slot[13] = &h->km;
    slot[14] = &h->kh;
}

int oc_bind_state(oc_handle* h, const oc_state_view* a, const oc_state_view* b) {
    if (!h) return OC_ERR_ARG;
    if (!h->has_domain) return fail(h, OC_ERR_STATE, "set the domain before binding a state");
    if (h->mixed)
        return fail(h, OC_ERR_UNSUPPORTED, "the mixed-precision step keeps FP32 state fields; bind needs fp64 ones");
    if ((a == nullptr) != (b == nullptr)) return fail(h, OC_ERR_ARG, "give both buffer sets, or neither");
    cudaSetDevice(h->cfg.device);
    // the step may still be writing the buffers about to be replaced
    cudaError_t err = cudaDeviceSynchronize();
    if (err != cudaSuccess) return cuda_fail(h, err, "oc_bind_state");
    double** slot[15];
    state_slots(h, slot);
    if (!a) {
        if (h->bound)
            for (int i = 0; i < 15; ++i) *slot[i] = h->own_state[i];
        h->bound = false;
        h->has_state = false;
        drop_graphs(h);
        return OC_OK;
    }
    const bool ts = h->cfg.tracers == OC_TRACERS_TS;
    const size_t fsize[6] = {h->n2, h->n3, h->n3, h->n3, h->n3, h->n3};
    struct Buf {
        double* p;
        size_t n;
        int slot;  // index into slot[] for the current parity's set (parity 0 numbering)
    };
    std::vector<Buf> bufs;
    const oc_state_view* sets[2] = {a, b};
    for (int which = 0; which < 2; ++which) {
        const oc_state_view* s = sets[which];
        double* f[6] = {s->eta, s->u, s->v, s->b, s->T, s->S};
        const int nf = ts ? 6 : 4;
        for (int i = 0; i < nf; ++i) {
            if (!f[i]) return fail(h, OC_ERR_ARG, "eta, u, v, b (and T, S with TS tracers) are required in both sets");
            bufs.push_back({f[i], fsize[i], 6 * which + i});
        }
    }
    double* opt[3] = {a->e, a->km, a->kh};
    for (int i = 0; i < 3; ++i)
        if (opt[i]) bufs.push_back({opt[i], h->n3i, 12 + i});
    for (const Buf& x : bufs) {
        if (reinterpret_cast<uintptr_t>(x.p) % alignof(double))
            return fail(h, OC_ERR_ARG, "a bound buffer is not 8-byte aligned");
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, x.p) != cudaSuccess ||
            (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) || at.device != h->cfg.device) {
            cudaGetLastError();
            return fail(h, OC_ERR_ARG, "a bound buffer is not device memory of the handle's device");
        }
    }
    for (size_t i = 0; i < bufs.size(); ++i)
        for (size_t j = i + 1; j < bufs.size(); ++j) {
            const char *p0 = reinterpret_cast<const char*>(bufs[i].p), *p1 = reinterpret_cast<const char*>(bufs[j].p);
            if (p0 < p1 + bufs[j].n * sizeof(double) && p1 < p0 + bufs[i].n * sizeof(double))
                return fail(h, OC_ERR_ARG, "two bound buffers overlap");
        }
    if (!h->bound)
        for (int i = 0; i < 15; ++i) h->own_state[i] = *slot[i];
    // set a becomes the current parity, set b the other one
    const int c = h->cur;
    for (int i = 0; i < 15; ++i) *slot[i] = h->own_state[i];
    for (const Buf& x : bufs) {
        int idx = x.slot;
        if (idx < 12) idx = 6 * ((idx / 6) ^ c) + idx % 6;
        *slot[idx] = x.p;
    }
    h->bound = true;
    h->bound_base = c;
    if (!a->e) fill(h->e, h->cfg.e_min, (int64_t)h->n3i, 0);
    launch_wcol(h->P, h->U[c], h->V[c], h->w, 0);
    if (a->km) {
        launch_qsolve(h->P, h->km, h->q, 0);
        launch_kukv(h->P, h->q, h->Ku, h->Kv, 0);
        if (h->solver) h->solver->rebuild(0);
    }
    drop_graphs(h);
    h->has_state = true;
    err = cudaDeviceSynchronize();
    return err == cudaSuccess ? check_launch(h, "oc_bind_state") : cuda_fail(h, err, "oc_bind_state");
}

int oc_state_parity(oc_handle* h, int32_t* which) {
    if (!h || !which) return OC_ERR_ARG;
    *which = h->bound ? (h->cur ^ h->bound_base) : 0;
    return OC_OK;
}

int oc_reset_mixing(oc_handle* h) {
    if (!h) return OC_ERR_ARG;
    if (!h->has_domain) return fail(h, OC_ERR_STATE, "set the domain first");
    cudaSetDevice(h->cfg.device);
    if (h->mixed) {
        int rc = mixed_reset_mixing(h, 0);
        if (rc) return rc;
        if (h->solver) h->solver->rebuild(0);
        const cudaError_t e = cudaDeviceSynchronize();
        return e == cudaSuccess ? OC_OK : cuda_fail(h, e, "oc_reset_mixing");
    }
    fill(h->km, h->cfg.nu, (int64_t)h->n3i, 0);
    fill(h->kh, h->cfg.kappa, (int64_t)h->n3i, 0);
    launch_qsolve(h->P, h->km, h->q, 0);
    launch_kukv(h->P, h->q, h->Ku, h->Kv, 0);
    if (h->solver) h->solver->rebuild(0);
    const cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? OC_OK : cuda_fail(h, e, "oc_reset_mixing");
}

static int device_status(oc_handle* h) {
    int st = 0;
    cudaMemcpy(&st, h->d_status, sizeof(int), cudaMemcpyDeviceToHost);
    return st;
}

// enqueue the copies of the current state on stream st
static int get_state_on(oc_handle* h, const oc_state_view* s, int32_t on_device, cudaStream_t st) {
    if (h->mixed) return mixed_get_state(h, s, on_device, st);
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    const int c = h->cur;
    const bool ts = h->cfg.tracers == OC_TRACERS_TS;
    struct {
        double* dst;
        const double* src;
        size_t n;
    } items[] = {{s->eta, h->ETA[c], h->n2}, {s->u, h->U[c], h->n3},   {s->v, h->V[c], h->n3},
                 {s->b, h->B[c], h->n3},     {ts ? s->T : nullptr, h->Tt[c], h->n3},
                 {ts ? s->S : nullptr, h->Ss[c], h->n3}, {s->e, h->e, h->n3i},
                 {s->km, h->km, h->n3i},     {s->kh, h->kh, h->n3i}};
    for (auto& it : items) {
        if (!it.dst || !it.src) continue;
        const cudaError_t e = cudaMemcpyAsync(it.dst, it.src, it.n * sizeof(double), kind, st);
        if (e != cudaSuccess) return cuda_fail(h, e, "oc_get_state copy");
    }
    return OC_OK;
}

int oc_get_state(oc_handle* h, const oc_state_view* s, int32_t on_device) {
    if (!h || !s) return OC_ERR_ARG;
    if (!h->has_state) return fail(h, OC_ERR_STATE, "no state has been set");
    cudaSetDevice(h->cfg.device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(h, e, "oc_get_state");
    const int dst = device_status(h);
    if (dst) return fail(h, dst, "a device-side wait ran out its bound");
    const int rc = get_state_on(h, s, on_device, 0);
    if (rc) return rc;
    e = cudaStreamSynchronize(0);
    return e == cudaSuccess ? OC_OK : cuda_fail(h, e, "oc_get_state");
}

int oc_get_state_async(oc_handle* h, const oc_state_view* s, int32_t on_device, void* stream) {
    if (!h || !s) return OC_ERR_ARG;
    if (!h->has_state) return fail(h, OC_ERR_STATE, "no state has been set");
    cudaSetDevice(h->cfg.device);
    return get_state_on(h, s, on_device, (cudaStream_t)stream);
}

int oc_step(oc_handle* h, int32_t n_steps, void* stream) {
    if (!h) return OC_ERR_ARG;
    if (!h->has_state) return fail(h, OC_ERR_STATE, "set the state before stepping");
    if (n_steps < 0) return fail(h, OC_ERR_ARG, "n_steps must be >= 0");
    cudaSetDevice(h->cfg.device);
    cudaStream_t s = (cudaStream_t)stream;
    h->last_stream = s;
    for (int n = 0; n < n_steps; ++n) {
        const int rc = step_once(h, s);
        if (rc) return rc;
    }
    return OC_OK;
}

int oc_step_graph(oc_handle* h, int32_t n_steps, void* stream) {
    if (!h) return OC_ERR_ARG;
    if (!h->has_state) return fail(h, OC_ERR_STATE, "set the state before stepping");
    if (n_steps < 0) return fail(h, OC_ERR_ARG, "n_steps must be >= 0");
    cudaSetDevice(h->cfg.device);
    cudaStream_t s = (cudaStream_t)stream;
    h->last_stream = s;
    if (h->profiling) return oc_step(h, n_steps, stream);  // per-kernel events need the launches one by one
    const int pairs = n_steps / 2;
    if (pairs > 0) {
        // the solve log must hold every solve of the launches without moving:
        // reserve it (and record again if it had to grow)
        const long long per_pair = h->solver ? 2LL * h->cfg.n_picard : 0;
        const long long need = h->solves + per_pair * pairs + per_pair;
        if (h->solver && need > h->solver->log_capacity()) {
            const int rc = ensure_log(h, 2 * need, s);
            if (rc) return rc;
            drop_graphs(h);
        }
        if (!h->graph[h->cur]) {
            const int rc = capture_graph(h);
            if (rc) return rc;
        }
        const int g = h->cur;
        const oc_handle::Counters& d = h->graph_delta[g];
        for (int i = 0; i < pairs; ++i) {
            const cudaError_t e = cudaGraphLaunch(h->graph[g], s);
            if (e != cudaSuccess) return cuda_fail(h, e, "graph launch");
            h->steps += d.steps;
            h->tridiag += d.tridiag;
            h->rebuilds += d.rebuilds;
            h->substeps += d.substeps;
            h->solves += d.solves;
            h->launches += d.launches;
        }
    }
    if (n_steps % 2) {
        const int rc = step_once(h, s);
        if (rc) return rc;
    }
    return OC_OK;
}

// ---------------------------------------------------------------------------- ensembles
struct oc_ensemble {
    std::vector<oc_handle*> members;
    std::vector<cudaStream_t> streams;  // one recording branch per member
    std::vector<cudaEvent_t> joins;
    cudaStream_t capture = nullptr;
    cudaEvent_t fork = nullptr, chain = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<int> parity;                    // each member's buffer index at recording
    std::vector<long long> version;             // each member's graph version at recording
    std::vector<oc_handle::Counters> delta;     // each member's counter increments per replay
    int device = 0;
    std::string err;
    // batched solves, when all members run the theta scheme with the same Picard
    // count: the members fall into groups whose systems fill the GPU together
    // (groups[g] lists its members); each solve of the recorded steps is one
    // cooperative launch per group, the groups one after another. plans[q * G + g]
    // is group g's launch for solve q.
    bool batched = false;
    std::vector<std::vector<int>> groups;
    std::vector<oc::HelmBatch> plans;
    ~oc_ensemble() {
        for (auto& b : plans) oc::helm_batch_free(b);
        if (exec) cudaGraphExecDestroy(exec);
        for (auto st : streams) cudaStreamDestroy(st);
        for (auto ev : joins) cudaEventDestroy(ev);
        if (capture) cudaStreamDestroy(capture);
        if (fork) cudaEventDestroy(fork);
        if (chain) cudaEventDestroy(chain);
    }
};

namespace {

oc_handle::Counters counters_of(const oc_handle* h) {
    return {h->steps, h->tridiag, h->rebuilds, h->substeps, h->solves, h->launches};
}

void set_counters(oc_handle* h, const oc_handle::Counters& c) {
    h->steps = c.steps;
    h->tridiag = c.tridiag;
    h->rebuilds = c.rebuilds;
    h->substeps = c.substeps;
    h->solves = c.solves;
    h->launches = c.launches;
}

// record two steps of every member into one graph: member m on branch m, the
// Helmholtz solves of all members chained in recording order
int ensemble_record(oc_ensemble* e) {
    if (e->exec) {
        cudaGraphExecDestroy(e->exec);
        e->exec = nullptr;
    }
    const size_t n = e->members.size();
    std::vector<oc_handle::Counters> before(n);
    std::vector<int> cur(n);
    for (size_t m = 0; m < n; ++m) {
        oc_handle* h = e->members[m];
        // the solve log must hold every solve of a replay without moving
        const long long per_pair = h->solver ? 2LL * h->cfg.n_picard : 0;
        if (h->solver && h->solves + 2 * per_pair > h->solver->log_capacity()) {
            const int rc = ensure_log(h, 2 * (h->solves + 2 * per_pair), 0);
            if (rc) return rc;
        }
        before[m] = counters_of(h);
        cur[m] = h->cur;
    }
    // batched solves: the members' systems and solution buffers of each solve of
    // the two recorded steps are known before recording (rhs2; eta of the other
    // buffer in the first step, of the current one in the second), so the plans
    // (device parameter arrays, CTA shares) are made here, outside the capture
    for (auto& b : e->plans) helm_batch_free(b);
    e->plans.clear();
    bool batched = n > 0;
    for (size_t m = 0; m < n && batched; ++m) {
        const oc_handle* h = e->members[m];
        batched = h->solver && h->cfg.scheme == OC_SCHEME_THETA && h->cfg.n_picard == e->members[0]->cfg.n_picard;
    }
    std::string why;
    e->groups.clear();
    if (batched) {
        // groups: members in order, each group's preferred CTAs (a member's solve
        // keeps about one CTA per 2048 cells of its grid busy) adding up to at most
        // the batched launch's grid
        const int grid = helm_batch_grid();
        int used = 0;
        for (size_t m = 0; m < n; ++m) {
            const int want = e->members[m]->solver->preferred_ctas();
            if (e->groups.empty() || used + want > grid) {
                e->groups.emplace_back();
                used = 0;
            }
            e->groups.back().push_back((int)m);
            used += want;
        }
        const int np = e->members[0]->cfg.n_picard;
        for (int q = 0; q < 2 * np && batched; ++q) {
            for (const auto& grp : e->groups) {
                std::vector<HelmSolver*> sv;
                std::vector<const double*> rh;
                std::vector<double*> xs;
                for (int m : grp) {
                    oc_handle* h = e->members[m];
                    sv.push_back(h->solver);
                    rh.push_back(h->rhs2);
                    xs.push_back(h->ETA[q < np ? 1 - h->cur : h->cur]);
                }
                e->plans.emplace_back();
                std::string perr;
                if (helm_batch_plan(sv.data(), rh.data(), xs.data(), (int)sv.size(), e->plans.back(), perr) != OC_OK) {
                    batched = false;  // e.g. a refined solver: chained solves instead
                    for (auto& b : e->plans) helm_batch_free(b);
                    e->plans.clear();
                    break;
                }
            }
        }
    }
    e->batched = batched;
    BatchRecorder rec;
    rec.per_member.resize(n);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamBeginCapture(e->capture, cudaStreamCaptureModeThreadLocal);
    int rc = ce == cudaSuccess ? OC_OK : OC_ERR_CUDA;
    if (rc) why = std::string("begin capture: ") + cudaGetErrorString(ce);
    if (rc == OC_OK) {
        cudaEventRecord(e->fork, e->capture);
        cudaEventRecord(e->chain, e->capture);  // the chain starts inside the recording
        for (size_t m = 0; m < n; ++m) cudaStreamWaitEvent(e->streams[m], e->fork, 0);
        for (int step = 0; step < 2 && rc == OC_OK; ++step)
            for (size_t m = 0; m < n && rc == OC_OK; ++m) {
                oc_handle* h = e->members[m];
                const bool prof = h->profiling;
                h->profiling = false;
                h->solve_chain = batched ? nullptr : e->chain;
                h->batch_rec = batched ? &rec : nullptr;
                rec.member = (int)m;
                rc = step_once(h, e->streams[m]);
                h->batch_rec = nullptr;
                h->solve_chain = nullptr;
                h->profiling = prof;
                if (rc) why = "member " + std::to_string(m) + ": " + h->err;
            }
        // the batched solves: group g's launch for solve q waits for its members'
        // placeholders before the solve and for the previous launch (two cooperative
        // grids never compete for the SMs)
        const size_t G = e->groups.size();
        const size_t rounds = G ? e->plans.size() / G : 0;
        std::vector<cudaGraphNode_t> solve_nodes;  // [q * G + g]
        if (batched && rc == OC_OK) {
            cudaGraphNode_t prev = nullptr;
            for (size_t q = 0; q < rounds && rc == OC_OK; ++q)
                for (size_t gi = 0; gi < G && rc == OC_OK; ++gi) {
                    std::vector<cudaGraphNode_t> pre;
                    for (int m : e->groups[gi]) {
                        if (rec.per_member[m].size() != rounds || rec.per_member[m][q].rhs != e->members[m]->rhs2 ||
                            rec.per_member[m][q].x != e->members[m]->ETA[q < rounds / 2 ? 1 - cur[m] : cur[m]]) {
                            rc = OC_ERR_STATE;
                            why = "member " + std::to_string(m) + ": its solves differ from the batched plan";
                            break;
                        }
                        pre.push_back(rec.per_member[m][q].pre);
                    }
                    if (rc) break;
                    if (prev) pre.push_back(prev);
                    ce = cudaStreamUpdateCaptureDependencies(e->capture, pre.data(), pre.size(),
                                                             cudaStreamSetCaptureDependencies);
                    if (ce == cudaSuccess) {
                        std::string lerr;
                        if (helm_batch_launch(e->plans[q * G + gi], e->capture, lerr) != OC_OK) {
                            rc = OC_ERR_CUDA;
                            why = lerr;
                        }
                    } else {
                        rc = OC_ERR_CUDA;
                        why = std::string("batched solve dependencies: ") + cudaGetErrorString(ce);
                    }
                    if (rc == OC_OK) {
                        cudaStreamCaptureStatus cs;
                        const cudaGraphNode_t* d = nullptr;
                        size_t nd = 0;
                        ce = cudaStreamGetCaptureInfo(e->capture, &cs, nullptr, nullptr, &d, &nd);
                        if (ce != cudaSuccess || nd != 1) {
                            rc = OC_ERR_CUDA;
                            why = "batched solve node not found in the recording";
                        } else {
                            solve_nodes.push_back(d[0]);
                            prev = d[0];
                        }
                    }
                }
        }
        for (size_t m = 0; m < n; ++m) {
            cudaEventRecord(e->joins[m], e->streams[m]);
            cudaStreamWaitEvent(e->capture, e->joins[m], 0);
        }
        ce = cudaStreamEndCapture(e->capture, &g);
        // each member's work after solve q waits for its group's launch of solve q
        for (size_t k = 0; k < solve_nodes.size() && rc == OC_OK && ce == cudaSuccess; ++k) {
            const size_t q = k / G, gi = k % G;
            for (int m : e->groups[gi]) {
                const cudaError_t ae = cudaGraphAddDependencies(g, &solve_nodes[k], &rec.per_member[m][q].post, 1);
                if (ae != cudaSuccess) {
                    rc = OC_ERR_CUDA;
                    why = std::string("batched solve edges: ") + cudaGetErrorString(ae);
                    break;
                }
            }
        }
    } else {
        ce = cudaStreamEndCapture(e->capture, &g);
    }
    if (rc == OC_OK && ce != cudaSuccess) {
        rc = OC_ERR_CUDA;
        why = std::string("end capture: ") + cudaGetErrorString(ce);
    }
    if (rc == OC_OK) {
        ce = cudaGraphInstantiate(&e->exec, g, 0);
        if (ce != cudaSuccess) {
            rc = OC_ERR_CUDA;
            why = std::string("instantiate: ") + cudaGetErrorString(ce);
        }
    }
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    e->parity = cur;
    e->version.assign(n, 0);
    e->delta.assign(n, {});
    for (size_t m = 0; m < n; ++m) {
        oc_handle* h = e->members[m];
        const oc_handle::Counters after = counters_of(h);
        e->delta[m] = {after.steps - before[m].steps, after.tridiag - before[m].tridiag,
                       after.rebuilds - before[m].rebuilds, after.substeps - before[m].substeps,
                       after.solves - before[m].solves, after.launches - before[m].launches};
        set_counters(h, before[m]);
        h->cur = cur[m];
        e->version[m] = h->graph_version;
    }
    if (rc) {
        if (e->exec) cudaGraphExecDestroy(e->exec);
        e->exec = nullptr;
        e->err = "the ensemble's steps could not be recorded (" + why + ")";
    }
    return rc;
}

}  // namespace

int oc_ensemble_create(oc_handle* const* members, int32_t n, oc_ensemble** out) {
    if (!members || n < 1 || !out) return OC_ERR_ARG;
    *out = nullptr;
    auto* e = new oc_ensemble();
    for (int32_t m = 0; m < n; ++m) {
        oc_handle* h = members[m];
        if (!h || !h->has_state || std::find(e->members.begin(), e->members.end(), h) != e->members.end() ||
            (m > 0 && h->cfg.device != e->members[0]->cfg.device)) {
            delete e;
            return OC_ERR_ARG;
        }
        e->members.push_back(h);
    }
    e->device = e->members[0]->cfg.device;
    cudaSetDevice(e->device);
    bool ok = cudaStreamCreateWithFlags(&e->capture, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&e->chain, cudaEventDisableTiming) == cudaSuccess;
    for (int32_t m = 0; m < n && ok; ++m) {
        cudaStream_t st = nullptr;
        cudaEvent_t ev = nullptr;
        ok = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess;
        if (st) e->streams.push_back(st);
        if (ev) e->joins.push_back(ev);
    }
    if (!ok) {
        delete e;
        return OC_ERR_CUDA;
    }
    *out = e;
    return OC_OK;
}

int oc_ensemble_step(oc_ensemble* e, int32_t n_steps, void* stream) {
    if (!e) return OC_ERR_ARG;
    if (n_steps < 0) return OC_ERR_ARG;
    cudaSetDevice(e->device);
    cudaStream_t s = (cudaStream_t)stream;
    bool profiling = false;
    for (auto* h : e->members) profiling = profiling || h->profiling;
    const int pairs = profiling ? 0 : n_steps / 2;
    if (pairs > 0) {
        bool stale = !e->exec;
        for (size_t m = 0; m < e->members.size() && !stale; ++m) {
            const oc_handle* h = e->members[m];
            const long long per_pair = h->solver ? 2LL * h->cfg.n_picard : 0;
            stale = h->cur != e->parity[m] || h->graph_version != e->version[m] ||
                    (h->solver && h->solves + per_pair * (pairs + 1) > h->solver->log_capacity());
        }
        if (stale) {
            for (auto* h : e->members) {
                const long long per_pair = h->solver ? 2LL * h->cfg.n_picard : 0;
                const int rc = ensure_log(h, h->solves + per_pair * (pairs + 2), s);
                if (rc) return rc;
            }
            const int rc = ensemble_record(e);
            if (rc) return rc;
        }
        for (int i = 0; i < pairs; ++i) {
            const cudaError_t ce = cudaGraphLaunch(e->exec, s);
            if (ce != cudaSuccess) {
                e->err = cudaGetErrorString(ce);
                return OC_ERR_CUDA;
            }
            for (size_t m = 0; m < e->members.size(); ++m) {
                oc_handle* h = e->members[m];
                const oc_handle::Counters c = counters_of(h), d = e->delta[m];
                set_counters(h, {c.steps + d.steps, c.tridiag + d.tridiag, c.rebuilds + d.rebuilds,
                                 c.substeps + d.substeps, c.solves + d.solves, c.launches + d.launches});
            }
        }
    }
    // a remaining odd step (or every step while a member profiles): one member after another
    for (int i = 2 * pairs; i < n_steps; ++i)
        for (auto* h : e->members) {
            h->last_stream = s;
            const int rc = step_once(h, s);
            if (rc) return rc;
        }
    return OC_OK;
}

const char* oc_ensemble_last_error(const oc_ensemble* e) { return e ? e->err.c_str() : "null ensemble"; }

int oc_ensemble_destroy(oc_ensemble* e) {
    if (!e) return OC_ERR_ARG;
    cudaSetDevice(e->device);
    cudaDeviceSynchronize();
    delete e;
    return OC_OK;
}

int oc_get_stats(oc_handle* h, oc_stats* out) {
    if (!h || !out) return OC_ERR_ARG;
    cudaSetDevice(h->cfg.device);
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(h, e, "oc_get_stats");
    std::memset(out, 0, sizeof(*out));
    out->steps = h->steps;
    out->tridiagonal_solves = h->tridiag;
    out->solver_rebuilds = h->rebuilds;
    out->barotropic_substeps = h->substeps;
    out->solves = h->solves;
    out->n_split = h->n_split;
    out->n_levels = h->solver ? h->solver->n_levels() : 0;
    out->device_bytes = (int64_t)(h->bytes + (h->solver ? h->solver->bytes() : 0));
    out->device_status = h->has_domain ? device_status(h) : 0;
    out->kernel_launches = h->launches;
    if (h->solver && h->solves > 0) {
        const int n = (int)std::min<long long>(h->solves, h->solver->log_capacity());
        std::vector<int> it(n), cv(n);
        cudaMemcpy(it.data(), h->solver->d_log_iters(), n * sizeof(int), cudaMemcpyDeviceToHost);
        cudaMemcpy(cv.data(), h->solver->d_log_conv(), n * sizeof(int), cudaMemcpyDeviceToHost);
        for (int k = 0; k < n; ++k) {
            out->solver_iterations += std::max(0, it[k]);
            out->solver_failures += cv[k] ? 0 : 1;
        }
    }
    if (h->has_state) {
        const int c = h->cur;
        oc::k_absmax_partial<<<64, 256>>>(h->ETA[c], (int64_t)h->n2, h->d_part);
        double part[64];
        cudaMemcpy(part, h->d_part, sizeof(part), cudaMemcpyDeviceToHost);
        double m = 0.0;
        for (double x : part) m = oc::nan_max(m, x);
        out->diverged = !(m < 1.0e6);
    }
    return out->device_status ? fail(h, out->device_status, "a device-side wait ran out its bound") : OC_OK;
}

int oc_get_solve_log(oc_handle* h, int32_t* iterations, int32_t capacity, int32_t* n_out) {
    if (!h || !n_out) return OC_ERR_ARG;
    cudaSetDevice(h->cfg.device);
    cudaDeviceSynchronize();
    const int n = h->solver ? (int)std::min<long long>(h->solves, h->solver->log_capacity()) : 0;
    *n_out = n;
    if (iterations && capacity > 0 && n > 0)
        cudaMemcpy(iterations, h->solver->d_log_iters(), std::min(n, capacity) * sizeof(int),
                   cudaMemcpyDeviceToHost);
    return OC_OK;
}

int oc_set_wait_bound(oc_handle* h, int64_t cycles) {
    if (!h) return OC_ERR_ARG;
    if (cycles < 1) return fail(h, OC_ERR_ARG, "the wait bound must be at least one cycle");
    if (!h->has_domain) return fail(h, OC_ERR_STATE, "set the domain first");
    cudaSetDevice(h->cfg.device);
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(h, e, "oc_set_wait_bound");
    if (h->solver) h->solver->set_wait_cycles(cycles);
    drop_graphs(h);  // recorded solve launches carry the old bound
    return OC_OK;
}

int oc_reset_stats(oc_handle* h) {
    if (!h) return OC_ERR_ARG;
    cudaSetDevice(h->cfg.device);
    cudaDeviceSynchronize();
    h->steps = h->tridiag = h->rebuilds = h->substeps = h->solves = h->launches = 0;
    if (h->solver) cudaMemset(h->solver->d_log_count(), 0, sizeof(int));
    return OC_OK;
}

int oc_helmholtz_solve(oc_handle* h, const double* rhs, double* x, int32_t* iterations, void* stream) {
    if (!h || !rhs || !x) return OC_ERR_ARG;
    if (!h->solver) return fail(h, OC_ERR_STATE, "the Helmholtz solver exists for the theta scheme only");
    cudaSetDevice(h->cfg.device);
    cudaStream_t s = (cudaStream_t)stream;
    int rc = ensure_log(h, h->solves + 1, s);
    if (rc) return rc;
    rc = h->solver->solve(rhs, x, s, h->err);
    if (rc) return rc;
    const long long idx = h->solves;
    h->solves += 1;
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(h, e, "oc_helmholtz_solve");
    const int dst = device_status(h);
    if (dst) return fail(h, dst, "a device-side wait ran out its bound");
    if (iterations) {
        cudaMemcpy(iterations, h->solver->d_log_iters() + idx, sizeof(int), cudaMemcpyDeviceToHost);
    }
    return OC_OK;
}

int oc_thomas(const double* sub, const double* diag, const double* sup, const double* rhs, double* x,
              int32_t n, int32_t ncols, void* stream) {
    if (!sub || !diag || !sup || !rhs || !x || n < 1 || ncols < 1) return OC_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    double* cstar = nullptr;
    if (cudaMallocAsync(&cstar, (size_t)n * ncols * sizeof(double), s) != cudaSuccess) return OC_ERR_CUDA;
    launch_thomas(sub, diag, sup, rhs, x, cstar, n, ncols, s);
    cudaFreeAsync(cstar, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? OC_OK : OC_ERR_CUDA;
}

int oc_buoyancy(oc_handle* h, const double* T, const double* S, const double* z, double* b, int64_t count,
                void* stream) {
    if (!h || !T || !S || !z || !b || count < 0) return OC_ERR_ARG;
    cudaSetDevice(h->cfg.device);
    cudaStream_t s = (cudaStream_t)stream;
    launch_buoyancy_flat(h->P, T, S, z, b, count, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? OC_OK : cuda_fail(h, e, "oc_buoyancy");
}

int oc_get_field(oc_handle* h, const char* name, double* out, int64_t count) {
    if (!h || !name || !out) return OC_ERR_ARG;
    if (!h->has_domain) return fail(h, OC_ERR_STATE, "no domain");
    cudaSetDevice(h->cfg.device);
    const std::string n(name);
    const std::vector<double>* src = nullptr;
    if (n == "dz3") src = &h->dz3;
    else if (n == "mask3") src = &h->mask3;
    else if (n == "mask3u") src = &h->mask3u;
    else if (n == "mask3v") src = &h->mask3v;
    else if (n == "dz3u") src = &h->dz3u;
    else if (n == "dz3v") src = &h->dz3v;
    else if (n == "zc") src = &h->zc;
    else if (n == "mask_u") src = &h->mask_u;
    else if (n == "mask_v") src = &h->mask_v;
    if (src) {
        if ((size_t)count != src->size()) return fail(h, OC_ERR_ARG, "wrong element count for " + n);
        std::memcpy(out, src->data(), src->size() * sizeof(double));
        return OC_OK;
    }
    const double* d = nullptr;
    size_t cnt = 0;
    if (n == "q" && h->mixed) return fail(h, OC_ERR_UNSUPPORTED, "q is an FP32 field on the mixed path");
    if (n == "q") d = h->q, cnt = h->n3;
    else if (n == "ku") d = h->Ku, cnt = h->n2;
    else if (n == "kv") d = h->Kv, cnt = h->n2;
    if (!d) return fail(h, OC_ERR_ARG, "unknown field " + n);
    if ((size_t)count != cnt) return fail(h, OC_ERR_ARG, "wrong element count for " + n);
    cudaDeviceSynchronize();
    const cudaError_t e = cudaMemcpy(out, d, cnt * sizeof(double), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? OC_OK : cuda_fail(h, e, "oc_get_field");
}

int oc_set_profiling(oc_handle* h, int32_t enable) {
    if (!h) return OC_ERR_ARG;
    cudaSetDevice(h->cfg.device);
    if (!enable) prof_harvest(h);
    h->profiling = enable != 0;
    return OC_OK;
}

int oc_get_kernel_times(oc_handle* h, oc_kernel_time* out, int32_t capacity, int32_t* n_out) {
    if (!h || !n_out) return OC_ERR_ARG;
    cudaSetDevice(h->cfg.device);
    cudaDeviceSynchronize();
    prof_harvest(h);
    const int n = (int)h->prof_names.size();
    *n_out = n;
    for (int i = 0; i < n && i < capacity && out; ++i) {
        std::memset(out[i].name, 0, sizeof(out[i].name));
        std::strncpy(out[i].name, h->prof_names[i].c_str(), sizeof(out[i].name) - 1);
        out[i].launches = h->prof_launches[i];
        out[i].total_ms = h->prof_ms[i];
    }
    for (int i = 0; i < n; ++i) {
        h->prof_launches[i] = 0;
        h->prof_ms[i] = 0.0;
    }
    return OC_OK;
}

const char* oc_last_error(const oc_handle* h) { return h ? h->err.c_str() : "null handle"; }

int oc_adjoint_step(oc_handle* h, const oc_state_view* x0, const oc_state_view* x1, const oc_state_view* x1_b,
                    oc_state_view* x0_b, double* taux_b, double* tauy_b, void* stream) {
    if (!h) return OC_ERR_ARG;
    if (!h->has_domain) return fail(h, OC_ERR_STATE, "set the domain first");
    cudaSetDevice(h->cfg.device);
    return adjoint_step(h, x0, x1, x1_b, x0_b, taux_b, tauy_b, (cudaStream_t)stream);
}

int oc_adjoint_eos(oc_handle* h, const double* T, const double* S, const double* b_b, double* T_b, double* S_b,
                   void* stream) {
    if (!h) return OC_ERR_ARG;
    if (!h->has_domain) return fail(h, OC_ERR_STATE, "set the domain first");
    cudaSetDevice(h->cfg.device);
    return adjoint_eos(h, T, S, b_b, T_b, S_b, (cudaStream_t)stream);
}

void oc_destroy(oc_handle* h) {
    if (!h) return;
    cudaSetDevice(h->cfg.device);
    cudaDeviceSynchronize();
    drop_graphs(h);
    if (h->capture_stream) cudaStreamDestroy(h->capture_stream);
    if (h->aux) cudaStreamDestroy(h->aux);
    if (h->fork) cudaEventDestroy(h->fork);
    if (h->join) cudaEventDestroy(h->join);
    adjoint_free(h);
    delete h->solver;
    for (void* p : h->allocs) cudaFree(p);
    for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
    delete h;
}

}  // extern "C"
