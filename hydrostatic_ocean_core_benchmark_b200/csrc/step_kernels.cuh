// Host-side launchers of the step kernels (step_kernels.cu).
#pragma once

#include "oc_internal.cuh"

namespace oc {

void launch_qsolve(const KP& P, const double* km, double* q, cudaStream_t s);
void launch_closure(const KP& P, const double* u, const double* v, const double* b, double* e,
                    double* km, double* kh, double* q, cudaStream_t s);
void launch_kukv(const KP& P, const double* q, double* Ku, double* Kv, cudaStream_t s);
void launch_wcol(const KP& P, const double* u, const double* v, double* w, cudaStream_t s);
void launch_phi(const KP& P, const double* b, double* phi, cudaStream_t s);
void launch_mom_explicit(const KP& P, const double* u, const double* v, const double* b,
                         const double* phi, const double* w, const double* km, double* pgx,
                         double* pgy, double* avpv, double* avpu, double* dzu, double* dzv,
                         double* stu, double* stv, cudaStream_t s);
// right-hand sides of the two momentum tridiagonals for one Picard pass (per cell)
void launch_predictor_rhs(const KP& P, const double* u, const double* v, const double* u_it,
                          const double* v_it, const double* pgx, const double* pgy, const double* avpv,
                          const double* avpu, const double* dzu, const double* dzv, const double* stu,
                          const double* stv, const double* gx2, const double* gy2, double* ru, double* rv,
                          cudaStream_t s);
// both column solves in place on gh_u/gh_v, then the transports
void launch_momentum_solve(const KP& P, const double* km, double* ghu, double* ghv, double* Ug, double* Vg,
                           cudaStream_t s);
void launch_backsub(const KP& P, const double* ghu, const double* ghv, const double* q,
                    const double* eta_new, double* u_out, double* v_out, cudaStream_t s);
void launch_tracer_rhs(const KP& P, const double* T, const double* S, const double* bold,
                       const double* u, const double* v, const double* w, const double* kh, double* rT,
                       double* rS, cudaStream_t s);
void launch_tracer_solve(const KP& P, const double* rT, const double* rS, const double* kh,
                         double* T_out, double* S_out, double* b_out, cudaStream_t s);
void launch_buoyancy_flat(const KP& P, const double* T, const double* S, const double* z, double* b,
                          int64_t n, cudaStream_t s);
void launch_diag_buoyancy(const KP& P, const double* T, const double* S, double* b, cudaStream_t s);
void launch_transport(const KP& P, const double* u, const double* v, double* U, double* V,
                      cudaStream_t s);
void launch_div2(const KP& P, const double* U, const double* V, double* out, cudaStream_t s);
void launch_grad2(const KP& P, const double* eta, double* gx, double* gy, cudaStream_t s);
void launch_helm_rhs(const KP& P, const double* eta, const double* div_old, const double* Ug,
                     const double* Vg, double* rhs, cudaStream_t s);
void launch_eta_fb(const KP& P, const double* eta, const double* U, const double* V, double* eta_new,
                   cudaStream_t s);
void launch_split_forcing(const KP& P, const double* U0, const double* V0, const double* Um,
                          const double* Vm, double* fx, double* fy, cudaStream_t s);
void launch_split_sub_avg(const KP& P, const double* U, const double* V, const double* e,
                          double* avv, double* avu, double* gxe, double* gye, cudaStream_t s);
void launch_split_sub_mom(const KP& P, double ddt, const double* U, const double* V, const double* Ui,
                          const double* Vi, const double* avv, const double* avu, const double* gxe,
                          const double* gye, const double* Ku, const double* Kv, const double* fx,
                          const double* fy, double* Uo, double* Vo, cudaStream_t s);
void launch_split_sub_eta(const KP& P, double ddt, const double* U, const double* V, double* e,
                          double* acc_u, double* acc_v, int first, cudaStream_t s);
void launch_split_mean(const KP& P, int n_split, double* acc_u, double* acc_v, cudaStream_t s);
void launch_split_correct(const KP& P, const double* ghu, const double* ghv, const double* Ug,
                          const double* Vg, const double* U, const double* V, double* u_out,
                          double* v_out, cudaStream_t s);
void launch_thomas(const double* sub, const double* diag, const double* sup, const double* rhs,
                   double* x, double* cstar, int n, int64_t ncols, cudaStream_t s);

}  // namespace oc
