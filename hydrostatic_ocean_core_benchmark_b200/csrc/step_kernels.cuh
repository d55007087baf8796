// Host-side launchers of the step kernels.
//
// The 3D kernels (step_kernels.cu) exist for two floating types of the 3D
// fields: double (the fp64 path, bit-identical to the reference) and float (the
// mixed-precision path). Their launchers are overloads on the parameter block
// KPT<R>; b, phi and every 2D field are double on both. The 2D kernels
// (step2d_kernels.cu) are fp64 only.
#pragma once

#include "oc_internal.cuh"

namespace oc {

#define OC_DECLARE_3D_LAUNCHERS(R)                                                                              \
    void launch_qsolve(const KPT<R>& P, const R* km, R* q, cudaStream_t s);                                     \
    void launch_closure(const KPT<R>& P, const R* u, const R* v, const double* b, R* e, R* km, R* kh, R* q,    \
                        cudaStream_t s);                                                                        \
    void launch_kukv(const KPT<R>& P, const R* q, double* Ku, double* Kv, cudaStream_t s);                      \
    void launch_wcol(const KPT<R>& P, const R* u, const R* v, R* w, cudaStream_t s);                            \
    void launch_phi(const KPT<R>& P, const double* b, double* phi, cudaStream_t s);                             \
    void launch_mom_explicit(const KPT<R>& P, const R* u, const R* v, const double* b, const double* phi,      \
                             const R* w, const R* km, R* pgx, R* pgy, R* avpv, R* avpu, R* dzu, R* dzv, R* stu, \
                             R* stv, cudaStream_t s);                                                           \
    /* right-hand sides of the two momentum tridiagonals for one Picard pass (per cell) */                     \
    void launch_predictor_rhs(const KPT<R>& P, const R* u, const R* v, const R* u_it, const R* v_it,           \
                              const R* pgx, const R* pgy, const R* avpv, const R* avpu, const R* dzu,           \
                              const R* dzv, const R* stu, const R* stv, const double* gx2, const double* gy2,   \
                              R* ru, R* rv, cudaStream_t s);                                                    \
    /* both column solves in place on gh_u/gh_v, then the transports */                                        \
    void launch_momentum_solve(const KPT<R>& P, const R* km, R* ghu, R* ghv, double* Ug, double* Vg,           \
                               cudaStream_t s);                                                                 \
    void launch_backsub(const KPT<R>& P, const R* ghu, const R* ghv, const R* q, const double* eta_new,         \
                        R* u_out, R* v_out, cudaStream_t s);                                                    \
    /* C0: T with TS tracers, else the buoyancy (fp64 path only) */                                             \
    void launch_tracer_rhs(const KPT<R>& P, const R* C0, const R* S, const R* u, const R* v, const R* w,        \
                           const R* kh, R* rT, R* rS, cudaStream_t s);                                          \
    void launch_tracer_solve(const KPT<R>& P, const R* rT, const R* rS, const R* kh, R* T_out, R* S_out,      \
                             double* b_out, cudaStream_t s);                                                    \
    void launch_diag_buoyancy(const KPT<R>& P, const R* T, const R* S, double* b, cudaStream_t s);             \
    void launch_transport(const KPT<R>& P, const R* u, const R* v, double* U, double* V, cudaStream_t s);

OC_DECLARE_3D_LAUNCHERS(double)
OC_DECLARE_3D_LAUNCHERS(float)
#undef OC_DECLARE_3D_LAUNCHERS

// fp64 only (step2d_kernels.cu)
void launch_buoyancy_flat(const KP& P, const double* T, const double* S, const double* z, double* b,
                          int64_t n, cudaStream_t s);
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
