// Two-dimensional kernels of the ocean-core step (sm_100a, fp64 on both paths):
// barotropic divergences and surface gradients, the right-hand side of the
// Helmholtz solve, the forward-backward surface update, the split-explicit
// barotropic mode, the batched Thomas solve of the unit entry point and the EOS
// on a flat buffer. The surface elevation and every depth-integrated field are
// fp64 in the mixed-precision path too, so these kernels serve both paths.
//
// Reference correspondence (paths inside the reference project):
//   div2 / grad2 / helm_rhs / eta_fb   model3d_v05.py:290-309, 376-384, 396-400, 410-413
//   split-explicit substeps            model3d_v05.py:312-335, 440-461
//   k_thomas_batched                   vertical.py:17-44
//   k_buoyancy                         eos.py:130-133

#include "oc_internal.cuh"
#include "step_common.cuh"
#include "step_kernels.cuh"

namespace oc {

// ------------------------------------------------------------------ EOS on a flat buffer
__global__ void k_buoyancy(KP P, const double* __restrict__ T, const double* __restrict__ S,
                           const double* __restrict__ z, double* __restrict__ b, int64_t n) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) b[t] = buoyancy_of(P, T[t], S[t], z[t]);
}

__device__ __forceinline__ double div2(const KP& P, const Nbr& nb, const double* __restrict__ U,
                                       const double* __restrict__ V) {
    const size_t c = nb.c;
    return P.mask[c] * ((U[c] - U[nb.at(0, -1)]) / P.dx + (V[c] - V[nb.at(-1, 0)]) / P.dy);
}

__global__ void k_div2(KP P, const double* __restrict__ U, const double* __restrict__ V,
                       double* __restrict__ out) {
    COLUMN_PROLOGUE
    out[nb.c] = div2(P, nb, U, V);
}

__global__ void k_grad2(KP P, const double* __restrict__ eta, double* __restrict__ gx,
                        double* __restrict__ gy) {
    COLUMN_PROLOGUE
    const size_t c = nb.c;
    gx[c] = P.mask_u[c] * (eta[nb.at(0, 1)] - eta[c]) / P.dx;
    gy[c] = P.mask_v[c] * (eta[nb.at(1, 0)] - eta[c]) / P.dy;
}

// rhs = eta - dt ((1 - theta) div_old + theta div(Ug, Vg))  (model3d_v05.py:398-400)
__global__ void k_helm_rhs(KP P, const double* __restrict__ eta, const double* __restrict__ div_old,
                           const double* __restrict__ Ug, const double* __restrict__ Vg,
                           double* __restrict__ rhs) {
    COLUMN_PROLOGUE
    const size_t c = nb.c;
    const double dg = div2(P, nb, Ug, Vg);
    rhs[c] = eta[c] - P.dt * (P.one_m_th * div_old[c] + P.theta * dg);
}

// forward-backward free surface eta_new = eta - dt div(U, V) (model3d_v05.py:410-413)
__global__ void k_eta_fb(KP P, const double* __restrict__ eta, const double* __restrict__ U,
                         const double* __restrict__ V, double* __restrict__ eta_new) {
    COLUMN_PROLOGUE
    eta_new[nb.c] = eta[nb.c] - P.dt * div2(P, nb, U, V);
}

// ---- split-explicit barotropic mode (model3d_v05.py:312-335, 440-461)
__device__ __forceinline__ double v_on_u2(const KP& P, const Nbr& nb, const double* __restrict__ V) {
    const double f0 = V[nb.at(0, 0)], f1 = V[nb.at(-1, 0)], f2 = V[nb.at(0, 1)], f3 = V[nb.at(-1, 1)];
    const double w0 = P.mask_v[nb.at(0, 0)], w1 = P.mask_v[nb.at(-1, 0)];
    const double w2 = P.mask_v[nb.at(0, 1)], w3 = P.mask_v[nb.at(-1, 1)];
    double num = 0.0 + w0 * f0;
    num = num + w1 * f1;
    num = num + w2 * f2;
    num = num + w3 * f3;
    double den = 0.0 + w0;
    den = den + w1;
    den = den + w2;
    den = den + w3;
    return (den > 0.0 ? num / den : 0.0) * P.mask_u[nb.c];
}

__device__ __forceinline__ double u_on_v2(const KP& P, const Nbr& nb, const double* __restrict__ U) {
    const double f0 = U[nb.at(0, 0)], f1 = U[nb.at(0, -1)], f2 = U[nb.at(1, 0)], f3 = U[nb.at(1, -1)];
    const double w0 = P.mask_u[nb.at(0, 0)], w1 = P.mask_u[nb.at(0, -1)];
    const double w2 = P.mask_u[nb.at(1, 0)], w3 = P.mask_u[nb.at(1, -1)];
    double num = 0.0 + w0 * f0;
    num = num + w1 * f1;
    num = num + w2 * f2;
    num = num + w3 * f3;
    double den = 0.0 + w0;
    den = den + w1;
    den = den + w2;
    den = den + w3;
    return (den > 0.0 ? num / den : 0.0) * P.mask_v[nb.c];
}

// barotropic forcing with the Coriolis of the 2D transport operator removed
__global__ void k_split_forcing(KP P, const double* __restrict__ U0, const double* __restrict__ V0,
                                const double* __restrict__ Um, const double* __restrict__ Vm,
                                double* __restrict__ fx, double* __restrict__ fy) {
    COLUMN_PROLOGUE
    const size_t c = nb.c;
    const double corx = P.f0 * (P.one_m_tc * v_on_u2(P, nb, V0) + P.theta_cor * v_on_u2(P, nb, Vm));
    const double cory = P.neg_f0 * (P.one_m_tc * u_on_v2(P, nb, U0) + P.theta_cor * u_on_v2(P, nb, Um));
    fx[c] = (Um[c] - U0[c]) / P.dt - corx;
    fy[c] = (Vm[c] - V0[c]) / P.dt - cory;
}

// substep set-up: the old-transport Coriolis averages and the surface gradient
__global__ void k_split_sub_avg(KP P, const double* __restrict__ U, const double* __restrict__ V,
                                const double* __restrict__ e, double* __restrict__ avv,
                                double* __restrict__ avu, double* __restrict__ gxe,
                                double* __restrict__ gye) {
    COLUMN_PROLOGUE
    const size_t c = nb.c;
    avv[c] = v_on_u2(P, nb, V);
    avu[c] = u_on_v2(P, nb, U);
    gxe[c] = P.mask_u[c] * (e[nb.at(0, 1)] - e[c]) / P.dx;
    gye[c] = P.mask_v[c] * (e[nb.at(1, 0)] - e[c]) / P.dy;
}

// one Picard pass of a substep: (Ui, Vi) from the previous iterate
__global__ void k_split_sub_mom(KP P, double ddt, const double* __restrict__ U,
                                const double* __restrict__ V, const double* __restrict__ Ui,
                                const double* __restrict__ Vi, const double* __restrict__ avv,
                                const double* __restrict__ avu, const double* __restrict__ gxe,
                                const double* __restrict__ gye, const double* __restrict__ Ku,
                                const double* __restrict__ Kv, const double* __restrict__ fx,
                                const double* __restrict__ fy, double* __restrict__ Uo,
                                double* __restrict__ Vo) {
    COLUMN_PROLOGUE
    const size_t c = nb.c;
    const double vcor = P.one_m_tc * avv[c] + P.theta_cor * v_on_u2(P, nb, Vi);
    const double ucor = P.one_m_tc * avu[c] + P.theta_cor * u_on_v2(P, nb, Ui);
    Uo[c] = (U[c] + ddt * (P.f0 * vcor - P.g * Ku[c] * gxe[c] + fx[c])) * P.mask_u[c];
    Vo[c] = (V[c] + ddt * (P.neg_f0 * ucor - P.g * Kv[c] * gye[c] + fy[c])) * P.mask_v[c];
}

// e -= ddt div(U, V); accumulate the substep transports
__global__ void k_split_sub_eta(KP P, double ddt, const double* __restrict__ U,
                                const double* __restrict__ V, double* __restrict__ e,
                                double* __restrict__ acc_u, double* __restrict__ acc_v, int first) {
    COLUMN_PROLOGUE
    const size_t c = nb.c;
    const double d = div2(P, nb, U, V);
    e[c] = e[c] - ddt * d;
    acc_u[c] = first ? 0.0 + U[c] : acc_u[c] + U[c];
    acc_v[c] = first ? 0.0 + V[c] : acc_v[c] + V[c];
}

__global__ void k_split_mean(KP P, int n_split, double* __restrict__ acc_u,
                             double* __restrict__ acc_v) {
    COLUMN_PROLOGUE
    acc_u[nb.c] = acc_u[nb.c] / n_split;
    acc_v[nb.c] = acc_v[nb.c] / n_split;
}

// replace the depth mean of the baroclinic velocity with the barotropic result
// (model3d_v05.py:452-461)
__global__ void k_split_correct(KP P, const double* __restrict__ ghu, const double* __restrict__ ghv,
                                const double* __restrict__ Ug, const double* __restrict__ Vg,
                                const double* __restrict__ U, const double* __restrict__ V,
                                double* __restrict__ u_out, double* __restrict__ v_out) {
    COLUMN_PROLOGUE
    const size_t c = nb.c;
    const ColGeo gc = ColGeo::load(P, (int)c), ge = ColGeo::load(P, nb.at(0, 1)), gn = ColGeo::load(P, nb.at(1, 0));
    const int2 kf = P.kface[c];
    double Hu = 0.0, Hv = 0.0;
    for (int k = 0; k < P.nz; ++k) {
        double m;
        const double dzc = gc.dz(P, k, m);
        const double du = face_dz(P, kf.x, k, dzc, ge.dz(P, k, m));
        const double dv = face_dz(P, kf.y, k, dzc, gn.dz(P, k, m));
        Hu = (k == 0) ? du : Hu + du;
        Hv = (k == 0) ? dv : Hv + dv;
    }
    const double ihu = inv_pos(Hu), ihv = inv_pos(Hv);
    for (int k = 0; k < P.nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        const double m3u_k = k < kf.x ? 1.0 : 0.0, m3v_k = k < kf.y ? 1.0 : 0.0;
        u_out[o] = (ghu[o] - Ug[c] * ihu + U[c] * ihu) * m3u_k;
        v_out[o] = (ghv[o] - Vg[c] * ihv + V[c] * ihv) * m3v_k;
    }
}

// ------------------------------------------------------------------ batched Thomas (unit entry)
__global__ void k_thomas_batched(const double* __restrict__ sub, const double* __restrict__ diag,
                                 const double* __restrict__ sup, const double* __restrict__ rhs,
                                 double* __restrict__ x, double* __restrict__ cstar, int n,
                                 int64_t ncols) {
    const int64_t col = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncols) return;
    double c_prev = sup[col] / diag[col];
    double d_prev = rhs[col] / diag[col];
    cstar[col] = c_prev;
    x[col] = d_prev;
    for (int k = 1; k < n; ++k) {
        const int64_t o = (int64_t)k * ncols + col;
        const double den = diag[o] - sub[o] * c_prev;
        c_prev = sup[o] / den;
        d_prev = (rhs[o] - sub[o] * d_prev) / den;
        cstar[o] = c_prev;
        x[o] = d_prev;
    }
    double xn = x[(int64_t)(n - 1) * ncols + col];
    for (int k = n - 2; k >= 0; --k) {
        const int64_t o = (int64_t)k * ncols + col;
        xn = x[o] - cstar[o] * xn;
        x[o] = xn;
    }
}

// ------------------------------------------------------------------ launchers
void launch_buoyancy_flat(const KP& P, const double* T, const double* S, const double* z, double* b,
                          int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    k_buoyancy<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P, T, S, z, b, n);
}

void launch_div2(const KP& P, const double* U, const double* V, double* out, cudaStream_t s) {
    k_div2<<<col_grid(P), col_block(), 0, s>>>(P, U, V, out);
}

void launch_grad2(const KP& P, const double* eta, double* gx, double* gy, cudaStream_t s) {
    k_grad2<<<col_grid(P), col_block(), 0, s>>>(P, eta, gx, gy);
}

void launch_helm_rhs(const KP& P, const double* eta, const double* div_old, const double* Ug,
                     const double* Vg, double* rhs, cudaStream_t s) {
    k_helm_rhs<<<col_grid(P), col_block(), 0, s>>>(P, eta, div_old, Ug, Vg, rhs);
}

void launch_eta_fb(const KP& P, const double* eta, const double* U, const double* V, double* eta_new,
                   cudaStream_t s) {
    k_eta_fb<<<col_grid(P), col_block(), 0, s>>>(P, eta, U, V, eta_new);
}

void launch_split_forcing(const KP& P, const double* U0, const double* V0, const double* Um,
                          const double* Vm, double* fx, double* fy, cudaStream_t s) {
    k_split_forcing<<<col_grid(P), col_block(), 0, s>>>(P, U0, V0, Um, Vm, fx, fy);
}

void launch_split_sub_avg(const KP& P, const double* U, const double* V, const double* e,
                          double* avv, double* avu, double* gxe, double* gye, cudaStream_t s) {
    k_split_sub_avg<<<col_grid(P), col_block(), 0, s>>>(P, U, V, e, avv, avu, gxe, gye);
}

void launch_split_sub_mom(const KP& P, double ddt, const double* U, const double* V, const double* Ui,
                          const double* Vi, const double* avv, const double* avu, const double* gxe,
                          const double* gye, const double* Ku, const double* Kv, const double* fx,
                          const double* fy, double* Uo, double* Vo, cudaStream_t s) {
    k_split_sub_mom<<<col_grid(P), col_block(), 0, s>>>(P, ddt, U, V, Ui, Vi, avv, avu, gxe, gye, Ku,
                                                       Kv, fx, fy, Uo, Vo);
}

void launch_split_sub_eta(const KP& P, double ddt, const double* U, const double* V, double* e,
                          double* acc_u, double* acc_v, int first, cudaStream_t s) {
    k_split_sub_eta<<<col_grid(P), col_block(), 0, s>>>(P, ddt, U, V, e, acc_u, acc_v, first);
}

void launch_split_mean(const KP& P, int n_split, double* acc_u, double* acc_v, cudaStream_t s) {
    k_split_mean<<<col_grid(P), col_block(), 0, s>>>(P, n_split, acc_u, acc_v);
}

void launch_split_correct(const KP& P, const double* ghu, const double* ghv, const double* Ug,
                          const double* Vg, const double* U, const double* V, double* u_out,
                          double* v_out, cudaStream_t s) {
    k_split_correct<<<col_grid(P), col_block(), 0, s>>>(P, ghu, ghv, Ug, Vg, U, V, u_out, v_out);
}

void launch_thomas(const double* sub, const double* diag, const double* sup, const double* rhs,
                   double* x, double* cstar, int n, int64_t ncols, cudaStream_t s) {
    k_thomas_batched<<<(unsigned)((ncols + 127) / 128), 128, 0, s>>>(sub, diag, sup, rhs, x, cstar, n,
                                                                    ncols);
}

}  // namespace oc
