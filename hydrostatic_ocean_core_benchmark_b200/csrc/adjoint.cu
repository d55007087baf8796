// Hand-written adjoint of the fp64 step (oc_adjoint_step): the transpose of
// the step's Jacobian applied to the cotangents of its outputs.
//
// Scope: the theta scheme with TS tracers and the closure off (constant
// viscosity and diffusivity), any advection, EOS, face rule and stress field.
// With the closure off every tridiagonal matrix and the Helmholtz operator are
// constant, so the step is linear except for the momentum advection, the
// tracer advection and the EOS; their adjoints take the forward values of the
// step (the state before and after it) and, for the TVD faces, the limiter
// branch the forward pass took, recomputed from those values.
//
// The forward step is reference model3d_v05.py:337-533 (the fp64 kernels of
// step_kernels.cu and the oracle give the same bits). The adjoint walks it
// backwards:
//   EOS -> implicit tracer solves (transposed Thomas) -> tracer right-hand
//   sides (explicit diffusion, horizontal diffusion, advection with the
//   limiter branches frozen) -> w -> for each Picard pass, last first:
//   back-substitution, Helmholtz solve (the operator is symmetric: the same
//   solver), its right-hand side, depth-integrated transports, momentum
//   column solves (transposed Thomas), predictor and Coriolis average of the
//   iterate -> explicit momentum terms (advection, horizontal viscosity,
//   explicit vertical diffusion with the surface stress, old Coriolis average,
//   pressure gradient) -> buoyancy potential -> the stress field.
// Stencils whose transposes gather are written as gathers; the advection
// faces scatter with atomic adds, so sums of the adjoint fields are formed in
// a run-dependent order (the forward step stays bit-exact).
//
// No reference counterpart: the reference has no adjoint.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "capi_internal.cuh"
#include "helmholtz.cuh"
#include "step_common.cuh"
#include "step_kernels.cuh"

namespace oc {
namespace {

// ---------------------------------------------------------------- dual numbers
// value and derivative, for the exact partial derivatives of the EOS
struct Dual {
    double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Dual sqrt(Dual a) {
    const double r = ::sqrt(a.v);
    return {r, a.d / (2.0 * r)};
}

// d b / d T and d b / d S of b = -g rho'(T, S, z) / rho0 (eos.py:103-133)
__device__ __forceinline__ void eos_partials(const KP& P, double T, double S, double z, double& dbdT,
                                             double& dbdS) {
    const double k = P.neg_g64 / P.rho0_64;
    const Dual zz{z, 0.0};
    dbdT = k * rho_anomaly_n<Dual>(P.eos, P.rho0_64, P.alpha_t64, P.beta_s64, P.t0_64, P.s0_64, Dual{T, 1.0},
                                   Dual{S, 0.0}, zz).d;
    dbdS = k * rho_anomaly_n<Dual>(P.eos, P.rho0_64, P.alpha_t64, P.beta_s64, P.t0_64, P.s0_64, Dual{T, 0.0},
                                   Dual{S, 1.0}, zz).d;
}

// ---------------------------------------------------------------- face values
// The face value between c0 and c1 (cm beyond c0, cp beyond c1) for the
// advecting velocity vel and the far cells' wet flags (advection_v06.py:21-74;
// the vertical faces map onto it with cm = the cell below the lower one, c0 =
// the lower cell, c1 = the upper cell, cp = the cell above the upper one), and
// its partial derivatives with respect to (cm, c0, c1, cp) with the limiter's
// branch held at the one the values select. scheme: advection code (1 centred,
// 2 upwind, 3 kappa = 1/3, 4 Superbee TVD).
struct Face {
    double f, dm, d0, d1, dp;
};

__device__ __forceinline__ Face face_lin(const KP& P, int scheme, double cm, double c0, double c1, double cp,
                                         double vel, bool wm, bool wp) {
    Face r{0.0, 0.0, 0.0, 0.0, 0.0};
    if (scheme == 1) {
        r.f = 0.5 * (c0 + c1);
        r.d0 = r.d1 = 0.5;
        return r;
    }
    const bool pos = vel > 0.0;
    if (scheme == 2) {
        r.f = pos ? c0 : c1;
        (pos ? r.d0 : r.d1) = 1.0;
        return r;
    }
    const double base = pos ? c0 : c1;
    const double far = pos ? (c0 - cm) : (cp - c1);
    const double d = c1 - c0;
    // t = beta * far + alpha * d to first order, frozen branch
    double t, alpha, beta;
    if (scheme == 4) {
        if (d == 0.0) {
            t = 0.0;
            alpha = beta = 0.0;
        } else {
            const double q = far / d;
            const double A = fmin(2.0 * q, 1.0), B = fmin(q, 2.0);
            const double inner = fmax(A, B);
            const double sb = fmax(0.0, inner);
            double dsb = 0.0;
            if (inner > 0.0) dsb = (A >= B) ? (2.0 * q < 1.0 ? 2.0 : 0.0) : (q < 2.0 ? 1.0 : 0.0);
            t = 0.5 * sb * d;
            alpha = 0.5 * (sb - dsb * q);
            beta = 0.5 * dsb;
        }
    } else {
        t = 0.25 * (P.one_m_kappa3 * far + P.one_p_kappa3 * d);
        alpha = 0.25 * P.one_p_kappa3;
        beta = 0.25 * P.one_m_kappa3;
    }
    if (pos) {
        if (!wm) {
            r.f = c0;
            r.d0 = 1.0;
            return r;
        }
        // f = c0 + t, far = c0 - cm, d = c1 - c0
        r.f = base + t;
        r.dm = -beta;
        r.d0 = 1.0 + beta - alpha;
        r.d1 = alpha;
    } else {
        if (!wp) {
            r.f = c1;
            r.d1 = 1.0;
            return r;
        }
        // f = c1 - t, far = cp - c1, d = c1 - c0
        r.f = base - t;
        r.dp = -beta;
        r.d1 = 1.0 + beta - alpha;
        r.d0 = alpha;
    }
    return r;
}

__device__ __forceinline__ void atomic_add(double* a, double v) {
    if (v != 0.0) atomicAdd(a, v);
}

// thickness of the east (x) or north (y) face of column c at level k
__device__ __forceinline__ double face_thick(const KP& P, int c, int cn, int kf, int k) {
    double m;
    return face_dz(P, kf, k, col_dz(P, c, k, m), col_dz(P, cn, k, m));
}

#define ADJ_PROLOGUE                                      \
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  \
    const int j = blockIdx.y * blockDim.y + threadIdx.y;  \
    if (i >= P.nx || j >= P.ny) return;                   \
    const int nx = P.nx, ny = P.ny, nz = P.nz;            \
    const size_t n2 = (size_t)P.n2;                       \
    const int c = j * nx + i;                             \
    const int cE = j * nx + (i + 1 == nx ? 0 : i + 1);    \
    const int cW = j * nx + (i == 0 ? nx - 1 : i - 1);    \
    const int cN = (j + 1 == ny ? 0 : j + 1) * nx + i;    \
    const int cS = (j == 0 ? ny - 1 : j - 1) * nx + i;    \
    (void)cE, (void)cW, (void)cN, (void)cS, (void)nz, (void)n2;

// ---------------------------------------------------------------- column solves
// x = M^-T y for the column's implicit rows (vertical_var.py:35-77) with the
// interface coefficient K (constant in this scope) and the bottom-row term
// thv_dt_drag = (theta_v dt) drag: the transposed matrix has sub'[k] = sup[k-1]
// and sup'[k] = sub[k+1]. y and x may alias.
template <int NZM>
__device__ void solve_transposed(const KP& P, int c, double K, double thv_dt_drag, const double* y, double* x,
                                 size_t n2) {
    const int nz = P.nz;
    const ColGeo g = ColGeo::load(P, c);
    double sub[NZM], dia[NZM], sup[NZM];
    double m3_k, dz_k = g.dz(P, 0, m3_k);
    double dzi_k = dz_k;
    for (int k = 0; k < nz; ++k) {
        double m3_k1 = 0.0, dz_k1 = 0.0;
        if (k + 1 < nz) dz_k1 = g.dz(P, k + 1, m3_k1);
        const double dzi_k1 = (k + 1 < nz) ? 0.5 * (dz_k + dz_k1) : dz_k;
        implicit_row(P, k, dz_k, m3_k, m3_k1, dzi_k, dzi_k1, K, K, thv_dt_drag, sub[k], dia[k], sup[k]);
        dz_k = dz_k1;
        m3_k = m3_k1;
        dzi_k = dzi_k1;
    }
    // Thomas on (sub' = sup[k-1], diag, sup' = sub[k+1])
    double cs[NZM];
    double cp = 0.0, dp = 0.0;
    for (int k = 0; k < nz; ++k) {
        const double a = k > 0 ? sup[k - 1] : 0.0;
        const double bsup = k + 1 < nz ? sub[k + 1] : 0.0;
        const double yk = y[(size_t)k * n2 + c];
        if (k == 0) {
            cp = bsup / dia[0];
            dp = yk / dia[0];
        } else {
            const double den = dia[k] - a * cp;
            cp = bsup / den;
            dp = (yk - a * dp) / den;
        }
        cs[k] = cp;
        x[(size_t)k * n2 + c] = dp;
    }
    double xn = dp;
    for (int k = nz - 2; k >= 0; --k) {
        const size_t o = (size_t)k * n2 + c;
        xn = x[o] - cs[k] * xn;
        x[o] = xn;
    }
}

// cotangent of the explicit vertical diffusion Dz[f] (vertical_var.py:80-106) of
// one face-velocity or tracer column with face thickness dzf[k], constant K,
// the cell column's bottom rule and drag: f_b += Dz^T r_b; returns the
// cotangent of the surface flux.
template <int NZM>
__device__ double explicit_dz_T(const KP& P, const double* dzf, const double* m3c, double K, double drag,
                                const double* r_b, double* f_b) {
    const int nz = P.nz;
    double flux_b[NZM + 1];
    for (int k = 0; k <= nz; ++k) flux_b[k] = 0.0;
    for (int k = 0; k < nz; ++k) {
        const double rb = m3c[k] > 0.0 ? r_b[k] : 0.0;
        const double idz = inv_pos(dzf[k]);
        const bool bottom = m3c[k] > 0.0 && (k + 1 >= nz || m3c[k + 1] == 0.0);
        flux_b[k] += rb * idz;
        flux_b[k + 1] -= rb * idz;
        if (bottom) f_b[k] -= drag * idz * rb;
    }
    for (int k = 1; k < nz; ++k) {
        const bool bottom_above = m3c[k - 1] > 0.0 && m3c[k] == 0.0;
        if (bottom_above) continue;
        const double coef = K * inv_pos(0.5 * (dzf[k - 1] + dzf[k]));
        f_b[k - 1] += coef * flux_b[k];
        f_b[k] -= coef * flux_b[k];
    }
    return flux_b[0];
}

// ---------------------------------------------------------------- kernels

// w = -cumsum from the bottom of the layer-transport divergence
// (vertical_var.py:109-121): td_b[k] = -sum_{k' <= k} w_b[k']
__global__ void k_wcol_T1(KP P, const double* __restrict__ w_b, double* __restrict__ td_b) {
    ADJ_PROLOGUE
    double acc = 0.0;
    for (int k = 0; k < nz; ++k) {
        acc += w_b[(size_t)k * n2 + c];
        td_b[(size_t)k * n2 + c] = -acc;
    }
}

// td = m3 ((dz3u u - W(dz3u u)) / dx + (dz3v v - S(dz3v v)) / dy): u_b, v_b += its transpose
__global__ void k_wcol_T2(KP P, const double* __restrict__ td_b, double* __restrict__ u_b, double* __restrict__ v_b) {
    ADJ_PROLOGUE
    const int2 kf = P.kface[c];
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2;
        const double mc = col_m3(P, c, k), me = col_m3(P, cE, k), mn = col_m3(P, cN, k);
        const double du = face_thick(P, c, cE, kf.x, k), dv = face_thick(P, c, cN, kf.y, k);
        u_b[o + c] += du / P.dx64 * (mc * td_b[o + c] - me * td_b[o + cE]);
        v_b[o + c] += dv / P.dy64 * (mc * td_b[o + c] - mn * td_b[o + cN]);
    }
}

// EOS and implicit tracer solves: r_b = M_b^-T ((X'_b + b'_b m3 db/dX) m3) for X = T, S
template <int NZM>
__global__ void k_tracer_solve_T(KP P, const double* __restrict__ Tn, const double* __restrict__ Sn,
                                 const double* __restrict__ Tn_b, const double* __restrict__ Sn_b,
                                 const double* __restrict__ bn_b, double* __restrict__ rT_b,
                                 double* __restrict__ rS_b) {
    ADJ_PROLOGUE
    const ColGeo g = ColGeo::load(P, c);
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        double m3;
        const double dz = g.dz(P, k, m3);
        double dT = 0.0, dS = 0.0;
        if (m3 > 0.0) eos_partials(P, Tn[o], Sn[o], g.above(P, k) + 0.5 * dz, dT, dS);
        const double bb = bn_b[o] * m3;
        rT_b[o] = (Tn_b[o] + bb * dT) * m3;
        rS_b[o] = (Sn_b[o] + bb * dS) * m3;
    }
    solve_transposed<NZM>(P, c, P.kappa, P.thv_dt_zero, rT_b, rT_b, n2);
    solve_transposed<NZM>(P, c, P.kappa, P.thv_dt_zero, rS_b, rS_b, n2);
}

// tracer right-hand side rhs = c + dt tend + c3 Dz[c] + surface terms: the
// identity and explicit vertical diffusion parts (per column; X_b written)
template <int NZM>
__global__ void k_tracer_rhs_T_col(KP P, const double* __restrict__ rT_b, const double* __restrict__ rS_b,
                                   double* __restrict__ T_b, double* __restrict__ S_b) {
    ADJ_PROLOGUE
    double dz[NZM], m3[NZM], rb[NZM], fb[NZM];
    for (int k = 0; k < nz; ++k) dz[k] = col_dz(P, c, k, m3[k]);
    for (int f = 0; f < 2; ++f) {
        const double* r = f == 0 ? rT_b : rS_b;
        double* out = f == 0 ? T_b : S_b;
        for (int k = 0; k < nz; ++k) {
            rb[k] = P.c3 * r[(size_t)k * n2 + c];
            fb[k] = r[(size_t)k * n2 + c];
        }
        explicit_dz_T<NZM>(P, dz, m3, P.kappa, 0.0, rb, fb);
        for (int k = 0; k < nz; ++k) out[(size_t)k * n2 + c] = fb[k];
    }
}

// tracer advection and horizontal diffusion (model3d_v05.py:466-512): tend =
// -adv(c; u, v, w) + k_h lap(c), rhs_b = dt tend_b. One thread per cell forms
// the cotangents of its east and north faces (scattered to the four cells of
// each face and to the face velocity) and, per column, of the vertical faces.
__global__ void k_tracer_adv_T(KP P, const double* __restrict__ T, const double* __restrict__ S,
                               const double* __restrict__ u, const double* __restrict__ v,
                               const double* __restrict__ w, const double* __restrict__ rT_b,
                               const double* __restrict__ rS_b, double* __restrict__ T_b, double* __restrict__ S_b,
                               double* __restrict__ u_b, double* __restrict__ v_b, double* __restrict__ w_b) {
    ADJ_PROLOGUE
    const int k = blockIdx.z;
    const size_t o = (size_t)k * n2;
    const int2 kf = P.kface[c];
    const int cEE = j * nx + (i + 2 >= nx ? i + 2 - nx : i + 2);
    const int cNN = ((j + 2 >= ny) ? j + 2 - ny : j + 2) * nx + i;
    const int scheme = P.advection;
    for (int f = 0; f < 2; ++f) {
        const double* C = f == 0 ? T : S;
        const double* R = f == 0 ? rT_b : rS_b;
        double* Cb = f == 0 ? T_b : S_b;
        // a = d rhs / d adv term per cell: adv enters as -dt adv, adv = (hdiv + vdiv) m3
        auto acoef = [&](int cc) {
            double m;
            const double dz = col_dz(P, cc, k, m);
            return -P.dt * R[o + cc] * m * inv_pos(dz);
        };
        const double a_c = acoef(c), a_e = acoef(cE), a_n = acoef(cN);
        if (scheme != 0) {
            // east face of cell c: flux dz3u u cx
            {
                const double fx_b = (a_c - a_e) / P.dx64;
                const double vel = u[o + c];
                const double dzf = face_thick(P, c, cE, kf.x, k);
                if (dzf != 0.0 && fx_b != 0.0) {
                    const Face fc = face_lin(P, scheme, C[o + cW], C[o + c], C[o + cE], C[o + cEE], vel,
                                             col_m3(P, cW, k) > 0.0, col_m3(P, cEE, k) > 0.0);
                    atomic_add(&u_b[o + c], fx_b * dzf * fc.f);
                    const double s = fx_b * dzf * vel;
                    atomic_add(&Cb[o + cW], s * fc.dm);
                    atomic_add(&Cb[o + c], s * fc.d0);
                    atomic_add(&Cb[o + cE], s * fc.d1);
                    atomic_add(&Cb[o + cEE], s * fc.dp);
                }
            }
            // north face
            {
                const double fy_b = (a_c - a_n) / P.dy64;
                const double vel = v[o + c];
                const double dzf = face_thick(P, c, cN, kf.y, k);
                if (dzf != 0.0 && fy_b != 0.0) {
                    const Face fc = face_lin(P, scheme, C[o + cS], C[o + c], C[o + cN], C[o + cNN], vel,
                                             col_m3(P, cS, k) > 0.0, col_m3(P, cNN, k) > 0.0);
                    atomic_add(&v_b[o + c], fy_b * dzf * fc.f);
                    const double s = fy_b * dzf * vel;
                    atomic_add(&Cb[o + cS], s * fc.dm);
                    atomic_add(&Cb[o + c], s * fc.d0);
                    atomic_add(&Cb[o + cN], s * fc.d1);
                    atomic_add(&Cb[o + cNN], s * fc.dp);
                }
            }
            // the top face of cell c (interface k): vdiv[k] = (w[k] cf[k] - w[k+1] cf[k+1]) inv
            {
                double wcf_b = a_c;
                if (k > 0) {
                    double m;
                    const double dzu = col_dz(P, c, k - 1, m);
                    wcf_b -= -P.dt * R[o - n2 + c] * m * inv_pos(dzu);
                }
                const double wv = w[o + c];
                if (wcf_b != 0.0) {
                    if (k == 0) {
                        atomic_add(&w_b[o + c], wcf_b * C[o + c]);
                        atomic_add(&Cb[o + c], wcf_b * wv);
                    } else {
                        const bool has_up = k >= 2 && col_m3(P, c, k - 2) > 0.0;
                        const bool has_dn = k + 1 <= nz - 1 && col_m3(P, c, k + 1) > 0.0;
                        const double far_up = k >= 2 ? C[o - 2 * n2 + c] : 0.0;
                        const double far_dn = k + 1 <= nz - 1 ? C[o + n2 + c] : 0.0;
                        const int sz = scheme == 2 ? 1 : scheme;  // upwind faces are centred vertically
                        const Face fc = face_lin(P, sz, far_dn, C[o + c], C[o - n2 + c], far_up, wv, has_dn, has_up);
                        atomic_add(&w_b[o + c], wcf_b * fc.f);
                        const double s = wcf_b * wv;
                        if (k + 1 <= nz - 1) atomic_add(&Cb[o + n2 + c], s * fc.dm);
                        atomic_add(&Cb[o + c], s * fc.d0);
                        atomic_add(&Cb[o - n2 + c], s * fc.d1);
                        if (k >= 2) atomic_add(&Cb[o - 2 * n2 + c], s * fc.dp);
                    }
                }
            }
        }
        if (P.k_h > 0.0) {
            // k_h lap(c) = k_h m3 ((gx - W gx) / dx + (gy - S gy) / dy), gx = m3u (E c - c) / dx
            auto lcoef = [&](int cc) { return P.dt * P.k_h * R[o + cc] * col_m3(P, cc, k); };
            const double l_c = lcoef(c), l_e = lcoef(cE), l_n = lcoef(cN);
            const double gx_b = (l_c - l_e) / P.dx64 * col_m3u(P, c, k) / P.dx64;
            const double gy_b = (l_c - l_n) / P.dy64 * col_m3v(P, c, k) / P.dy64;
            atomic_add(&Cb[o + cE], gx_b);
            atomic_add(&Cb[o + c], -gx_b - gy_b);
            atomic_add(&Cb[o + cN], gy_b);
        }
    }
}

// back-substitution u = (gh_u - c2 q gx(eta_new) m3u) m3 (model3d_v05.py:404-406):
// gh_b = u_b m3 and the per-column cotangent of the surface gradient
__global__ void k_backsub_T(KP P, const double* __restrict__ uo_b, const double* __restrict__ vo_b,
                            const double* __restrict__ q, double* __restrict__ ghu_b, double* __restrict__ ghv_b,
                            double* __restrict__ gx_b, double* __restrict__ gy_b) {
    ADJ_PROLOGUE
    const int kb = P.kinfo[c].y;
    const int2 kf = P.kface[c];
    double sx = 0.0, sy = 0.0;
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        const double m3 = k < kb ? 1.0 : 0.0;
        const double ub = uo_b[o] * m3, vb = vo_b[o] * m3;
        ghu_b[o] = ub;
        ghv_b[o] = vb;
        sx += q[o] * (k < kf.x ? 1.0 : 0.0) * ub;
        sy += q[o] * (k < kf.y ? 1.0 : 0.0) * vb;
    }
    gx_b[c] = -P.c2 * sx;
    gy_b[c] = -P.c2 * sy;
}

// eta_b += the transpose of the masked surface gradient (mask_u (E eta - eta) / dx, ...)
__global__ void k_grad2_T(KP P, const double* __restrict__ gx_b, const double* __restrict__ gy_b,
                          double* __restrict__ eta_b, int overwrite, const double* __restrict__ base) {
    ADJ_PROLOGUE
    const double t = (P.mask_u[cW] * gx_b[cW] - P.mask_u[c] * gx_b[c]) / P.dx64 +
                     (P.mask_v[cS] * gy_b[cS] - P.mask_v[c] * gy_b[c]) / P.dy64;
    if (overwrite)
        eta_b[c] = (base ? base[c] : 0.0) + t;
    else
        eta_b[c] += t;
}

// rhs = eta - dt ((1 - theta) div_old + theta div(Ug, Vg)) (model3d_v05.py:398-400):
// eta_b += rhs_b, div_old_b += ..., and (Ug_b, Vg_b) = div^T(-dt theta rhs_b)
__global__ void k_helm_rhs_T(KP P, const double* __restrict__ rhs_b, double* __restrict__ eta_b,
                             double* __restrict__ divold_b, double* __restrict__ Ug_b, double* __restrict__ Vg_b) {
    ADJ_PROLOGUE
    eta_b[c] += rhs_b[c];
    divold_b[c] += -P.dt * P.one_m_th * rhs_b[c];
    const double s = -P.dt * P.theta;
    Ug_b[c] = s * (P.mask[c] * rhs_b[c] - P.mask[cE] * rhs_b[cE]) / P.dx64;
    Vg_b[c] = s * (P.mask[c] * rhs_b[c] - P.mask[cN] * rhs_b[cN]) / P.dy64;
}

// (U, V) = div^T(d_b) for the old-state transports: U_b = (m d_b - m_E d_b_E) / dx
__global__ void k_div2_T(KP P, const double* __restrict__ d_b, double* __restrict__ U_b, double* __restrict__ V_b) {
    ADJ_PROLOGUE
    U_b[c] = (P.mask[c] * d_b[c] - P.mask[cE] * d_b[cE]) / P.dx64;
    V_b[c] = (P.mask[c] * d_b[c] - P.mask[cN] * d_b[cN]) / P.dy64;
}

// u_b += dz3u U_b (the depth-integrated transport sum_k dz3u u)
__global__ void k_transport_T(KP P, const double* __restrict__ U_b, const double* __restrict__ V_b,
                              double* __restrict__ u_b, double* __restrict__ v_b) {
    ADJ_PROLOGUE
    const int2 kf = P.kface[c];
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        u_b[o] += face_thick(P, c, cE, kf.x, k) * U_b[c];
        v_b[o] += face_thick(P, c, cN, kf.y, k) * V_b[c];
    }
}

// gh = M_m^-1 (rhs) m3 with the transports Ug = sum_k dz3u gh: r_b = M_m^-T ((gh_b + dz3u Ug_b) m3)
template <int NZM>
__global__ void k_momentum_solve_T(KP P, double* __restrict__ ghu_b, double* __restrict__ ghv_b,
                                   const double* __restrict__ Ug_b, const double* __restrict__ Vg_b,
                                   double* __restrict__ ru_b, double* __restrict__ rv_b) {
    ADJ_PROLOGUE
    const int2 kf = P.kface[c];
    const int kb = P.kinfo[c].y;
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        const double m3 = k < kb ? 1.0 : 0.0;
        ru_b[o] = (ghu_b[o] + face_thick(P, c, cE, kf.x, k) * Ug_b[c]) * m3;
        rv_b[o] = (ghv_b[o] + face_thick(P, c, cN, kf.y, k) * Vg_b[c]) * m3;
    }
    solve_transposed<NZM>(P, c, P.nu, P.thv_dt_drag, ru_b, ru_b, n2);
    solve_transposed<NZM>(P, c, P.nu, P.thv_dt_drag, rv_b, rv_b, n2);
}

// Coriolis averages (operators_masked.py:45-61): av[c] = sum_q w_q f_q / sum_q w_q * m,
// transposed by scattering to the four points
__device__ __forceinline__ void v_on_u_T(const KP& P, size_t o, int k, int c, int cS, int cE, int cSE, double m,
                                         double av_b, double* v_b) {
    if (av_b == 0.0 || m == 0.0) return;
    const double w0 = col_m3v(P, c, k), w1 = col_m3v(P, cS, k), w2 = col_m3v(P, cE, k), w3 = col_m3v(P, cSE, k);
    const double den = w0 + w1 + w2 + w3;
    if (!(den > 0.0)) return;
    const double s = av_b * m / den;
    atomic_add(&v_b[o + c], s * w0);
    atomic_add(&v_b[o + cS], s * w1);
    atomic_add(&v_b[o + cE], s * w2);
    atomic_add(&v_b[o + cSE], s * w3);
}

__device__ __forceinline__ void u_on_v_T(const KP& P, size_t o, int k, int c, int cW, int cN, int cNW, double m,
                                         double av_b, double* u_b) {
    if (av_b == 0.0 || m == 0.0) return;
    const double w0 = col_m3u(P, c, k), w1 = col_m3u(P, cW, k), w2 = col_m3u(P, cN, k), w3 = col_m3u(P, cNW, k);
    const double den = w0 + w1 + w2 + w3;
    if (!(den > 0.0)) return;
    const double s = av_b * m / den;
    atomic_add(&u_b[o + c], s * w0);
    atomic_add(&u_b[o + cW], s * w1);
    atomic_add(&u_b[o + cN], s * w2);
    atomic_add(&u_b[o + cNW], s * w3);
}

// predictor gu = u + dt (f0 v_cor + pgx) - c1 gx m3u + c3 dzu, rhs = gu + st_u,
// v_cor = (1 - tc) av(v) + tc av(v_it): cotangents of its inputs. The old
// average's cotangent is accumulated in avpv_b; the iterate's is scattered to
// it_b (u_b for the first pass, whose iterate is the old state).
__global__ void k_predictor_T(KP P, const double* __restrict__ ru_b, const double* __restrict__ rv_b,
                              double* __restrict__ u_b, double* __restrict__ v_b, double* __restrict__ uit_b,
                              double* __restrict__ vit_b, double* __restrict__ avpv_b, double* __restrict__ avpu_b,
                              double* __restrict__ pgx_b, double* __restrict__ pgy_b, double* __restrict__ dzu_b,
                              double* __restrict__ dzv_b, double* __restrict__ stu_b, double* __restrict__ stv_b,
                              double* __restrict__ gx2_b, double* __restrict__ gy2_b) {
    ADJ_PROLOGUE
    const int cSE = (j == 0 ? ny - 1 : j - 1) * nx + (i + 1 == nx ? 0 : i + 1);
    const int cNW = (j + 1 == ny ? 0 : j + 1) * nx + (i == 0 ? nx - 1 : i - 1);
    const int2 kf = P.kface[c];
    double sx = 0.0, sy = 0.0;
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2;
        const double rb = ru_b[o + c], rvb = rv_b[o + c];
        u_b[o + c] += rb;
        v_b[o + c] += rvb;
        stu_b[o + c] += rb;
        stv_b[o + c] += rvb;
        pgx_b[o + c] += P.dt * rb;
        pgy_b[o + c] += P.dt * rvb;
        dzu_b[o + c] += P.c3 * rb;
        dzv_b[o + c] += P.c3 * rvb;
        sx += (k < kf.x ? 1.0 : 0.0) * rb;
        sy += (k < kf.y ? 1.0 : 0.0) * rvb;
        const double vcor_b = P.dt * P.f0 * rb;
        const double ucor_b = P.dt * P.neg_f0 * rvb;
        avpv_b[o + c] += P.one_m_tc * vcor_b;
        avpu_b[o + c] += P.one_m_tc * ucor_b;
        v_on_u_T(P, o, k, c, cS, cE, cSE, k < kf.x ? 1.0 : 0.0, P.theta_cor * vcor_b, vit_b);
        u_on_v_T(P, o, k, c, cW, cN, cNW, k < kf.y ? 1.0 : 0.0, P.theta_cor * ucor_b, uit_b);
    }
    gx2_b[c] += -P.c1 * sx;
    gy2_b[c] += -P.c1 * sy;
}

// the old-state Coriolis averages (avpv = av(v), avpu = av(u)): scatter
__global__ void k_coriolis_old_T(KP P, const double* __restrict__ avpv_b, const double* __restrict__ avpu_b,
                                 double* __restrict__ u_b, double* __restrict__ v_b) {
    ADJ_PROLOGUE
    const int cSE = (j == 0 ? ny - 1 : j - 1) * nx + (i + 1 == nx ? 0 : i + 1);
    const int cNW = (j + 1 == ny ? 0 : j + 1) * nx + (i == 0 ? nx - 1 : i - 1);
    const int2 kf = P.kface[c];
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2;
        v_on_u_T(P, o, k, c, cS, cE, cSE, k < kf.x ? 1.0 : 0.0, avpv_b[o + c], v_b);
        u_on_v_T(P, o, k, c, cW, cN, cNW, k < kf.y ? 1.0 : 0.0, avpu_b[o + c], u_b);
    }
}

// explicit vertical diffusion of the face velocities with the surface stress
// (dzu = Dz[u; K_m, dz3u, tau_u, drag]) and the stress increment st_u[0] =
// thv dt tau_u / dz3u[0]: u_b += Dz^T dzu_b, tau_u_b = its surface cotangent
template <int NZM>
__global__ void k_explicit_dz_T(KP P, const double* __restrict__ dzu_b, const double* __restrict__ dzv_b,
                                const double* __restrict__ stu_b, const double* __restrict__ stv_b,
                                double* __restrict__ u_b, double* __restrict__ v_b, double* __restrict__ tau_u_b,
                                double* __restrict__ tau_v_b) {
    ADJ_PROLOGUE
    const int2 kf = P.kface[c];
    double dzf[NZM], m3c[NZM], rb[NZM], fb[NZM];
    for (int k = 0; k < nz; ++k) {
        double m;
        col_dz(P, c, k, m);
        m3c[k] = m;
    }
    for (int f = 0; f < 2; ++f) {
        const double* src = f == 0 ? dzu_b : dzv_b;
        double* dst = f == 0 ? u_b : v_b;
        const int cn = f == 0 ? cE : cN;
        const int kk = f == 0 ? kf.x : kf.y;
        for (int k = 0; k < nz; ++k) {
            dzf[k] = face_thick(P, c, cn, kk, k);
            rb[k] = src[(size_t)k * n2 + c];
            fb[k] = 0.0;
        }
        const double surf_b = explicit_dz_T<NZM>(P, dzf, m3c, P.nu, P.bottom_drag, rb, fb);
        for (int k = 0; k < nz; ++k) dst[(size_t)k * n2 + c] += fb[k];
        const double st0 = (f == 0 ? stu_b : stv_b)[c];
        const double t = surf_b + P.thv_dt * inv_pos(dzf[0]) * st0;
        (f == 0 ? tau_u_b : tau_v_b)[c] = t;
    }
}

// momentum advection and horizontal viscosity (advection_v06.py:77-108,
// model3d_v05.py:241-260): ex = -adv(u, v, w) m3u + a_h lap(u); the cotangent
// exu_b = dt st_u_b. One thread per cell handles the fluxes it owns: for u the
// centre flux at the T-cell c (between u faces W and c), the corner flux north
// of u face c and the vertical flux at the top of u face c; for v likewise.
__global__ void k_mom_adv_T(KP P, const double* __restrict__ u, const double* __restrict__ v,
                            const double* __restrict__ w, const double* __restrict__ stu_b,
                            const double* __restrict__ stv_b, double* __restrict__ u_b, double* __restrict__ v_b,
                            double* __restrict__ w_b) {
    ADJ_PROLOGUE
    const int k = blockIdx.z;
    const size_t o = (size_t)k * n2;
    const int scheme = P.advection;
    const int cWW = j * nx + (i <= 1 ? i - 2 + nx : i - 2);
    const int cEE = j * nx + (i + 2 >= nx ? i + 2 - nx : i + 2);
    const int cSS = ((j <= 1) ? j - 2 + ny : j - 2) * nx + i;
    const int cNN = ((j + 2 >= ny) ? j + 2 - ny : j + 2) * nx + i;
    const int cSE = (j == 0 ? ny - 1 : j - 1) * nx + (i + 1 == nx ? 0 : i + 1);
    const int cNW = (j + 1 == ny ? 0 : j + 1) * nx + (i == 0 ? nx - 1 : i - 1);
    const double dz_nom = P.dz_nom[k];
    // adv cotangents: ex = -adv m3f, ex_b = dt st_b
    auto au_b = [&](int cc, int kk) { return -P.dt * stu_b[(size_t)kk * n2 + cc] * col_m3u(P, cc, kk); };
    auto av_b = [&](int cc, int kk) { return -P.dt * stv_b[(size_t)kk * n2 + cc] * col_m3v(P, cc, kk); };
    const bool kap = scheme >= 3;
    if (scheme != 0) {
        // ---- u: centre flux F[c] = ub_c uc_c, ub_c = (u_W + u_c)/2; ax = (F_E - F)/dx at u face c
        {
            const double F_b = (au_b(cW, k) - au_b(c, k)) / P.dx64;
            if (F_b != 0.0) {
                const double ub = 0.5 * (u[o + cW] + u[o + c]);
                double val;
                if (kap) {
                    const Face fc = face_lin(P, scheme, u[o + cWW], u[o + cW], u[o + c], u[o + cE], ub,
                                             col_m3u(P, cWW, k) > 0.0, col_m3u(P, cE, k) > 0.0);
                    val = fc.f;
                    const double s = F_b * ub;
                    atomic_add(&u_b[o + cWW], s * fc.dm);
                    atomic_add(&u_b[o + cW], s * fc.d0);
                    atomic_add(&u_b[o + c], s * fc.d1);
                    atomic_add(&u_b[o + cE], s * fc.dp);
                } else {
                    val = ub;
                    atomic_add(&u_b[o + cW], F_b * ub * 0.5);
                    atomic_add(&u_b[o + c], F_b * ub * 0.5);
                }
                atomic_add(&u_b[o + cW], 0.5 * F_b * val);
                atomic_add(&u_b[o + c], 0.5 * F_b * val);
            }
        }
        // ---- u: corner flux fy north of u face c: vbar = (v_c + v_E)/2, face of u between c and N
        {
            const double fy_b = (au_b(c, k) - au_b(cN, k)) / P.dy64;
            if (fy_b != 0.0) {
                const double vb = 0.5 * (v[o + c] + v[o + cE]);
                double val;
                if (kap) {
                    const Face fc = face_lin(P, scheme, u[o + cS], u[o + c], u[o + cN], u[o + cNN], vb,
                                             col_m3u(P, cS, k) > 0.0, col_m3u(P, cNN, k) > 0.0);
                    val = fc.f;
                    const double s = fy_b * vb;
                    atomic_add(&u_b[o + cS], s * fc.dm);
                    atomic_add(&u_b[o + c], s * fc.d0);
                    atomic_add(&u_b[o + cN], s * fc.d1);
                    atomic_add(&u_b[o + cNN], s * fc.dp);
                } else {
                    val = 0.5 * (u[o + c] + u[o + cN]);
                    atomic_add(&u_b[o + c], fy_b * vb * 0.5);
                    atomic_add(&u_b[o + cN], fy_b * vb * 0.5);
                }
                atomic_add(&v_b[o + c], 0.5 * fy_b * val);
                atomic_add(&v_b[o + cE], 0.5 * fy_b * val);
            }
        }
        // ---- u: vertical flux at interface k of u face c (1 <= k <= nz-1)
        if (k >= 1) {
            const double fz_b = (au_b(c, k) - au_b(c, k - 1)) / dz_nom;
            if (fz_b != 0.0) {
                const double wb = 0.5 * (w[o + c] + w[o + cE]);
                const double ab = u[o - n2 + c], bl = u[o + c];
                double val;
                if (kap) {
                    const int kf = P.kface[c].x;
                    const bool hu = k >= 2 && k - 2 < kf, hd = k + 1 <= nz - 1 && k + 1 < kf;
                    const double fu = k >= 2 ? u[o - 2 * n2 + c] : 0.0, fd = k + 1 <= nz - 1 ? u[o + n2 + c] : 0.0;
                    const Face fc = face_lin(P, scheme, fd, bl, ab, fu, wb, hd, hu);
                    val = fc.f;
                    const double s = fz_b * wb;
                    if (k + 1 <= nz - 1) atomic_add(&u_b[o + n2 + c], s * fc.dm);
                    atomic_add(&u_b[o + c], s * fc.d0);
                    atomic_add(&u_b[o - n2 + c], s * fc.d1);
                    if (k >= 2) atomic_add(&u_b[o - 2 * n2 + c], s * fc.dp);
                } else {
                    val = 0.5 * (ab + bl);
                    atomic_add(&u_b[o + c], fz_b * wb * 0.5);
                    atomic_add(&u_b[o - n2 + c], fz_b * wb * 0.5);
                }
                atomic_add(&w_b[o + c], 0.5 * fz_b * val);
                atomic_add(&w_b[o + cE], 0.5 * fz_b * val);
            }
        }
        // ---- v: centre flux G[c] = vb_c vc_c, vb_c = (v_S + v_c)/2; by = (G_N - G)/dy at v face c
        {
            const double G_b = (av_b(cS, k) - av_b(c, k)) / P.dy64;
            if (G_b != 0.0) {
                const double vb = 0.5 * (v[o + cS] + v[o + c]);
                double val;
                if (kap) {
                    const Face fc = face_lin(P, scheme, v[o + cSS], v[o + cS], v[o + c], v[o + cN], vb,
                                             col_m3v(P, cSS, k) > 0.0, col_m3v(P, cN, k) > 0.0);
                    val = fc.f;
                    const double s = G_b * vb;
                    atomic_add(&v_b[o + cSS], s * fc.dm);
                    atomic_add(&v_b[o + cS], s * fc.d0);
                    atomic_add(&v_b[o + c], s * fc.d1);
                    atomic_add(&v_b[o + cN], s * fc.dp);
                } else {
                    val = vb;
                    atomic_add(&v_b[o + cS], G_b * vb * 0.5);
                    atomic_add(&v_b[o + c], G_b * vb * 0.5);
                }
                atomic_add(&v_b[o + cS], 0.5 * G_b * val);
                atomic_add(&v_b[o + c], 0.5 * G_b * val);
            }
        }
        // ---- v: corner flux fx east of v face c: ubar = (u_c + u_N)/2, face of v between c and E
        {
            const double fx_b = (av_b(c, k) - av_b(cE, k)) / P.dx64;
            if (fx_b != 0.0) {
                const double ub = 0.5 * (u[o + c] + u[o + cN]);
                double val;
                if (kap) {
                    const Face fc = face_lin(P, scheme, v[o + cW], v[o + c], v[o + cE], v[o + cEE], ub,
                                             col_m3v(P, cW, k) > 0.0, col_m3v(P, cEE, k) > 0.0);
                    val = fc.f;
                    const double s = fx_b * ub;
                    atomic_add(&v_b[o + cW], s * fc.dm);
                    atomic_add(&v_b[o + c], s * fc.d0);
                    atomic_add(&v_b[o + cE], s * fc.d1);
                    atomic_add(&v_b[o + cEE], s * fc.dp);
                } else {
                    val = 0.5 * (v[o + c] + v[o + cE]);
                    atomic_add(&v_b[o + c], fx_b * ub * 0.5);
                    atomic_add(&v_b[o + cE], fx_b * ub * 0.5);
                }
                atomic_add(&u_b[o + c], 0.5 * fx_b * val);
                atomic_add(&u_b[o + cN], 0.5 * fx_b * val);
            }
        }
        // ---- v: vertical flux at interface k of v face c
        if (k >= 1) {
            const double fz_b = (av_b(c, k) - av_b(c, k - 1)) / dz_nom;
            if (fz_b != 0.0) {
                const double wb = 0.5 * (w[o + c] + w[o + cN]);
                const double ab = v[o - n2 + c], bl = v[o + c];
                double val;
                if (kap) {
                    const int kf = P.kface[c].y;
                    const bool hu = k >= 2 && k - 2 < kf, hd = k + 1 <= nz - 1 && k + 1 < kf;
                    const double fu = k >= 2 ? v[o - 2 * n2 + c] : 0.0, fd = k + 1 <= nz - 1 ? v[o + n2 + c] : 0.0;
                    const Face fc = face_lin(P, scheme, fd, bl, ab, fu, wb, hd, hu);
                    val = fc.f;
                    const double s = fz_b * wb;
                    if (k + 1 <= nz - 1) atomic_add(&v_b[o + n2 + c], s * fc.dm);
                    atomic_add(&v_b[o + c], s * fc.d0);
                    atomic_add(&v_b[o - n2 + c], s * fc.d1);
                    if (k >= 2) atomic_add(&v_b[o - 2 * n2 + c], s * fc.dp);
                } else {
                    val = 0.5 * (ab + bl);
                    atomic_add(&v_b[o + c], fz_b * wb * 0.5);
                    atomic_add(&v_b[o - n2 + c], fz_b * wb * 0.5);
                }
                atomic_add(&w_b[o + c], 0.5 * fz_b * val);
                atomic_add(&w_b[o + cN], 0.5 * fz_b * val);
            }
        }
    }
    if (P.a_h > 0.0) {
        // a_h lap(f) with face masks m3u (x) and m3v (y) and cell mask m of the component:
        // lap = m ((gx - W gx)/dx + (gy - S gy)/dy), gx = m3u (E f - f)/dx, gy = m3v (N f - f)/dy
        for (int comp = 0; comp < 2; ++comp) {
            const double* st_b = comp ? stv_b : stu_b;
            double* fb = comp ? v_b : u_b;
            auto lc = [&](int cc) {
                const double m = comp ? col_m3v(P, cc, k) : col_m3u(P, cc, k);
                return P.dt * P.a_h * st_b[o + cc] * m;
            };
            const double l_c = lc(c), l_e = lc(cE), l_n = lc(cN);
            const double gx_b = (l_c - l_e) / P.dx64 * col_m3u(P, c, k) / P.dx64;
            const double gy_b = (l_c - l_n) / P.dy64 * col_m3v(P, c, k) / P.dy64;
            atomic_add(&fb[o + cE], gx_b);
            atomic_add(&fb[o + c], -gx_b - gy_b);
            atomic_add(&fb[o + cN], gy_b);
        }
    }
    (void)cSE;
    (void)cNW;
}

// pressure gradient (model3d_v05.py:211-230): pg = m3f ((phi_F + b_F (zf - zc_F)) -
// (phi + b (zf - zc))) / dx at the east / north face: phi_b and b_b gathered
__global__ void k_pgf_T(KP P, const double* __restrict__ pgx_b, const double* __restrict__ pgy_b,
                        double* __restrict__ phi_b, double* __restrict__ b_b) {
    ADJ_PROLOGUE
    const ColGeo gc = ColGeo::load(P, c), gw = ColGeo::load(P, cW), ge = ColGeo::load(P, cE);
    const ColGeo gs = ColGeo::load(P, cS), gn = ColGeo::load(P, cN);
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2;
        double m;
        const double zc = gc.above(P, k) + 0.5 * gc.dz(P, k, m);
        const double zw = gw.above(P, k) + 0.5 * gw.dz(P, k, m);
        const double ze = ge.above(P, k) + 0.5 * ge.dz(P, k, m);
        const double zs = gs.above(P, k) + 0.5 * gs.dz(P, k, m);
        const double zn = gn.above(P, k) + 0.5 * gn.dz(P, k, m);
        // faces: east of c (c is the left cell), east of W (c is the right cell), same in y
        const double ge_b = col_m3u(P, c, k) * pgx_b[o + c] / P.dx64;
        const double gw_b = col_m3u(P, cW, k) * pgx_b[o + cW] / P.dx64;
        const double gn_b = col_m3v(P, c, k) * pgy_b[o + c] / P.dy64;
        const double gs_b = col_m3v(P, cS, k) * pgy_b[o + cS] / P.dy64;
        double pb, bb;
        if (P.pgf_correction) {
            pb = gw_b - ge_b + gs_b - gn_b;
            bb = -ge_b * (0.5 * (zc + ze) - zc) + gw_b * (0.5 * (zw + zc) - zc) - gn_b * (0.5 * (zc + zn) - zc) +
                 gs_b * (0.5 * (zs + zc) - zc);
        } else {
            // pg = m3f (phi_F - phi) / dx m3f
            pb = col_m3u(P, cW, k) * gw_b - col_m3u(P, c, k) * ge_b + col_m3v(P, cS, k) * gs_b -
                 col_m3v(P, c, k) * gn_b;
            bb = 0.0;
        }
        phi_b[o + c] = pb;
        b_b[o + c] += bb;
    }
}

// phi[k] = 0.5 dz b[k] + sum_{k' < k} dz b[k'] (vertical_var.py:132-136):
// b_b[k] += dz[k] (0.5 phi_b[k] + sum_{k' > k} phi_b[k'])
__global__ void k_phi_T(KP P, const double* __restrict__ phi_b, double* __restrict__ b_b) {
    ADJ_PROLOGUE
    double below = 0.0;
    for (int k = nz - 1; k >= 0; --k) {
        const size_t o = (size_t)k * n2 + c;
        double m;
        const double dz = col_dz(P, c, k, m);
        b_b[o] += dz * (0.5 * phi_b[o] + below);
        below += phi_b[o];
    }
}

// tau_u = 0.5 (tx + E tx) / rho0 m3u[0], tau_v = 0.5 (ty + N ty) / rho0 m3v[0]:
// the stress field's cotangent at the centres (accumulated)
__global__ void k_stress_T(KP P, const double* __restrict__ tau_u_b, const double* __restrict__ tau_v_b,
                           double* __restrict__ tx_b, double* __restrict__ ty_b) {
    ADJ_PROLOGUE
    const double s = 0.5 / P.rho0_64;
    tx_b[c] += s * (col_m3u(P, c, 0) * tau_u_b[c] + col_m3u(P, cW, 0) * tau_u_b[cW]);
    if (ty_b) ty_b[c] += s * (col_m3v(P, c, 0) * tau_v_b[c] + col_m3v(P, cS, 0) * tau_v_b[cS]);
}

// b_b of a buoyancy diagnosed from T and S (b = EOS(T, S, zc) m3): T_b += b_b m3 db/dT
__global__ void k_eos_T(KP P, const double* __restrict__ T, const double* __restrict__ S,
                        const double* __restrict__ b_b, double* __restrict__ T_b, double* __restrict__ S_b) {
    ADJ_PROLOGUE
    const ColGeo g = ColGeo::load(P, c);
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        double m3;
        const double dz = g.dz(P, k, m3);
        if (m3 == 0.0) continue;
        double dT, dS;
        eos_partials(P, T[o], S[o], g.above(P, k) + 0.5 * dz, dT, dS);
        T_b[o] += b_b[o] * dT;
        S_b[o] += b_b[o] * dS;
    }
}

#define NZ_DISPATCH_ADJ(NZ, CALL)             \
    do {                                      \
        if ((NZ) + 1 <= 33) {                 \
            constexpr int NZM = 33;           \
            CALL;                             \
        } else if ((NZ) + 1 <= 65) {          \
            constexpr int NZM = 65;           \
            CALL;                             \
        } else {                              \
            constexpr int NZM = OC_MAXNZ + 1; \
            CALL;                             \
        }                                     \
    } while (0)

}  // namespace

// ---------------------------------------------------------------- the adjoint step
struct AdjointWork {
    size_t n2 = 0, n3 = 0, n3i = 0;
    std::vector<void*> allocs;
    double *w_old = nullptr, *w_new = nullptr, *w_b = nullptr, *td_b = nullptr;
    double *rT_b = nullptr, *rS_b = nullptr;
    double *it_u[2] = {}, *it_v[2] = {};
    double *ghu_b = nullptr, *ghv_b = nullptr, *ru_b = nullptr, *rv_b = nullptr;
    double *stu_b = nullptr, *stv_b = nullptr, *pgx_b = nullptr, *pgy_b = nullptr;
    double *dzu_b = nullptr, *dzv_b = nullptr, *avpv_b = nullptr, *avpu_b = nullptr, *phi_b = nullptr;
    double *gx_b = nullptr, *gy_b = nullptr, *eta_m_b = nullptr, *rhs_b = nullptr, *Ug_b = nullptr,
           *Vg_b = nullptr, *divold_b = nullptr, *gx2_b = nullptr, *gy2_b = nullptr, *tau_u_b = nullptr,
           *tau_v_b = nullptr;
    HelmSolver* solver = nullptr;
    ~AdjointWork() {
        delete solver;
        for (void* p : allocs) cudaFree(p);
    }
};

static double* adj_alloc(AdjointWork* a, size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, n * sizeof(double)) != cudaSuccess) return nullptr;
    a->allocs.push_back(p);
    return (double*)p;
}

void adjoint_free(oc_handle* h) {
    delete h->adj;
    h->adj = nullptr;
}

static int adjoint_setup(oc_handle* h) {
    if (h->adj) return OC_OK;
    AdjointWork* a = new AdjointWork();
    a->n2 = h->n2;
    a->n3 = h->n3;
    a->n3i = h->n3i;
    const size_t n2 = h->n2, n3 = h->n3, n3i = h->n3i;
    bool ok = true;
    for (double** p : {&a->w_old, &a->w_new, &a->w_b}) ok = ok && (*p = adj_alloc(a, n3i));
    for (double** p : {&a->td_b, &a->rT_b, &a->rS_b, &a->it_u[0], &a->it_u[1], &a->it_v[0], &a->it_v[1], &a->ghu_b,
                       &a->ghv_b, &a->ru_b, &a->rv_b, &a->stu_b, &a->stv_b, &a->pgx_b, &a->pgy_b, &a->dzu_b,
                       &a->dzv_b, &a->avpv_b, &a->avpu_b, &a->phi_b})
        ok = ok && (*p = adj_alloc(a, n3));
    for (double** p : {&a->gx_b, &a->gy_b, &a->eta_m_b, &a->rhs_b, &a->Ug_b, &a->Vg_b, &a->divold_b, &a->gx2_b,
                       &a->gy2_b, &a->tau_u_b, &a->tau_v_b})
        ok = ok && (*p = adj_alloc(a, n2));
    if (!ok) {
        delete a;
        return fail(h, OC_ERR_CUDA, "cudaMalloc failed (adjoint work)");
    }
    // a solver of its own (same operator), so the adjoint solves stay out of the
    // forward solve log and counters
    a->solver = new HelmSolver();
    const oc_config& c = h->cfg;
    const double coef = c.g * std::pow(c.theta, 2.0) * std::pow(c.dt, 2.0);
    // its systems solved to a tighter tolerance than the forward's (at most 1e-13)
    const double rtol = std::min(c.rtol, 1.0e-13);
    const int rc = a->solver->init(h->nx, h->ny, c.lx / h->nx, c.ly / h->ny, coef, c.solver, rtol, c.max_iter,
                                   h->mask.data(), h->Ku, h->Kv, 1 << 20, h->d_status, h->err);
    if (rc) {
        delete a;
        return rc;
    }
    a->solver->rebuild(0);
    h->adj = a;
    return OC_OK;
}

int adjoint_step(oc_handle* h, const oc_state_view* x0, const oc_state_view* x1, const oc_state_view* x1_b,
                 const oc_state_view* x0_b, double* taux_b, double* tauy_b, cudaStream_t s) {
    const oc_config& cf = h->cfg;
    if (h->mixed || cf.scheme != OC_SCHEME_THETA || cf.tracers != OC_TRACERS_TS || cf.closure != OC_CLOSURE_NONE ||
        cf.pgf != OC_PGF_KEEP)
        return fail(h, OC_ERR_UNSUPPORTED,
                    "the adjoint covers the fp64 theta scheme with TS tracers, the closure off and pgf keep");
    if (!x0 || !x1 || !x1_b || !x0_b || !x0->u || !x0->v || !x0->T || !x0->S || !x0->eta || !x1->u || !x1->v ||
        !x1->T || !x1->S || !x1_b->u || !x1_b->v || !x1_b->b || !x1_b->eta || !x1_b->T || !x1_b->S || !x0_b->u ||
        !x0_b->v || !x0_b->b || !x0_b->eta || !x0_b->T || !x0_b->S || !taux_b)
        return fail(h, OC_ERR_ARG, "every state and cotangent field is required (device pointers)");
    int rc = adjoint_setup(h);
    if (rc) return rc;
    AdjointWork& A = *h->adj;
    const KP& P = h->P;
    const size_t n2 = h->n2, n3 = h->n3, n3i = h->n3i;
    const dim3 cb = col_block(), cg = col_grid(P);
    const dim3 vb(32, 4, 1), vg((P.nx + 31) / 32, (P.ny + 3) / 4, P.nz);
    auto zero = [&](double* p, size_t n) { cudaMemsetAsync(p, 0, n * sizeof(double), s); };
    // forward values: w of the state before and after the step
    launch_wcol(P, x0->u, x0->v, A.w_old, s);
    launch_wcol(P, x1->u, x1->v, A.w_new, s);
    // outputs start from zero
    for (double* p : {x0_b->u, x0_b->v, x0_b->b, x0_b->T, x0_b->S}) zero(p, n3);
    zero(x0_b->eta, n2);
    for (double* p : {A.stu_b, A.stv_b, A.pgx_b, A.pgy_b, A.dzu_b, A.dzv_b, A.avpv_b, A.avpu_b}) zero(p, n3);
    for (double* p : {A.divold_b, A.gx2_b, A.gy2_b}) zero(p, n2);
    zero(A.w_b, n3i);
    // ---- EOS and the implicit tracer solves
    NZ_DISPATCH_ADJ(P.nz, (k_tracer_solve_T<NZM><<<cg, cb, 0, s>>>(P, x1->T, x1->S, x1_b->T, x1_b->S, x1_b->b,
                                                                    A.rT_b, A.rS_b)));
    // ---- tracer right-hand sides: the identity and vertical diffusion, then advection
    NZ_DISPATCH_ADJ(P.nz, (k_tracer_rhs_T_col<NZM><<<cg, cb, 0, s>>>(P, A.rT_b, A.rS_b, x0_b->T, x0_b->S)));
    // the last iterate's cotangent starts as the output's
    double* uit_b = A.it_u[0];
    double* vit_b = A.it_v[0];
    cudaMemcpyAsync(uit_b, x1_b->u, n3 * sizeof(double), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(vit_b, x1_b->v, n3 * sizeof(double), cudaMemcpyDeviceToDevice, s);
    k_tracer_adv_T<<<vg, vb, 0, s>>>(P, x0->T, x0->S, x1->u, x1->v, A.w_new, A.rT_b, A.rS_b, x0_b->T, x0_b->S,
                                     uit_b, vit_b, A.w_b);
    // w of the new velocities
    k_wcol_T1<<<cg, cb, 0, s>>>(P, A.w_b, A.td_b);
    k_wcol_T2<<<cg, cb, 0, s>>>(P, A.td_b, uit_b, vit_b);
    // ---- Picard passes, last first
    for (int m = cf.n_picard - 1; m >= 0; --m) {
        k_backsub_T<<<cg, cb, 0, s>>>(P, uit_b, vit_b, h->q, A.ghu_b, A.ghv_b, A.gx_b, A.gy_b);
        k_grad2_T<<<cg, cb, 0, s>>>(P, A.gx_b, A.gy_b, A.eta_m_b, 1, m == cf.n_picard - 1 ? x1_b->eta : nullptr);
        rc = A.solver->solve(A.eta_m_b, A.rhs_b, s, h->err);
        if (rc) return rc;
        k_helm_rhs_T<<<cg, cb, 0, s>>>(P, A.rhs_b, x0_b->eta, A.divold_b, A.Ug_b, A.Vg_b);
        NZ_DISPATCH_ADJ(P.nz, (k_momentum_solve_T<NZM><<<cg, cb, 0, s>>>(P, A.ghu_b, A.ghv_b, A.Ug_b, A.Vg_b,
                                                                          A.ru_b, A.rv_b)));
        // the iterate of pass m is the output of pass m - 1, or the old state
        double* nu_b = m > 0 ? A.it_u[(cf.n_picard - m) % 2] : x0_b->u;
        double* nv_b = m > 0 ? A.it_v[(cf.n_picard - m) % 2] : x0_b->v;
        if (m > 0) {
            zero(nu_b, n3);
            zero(nv_b, n3);
        }
        k_predictor_T<<<cg, cb, 0, s>>>(P, A.ru_b, A.rv_b, x0_b->u, x0_b->v, nu_b, nv_b, A.avpv_b, A.avpu_b,
                                        A.pgx_b, A.pgy_b, A.dzu_b, A.dzv_b, A.stu_b, A.stv_b, A.gx2_b, A.gy2_b);
        uit_b = nu_b;
        vit_b = nv_b;
    }
    // ---- the old state's terms
    k_grad2_T<<<cg, cb, 0, s>>>(P, A.gx2_b, A.gy2_b, x0_b->eta, 0, nullptr);
    k_div2_T<<<cg, cb, 0, s>>>(P, A.divold_b, A.Ug_b, A.Vg_b);
    k_transport_T<<<cg, cb, 0, s>>>(P, A.Ug_b, A.Vg_b, x0_b->u, x0_b->v);
    zero(A.w_b, n3i);
    k_mom_adv_T<<<vg, vb, 0, s>>>(P, x0->u, x0->v, A.w_old, A.stu_b, A.stv_b, x0_b->u, x0_b->v, A.w_b);
    k_wcol_T1<<<cg, cb, 0, s>>>(P, A.w_b, A.td_b);
    k_wcol_T2<<<cg, cb, 0, s>>>(P, A.td_b, x0_b->u, x0_b->v);
    NZ_DISPATCH_ADJ(P.nz, (k_explicit_dz_T<NZM><<<cg, cb, 0, s>>>(P, A.dzu_b, A.dzv_b, A.stu_b, A.stv_b, x0_b->u,
                                                                   x0_b->v, A.tau_u_b, A.tau_v_b)));
    k_coriolis_old_T<<<cg, cb, 0, s>>>(P, A.avpv_b, A.avpu_b, x0_b->u, x0_b->v);
    k_pgf_T<<<cg, cb, 0, s>>>(P, A.pgx_b, A.pgy_b, A.phi_b, x0_b->b);
    k_phi_T<<<cg, cb, 0, s>>>(P, A.phi_b, x0_b->b);
    k_stress_T<<<cg, cb, 0, s>>>(P, A.tau_u_b, A.tau_v_b, taux_b, tauy_b);
    return check_launch(h, "oc_adjoint_step");
}

int adjoint_eos(oc_handle* h, const double* T, const double* S, const double* b_b, double* T_b, double* S_b,
                cudaStream_t s) {
    if (!T || !S || !b_b || !T_b || !S_b) return fail(h, OC_ERR_ARG, "T, S, b_b, T_b and S_b are required");
    const KP& P = h->P;
    k_eos_T<<<col_grid(P), col_block(), 0, s>>>(P, T, S, b_b, T_b, S_b);
    return check_launch(h, "oc_adjoint_eos");
}

}  // namespace oc
