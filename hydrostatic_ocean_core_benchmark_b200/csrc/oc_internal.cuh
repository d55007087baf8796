// Internal definitions of the sm_100a ocean-core step.
//
// Bit-for-bit parity with the reference NumPy step (libs/core/model3d_v05.py)
// is a design rule: every expression below performs the same IEEE-754 fp64
// operations in the same order as the reference, the library is compiled with
// -fmad=false (no contraction into FMA) and reductions follow the reference's
// summation order (sequential over k for column sums; NumPy's pairwise tree
// for the global dot products of the Helmholtz solver).
//
// Static geometry is never stored as 3D arrays on the device: the z-level
// thickness of a cell is a function of its column's depth H and the level
// table (reference libs/core/domain.py:113-129), so each kernel derives dz3,
// mask3 and the face thicknesses of the columns it touches in registers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define OC_MAXNZ 128
#define OC_MAX_LEVELS 16

namespace oc {

// Everything a step kernel needs, passed by value (lives in the kernel
// parameter bank, constant-cached).
struct KP {
    int nx, ny, nz, n2, n3, n3i;
    double dx, dy;
    // options
    int eos, pgf_remove, pgf_correction, advection, tracers_ts, closure_tke, mxl_recursive;
    int scheme;  // 0 fb, 1 theta, 2 split
    // physical constants
    double dt, g, f0, rho0, N2, nu, kappa, bottom_drag, a_h, k_h;
    double alpha_t, beta_s, t0, s0;
    double c_k, c_eps, pr_t, z_0, e_min, l_min, e_bb, n2_min;
    double theta, theta_cor, theta_v;
    // host-precomputed scalar products, formed in the reference's order
    double thv_dt;        // theta_v * dt
    double thv_dt_drag;   // (theta_v * dt) * bottom_drag
    double thv_dt_zero;   // (theta_v * dt) * 0.0 (tracer rows have no drag)
    double c1;            // (g * dt) * (1 - theta_eff)   explicit surface gradient
    double c2;            // (g * dt) * theta_eff         back-substitution
    double c3;            // (1 - theta_v) * dt           explicit vertical diffusion
    double one_m_tc;      // 1 - theta_cor
    double one_m_th;      // 1 - theta_eff
    double neg_f0;        // -f0
    double neg_g;         // -g
    double neg_n2;        // -N2
    double flux_t, flux_s;  // surface tracer fluxes
    double one_m_kappa3, one_p_kappa3;  // 1 - 1/3, 1 + 1/3
    // level table
    double edge[OC_MAXNZ + 1];   // depth of level tops, cumsum of dzr
    double dzr[OC_MAXNZ];
    double thin[OC_MAXNZ];       // min_partial * dzr
    double dz_nom[OC_MAXNZ];     // spacing of the momentum vertical advection per level
    // static 2D fields
    const double* H;
    const double* mask;
    const double* mask_u;
    const double* mask_v;
    const double* tau_u;   // surface stress / rho0 at u faces, masked
    const double* tau_v;
    const double* ustar2;  // closure surface u*^2
    const int2* kinfo;     // per column: (levels of exact thickness dzr, wet levels)
    const double2* dzx;    // per column: thickness of wet levels kfull and kfull + 1
    const int2* kface;     // per column: wet levels of its east (x) and north (y) face
    int face_rule;         // 0 min, 1 mean, 2 harmonic
    // levels one CTA marches in k_mom_column and k_tracer_rhs (1..nz); every
    // value gives the same results, only the speed depends on it
    int mom_kl, tr_kl;
};

__device__ __forceinline__ int wrapi(int i, int n) {
    if (i < 0) i += n;
    if (i >= n) i -= n;
    if (i < 0 || i >= n) {  // only for grids narrower than the offset
        i %= n;
        if (i < 0) i += n;
    }
    return i;
}

__device__ __forceinline__ double inv_pos(double a) { return a > 0.0 ? 1.0 / a : 0.0; }

// z-level partial-cell thickness of level k of column c and its wet mask
// (reference domain.py:113-129: dz3_ref = clip(H - edge, 0, dzr) with thin
// cells removed, times the wet mask). The host stores each column in compact
// form -- kinfo = (kfull, kb): levels below kfull are full (thickness dzr[k]
// exactly), levels kfull..kb-1 are wet with the explicit thicknesses dzx, levels
// from kb on are dry -- after checking that it reproduces the formula bit for
// bit, so no 3D geometry array is ever read.
__device__ __forceinline__ double col_dz(const KP& P, int c, int k, double& m3) {
    const int2 ki = P.kinfo[c];
    if (k >= ki.y) {
        m3 = 0.0;
        return 0.0;
    }
    m3 = 1.0;
    if (k < ki.x) return P.dzr[k];
    const double2 dx = P.dzx[c];
    return k == ki.x ? dx.x : dx.y;
}

// the compact geometry of one column held in registers; dz() equals col_dz()
struct ColGeo {
    int kf, kb;
    double d0, d1;
    __device__ __forceinline__ static ColGeo load(const KP& P, int c) {
        const int2 ki = P.kinfo[c];
        const double2 dx = P.dzx[c];
        return ColGeo{ki.x, ki.y, dx.x, dx.y};
    }
    __device__ __forceinline__ double dz(const KP& P, int k, double& m3) const {
        if (k >= kb) {
            m3 = 0.0;
            return 0.0;
        }
        m3 = 1.0;
        if (k < kf) return P.dzr[k];
        return k == kf ? d0 : d1;
    }
    // depth of the top of level k: the sequential sum of the thicknesses above
    // (col_above with the column's geometry in registers)
    __device__ __forceinline__ double above(const KP& P, int k) const {
        const int m = k < kf ? k : kf;
        double a = P.edge[m];
        if (k > kf && kf < kb) {
            a = (m == 0) ? d0 : a + d0;
            if (k > kf + 1 && kf + 1 < kb) a = a + d1;
        }
        return a;
    }
};

__device__ __forceinline__ double col_m3(const KP& P, int c, int k) { return k < P.kinfo[c].y ? 1.0 : 0.0; }

// 3D face masks m3 * m3(neighbour) * mask_face (domain.py:93-96): the wet levels
// of a face are the top min(kb, kb of the neighbour) levels when the 2D face
// is open, so one integer per face and column (checked on the host) gives them
__device__ __forceinline__ double col_m3u(const KP& P, int c, int k) { return k < P.kface[c].x ? 1.0 : 0.0; }
__device__ __forceinline__ double col_m3v(const KP& P, int c, int k) { return k < P.kface[c].y ? 1.0 : 0.0; }

// depth of the top of level k (the sequential sum of dz3 above it) and of the
// level centre (reference domain.py:148-154)
__device__ __forceinline__ double col_above(const KP& P, int c, int k) {
    const int2 ki = P.kinfo[c];
    const int m = k < ki.x ? k : ki.x;
    double above = P.edge[m];
    if (k > ki.x && ki.x < ki.y) {
        const double2 dx = P.dzx[c];
        above = (m == 0) ? dx.x : above + dx.x;
        if (k > ki.x + 1 && ki.x + 1 < ki.y) above = above + dx.y;
    }
    return above;
}


__device__ __forceinline__ double face_combine(const KP& P, double a, double b) {
    if (P.face_rule == 0) return fmin(a, b);
    if (P.face_rule == 1) return 0.5 * (a + b);
    double tot = a + b;
    return tot > 0.0 ? 2.0 * a * b / tot : 0.0;
}

// Superbee limiter of the TVD face (reference advection_v06.py:35-43)
__device__ __forceinline__ double superbee(double r) {
    return fmax(0.0, fmax(fmin(2.0 * r, 1.0), fmin(r, 2.0)));
}

// Upwind-biased value on the face between c0 and c1 (c_m = left of c0,
// c_p = right of c1), advecting velocity vel, far-cell wet flags wm (left of
// c0) and wp (right of c1). Reference advection_v06.py:21-47. The reference
// forms both one-sided values and selects by the sign of vel. Here the inputs
// are selected first and one value is formed: for vel <= 0 the reference's
// c1 - t equals c1 + (-t) exactly, so the bits are the same, with one division
// instead of two and no divergent branch.
__device__ __forceinline__ double kappa_face(const KP& P, double cm, double c0, double c1, double cp,
                                             double vel, double wm, double wp, bool limited) {
    const bool pos = vel > 0.0;
    const double base = pos ? c0 : c1;
    const double far = pos ? (c0 - cm) : (cp - c1);
    const double d = c1 - c0;
    double t;
    if (limited) {
        const double eps = d == 0.0 ? 1.0 : d;
        const double r = d == 0.0 ? 0.0 : far / eps;
        t = 0.5 * superbee(r) * d;
    } else {
        t = 0.25 * (P.one_m_kappa3 * far + P.one_p_kappa3 * d);
    }
    const double f = base + (pos ? t : -t);
    return ((pos ? wm : wp) > 0.0) ? f : base;
}

// Interior vertical face value at an interface with `above` (layer k-1),
// `below` (layer k), far_up (k-2, 0 when absent), far_dn (k+1, 0 when absent)
// and wet flags of the far cells; w positive upward. advection_v06.py:50-74,
// selected before forming as in kappa_face.
__device__ __forceinline__ double kappa_face_z(const KP& P, double far_up, double above, double below,
                                               double far_dn, double w, bool has_up, bool has_dn,
                                               bool limited) {
    const bool up = w > 0.0;
    const double base = up ? below : above;
    const double far = up ? (below - far_dn) : (far_up - above);
    const double d = above - below;
    double t;
    if (limited) {
        const double eps = d == 0.0 ? 1.0 : d;
        const double r = d == 0.0 ? 0.0 : far / eps;
        t = 0.5 * superbee(r) * d;
    } else {
        t = 0.25 * (P.one_m_kappa3 * far + P.one_p_kappa3 * d);
    }
    const double f = base + (up ? t : -t);
    return (up ? has_dn : has_up) ? f : base;
}

// ---------------------------------------------------------------- EOS
// polyTEOS10-bsq (Roquet et al. 2015, Table 4) and the S-EOS of their eq. (25):
// the published coefficients, in the Horner form of reference eos.py:68-111.
__device__ __forceinline__ double rho_teos10(double CT, double SA, double z) {
    const double zh = z * 1.0e-4;
    const double ss = sqrt((SA + 32.0) * (0.875 / 35.16504));
    const double tt = CT * (1.0 / 40.0);
    const double r0 = (((((-1.7243708991e-03 * zh + 1.5616995503e-02) * zh + 6.4326772569e-02) * zh
                         + 2.2601900708e-01) * zh + -5.2099962525e+00) * zh + 4.6494977072e+01) * zh;
    const double rz3 = 3.7969820455e-01 * tt + -1.8507636718e-02 * ss + -2.3342758797e-02;
    const double rz2 = ((-1.2419983026e+00 * tt + -2.1311365518e-01 * ss + 2.0564311499e+00) * tt
                        + (2.5019633803e+00 * ss + -4.9527603989e+00) * ss + 2.0660924175e+00);
    const double rz1 = ((((5.5927935970e-01 * tt + -5.5077101279e-01 * ss + -2.4649669534e+00) * tt
                          + (-1.8795372996e+00 * ss + 3.5063081279e+00) * ss + 6.7080479603e+00) * tt
                         + ((-6.5399043664e-01 * ss + 5.0042598061e+00) * ss + -4.4870114575e+00) * ss
                         + -1.3336301113e+01) * tt
                        + (((6.6051753097e+00 * ss + -3.0938076334e+01) * ss + 5.0774768218e+01) * ss
                           + -4.2549998214e+01) * ss
                        + 1.9681925209e+01);
    const double rz0 = ((((((-1.9098268277e-01 * tt + 4.5111434961e-01 * ss + 5.4048723791e-01) * tt
                            + (-5.3563304045e+00 * ss + 1.1311538584e+01) * ss + -8.3627885467e+00) * tt
                           + ((-3.1742946532e+00 * ss + 1.9717078466e+01) * ss + -3.3449108469e+01) * ss
                           + 2.1661789529e+01) * tt
                          + (((-5.4723692739e+00 * ss + 2.9130021253e+01) * ss + -6.0362551501e+01) * ss
                             + 6.1548258127e+01) * ss
                          + -3.7074170417e+01) * tt
                         + ((((-1.9193502195e+00 * ss + 1.7681814114e+01) * ss + -5.6888046321e+01) * ss
                             + 8.1770425108e+01) * ss
                            + -6.5281885265e+01) * ss
                         + 2.6010145068e+01) * tt
                        + (((((-6.0579916612e+01 * ss + 4.3227585684e+02) * ss + -1.2849161071e+03) * ss
                             + 2.0375295546e+03) * ss
                            + -1.7864682637e+03) * ss
                           + 8.6672408165e+02) * ss
                        + 8.0189615746e+02);
    return ((rz3 * zh + rz2) * zh + rz1) * zh + rz0 + r0;
}

// density anomaly rho' (eos.py:103-127): linear with the given constants, the
// simplified EOS, or polyTEOS10-bsq about rho0
__device__ __forceinline__ double rho_anomaly_of(int eos, double rho0, double alpha_t, double beta_s,
                                                 double t0, double s0, double T, double S, double z) {
    if (eos == 0) return rho0 * (-alpha_t * (T - t0) + beta_s * (S - s0));
    if (eos == 1) {
        const double Ta = T - 10.0, Sa = S - 35.0;
        return (-1.6550e-1 * (1.0 + (0.5 * 5.9520e-2) * Ta + 1.4970e-4 * z) * Ta
                + 7.6554e-1 * (1.0 - (0.5 * 7.4914e-4) * Sa - 1.1090e-5 * z) * Sa
                - 2.4341e-3 * Ta * Sa);
    }
    return rho_teos10(T, S, z) - rho0;
}

__device__ __forceinline__ double rho_anomaly(const KP& P, double T, double S, double z) {
    return rho_anomaly_of(P.eos, P.rho0, P.alpha_t, P.beta_s, P.t0, P.s0, T, S, z);
}

__device__ __forceinline__ double buoyancy_of(const KP& P, double T, double S, double z) {
    return P.neg_g * rho_anomaly(P, T, S, z) / P.rho0;
}

// ---------------------------------------------------------------- launch helpers
void launch_check(const char* where);

}  // namespace oc
