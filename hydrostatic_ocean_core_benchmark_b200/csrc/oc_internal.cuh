// Internal definitions of the sm_100a ocean-core step.
//
// Bit-for-bit parity with the reference NumPy step (libs/core/model3d_v05.py)
// is a design rule of the fp64 path: every expression below performs the same
// IEEE-754 fp64 operations in the same order as the reference, the fp64 build
// is compiled with -fmad=false (no contraction into FMA) and reductions follow
// the reference's summation order (sequential over k for column sums; NumPy's
// pairwise tree for the global dot products of the Helmholtz solver).
//
// The helpers are templates on the floating type T of the step's 3D fields:
// T = double is the fp64 path (every literal T(x) is then the same double, so
// the operations are exactly the reference's); T = float is the mixed-precision
// path, whose stencils and column solves run in FP32 (compiled separately, with
// contraction).
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

template <class T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// Everything a step kernel needs, passed by value (lives in the kernel
// parameter bank, constant-cached). T is the floating type of the 3D fields.
// The fp64 copies (dx64, dy64, edge64, dzx64, eos constants) serve the few
// quantities the mixed path keeps in FP64 (pressure-gradient depths, the EOS,
// the surface-elevation gradient); in the fp64 path they equal the T fields.
template <class T>
struct KPT {
    int nx, ny, nz, n2, n3, n3i;
    T dx, dy;
    // options
    int eos, pgf_remove, pgf_correction, advection, tracers_ts, closure_tke, mxl_recursive;
    int scheme;  // 0 fb, 1 theta, 2 split
    // physical constants
    T dt, g, f0, rho0, N2, nu, kappa, bottom_drag, a_h, k_h;
    T alpha_t, beta_s, t0, s0;
    T c_k, c_eps, pr_t, z_0, e_min, l_min, e_bb, n2_min;
    T theta, theta_cor, theta_v;
    // host-precomputed scalar products, formed in the reference's order
    T thv_dt;        // theta_v * dt
    T thv_dt_drag;   // (theta_v * dt) * bottom_drag
    T thv_dt_zero;   // (theta_v * dt) * 0.0 (tracer rows have no drag)
    T c1;            // (g * dt) * (1 - theta_eff)   explicit surface gradient
    T c2;            // (g * dt) * theta_eff         back-substitution
    T c3;            // (1 - theta_v) * dt           explicit vertical diffusion
    T one_m_tc;      // 1 - theta_cor
    T one_m_th;      // 1 - theta_eff
    T neg_f0;        // -f0
    T neg_g;         // -g
    T neg_n2;        // -N2
    T flux_t, flux_s;  // surface tracer fluxes
    T one_m_kappa3, one_p_kappa3;  // 1 - 1/3, 1 + 1/3
    // level table
    T edge[OC_MAXNZ + 1];   // depth of level tops, cumsum of dzr
    T dzr[OC_MAXNZ];
    T thin[OC_MAXNZ];       // min_partial * dzr
    T dz_nom[OC_MAXNZ];     // spacing of the momentum vertical advection per level
    // static 2D fields
    const T* H;
    const T* mask;
    const T* mask_u;
    const T* mask_v;
    const T* tau_u;   // surface stress / rho0 at u faces, masked
    const T* tau_v;
    const T* ustar2;  // closure surface u*^2
    const int2* kinfo;     // per column: (levels of exact thickness dzr, wet levels)
    const typename Vec2<T>::type* dzx;  // per column: thickness of wet levels kfull and kfull + 1
    const int2* kface;     // per column: wet levels of its east (x) and north (y) face
    int face_rule;         // 0 min, 1 mean, 2 harmonic
    // levels one CTA marches in k_mom_column and k_tracer_rhs (1..nz); every
    // value gives the same results, only the speed depends on it
    int mom_kl, tr_kl;
    // fp64 copies (see above)
    double dx64, dy64;
    double rho0_64, alpha_t64, beta_s64, t0_64, s0_64, neg_g64;
    const double* mask_u64;
    const double* mask_v64;
    const double2* dzx64;
    double edge64[OC_MAXNZ + 1];
    double dzr64[OC_MAXNZ];
};
using KP = KPT<double>;

__device__ __forceinline__ int wrapi(int i, int n) {
    if (i < 0) i += n;
    if (i >= n) i -= n;
    if (i < 0 || i >= n) {  // only for grids narrower than the offset
        i %= n;
        if (i < 0) i += n;
    }
    return i;
}

template <class T>
__device__ __forceinline__ T inv_pos(T a) { return a > T(0.0) ? T(1.0) / a : T(0.0); }

// z-level partial-cell thickness of level k of column c and its wet mask
// (reference domain.py:113-129: dz3_ref = clip(H - edge, 0, dzr) with thin
// cells removed, times the wet mask). The host stores each column in compact
// form -- kinfo = (kfull, kb): levels below kfull are full (thickness dzr[k]
// exactly), levels kfull..kb-1 are wet with the explicit thicknesses dzx, levels
// from kb on are dry -- after checking that it reproduces the formula bit for
// bit, so no 3D geometry array is ever read.
template <class T>
__device__ __forceinline__ T col_dz(const KPT<T>& P, int c, int k, T& m3) {
    const int2 ki = P.kinfo[c];
    if (k >= ki.y) {
        m3 = T(0.0);
        return T(0.0);
    }
    m3 = T(1.0);
    if (k < ki.x) return P.dzr[k];
    const auto dx = P.dzx[c];
    return k == ki.x ? dx.x : dx.y;
}

// the compact geometry of one column held in registers; dz() equals col_dz()
template <class T>
struct ColGeoT {
    int kf, kb;
    T d0, d1;
    __device__ __forceinline__ static ColGeoT load(const KPT<T>& P, int c) {
        const int2 ki = P.kinfo[c];
        const auto dx = P.dzx[c];
        return ColGeoT{ki.x, ki.y, dx.x, dx.y};
    }
    __device__ __forceinline__ T dz(const KPT<T>& P, int k, T& m3) const {
        if (k >= kb) {
            m3 = T(0.0);
            return T(0.0);
        }
        m3 = T(1.0);
        if (k < kf) return P.dzr[k];
        return k == kf ? d0 : d1;
    }
    // depth of the top of level k: the sequential sum of the thicknesses above
    // (col_above with the column's geometry in registers)
    __device__ __forceinline__ T above(const KPT<T>& P, int k) const {
        const int m = k < kf ? k : kf;
        T a = P.edge[m];
        if (k > kf && kf < kb) {
            a = (m == 0) ? d0 : a + d0;
            if (k > kf + 1 && kf + 1 < kb) a = a + d1;
        }
        return a;
    }
};

using ColGeo = ColGeoT<double>;

// the same column geometry in fp64 from the fp64 copies (the fp64 path's values
// exactly): the depths the mixed path's pressure gradient and EOS are formed at
struct ColGeo64 {
    int kf, kb;
    double d0, d1;
    template <class T>
    __device__ __forceinline__ static ColGeo64 load(const KPT<T>& P, int c) {
        const int2 ki = P.kinfo[c];
        const double2 dx = P.dzx64[c];
        return ColGeo64{ki.x, ki.y, dx.x, dx.y};
    }
    template <class T>
    __device__ __forceinline__ double dz(const KPT<T>& P, int k) const {
        if (k >= kb) return 0.0;
        if (k < kf) return P.dzr64[k];
        return k == kf ? d0 : d1;
    }
    template <class T>
    __device__ __forceinline__ double above(const KPT<T>& P, int k) const {
        const int m = k < kf ? k : kf;
        double a = P.edge64[m];
        if (k > kf && kf < kb) {
            a = (m == 0) ? d0 : a + d0;
            if (k > kf + 1 && kf + 1 < kb) a = a + d1;
        }
        return a;
    }
};

template <class T>
__device__ __forceinline__ T col_m3(const KPT<T>& P, int c, int k) { return k < P.kinfo[c].y ? T(1.0) : T(0.0); }

// 3D face masks m3 * m3(neighbour) * mask_face (domain.py:93-96): the wet levels
// of a face are the top min(kb, kb of the neighbour) levels when the 2D face
// is open, so one integer per face and column (checked on the host) gives them
template <class T>
__device__ __forceinline__ T col_m3u(const KPT<T>& P, int c, int k) { return k < P.kface[c].x ? T(1.0) : T(0.0); }
template <class T>
__device__ __forceinline__ T col_m3v(const KPT<T>& P, int c, int k) { return k < P.kface[c].y ? T(1.0) : T(0.0); }

// depth of the top of level k (the sequential sum of dz3 above it) and of the
// level centre (reference domain.py:148-154)
template <class T>
__device__ __forceinline__ T col_above(const KPT<T>& P, int c, int k) {
    const int2 ki = P.kinfo[c];
    const int m = k < ki.x ? k : ki.x;
    T above = P.edge[m];
    if (k > ki.x && ki.x < ki.y) {
        const auto dx = P.dzx[c];
        above = (m == 0) ? dx.x : above + dx.x;
        if (k > ki.x + 1 && ki.x + 1 < ki.y) above = above + dx.y;
    }
    return above;
}


template <class T>
__device__ __forceinline__ T face_combine(const KPT<T>& P, T a, T b) {
    if (P.face_rule == 0) return fmin(a, b);
    if (P.face_rule == 1) return T(0.5) * (a + b);
    T tot = a + b;
    return tot > T(0.0) ? T(2.0) * a * b / tot : T(0.0);
}

// Superbee limiter of the TVD face (reference advection_v06.py:35-43)
template <class T>
__device__ __forceinline__ T superbee(T r) {
    return fmax(T(0.0), fmax(fmin(T(2.0) * r, T(1.0)), fmin(r, T(2.0))));
}

// Upwind-biased value on the face between c0 and c1 (c_m = left of c0,
// c_p = right of c1), advecting velocity vel, far-cell wet flags wm (left of
// c0) and wp (right of c1). Reference advection_v06.py:21-47. The reference
// forms both one-sided values and selects by the sign of vel. Here the inputs
// are selected first and one value is formed: for vel <= 0 the reference's
// c1 - t equals c1 + (-t) exactly, so the bits are the same, with one division
// instead of two and no divergent branch.
template <class T>
__device__ __forceinline__ T kappa_face(const KPT<T>& P, T cm, T c0, T c1, T cp, T vel, T wm, T wp, bool limited) {
    const bool pos = vel > T(0.0);
    const T base = pos ? c0 : c1;
    const T far = pos ? (c0 - cm) : (cp - c1);
    const T d = c1 - c0;
    T t;
    if (limited) {
        const T eps = d == T(0.0) ? T(1.0) : d;
        const T r = d == T(0.0) ? T(0.0) : far / eps;
        t = T(0.5) * superbee(r) * d;
    } else {
        t = T(0.25) * (P.one_m_kappa3 * far + P.one_p_kappa3 * d);
    }
    const T f = base + (pos ? t : -t);
    return ((pos ? wm : wp) > T(0.0)) ? f : base;
}

// Interior vertical face value at an interface with `above` (layer k-1),
// `below` (layer k), far_up (k-2, 0 when absent), far_dn (k+1, 0 when absent)
// and wet flags of the far cells; w positive upward. advection_v06.py:50-74,
// selected before forming as in kappa_face.
template <class T>
__device__ __forceinline__ T kappa_face_z(const KPT<T>& P, T far_up, T above, T below, T far_dn, T w, bool has_up,
                                          bool has_dn, bool limited) {
    const bool up = w > T(0.0);
    const T base = up ? below : above;
    const T far = up ? (below - far_dn) : (far_up - above);
    const T d = above - below;
    T t;
    if (limited) {
        const T eps = d == T(0.0) ? T(1.0) : d;
        const T r = d == T(0.0) ? T(0.0) : far / eps;
        t = T(0.5) * superbee(r) * d;
    } else {
        t = T(0.25) * (P.one_m_kappa3 * far + P.one_p_kappa3 * d);
    }
    const T f = base + (up ? t : -t);
    return (up ? has_dn : has_up) ? f : base;
}
// ---------------------------------------------------------------- EOS
// polyTEOS10-bsq (Roquet et al. 2015, Table 4) and the S-EOS of their eq. (25):
// the published coefficients, in the Horner form of reference eos.py:68-111.
// N is double for the step; the adjoint evaluates the same expressions on a
// dual number (value and derivative) to get the exact partial derivatives
template <class N>
__device__ __forceinline__ N rho_teos10_n(N CT, N SA, N z) {
    const N zh = z * 1.0e-4;
    const N ss = sqrt((SA + 32.0) * (0.875 / 35.16504));
    const N tt = CT * (1.0 / 40.0);
    const N r0 = (((((-1.7243708991e-03 * zh + 1.5616995503e-02) * zh + 6.4326772569e-02) * zh
                         + 2.2601900708e-01) * zh + -5.2099962525e+00) * zh + 4.6494977072e+01) * zh;
    const N rz3 = 3.7969820455e-01 * tt + -1.8507636718e-02 * ss + -2.3342758797e-02;
    const N rz2 = ((-1.2419983026e+00 * tt + -2.1311365518e-01 * ss + 2.0564311499e+00) * tt
                        + (2.5019633803e+00 * ss + -4.9527603989e+00) * ss + 2.0660924175e+00);
    const N rz1 = ((((5.5927935970e-01 * tt + -5.5077101279e-01 * ss + -2.4649669534e+00) * tt
                          + (-1.8795372996e+00 * ss + 3.5063081279e+00) * ss + 6.7080479603e+00) * tt
                         + ((-6.5399043664e-01 * ss + 5.0042598061e+00) * ss + -4.4870114575e+00) * ss
                         + -1.3336301113e+01) * tt
                        + (((6.6051753097e+00 * ss + -3.0938076334e+01) * ss + 5.0774768218e+01) * ss
                           + -4.2549998214e+01) * ss
                        + 1.9681925209e+01);
    const N rz0 = ((((((-1.9098268277e-01 * tt + 4.5111434961e-01 * ss + 5.4048723791e-01) * tt
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

__device__ __forceinline__ double rho_teos10(double CT, double SA, double z) { return rho_teos10_n<double>(CT, SA, z); }

// density anomaly rho' (eos.py:103-127): linear with the given constants, the
// simplified EOS, or polyTEOS10-bsq about rho0
template <class N>
__device__ __forceinline__ N rho_anomaly_n(int eos, double rho0, double alpha_t, double beta_s, double t0, double s0,
                                           N T, N S, N z) {
    if (eos == 0) return rho0 * (-alpha_t * (T - t0) + beta_s * (S - s0));
    if (eos == 1) {
        const N Ta = T - 10.0, Sa = S - 35.0;
        return (-1.6550e-1 * (1.0 + (0.5 * 5.9520e-2) * Ta + 1.4970e-4 * z) * Ta
                + 7.6554e-1 * (1.0 - (0.5 * 7.4914e-4) * Sa - 1.1090e-5 * z) * Sa
                - 2.4341e-3 * Ta * Sa);
    }
    return rho_teos10_n<N>(T, S, z) - rho0;
}

__device__ __forceinline__ double rho_anomaly_of(int eos, double rho0, double alpha_t, double beta_s,
                                                 double t0, double s0, double T, double S, double z) {
    return rho_anomaly_n<double>(eos, rho0, alpha_t, beta_s, t0, s0, T, S, z);
}

// The EOS is evaluated in fp64 on both paths, with the fp64 copies of the
// constants (in the fp64 path they are the constants themselves): in FP32 the
// anomaly rho - rho0 of a ~1027 kg m-3 density would keep only ~3 digits.
template <class T>
__device__ __forceinline__ double rho_anomaly(const KPT<T>& P, double Tc, double Sa, double z) {
    return rho_anomaly_of(P.eos, P.rho0_64, P.alpha_t64, P.beta_s64, P.t0_64, P.s0_64, Tc, Sa, z);
}

template <class T>
__device__ __forceinline__ double buoyancy_of(const KPT<T>& P, double Tc, double Sa, double z) {
    return P.neg_g64 * rho_anomaly(P, Tc, Sa, z) / P.rho0_64;
}

// ---------------------------------------------------------------- launch helpers
void launch_check(const char* where);

}  // namespace oc
