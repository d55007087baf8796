// Column and stencil kernels of the ocean-core step (sm_100a, fp64).
//
// The column kernels map one thread to one water column (i, j) and march over
// the levels k, so every vertical recurrence of the reference (cumulative sums,
// Thomas sweeps, the closure's mixing-length marches) runs in the reference's
// order; the 32 threads of a warp read 32 consecutive i of each level plane
// (coalesced 256-byte rows). The stencil kernels (k_mom_column, k_tracer_rhs,
// k_predictor_rhs) work on tiles of columns over a range of levels.
//
// Reference correspondence (paths inside the reference project):
//   k_closure         libs/core/closure.py:43-205 + model3d_v05.py:141-157 (q = A^-1 1)
//   k_qsolve          model3d_v05.py:147-153 (constant-coefficient q)
//   k_kukv            model3d_v05.py:154-157
//   k_wcol            vertical_var.py:109-121 + model3d_v05.py:232-235
//   k_phi             vertical_var.py:132-145
//   k_mom_column      model3d_v05.py:195-230, 241-260, 352-370; advection_v06.py:77-108;
//                     advection.py:62-95; operators_masked.py:45-68; vertical_var.py:80-106
//   k_predictor_rhs   model3d_v05.py:387-393
//   k_momentum_solve  model3d_v05.py:394-395, 426-433 + vertical.py:17-44
//   k_backsub         model3d_v05.py:404-406
//   k_tracer_rhs      model3d_v05.py:466-512
//   k_tracer_solve    model3d_v05.py:514-533 + eos.py:68-133
//   2D kernels        model3d_v05.py:290-335, 376-384, 396-400, 410-413, 440-461

#include "oc_internal.cuh"
#include "step_kernels.cuh"

namespace oc {

// ------------------------------------------------------------------ helpers

// Row k of A = I - thv dt Dz for a column (reference vertical_var.py:35-77).
__device__ __forceinline__ void implicit_row(const KP& P, int k, double dzk, double m3k, double m3k1,
                                             double dzi_k, double dzi_k1, double Kk, double Kk1,
                                             double thv_dt_drag, double& sub, double& diag,
                                             double& sup) {
    const double inv_dz = inv_pos(dzk);
    const double fac = P.thv_dt * inv_dz;
    const double at = fac * Kk * inv_pos(dzi_k);
    const double ab = fac * Kk1 * inv_pos(dzi_k1);
    sub = -at;
    sup = -ab;
    diag = 1.0 + at + ab;
    if (k == 0) {
        diag = 1.0 + ab;
        sub = 0.0;
    }
    if (m3k > 0.0 && m3k1 == 0.0) {
        diag = 1.0 + at + thv_dt_drag * inv_dz;
        sup = 0.0;
    }
    if (m3k == 0.0) {
        diag = 1.0;
        sub = 0.0;
        sup = 0.0;
    }
}

// neighbour offsets of one column, wrapped once (periodic index layout, up to
// three cells away)
struct Nbr {
    int i, j, c;
    int nx, ny;
    int ix[7], jy[7];  // i-3..i+3 and (j-3..j+3) * nx, wrapped
    __device__ __forceinline__ void init(int i_, int j_, int nx_, int ny_) {
        i = i_;
        j = j_;
        nx = nx_;
        ny = ny_;
        c = j * nx + i;
#pragma unroll
        for (int d = -3; d <= 3; ++d) {
            ix[d + 3] = wrapi(i + d, nx);
            jy[d + 3] = wrapi(j + d, ny) * nx;
        }
    }
    __device__ __forceinline__ int at(int dj, int di) const { return jy[dj + 3] + ix[di + 3]; }
};

__device__ __forceinline__ double m3u_at(const KP& P, const Nbr& n, int dj, int di, int k) {
    return col_m3u(P, n.at(dj, di), k);
}

__device__ __forceinline__ double m3v_at(const KP& P, const Nbr& n, int dj, int di, int k) {
    return col_m3v(P, n.at(dj, di), k);
}

__device__ __forceinline__ double m3_at(const KP& P, const Nbr& n, int dj, int di, int k) {
    return col_m3(P, n.at(dj, di), k);
}

// face thickness at level k of a face whose wet levels are the top kf ones,
// between cells of thickness dza and dzb: mask3_face x face_combine(dza, dzb)
// (reference domain.py:93-96, 142-146)
__device__ __forceinline__ double face_dz(const KP& P, int kf, int k, double dza, double dzb) {
    return (k < kf ? 1.0 : 0.0) * face_combine(P, dza, dzb);
}

#define COLUMN_PROLOGUE                                  \
    const int i = blockIdx.x * blockDim.x + threadIdx.x; \
    const int j = blockIdx.y * blockDim.y + threadIdx.y; \
    if (i >= P.nx || j >= P.ny) return;                  \
    Nbr nb;                                              \
    nb.init(i, j, P.nx, P.ny);                           \
    const size_t n2 = (size_t)P.n2;                      \
    (void)n2;

// ------------------------------------------------------------------ q = A^-1 1 on a column
// interface spacing of the column (closure.py:43-62): dz[0] at the surface,
// dz[nz-1] at the bottom, the mean of the two levels elsewhere
__device__ __forceinline__ double col_dzi(const KP& P, const ColGeo& g, int k) {
    double m;
    if (k == 0) return g.dz(P, 0, m);
    if (k == P.nz) return g.dz(P, P.nz - 1, m);
    const double a = g.dz(P, k - 1, m);
    return 0.5 * (a + g.dz(P, k, m));
}

// Momentum tridiagonal with a unit right-hand side for the column's interface
// viscosity Km(k), k = 0..nz (reference model3d_v05.py:147-153). The forward
// elimination keeps its coefficients in cs and its right-hand sides in q, which
// the back substitution then overwrites with the solution.
template <class KM>
__device__ __forceinline__ void column_q(const KP& P, const ColGeo& g, KM Km, double* cs,
                                         double* __restrict__ q, int c, size_t n2) {
    const int nz = P.nz;
    double m3_k, dz_k = g.dz(P, 0, m3_k);
    double dzi_k = dz_k;
    double km_k = Km(0);
    double ds = 0.0, cp = 0.0;
#pragma unroll 2
    for (int k = 0; k < nz; ++k) {
        double m3_k1 = 0.0, dz_k1 = 0.0;
        if (k + 1 < nz) dz_k1 = g.dz(P, k + 1, m3_k1);
        const double dzi_k1 = (k + 1 < nz) ? 0.5 * (dz_k + dz_k1) : dz_k;
        const double km_k1 = Km(k + 1);
        double sub, diag, sup;
        implicit_row(P, k, dz_k, m3_k, m3_k1, dzi_k, dzi_k1, km_k, km_k1, P.thv_dt_drag, sub, diag, sup);
        if (k == 0) {
            cp = sup / diag;
            ds = 1.0 / diag;
        } else {
            const double den = diag - sub * cp;
            cp = sup / den;
            ds = (1.0 - sub * ds) / den;
        }
        cs[k] = cp;
        if (k + 1 < nz) q[(size_t)k * n2 + c] = ds;
        km_k = km_k1;
        dz_k = dz_k1;
        m3_k = m3_k1;
        dzi_k = dzi_k1;
    }
    double x = ds;
    q[(size_t)(nz - 1) * n2 + c] = x;
#pragma unroll 4
    for (int k = nz - 2; k >= 0; --k) {
        const size_t o = (size_t)k * n2 + c;
        x = q[o] - cs[k] * x;
        q[o] = x;
    }
}

template <int NZM>
__global__ void __launch_bounds__(128) k_qsolve(KP P, const double* __restrict__ km,
                                                double* __restrict__ q) {
    COLUMN_PROLOGUE
    const int c = nb.c;
    const ColGeo g = ColGeo::load(P, c);
    double cs[NZM];
    column_q(P, g, [&](int k) { return km[(size_t)k * n2 + c]; }, cs, q, c, n2);
}

// ------------------------------------------------------------------ TKE closure
// One thread per column (closure.py:141-205): shear and N^2 on interfaces, the
// mixing lengths, the implicit TKE tridiagonal (nz+1 rows), K_m/K_h, then q for
// the new K_m. Only N^2, shear^2, the new K_m and the elimination coefficients
// are kept per thread; the elimination right-hand sides go to e (whose old value
// at a level is read just before) and q. With the Gaspar lengths, the lengths
// of interface k are formed inside the forward sweep.
template <int NZM>
__global__ void __launch_bounds__(128, 8) k_closure(KP P, const double* __restrict__ u,
                                                 const double* __restrict__ v,
                                                 const double* __restrict__ b,
                                                 double* __restrict__ e, double* __restrict__ km,
                                                 double* __restrict__ kh, double* __restrict__ q) {
    COLUMN_PROLOGUE
    const int nz = P.nz;
    const int c = nb.c;
    const size_t cw = nb.at(0, -1), cs_ = nb.at(-1, 0);
    const ColGeo g = ColGeo::load(P, c);
    double nn2[NZM + 1], sh2[NZM + 1], lk[NZM + 1], le[NZM + 1], cst[NZM + 1];
    double depth = 0.0;
    for (int k = 0; k < nz; ++k) {
        double m;
        const double dz = g.dz(P, k, m);
        depth = (k == 0) ? dz : depth + dz;
    }
    // shear^2 and N^2 on interfaces (closure.py:150-161)
    {
        double uc_prev = 0.0, vc_prev = 0.0, b_prev = 0.0, dz_prev = 0.0, m3_prev = 0.0;
#pragma unroll 2
        for (int k = 0; k < nz; ++k) {
            const size_t o = (size_t)k * n2;
            const double uc = 0.5 * (u[o + c] + u[o + cw]);
            const double vc = 0.5 * (v[o + c] + v[o + cs_]);
            const double bk = b[o + c];
            double m3k;
            const double dzk = g.dz(P, k, m3k);
            if (k >= 1) {
                const double wk = m3_prev * m3k;
                const double idz = inv_pos(0.5 * (dz_prev + dzk));
                const double du = (uc_prev - uc) * idz;
                const double dv = (vc_prev - vc) * idz;
                const double db = (b_prev - bk) * idz;
                sh2[k] = (du * du + dv * dv) * wk;
                nn2[k] = db * wk;
            }
            uc_prev = uc;
            vc_prev = vc;
            b_prev = bk;
            dz_prev = dzk;
            m3_prev = m3k;
        }
    }
    sh2[0] = 0.0;
    nn2[0] = 0.0;
    sh2[nz] = 0.0;
    nn2[nz] = 0.0;
    // recursive lengths (closure.py:106-129) need whole-column sweeps first
    if (P.mxl_recursive) {
        double zi = 0.0;
        for (int k = 0; k <= nz; ++k) {
            double m;
            if (k >= 1) zi = (k == 1) ? g.dz(P, 0, m) : zi + g.dz(P, k - 1, m);
            const double zb = fmax(depth - zi, 0.0);
            const double ek = fmax(e[(size_t)k * n2 + c], P.e_min);
            const double n2c = fmax(nn2[k], P.n2_min);
            const double ell = sqrt(2.0 * ek / n2c);
            le[k] = fmin(ell, fmin(zi + P.z_0, zb + P.z_0));
        }
        for (int k = 1; k <= nz; ++k) le[k] = fmin(le[k], le[k - 1] + col_dzi(P, g, k));
        for (int k = nz - 1; k >= 0; --k) le[k] = fmin(le[k], le[k + 1] + col_dzi(P, g, k + 1));
        for (int k = 0; k <= nz; ++k) {
            double m0, m1;
            g.dz(P, k >= 1 ? k - 1 : 0, m0);
            g.dz(P, k, m1);
            const double wk = (k >= 1 && k <= nz - 1) ? m0 * m1 : 0.0;
            const double ell = le[k] * wk;
            lk[k] = fmax(P.l_min, sqrt(ell * ell));
            le[k] = fmax(P.l_min, fmin(ell, ell));
        }
    }
    // implicit TKE rows and forward sweep (closure.py:171-198)
    double rhs0 = 0.0, ds = 0.0, cp = 0.0, zi = 0.0;
    double km_prev = 0.0, km_cur = km[c];
    double m3_km1 = 0.0, dz_km1 = 0.0;  // level k-1
    double m3_k, dz_k = g.dz(P, 0, m3_k);
    for (int k = 0; k <= nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        const double km_next = (k < nz) ? km[o + n2] : 0.0;
        const double wk = (k >= 1 && k <= nz - 1) ? m3_km1 * m3_k : 0.0;
        const double e_old = e[o];
        double le_k;
        if (!P.mxl_recursive) {
            // Gaspar lengths (closure.py:65-104): march away from interface k
            // until the energy budget is spent; once the budget is zero the
            // reference's remaining steps add exactly 0
            if (k >= 1) zi = (k == 1) ? dz_km1 : zi + dz_km1;
            const double zb = fmax(depth - zi, 0.0);
            const double ek = fmax(e_old, P.e_min);
            double lu = 0.0, bud = ek;
            for (int kk = k - 1; kk >= 0 && bud > 0.0; --kk) {
                const double n2j = fmax(nn2[kk], 0.0), dzj = col_dzi(P, g, kk);
                const double cost = n2j * dzj * (lu + 0.5 * dzj);
                const bool full = cost <= bud;
                double step = dzj;
                if (!full && n2j > 0.0) {
                    const double part = sqrt(fmax(lu * lu + 2.0 * bud / n2j, 0.0)) - lu;
                    step = fmin(fmax(part, 0.0), dzj);
                }
                lu = lu + step;
                bud = full ? bud - cost : 0.0;
            }
            double ld = 0.0;
            bud = ek;
            for (int kk = k + 1; kk <= nz && bud > 0.0; ++kk) {
                const double n2j = fmax(nn2[kk], 0.0), dzj = col_dzi(P, g, kk);
                const double cost = n2j * dzj * (ld + 0.5 * dzj);
                const bool full = cost <= bud;
                double step = dzj;
                if (!full && n2j > 0.0) {
                    const double part = sqrt(fmax(ld * ld + 2.0 * bud / n2j, 0.0)) - ld;
                    step = fmin(fmax(part, 0.0), dzj);
                }
                ld = ld + step;
                bud = full ? bud - cost : 0.0;
            }
            lu = fmin(lu, zi + P.z_0) * wk;
            ld = fmin(ld, zb + P.z_0) * wk;
            lk[k] = fmax(P.l_min, sqrt(lu * ld));
            le_k = fmax(P.l_min, fmin(lu, ld));
        } else {
            le_k = le[k];
        }
        const double prod = (km_cur - P.nu) * sh2[k] - (kh[o] - P.kappa) * nn2[k];
        const double diss = P.c_eps * sqrt(fmax(e_old, P.e_min)) / le_k;
        double a_up = 0.0, a_dn = 0.0;
        if (k >= 1 && k <= nz - 1) {
            const double idzi = inv_pos(0.5 * (dz_km1 + dz_k));
            a_up = P.dt * (0.5 * (km_prev + km_cur)) * inv_pos(dz_km1) * idzi;
            a_dn = P.dt * (0.5 * (km_cur + km_next)) * inv_pos(dz_k) * idzi;
        }
        double sub = -a_up, sup = -a_dn;
        double diag = 1.0 + a_up + a_dn + P.dt * diss;
        double rhs = e_old + P.dt * prod;
        if (wk <= 0.0) {
            diag = 1.0;
            sub = 0.0;
            sup = 0.0;
            rhs = P.e_min;
        }
        if (k == 0) {
            rhs = (g.kb > 0) ? P.e_bb * P.ustar2[c] : P.e_min;
            rhs0 = rhs;
            cp = sup / diag;
            ds = rhs / diag;
        } else {
            const double den = diag - sub * cp;
            cp = sup / den;
            ds = (rhs - sub * ds) / den;
        }
        cst[k] = cp;
        e[o] = ds;
        km_prev = km_cur;
        km_cur = km_next;
        m3_km1 = m3_k;
        dz_km1 = dz_k;
        if (k + 1 < nz) {
            dz_k = g.dz(P, k + 1, m3_k);
        } else {
            dz_k = 0.0;
            m3_k = 0.0;
        }
    }
    // back substitution, e/K update (closure.py:198-205)
    double x = 0.0;
    for (int k = nz; k >= 0; --k) {
        const size_t o = (size_t)k * n2 + c;
        x = (k == nz) ? ds : e[o] - cst[k] * x;
        double m0, m1;
        g.dz(P, k >= 1 ? k - 1 : 0, m0);
        g.dz(P, k < nz ? k : 0, m1);
        const double wk = (k >= 1 && k <= nz - 1) ? m0 * m1 : 0.0;
        double en = fmax(x, P.e_min);
        en = (wk > 0.0) ? en : P.e_min;
        if (k == 0) en = rhs0;
        const double kmn = P.c_k * lk[k] * sqrt(en) * wk + P.nu;
        const double khn = (kmn - P.nu) / P.pr_t + P.kappa;
        e[o] = en;
        km[o] = kmn;
        kh[o] = khn;
        lk[k] = kmn;
    }
    column_q(P, g, [&](int k) { return lk[k]; }, cst, q, c, n2);
}

// ------------------------------------------------------------------ Ku, Kv
// Ku = sum_k dz3u * min(q, q_east) * mask_u (model3d_v05.py:154-157)
__global__ void k_kukv(KP P, const double* __restrict__ q, double* __restrict__ Ku,
                       double* __restrict__ Kv) {
    COLUMN_PROLOGUE
    const size_t c = nb.c;
    const size_t ce = nb.at(0, 1), cn = nb.at(1, 0);
    const ColGeo gc = ColGeo::load(P, (int)c), ge = ColGeo::load(P, (int)ce), gn = ColGeo::load(P, (int)cn);
    const int2 kf = P.kface[c];
    double su = 0.0, sv = 0.0;
#pragma unroll 4
    for (int k = 0; k < P.nz; ++k) {
        const size_t o = (size_t)k * n2;
        double m;
        const double dzc = gc.dz(P, k, m), dze = ge.dz(P, k, m), dzn = gn.dz(P, k, m);
        const double qc = q[o + c];
        const double tu = face_dz(P, kf.x, k, dzc, dze) * fmin(qc, q[o + ce]);
        const double tv = face_dz(P, kf.y, k, dzc, dzn) * fmin(qc, q[o + cn]);
        su = (k == 0) ? tu : su + tu;
        sv = (k == 0) ? tv : sv + tv;
    }
    Ku[c] = su * P.mask_u[c];
    Kv[c] = sv * P.mask_v[c];
}

// ------------------------------------------------------------------ w from transport divergence
// w[k] = -sum_{k'>=k} div(dz3u u, dz3v v)[k'], accumulated from the bottom
// (vertical_var.py:109-121); w[nz] = 0.
__global__ void __launch_bounds__(128, 8) k_wcol(KP P, const double* __restrict__ u, const double* __restrict__ v,
                       double* __restrict__ w) {
    COLUMN_PROLOGUE
    const int nz = P.nz;
    const size_t c = nb.c, cw = nb.at(0, -1), cs_ = nb.at(-1, 0);
    const ColGeo gc = ColGeo::load(P, (int)c), ge = ColGeo::load(P, nb.at(0, 1)),
                 gw = ColGeo::load(P, (int)cw), gn = ColGeo::load(P, nb.at(1, 0)), gs = ColGeo::load(P, (int)cs_);
    const int2 kf = P.kface[c];
    const int kuw = P.kface[cw].x, kvs = P.kface[cs_].y;
    double acc = 0.0;
    w[(size_t)nz * n2 + c] = 0.0;
#pragma unroll 2
    for (int k = nz - 1; k >= 0; --k) {
        const size_t o = (size_t)k * n2;
        double m3, m;
        const double dzc = gc.dz(P, k, m3);
        const double dzu_c = face_dz(P, kf.x, k, dzc, ge.dz(P, k, m));
        const double dzu_w = face_dz(P, kuw, k, gw.dz(P, k, m), dzc);
        const double dzv_c = face_dz(P, kf.y, k, dzc, gn.dz(P, k, m));
        const double dzv_s = face_dz(P, kvs, k, gs.dz(P, k, m), dzc);
        const double td = m3 * ((dzu_c * u[o + c] - dzu_w * u[o + cw]) / P.dx +
                                (dzv_c * v[o + c] - dzv_s * v[o + cs_]) / P.dy);
        acc = (k == nz - 1) ? td : acc + td;
        w[o + c] = -acc;
    }
}

// ------------------------------------------------------------------ buoyancy potential
// phi[k] = 0.5 dz3 b + sum_{k'<k} dz3 b, optionally minus its thickness-weighted
// column mean (vertical_var.py:132-145).
__global__ void k_phi(KP P, const double* __restrict__ b, double* __restrict__ phi) {
    COLUMN_PROLOGUE
    const int nz = P.nz;
    const size_t c = nb.c;
    const ColGeo g = ColGeo::load(P, (int)c);
    double above = 0.0, total = 0.0;
#pragma unroll 4
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        double m3;
        const double dz = g.dz(P, k, m3);
        const double bk = b[o];
        phi[o] = 0.5 * dz * bk + above;
        const double t = dz * bk;
        above = (k == 0) ? t : above + t;
        total = (k == 0) ? dz : total + dz;
    }
    if (P.pgf_remove) {
        double s = 0.0;
        for (int k = 0; k < nz; ++k) {
            double m3;
            const double dz = g.dz(P, k, m3);
            const double t = dz * phi[(size_t)k * n2 + c];
            s = (k == 0) ? t : s + t;
        }
        const double mean = s * inv_pos(total);
        for (int k = 0; k < nz; ++k) {
            const size_t o = (size_t)k * n2 + c;
            phi[o] = phi[o] - mean;
        }
    }
}

// ------------------------------------------------------------------ stencil accessors
// The horizontal stencils below read the face velocities and face masks of one
// level through an accessor: U(dj, di) / V(dj, di) are u / v of column
// (j + dj, i + di), MU / MV the 0/1 wet flags of its east / north face.
struct GlobalLevel {  // straight from the level planes in global memory
    const KP& P;
    const Nbr& nb;
    const double* __restrict__ u;
    const double* __restrict__ v;
    size_t o;
    int k;
    __device__ __forceinline__ double U(int dj, int di) const { return u[o + nb.at(dj, di)]; }
    __device__ __forceinline__ double V(int dj, int di) const { return v[o + nb.at(dj, di)]; }
    __device__ __forceinline__ double MU(int dj, int di) const { return col_m3u(P, nb.at(dj, di), k); }
    __device__ __forceinline__ double MV(int dj, int di) const { return col_m3v(P, nb.at(dj, di), k); }
};

// ------------------------------------------------------------------ Coriolis averages
// v averaged onto u points over wet v faces (operators_masked.py:45-52)
template <class A>
__device__ __forceinline__ double v_on_u_at(const A& a) {
    const double f0 = a.V(0, 0), f1 = a.V(-1, 0), f2 = a.V(0, 1), f3 = a.V(-1, 1);
    const double w0 = a.MV(0, 0), w1 = a.MV(-1, 0), w2 = a.MV(0, 1), w3 = a.MV(-1, 1);
    double num = 0.0 + w0 * f0;
    num = num + w1 * f1;
    num = num + w2 * f2;
    num = num + w3 * f3;
    double den = 0.0 + w0;
    den = den + w1;
    den = den + w2;
    den = den + w3;
    const double avg = den > 0.0 ? num / den : 0.0;
    return avg * a.MU(0, 0);
}

// u averaged onto v points over wet u faces (operators_masked.py:55-61)
template <class A>
__device__ __forceinline__ double u_on_v_at(const A& a) {
    const double f0 = a.U(0, 0), f1 = a.U(0, -1), f2 = a.U(1, 0), f3 = a.U(1, -1);
    const double w0 = a.MU(0, 0), w1 = a.MU(0, -1), w2 = a.MU(1, 0), w3 = a.MU(1, -1);
    double num = 0.0 + w0 * f0;
    num = num + w1 * f1;
    num = num + w2 * f2;
    num = num + w3 * f3;
    double den = 0.0 + w0;
    den = den + w1;
    den = den + w2;
    den = den + w3;
    const double avg = den > 0.0 ? num / den : 0.0;
    return avg * a.MV(0, 0);
}

__device__ __forceinline__ double v_on_u(const KP& P, const Nbr& nb, const double* __restrict__ v, size_t o,
                                         int k) {
    return v_on_u_at(GlobalLevel{P, nb, nullptr, v, o, k});
}

__device__ __forceinline__ double u_on_v(const KP& P, const Nbr& nb, const double* __restrict__ u, size_t o,
                                         int k) {
    return u_on_v_at(GlobalLevel{P, nb, u, nullptr, o, k});
}

// horizontal Laplacian D o G with the given face masks (operators_masked.py:64-68);
// which = 0: u (x-mask m3u, y-mask m3v, cell mask m3u), 1: v (cell mask m3v),
// 2: tracer (cell mask m3)
__device__ double hlap(const KP& P, const Nbr& nb, const double* __restrict__ f, int k, int which) {
    const size_t o = (size_t)k * P.n2;
    auto F = [&](int dj, int di) { return f[o + nb.at(dj, di)]; };
    const double gx0 = m3u_at(P, nb, 0, 0, k) * (F(0, 1) - F(0, 0)) / P.dx;
    const double gxw = m3u_at(P, nb, 0, -1, k) * (F(0, 0) - F(0, -1)) / P.dx;
    const double gy0 = m3v_at(P, nb, 0, 0, k) * (F(1, 0) - F(0, 0)) / P.dy;
    const double gys = m3v_at(P, nb, -1, 0, k) * (F(0, 0) - F(-1, 0)) / P.dy;
    const double m = which == 0 ? m3u_at(P, nb, 0, 0, k)
                                : (which == 1 ? m3v_at(P, nb, 0, 0, k) : m3_at(P, nb, 0, 0, k));
    return m * ((gx0 - gxw) / P.dx + (gy0 - gys) / P.dy);
}

// explicit vertical diffusion of a face velocity (vertical_var.py:80-106) with
// the column's interface viscosity, the face thickness table dzf[k-1..k+1], the
// cell mask's bottom rule and surface flux `surf`
__device__ __forceinline__ double explicit_dz(const KP& P, int k, double fkm1, double fk, double fkp1,
                                              double Kk, double Kk1, double dzf_m1, double dzf_k,
                                              double dzf_p1, double m3k_m1_bottom,
                                              double m3k_bottom, double m3k, double surf,
                                              double drag) {
    const int nz = P.nz;
    double flux_k, flux_k1;
    if (k == 0) {
        flux_k = surf;
    } else {
        const double dzi = 0.5 * (dzf_m1 + dzf_k);
        flux_k = Kk * (fkm1 - fk) * inv_pos(dzi);
        if (m3k_m1_bottom > 0.0) flux_k = 0.0;
    }
    if (k == nz - 1) {
        flux_k1 = 0.0;
    } else {
        const double dzi = 0.5 * (dzf_k + dzf_p1);
        flux_k1 = Kk1 * (fk - fkp1) * inv_pos(dzi);
        if (m3k_bottom > 0.0) flux_k1 = 0.0;
    }
    const double idz = inv_pos(dzf_k);
    const double out = (flux_k - flux_k1) * idz;
    const double dragc = drag * fk * m3k_bottom;
    return (out - dragc * idz) * (m3k > 0.0 ? 1.0 : 0.0);
}

// ------------------------------------------------------------------ momentum advection
// x- and y-flux divergence of u at its east face (advection_v06.py:77-99 for the
// kappa/TVD scheme, advection.py:62-79 for the centred one); the reference forms
// ax + ay + az left to right, so (ax + ay) + az is its sum
template <class A>
__device__ __forceinline__ double mom_adv_u_xy(const KP& P, const A& a) {
    if (P.advection >= 3) {
        const bool lim = P.advection == 4;
        const double ub_c0 = 0.5 * (a.U(0, -1) + a.U(0, 0));
        const double ub_c1 = 0.5 * (a.U(0, 0) + a.U(0, 1));
        const double uc0 = kappa_face(P, a.U(0, -2), a.U(0, -1), a.U(0, 0), a.U(0, 1), ub_c0, a.MU(0, -2),
                                      a.MU(0, 1), lim);
        const double uc1 = kappa_face(P, a.U(0, -1), a.U(0, 0), a.U(0, 1), a.U(0, 2), ub_c1, a.MU(0, -1),
                                      a.MU(0, 2), lim);
        const double ax = (ub_c1 * uc1 - ub_c0 * uc0) / P.dx;
        const double vb0 = 0.5 * (a.V(0, 0) + a.V(0, 1));
        const double vbm = 0.5 * (a.V(-1, 0) + a.V(-1, 1));
        const double fy0 = vb0 * kappa_face(P, a.U(-1, 0), a.U(0, 0), a.U(1, 0), a.U(2, 0), vb0, a.MU(-1, 0),
                                            a.MU(2, 0), lim);
        const double fym = vbm * kappa_face(P, a.U(-2, 0), a.U(-1, 0), a.U(0, 0), a.U(1, 0), vbm, a.MU(-2, 0),
                                            a.MU(1, 0), lim);
        return ax + (fy0 - fym) / P.dy;
    }
    const double ub_c0 = 0.5 * (a.U(0, -1) + a.U(0, 0));
    const double ub_c1 = 0.5 * (a.U(0, 0) + a.U(0, 1));
    const double ax = (ub_c1 * ub_c1 - ub_c0 * ub_c0) / P.dx;
    const double vb0 = 0.5 * (a.V(0, 0) + a.V(0, 1));
    const double vbm = 0.5 * (a.V(-1, 0) + a.V(-1, 1));
    const double fy0 = vb0 * (0.5 * (a.U(0, 0) + a.U(1, 0)));
    const double fym = vbm * (0.5 * (a.U(-1, 0) + a.U(0, 0)));
    return ax + (fy0 - fym) / P.dy;
}

// the same for v at its north face (advection_v06.py:100-108, advection.py:81-95):
// bx + by, formed in that order
template <class A>
__device__ __forceinline__ double mom_adv_v_xy(const KP& P, const A& a) {
    if (P.advection >= 3) {
        const bool lim = P.advection == 4;
        const double vb_c0 = 0.5 * (a.V(-1, 0) + a.V(0, 0));
        const double vb_c1 = 0.5 * (a.V(0, 0) + a.V(1, 0));
        const double vc0 = kappa_face(P, a.V(-2, 0), a.V(-1, 0), a.V(0, 0), a.V(1, 0), vb_c0, a.MV(-2, 0),
                                      a.MV(1, 0), lim);
        const double vc1 = kappa_face(P, a.V(-1, 0), a.V(0, 0), a.V(1, 0), a.V(2, 0), vb_c1, a.MV(-1, 0),
                                      a.MV(2, 0), lim);
        const double by = (vb_c1 * vc1 - vb_c0 * vc0) / P.dy;
        const double ub0 = 0.5 * (a.U(0, 0) + a.U(1, 0));
        const double ubm = 0.5 * (a.U(0, -1) + a.U(1, -1));
        const double fx0 = ub0 * kappa_face(P, a.V(0, -1), a.V(0, 0), a.V(0, 1), a.V(0, 2), ub0, a.MV(0, -1),
                                            a.MV(0, 2), lim);
        const double fxm = ubm * kappa_face(P, a.V(0, -2), a.V(0, -1), a.V(0, 0), a.V(0, 1), ubm, a.MV(0, -2),
                                            a.MV(0, 1), lim);
        return (fx0 - fxm) / P.dx + by;
    }
    const double vb_c0 = 0.5 * (a.V(-1, 0) + a.V(0, 0));
    const double vb_c1 = 0.5 * (a.V(0, 0) + a.V(1, 0));
    const double by = (vb_c1 * vb_c1 - vb_c0 * vb_c0) / P.dy;
    const double ub0 = 0.5 * (a.U(0, 0) + a.U(1, 0));
    const double ubm = 0.5 * (a.U(0, -1) + a.U(1, -1));
    const double fx0 = ub0 * (0.5 * (a.V(0, 0) + a.V(0, 1)));
    const double fxm = ubm * (0.5 * (a.V(0, -1) + a.V(0, 0)));
    return (fx0 - fxm) / P.dx + by;
}

// advective flux of a face velocity through interface kk of its column (0 =
// surface), from the velocity at kk-2 .. kk+1, the interface w averaged over
// the two cells of the face, and the face's wet levels kf
// (advection_v06.py:50-74 and :86-99; advection.py:75-79)
__device__ __forceinline__ double mom_vflux(const KP& P, int kk, int kf, double f_m2, double f_m1, double f_0,
                                            double f_p1, double wa, double wb_) {
    const int nz = P.nz;
    if (kk == 0 || kk == nz) return 0.0;
    const double wb = 0.5 * (wa + wb_);
    if (P.advection >= 3) {
        const double fu = (kk >= 2) ? f_m2 : 0.0;
        const double fd = (kk + 1 <= nz - 1) ? f_p1 : 0.0;
        const bool hu = (kk >= 2) && kk - 2 < kf;
        const bool hd = (kk + 1 <= nz - 1) && kk + 1 < kf;
        return wb * kappa_face_z(P, fu, f_m1, f_0, fd, wb, hu, hd, P.advection == 4);
    }
    return wb * 0.5 * (f_m1 + f_0);
}

// the diffusive flux K (f_above - f_below) / dzi through interface k of a face
// velocity column (vertical_var.py:80-106), zero when the level above is the
// column's last wet one
__device__ __forceinline__ double diff_flux(double Kk, double f_above, double f_below, double dzf_above,
                                           double dzf_below, double bottom_above) {
    const double dzi = 0.5 * (dzf_above + dzf_below);
    const double flux = Kk * (f_above - f_below) * inv_pos(dzi);
    return bottom_above > 0.0 ? 0.0 : flux;
}

// ------------------------------------------------------------------ explicit momentum terms
// Everything of the predictor that depends on the old state only: the
// common-depth pressure gradient, the old-state Coriolis average, the explicit
// vertical diffusion and the stress + advection/viscosity increment
// (model3d_v05.py:352-370), in level-marching form: two threads per column of
// a 32 x 8 tile, one for the u terms and one for the v terms, march P.mom_kl
// levels over the level planes the CTA stages in shared memory. The compact
// geometry of the column and of its face's far neighbour is formed once; the
// component's velocity and face thickness at the levels above and below roll
// in registers; the vertical advective flux at the bottom of a level and the
// diffusive flux there are carried to the next level as the fluxes at its top
// (a per-cell form forms each of them twice). Every value is formed by the
// reference's operations in its order.
constexpr int MOM_TX = 32, MOM_TY = 8, MOM_RX = MOM_TX + 4, MOM_RY = MOM_TY + 4, MOM_RN = MOM_RX * MOM_RY;

// the level's u, v and face masks of a tile plus a 2-column ring, in shared memory
struct TileLevel {
    const double* su;
    const double* sv;
    const int* sku;
    const int* skv;
    int rc;  // the thread's column in the region
    int k;
    __device__ __forceinline__ double U(int dj, int di) const { return su[rc + dj * MOM_RX + di]; }
    __device__ __forceinline__ double V(int dj, int di) const { return sv[rc + dj * MOM_RX + di]; }
    __device__ __forceinline__ double MU(int dj, int di) const { return k < sku[rc + dj * MOM_RX + di] ? 1.0 : 0.0; }
    __device__ __forceinline__ double MV(int dj, int di) const { return k < skv[rc + dj * MOM_RX + di] ? 1.0 : 0.0; }
};

__global__ void __launch_bounds__(MOM_TX * MOM_TY * 2, 2) k_mom_column(
    KP P, const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ b,
    const double* __restrict__ phi, const double* __restrict__ w, const double* __restrict__ km,
    double* __restrict__ pgx, double* __restrict__ pgy, double* __restrict__ avpv,
    double* __restrict__ avpu, double* __restrict__ dzu, double* __restrict__ dzv,
    double* __restrict__ stu, double* __restrict__ stv) {
    __shared__ int s_g[MOM_RN], s_ku[MOM_RN], s_kv[MOM_RN];
    __shared__ double s_u[MOM_RN], s_v[MOM_RN];
    // threadIdx.z selects the component: 0 the u terms at the column's east face,
    // 1 the v terms at its north face (whole warps, so no divergence)
    const int tx = threadIdx.x, ty = threadIdx.y, comp = threadIdx.z;
    const int tid = (comp * MOM_TY + ty) * MOM_TX + tx;
    const int nthreads = MOM_TX * MOM_TY * 2;
    const int i0 = blockIdx.x * MOM_TX, j0 = blockIdx.y * MOM_TY;
    const int i = i0 + tx, j = j0 + ty;
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const bool live = i < nx && j < ny;
    const int kbeg = blockIdx.z * P.mom_kl;
    const int kend = kbeg + P.mom_kl < nz ? kbeg + P.mom_kl : nz;
    for (int r = tid; r < MOM_RN; r += nthreads) {
        const int rj = r / MOM_RX, ri = r - rj * MOM_RX;
        const int gcol = wrapi(j0 - 2 + rj, ny) * nx + wrapi(i0 - 2 + ri, nx);
        const int2 kfc = P.kface[gcol];
        s_g[r] = gcol;
        s_ku[r] = kfc.x;
        s_kv[r] = kfc.y;
    }
    const int rc = (ty + 2) * MOM_RX + tx + 2;
    const size_t n2 = (size_t)P.n2;
    const int wi = wrapi(i, nx), wj = wrapi(j, ny);
    const int c = wj * nx + wi;
    // the face's far column (east for u, north for v) and its wet levels
    const int cf = comp ? wrapi(j + 1, ny) * nx + wi : wj * nx + wrapi(i + 1, nx);
    const ColGeo gc = ColGeo::load(P, c), gf = ColGeo::load(P, cf);
    const int kff = comp ? P.kface[c].y : P.kface[c].x;
    const double tau = comp ? P.tau_v[c] : P.tau_u[c];
    const double* __restrict__ X = comp ? v : u;
    // face thickness of the column's face at level kk (0 outside)
    auto dzf_at = [&](int kk) {
        if (kk < 0 || kk >= nz) return 0.0;
        double m;
        return face_dz(P, kff, kk, gc.dz(P, kk, m), gf.dz(P, kk, m));
    };
    auto m3c_at = [&](int kk) { return (kk >= 0 && kk < gc.kb) ? 1.0 : 0.0; };
    auto Xc = [&](int kk) { return (kk >= 0 && kk < nz) ? X[(size_t)kk * n2 + c] : 0.0; };
    // rolling values of the component at k-1, k, k+1 (and k+2 for advection)
    double x_m1 = 0.0, x_0 = 0.0, x_p1 = 0.0, dz_0 = 0.0;
    // fluxes through the top of level kbeg
    double fz = 0.0, df = 0.0;
    if (live) {
        x_m1 = Xc(kbeg - 1);
        x_0 = Xc(kbeg);
        x_p1 = Xc(kbeg + 1);
        const double dz_m1 = dzf_at(kbeg - 1);
        dz_0 = dzf_at(kbeg);
        const int kk = kbeg;
        if (P.advection != 0)
            fz = mom_vflux(P, kk, kff, Xc(kk - 2), x_m1, x_0, x_p1, w[(size_t)kk * n2 + c], w[(size_t)kk * n2 + cf]);
        if (kk == 0) {
            df = tau;
        } else {
            const double bot = (m3c_at(kk - 1) > 0.0 && m3c_at(kk) == 0.0) ? 1.0 : 0.0;
            df = diff_flux(km[(size_t)kbeg * n2 + c], x_m1, x_0, dz_m1, dz_0, bot);
        }
    }
    for (int k = kbeg; k < kend; ++k) {
        const size_t o = (size_t)k * n2;
        // stage the level's u and v of the region (the previous level is done)
        __syncthreads();
        for (int r = tid; r < MOM_RN; r += nthreads) {
            s_u[r] = u[o + s_g[r]];
            s_v[r] = v[o + s_g[r]];
        }
        __syncthreads();
        if (!live) continue;
        const TileLevel lv{s_u, s_v, s_ku, s_kv, rc, k};
        const double x_p2 = Xc(k + 2);
        const double dz_p1 = dzf_at(k + 1);
        const double K_1 = km[o + n2 + c];
        double m3c, m3f;
        const double dz_c = gc.dz(P, k, m3c), dz_f = gf.dz(P, k, m3f);
        const double m3f_k = k < kff ? 1.0 : 0.0;
        const double bottom_k = (m3c > 0.0 && m3c_at(k + 1) == 0.0) ? 1.0 : 0.0;
        // ---- pressure gradient at a common depth (model3d_v05.py:211-230)
        const double phc = phi[o + c], phf = phi[o + cf];
        const double bc = b[o + c], bf = b[o + cf];
        const double dxy = comp ? P.dy : P.dx;
        double pg;
        if (P.pgf_correction) {
            const double zc_c = gc.above(P, k) + 0.5 * dz_c;
            const double zc_f = gf.above(P, k) + 0.5 * dz_f;
            const double zf = 0.5 * (zc_c + zc_f);
            pg = m3f_k * ((phf + bf * (zf - zc_f)) - (phc + bc * (zf - zc_c))) / dxy;
        } else {
            pg = m3f_k * (phf - phc) / dxy * m3f_k;
        }
        (comp ? pgy : pgx)[o + c] = pg;
        // ---- Coriolis average of the old state (v at u points, u at v points)
        if (comp)
            avpu[o + c] = u_on_v_at(lv);
        else
            avpv[o + c] = v_on_u_at(lv);
        // ---- explicit vertical diffusion: top flux carried, bottom flux formed here
        const double db = (k < nz - 1) ? diff_flux(K_1, x_0, x_p1, dz_0, dz_p1, bottom_k) : 0.0;
        {
            const double mk = m3c > 0.0 ? 1.0 : 0.0;
            const double id = inv_pos(dz_0);
            const double out = (df - db) * id;
            const double drag = P.bottom_drag * x_0 * bottom_k;
            (comp ? dzv : dzu)[o + c] = (out - drag * id) * mk;
        }
        // ---- advection and horizontal viscosity, then the stress increment
        double ex = 0.0, fb = 0.0;
        if (P.advection != 0) {
            fb = mom_vflux(P, k + 1, kff, x_m1, x_0, x_p1, x_p2, w[o + n2 + c], w[o + n2 + cf]);
            const double a = (comp ? mom_adv_v_xy(P, lv) : mom_adv_u_xy(P, lv)) + (fz - fb) / P.dz_nom[k];
            ex = ex - a * m3f_k;
        }
        if (P.a_h > 0.0) {
            Nbr nb;
            nb.init(wi, wj, nx, ny);
            ex = ex + P.a_h * hlap(P, nb, X, k, comp);
        }
        (comp ? stv : stu)[o + c] = (k == 0) ? P.thv_dt * tau * inv_pos(dz_0) + P.dt * ex : 0.0 + P.dt * ex;
        // roll down one level
        fz = fb;
        df = db;
        x_m1 = x_0;
        x_0 = x_p1;
        x_p1 = x_p2;
        dz_0 = dz_p1;
    }
}

// ------------------------------------------------------------------ predictor + column solves
// Per cell, for one Picard iteration: the explicit predictors with the iterate's
// Coriolis average plus the stress/advection increment -- the right-hand sides
// of the two momentum tridiagonals (model3d_v05.py:387-393).
__global__ void __launch_bounds__(256) k_predictor_rhs(
    KP P, const double* __restrict__ u, const double* __restrict__ v,
    const double* __restrict__ u_it, const double* __restrict__ v_it,
    const double* __restrict__ pgx, const double* __restrict__ pgy,
    const double* __restrict__ avpv, const double* __restrict__ avpu,
    const double* __restrict__ dzu, const double* __restrict__ dzv,
    const double* __restrict__ stu, const double* __restrict__ stv,
    const double* __restrict__ gx2, const double* __restrict__ gy2, double* __restrict__ ru,
    double* __restrict__ rv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= P.nx || j >= P.ny) return;
    const int c = j * P.nx + i;
    const size_t o = (size_t)k * P.n2;
    const double av_v = avpv[o + c], av_u = avpu[o + c];
    // the iterate's averages; in the first pass the iterate is the old state,
    // whose averages the explicit-terms kernel formed already by the same function
    double it_v = av_v, it_u = av_u;
    if (u_it != u || v_it != v) {
        Nbr nb;
        nb.init(i, j, P.nx, P.ny);
        it_v = v_on_u(P, nb, v_it, o, k);
        it_u = u_on_v(P, nb, u_it, o, k);
    }
    const double vcor = P.one_m_tc * av_v + P.theta_cor * it_v;
    const double ucor = P.one_m_tc * av_u + P.theta_cor * it_u;
    double gu, gv;
    if (P.scheme != 2) {
        const double m3u_k = col_m3u(P, c, k), m3v_k = col_m3v(P, c, k);
        gu = u[o + c] + P.dt * (P.f0 * vcor + pgx[o + c]) - P.c1 * (gx2[c] * m3u_k) + P.c3 * dzu[o + c];
        gv = v[o + c] + P.dt * (P.neg_f0 * ucor + pgy[o + c]) - P.c1 * (gy2[c] * m3v_k) + P.c3 * dzv[o + c];
    } else {
        gu = u[o + c] + P.dt * (P.f0 * vcor + pgx[o + c]) + P.c3 * dzu[o + c];
        gv = v[o + c] + P.dt * (P.neg_f0 * ucor + pgy[o + c]) + P.c3 * dzv[o + c];
    }
    ru[o + c] = gu + stu[o + c];
    rv[o + c] = gv + stv[o + c];
}

// Per column: both momentum tridiagonals with the cell column's rows
// (vertical.py:17-44 on vertical_var.py:35-77 coefficients), the cell-mask
// multiply and the depth-integrated transports (model3d_v05.py:426-433). The
// right-hand sides arrive in gh_u/gh_v; the forward elimination overwrites them
// with its intermediate values, the back substitution with the solution, and
// the transports are summed in a last, downward pass to keep the reference's
// order. Only the elimination coefficients stay in the thread.
template <int NZM>
__global__ void __launch_bounds__(128) k_momentum_solve(KP P, const double* __restrict__ km,
                                                        double* __restrict__ ghu,
                                                        double* __restrict__ ghv,
                                                        double* __restrict__ Ug,
                                                        double* __restrict__ Vg) {
    COLUMN_PROLOGUE
    const int nz = P.nz;
    const int c = nb.c;
    const ColGeo g = ColGeo::load(P, c);
    double cs[NZM];
    double m3_k, dz_k = g.dz(P, 0, m3_k);
    double dzi_k = dz_k;
    double km_k = km[c];
    double du = 0.0, dv = 0.0, cp = 0.0;
#pragma unroll 4
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        const double km_k1 = km[o + n2];
        const double ru = ghu[o], rv = ghv[o];
        double m3_k1 = 0.0, dz_k1 = 0.0;
        if (k + 1 < nz) dz_k1 = g.dz(P, k + 1, m3_k1);
        const double dzi_k1 = (k + 1 < nz) ? 0.5 * (dz_k + dz_k1) : dz_k;
        double sub, diag, sup;
        implicit_row(P, k, dz_k, m3_k, m3_k1, dzi_k, dzi_k1, km_k, km_k1, P.thv_dt_drag, sub, diag, sup);
        if (k == 0) {
            cp = sup / diag;
            du = ru / diag;
            dv = rv / diag;
        } else {
            const double den = diag - sub * cp;
            cp = sup / den;
            du = (ru - sub * du) / den;
            dv = (rv - sub * dv) / den;
        }
        cs[k] = cp;
        ghu[o] = du;
        ghv[o] = dv;
        km_k = km_k1;
        dz_k = dz_k1;
        m3_k = m3_k1;
        dzi_k = dzi_k1;
    }
    double xu = du, xv = dv;
    {
        const size_t o = (size_t)(nz - 1) * n2 + c;
        const double m = (nz - 1 < g.kb) ? 1.0 : 0.0;
        ghu[o] = xu * m;
        ghv[o] = xv * m;
    }
#pragma unroll 4
    for (int k = nz - 2; k >= 0; --k) {
        const size_t o = (size_t)k * n2 + c;
        const double m = (k < g.kb) ? 1.0 : 0.0;
        xu = ghu[o] - cs[k] * xu;
        xv = ghv[o] - cs[k] * xv;
        ghu[o] = xu * m;
        ghv[o] = xv * m;
    }
    const ColGeo ge = ColGeo::load(P, nb.at(0, 1)), gn = ColGeo::load(P, nb.at(1, 0));
    const int2 kfc = P.kface[c];
    double su = 0.0, sv = 0.0;
#pragma unroll 4
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        double m3c, m3e, m3n;
        const double dzc = g.dz(P, k, m3c);
        const double dze = ge.dz(P, k, m3e);
        const double dzn = gn.dz(P, k, m3n);
        const double tu = (k < kfc.x ? 1.0 : 0.0) * face_combine(P, dzc, dze) * ghu[o];
        const double tv = (k < kfc.y ? 1.0 : 0.0) * face_combine(P, dzc, dzn) * ghv[o];
        su = (k == 0) ? tu : su + tu;
        sv = (k == 0) ? tv : sv + tv;
    }
    Ug[c] = su;
    Vg[c] = sv;
}

// ------------------------------------------------------------------ back substitution
// u = (gh_u - g dt theta q dx(eta_new) m3u) m3   (model3d_v05.py:404-406)
__global__ void k_backsub(KP P, const double* __restrict__ ghu, const double* __restrict__ ghv,
                          const double* __restrict__ q, const double* __restrict__ eta_new,
                          double* __restrict__ u_out, double* __restrict__ v_out) {
    COLUMN_PROLOGUE
    const size_t c = nb.c, ce = nb.at(0, 1), cn = nb.at(1, 0);
    const double gx = P.mask_u[c] * (eta_new[ce] - eta_new[c]) / P.dx;
    const double gy = P.mask_v[c] * (eta_new[cn] - eta_new[c]) / P.dy;
    const int kb = P.kinfo[c].y;
    const int2 kf = P.kface[c];
#pragma unroll 4
    for (int k = 0; k < P.nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        const double m3 = k < kb ? 1.0 : 0.0;
        const double m3u_k = k < kf.x ? 1.0 : 0.0;
        const double m3v_k = k < kf.y ? 1.0 : 0.0;
        const double qk = q[o];
        u_out[o] = (ghu[o] - P.c2 * qk * gx * m3u_k) * m3;
        v_out[o] = (ghv[o] - P.c2 * qk * gy * m3v_k) * m3;
    }
}

// ------------------------------------------------------------------ tracers + EOS
// Tiled right-hand sides of the implicit tracer solves (model3d_v05.py:466-512).
// A CTA owns a TRX x TRY tile of columns and P.tr_kl levels and marches down the
// levels. At each level the horizontal face fluxes of the tile -- TRX + 1 east
// faces per row, TRY + 1 north faces per column -- are formed once into shared
// memory (double-buffered, one barrier per level); a per-cell form would form
// every face twice, once from each side. The vertical face at the bottom of a
// cell is carried to the next level as the face at its top, and the column's
// tracer values, w and K_h roll in registers. Every face and cell value is
// formed by the reference's operations in the reference's order.
constexpr int TRX = 32, TRY = 8;

struct Stencil4 {
    int cm, c0, c1, cp;  // far upstream, the two cells of the face, far downstream (flat 2D)
};

// the east face of column i in row j (cells i-1, i, i+1, i+2), periodic index layout
__device__ __forceinline__ Stencil4 xstencil(int j, int i, int nx, int ny) {
    const int r = wrapi(j, ny) * nx;
    return Stencil4{r + wrapi(i - 1, nx), r + wrapi(i, nx), r + wrapi(i + 1, nx), r + wrapi(i + 2, nx)};
}

// the north face of row j in column i (rows j-1, j, j+1, j+2)
__device__ __forceinline__ Stencil4 ystencil(int j, int i, int nx, int ny) {
    const int ii = wrapi(i, nx);
    return Stencil4{wrapi(j - 1, ny) * nx + ii, wrapi(j, ny) * nx + ii, wrapi(j + 1, ny) * nx + ii,
                    wrapi(j + 2, ny) * nx + ii};
}

// tracer value on a horizontal face: centred, kappa/TVD with the dry far-cell
// fallback, or first-order upwind (model3d_v05.py:482-497)
__device__ __forceinline__ double tracer_face(const KP& P, const double* __restrict__ C, size_t o,
                                              const Stencil4& s, double vel, int k) {
    const double a = C[o + s.c0], b = C[o + s.c1];
    if (P.advection == 1) return 0.5 * (a + b);
    if (P.advection >= 3)
        return kappa_face(P, C[o + s.cm], a, b, C[o + s.cp], vel, col_m3(P, s.cm, k), col_m3(P, s.cp, k),
                          P.advection == 4);
    return vel > 0.0 ? a : b;
}

// flux through an east (ax = 0) or north (ax = 1) face: face thickness x
// normal velocity x face value (model3d_v05.py:498-501)
__device__ __forceinline__ double tracer_flux(const KP& P, const double* __restrict__ C,
                                              const double* __restrict__ vel_f, size_t o,
                                              const Stencil4& s, int k, int ax) {
    const double vel = vel_f[o + s.c0];
    const int2 kf = P.kface[s.c0];
    double m;
    const double dzf = face_dz(P, ax == 0 ? kf.x : kf.y, k, col_dz(P, s.c0, k, m), col_dz(P, s.c1, k, m));
    return dzf * vel * tracer_face(P, C, o, s, vel, k);
}

// tracer value on interface kk of a column (0 = surface) from the column values
// at kk-2, kk-1, kk, kk+1 and w there (model3d_v05.py:502-510)
__device__ __forceinline__ double tracer_vface(const KP& P, const ColGeo& g, int kk, double f_m2, double f_m1,
                                               double f_0, double f_p1, double wv) {
    const int nz = P.nz;
    if (kk == 0) return f_0;
    if (kk == nz) return 0.0;
    if (P.advection >= 3) {
        const double fu = (kk >= 2) ? f_m2 : 0.0;
        const double fd = (kk + 1 <= nz - 1) ? f_p1 : 0.0;
        const bool hu = (kk >= 2) && kk - 2 < g.kb;
        const bool hd = (kk + 1 <= nz - 1) && kk + 1 < g.kb;
        return kappa_face_z(P, fu, f_m1, f_0, fd, wv, hu, hd, P.advection == 4);
    }
    return 0.5 * (f_m1 + f_0);
}

__global__ void __launch_bounds__(TRX * TRY, 4) k_tracer_rhs(KP P, const double* __restrict__ T,
                                                             const double* __restrict__ S,
                                                             const double* __restrict__ bold,
                                                             const double* __restrict__ u,
                                                             const double* __restrict__ v,
                                                             const double* __restrict__ w,
                                                             const double* __restrict__ kh,
                                                             double* __restrict__ rT,
                                                             double* __restrict__ rS) {
    // the tile's columns plus a 2-column ring: flat 2D index and compact geometry
    // (once), then each level's tracers and face velocities (staged per level)
    constexpr int RX = TRX + 4, RY = TRY + 4, RNC = RX * RY;
    __shared__ int s_g[RNC], s_kf[RNC], s_kb[RNC], s_ku[RNC], s_kv[RNC];
    __shared__ double s_d0[RNC], s_d1[RNC];
    __shared__ double s_f[2][RNC], s_u[RNC], s_v[RNC];
    __shared__ double sfx[2][TRY][TRX + 1];  // [field][row][west face of column]
    __shared__ double sfy[2][TRY + 1][TRX];  // [field][south face of row][column]
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * TRX + tx;
    const int i0 = blockIdx.x * TRX, j0 = blockIdx.y * TRY;
    const int i = i0 + tx, j = j0 + ty;
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const size_t n2 = P.n2;
    const bool live = i < nx && j < ny;
    const bool ts = P.tracers_ts;
    const int nf = ts ? 2 : 1;
    const bool adv = P.advection != 0;
    const int kbeg = blockIdx.z * P.tr_kl;
    const int kend = kbeg + P.tr_kl < nz ? kbeg + P.tr_kl : nz;
    // faces this thread forms: the west and south faces of its cell, and for two
    // warps the east faces of the tile's last column / north faces of its last row
    const bool xextra = ty == TRY - 2 && tx < TRY, yextra = ty == TRY - 1;
    const int c = wrapi(j, ny) * nx + wrapi(i, nx);
    const ColGeo g = ColGeo::load(P, c);
    const double* __restrict__ C0 = ts ? T : bold;
    double* __restrict__ R0 = rT;
    for (int r = tid; r < RNC; r += TRX * TRY) {
        const int rj = r / RX, ri = r - rj * RX;
        const int gc = wrapi(j0 - 2 + rj, ny) * nx + wrapi(i0 - 2 + ri, nx);
        const int2 ki = P.kinfo[gc], kfc = P.kface[gc];
        const double2 dx = P.dzx[gc];
        s_g[r] = gc;
        s_kf[r] = ki.x;
        s_kb[r] = ki.y;
        s_ku[r] = kfc.x;
        s_kv[r] = kfc.y;
        s_d0[r] = dx.x;
        s_d1[r] = dx.y;
    }
    // thickness and wet flag of region column r at level k (col_dz from the staged geometry)
    auto sdz = [&](int r, int k, double& m3) {
        if (k >= s_kb[r]) {
            m3 = 0.0;
            return 0.0;
        }
        m3 = 1.0;
        if (k < s_kf[r]) return P.dzr[k];
        return k == s_kf[r] ? s_d0[r] : s_d1[r];
    };
    // flux through a face with stencil cells (cm, c0, c1, cp) of the region,
    // normal velocity vel and face wet levels kfa (tracer_flux from shared memory)
    auto sflux = [&](const double* F, int cm, int c0, int c1, int cp, double vel, int kfa, int k) {
        double m;
        const double dzf = face_dz(P, kfa, k, sdz(c0, k, m), sdz(c1, k, m));
        const double a = F[c0], b = F[c1];
        double val;
        if (P.advection == 1)
            val = 0.5 * (a + b);
        else if (P.advection >= 3)
            val = kappa_face(P, F[cm], a, b, F[cp], vel, k < s_kb[cm] ? 1.0 : 0.0, k < s_kb[cp] ? 1.0 : 0.0,
                             P.advection == 4);
        else
            val = vel > 0.0 ? a : b;
        return dzf * vel * val;
    };
    const int rc = (ty + 2) * RX + tx + 2;                    // this thread's cell in the region
    const int rce = (tx + 2) * RX + TRX + 1;                  // east-column cell of row tx (x extras)
    const int rcn = (TRY + 1) * RX + tx + 2;                  // north-row cell of column tx (y extras)
    // rolling column values of each field at k-1, k, k+1 and the face at the top of level k
    double fm1[2] = {0.0, 0.0}, f0[2] = {0.0, 0.0}, fp1[2] = {0.0, 0.0}, ftop[2] = {0.0, 0.0};
    double w_k = 0.0, kh_k = 0.0;
    if (live) {
#pragma unroll
        for (int f = 0; f < 2; ++f) {
            if (f >= nf) break;
            const double* __restrict__ C = f == 0 ? C0 : S;
            const double fm2 = kbeg >= 2 ? C[(size_t)(kbeg - 2) * n2 + c] : 0.0;
            fm1[f] = kbeg >= 1 ? C[(size_t)(kbeg - 1) * n2 + c] : 0.0;
            f0[f] = C[(size_t)kbeg * n2 + c];
            fp1[f] = kbeg + 1 < nz ? C[(size_t)(kbeg + 1) * n2 + c] : 0.0;
            if (adv) ftop[f] = tracer_vface(P, g, kbeg, fm2, fm1[f], f0[f], fp1[f], w[(size_t)kbeg * n2 + c]);
        }
        w_k = w[(size_t)kbeg * n2 + c];
        kh_k = kh[(size_t)kbeg * n2 + c];
    }
    for (int k = kbeg; k < kend; ++k) {
        const size_t o = (size_t)k * n2;
        if (adv) {
            // stage the level (the previous level's faces and cells are done)
            __syncthreads();
            for (int r = tid; r < RNC; r += TRX * TRY) {
                const size_t g = o + s_g[r];
                s_f[0][r] = C0[g];
                if (ts) s_f[1][r] = S[g];
                s_u[r] = u[g];
                s_v[r] = v[g];
            }
            __syncthreads();
#pragma unroll 1
            for (int f = 0; f < nf; ++f) {
                const double* F = s_f[f];
                // west face of this cell (cells rc-2 .. rc+1), south face (rc-2RX .. rc+RX)
                sfx[f][ty][tx] = sflux(F, rc - 2, rc - 1, rc, rc + 1, s_u[rc - 1], s_ku[rc - 1], k);
                sfy[f][ty][tx] = sflux(F, rc - 2 * RX, rc - RX, rc, rc + RX, s_v[rc - RX], s_kv[rc - RX], k);
                if (xextra) sfx[f][tx][TRX] = sflux(F, rce - 1, rce, rce + 1, rce + 2, s_u[rce], s_ku[rce], k);
                if (yextra)
                    sfy[f][TRY][tx] = sflux(F, rcn - RX, rcn, rcn + RX, rcn + 2 * RX, s_v[rcn], s_kv[rcn], k);
            }
            __syncthreads();
        }
        if (!live) continue;
        double m3k, m3_m1 = 0.0, m3_p1 = 0.0;
        const double dzk = g.dz(P, k, m3k);
        const double dz_m1 = (k > 0) ? g.dz(P, k - 1, m3_m1) : 0.0;
        const double dz_p1 = (k + 1 < nz) ? g.dz(P, k + 1, m3_p1) : 0.0;
        const double bottom_m1 = (k > 0 && m3_m1 > 0.0 && m3k == 0.0) ? 1.0 : 0.0;
        const double bottom_k = (m3k > 0.0 && m3_p1 == 0.0) ? 1.0 : 0.0;
        const double w_k1 = w[o + n2 + c];
        const double kh_k1 = kh[o + n2 + c];
        const double inv = inv_pos(dzk);
#pragma unroll
        for (int f = 0; f < 2; ++f) {
            if (f >= nf) break;
            const double* __restrict__ C = f == 0 ? C0 : S;
            const double fp2 = (k + 2 < nz) ? C[o + 2 * n2 + c] : 0.0;
            const double surf = ts ? (f == 0 ? P.flux_t : P.flux_s) : 0.0;
            double tend = ts ? 0.0 : P.neg_n2 * (0.5 * (w_k + w_k1));
            double fbot = 0.0;
            if (adv) {
                fbot = tracer_vface(P, g, k + 1, fm1[f], f0[f], fp1[f], fp2, w_k1);
                const double hdiv = ((sfx[f][ty][tx + 1] - sfx[f][ty][tx]) / P.dx +
                                     (sfy[f][ty + 1][tx] - sfy[f][ty][tx]) / P.dy) *
                                    inv;
                const double vdiv = (w_k * ftop[f] - w_k1 * fbot) * inv;
                tend = tend - (hdiv + vdiv) * m3k;
            }
            if (P.k_h > 0.0) {
                Nbr nb;
                nb.init(wrapi(i, nx), wrapi(j, ny), nx, ny);
                tend = tend + P.k_h * hlap(P, nb, C, k, 2);
            }
            // explicit vertical diffusion with zero drag (vertical_var.py:80-106)
            const double diff = explicit_dz(P, k, k > 0 ? fm1[f] : 0.0, f0[f], k + 1 < nz ? fp1[f] : 0.0, kh_k,
                                            kh_k1, dz_m1, dzk, dz_p1, bottom_m1, bottom_k, m3k, surf, 0.0);
            double rhs = f0[f] + P.dt * tend + P.c3 * diff;
            if (k == 0) rhs = rhs + P.thv_dt * surf * inv_pos(dzk);
            (f == 0 ? R0 : rS)[o + c] = rhs;
            ftop[f] = fbot;
            fm1[f] = f0[f];
            f0[f] = fp1[f];
            fp1[f] = fp2;
        }
        w_k = w_k1;
        kh_k = kh_k1;
    }
}

// One thread per column: the implicit solves with the diffusivity rows
// (shared by T and S), the cell mask, and the EOS of the new T/S
// (model3d_v05.py:514-533). The forward elimination stores its right-hand sides
// in the outputs; the back substitution finishes each level there, EOS
// included, with the level-centre depth in closed form (col_above is the
// sequential sum of the thicknesses above, bit for bit).
template <int NZM>
__global__ void __launch_bounds__(128) k_tracer_solve(KP P, const double* __restrict__ rT,
                                                      const double* __restrict__ rS,
                                                      const double* __restrict__ kh,
                                                      double* __restrict__ T_out,
                                                      double* __restrict__ S_out,
                                                      double* __restrict__ b_out) {
    COLUMN_PROLOGUE
    const int nz = P.nz;
    const int c = nb.c;
    const ColGeo g = ColGeo::load(P, c);
    double cs[NZM];
    const bool ts = P.tracers_ts;
    double* __restrict__ o1 = ts ? T_out : b_out;
    double m3_k, dz_k = g.dz(P, 0, m3_k);
    double dzi_k = dz_k;
    double kh_k = kh[c];
    double d1 = 0.0, d2 = 0.0, cp = 0.0;
#pragma unroll 4
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        const double kh_k1 = kh[o + n2];
        double m3_k1 = 0.0, dz_k1 = 0.0;
        if (k + 1 < nz) dz_k1 = g.dz(P, k + 1, m3_k1);
        const double dzi_k1 = (k + 1 < nz) ? 0.5 * (dz_k + dz_k1) : dz_k;
        const double r1 = rT[o];
        const double r2 = ts ? rS[o] : 0.0;
        double sub, diag, sup;
        implicit_row(P, k, dz_k, m3_k, m3_k1, dzi_k, dzi_k1, kh_k, kh_k1, P.thv_dt_zero, sub, diag, sup);
        if (k == 0) {
            cp = sup / diag;
            d1 = r1 / diag;
            d2 = r2 / diag;
        } else {
            const double den = diag - sub * cp;
            cp = sup / den;
            d1 = (r1 - sub * d1) / den;
            d2 = (r2 - sub * d2) / den;
        }
        cs[k] = cp;
        if (k + 1 < nz) {
            o1[o] = d1;
            if (ts) S_out[o] = d2;
        }
        kh_k = kh_k1;
        dz_k = dz_k1;
        m3_k = m3_k1;
        dzi_k = dzi_k1;
    }
    double x1 = d1, x2 = d2;
#pragma unroll 4
    for (int k = nz - 1; k >= 0; --k) {
        const size_t o = (size_t)k * n2 + c;
        if (k < nz - 1) {
            x1 = o1[o] - cs[k] * x1;
            if (ts) x2 = S_out[o] - cs[k] * x2;
        }
        double m3;
        const double dz = g.dz(P, k, m3);
        if (ts) {
            const double Tn = x1 * m3;
            const double Sn = x2 * m3;
            const double zc = col_above(P, c, k) + 0.5 * dz;
            T_out[o] = Tn;
            S_out[o] = Sn;
            b_out[o] = buoyancy_of(P, Tn, Sn, zc) * m3;
        } else {
            b_out[o] = x1 * m3;
        }
    }
}


// ------------------------------------------------------------------ EOS on a flat buffer
__global__ void k_buoyancy(KP P, const double* __restrict__ T, const double* __restrict__ S,
                           const double* __restrict__ z, double* __restrict__ b, int64_t n) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) b[t] = buoyancy_of(P, T[t], S[t], z[t]);
}

// diagnose b = EOS(T, S, zc) * m3 on the model grid (initial states)
__global__ void k_diag_buoyancy(KP P, const double* __restrict__ T, const double* __restrict__ S,
                                double* __restrict__ b) {
    COLUMN_PROLOGUE
    const size_t c = nb.c;
    double above = 0.0;
    for (int k = 0; k < P.nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        double m3;
        const double dz = col_dz(P, (int)c, k, m3);
        const double zc = above + 0.5 * dz;
        above = (k == 0) ? dz : above + dz;
        b[o] = buoyancy_of(P, T[o], S[o], zc) * m3;
    }
}

// ------------------------------------------------------------------ 2D kernels
// depth-integrated transports sum_k dz3u u, sum_k dz3v v
__global__ void k_transport(KP P, const double* __restrict__ u, const double* __restrict__ v,
                            double* __restrict__ U, double* __restrict__ V) {
    COLUMN_PROLOGUE
    const size_t c = nb.c;
    const ColGeo gc = ColGeo::load(P, (int)c), ge = ColGeo::load(P, nb.at(0, 1)), gn = ColGeo::load(P, nb.at(1, 0));
    const int2 kf = P.kface[c];
    double su = 0.0, sv = 0.0;
#pragma unroll 4
    for (int k = 0; k < P.nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        double m;
        const double dzc = gc.dz(P, k, m);
        const double tu = face_dz(P, kf.x, k, dzc, ge.dz(P, k, m)) * u[o];
        const double tv = face_dz(P, kf.y, k, dzc, gn.dz(P, k, m)) * v[o];
        su = (k == 0) ? tu : su + tu;
        sv = (k == 0) ? tv : sv + tv;
    }
    U[c] = su;
    V[c] = sv;
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
#define NZ_DISPATCH(NZ, CALL)                \
    do {                                     \
        if ((NZ) + 1 <= 33) {                \
            constexpr int NZM = 33;          \
            CALL;                            \
        } else if ((NZ) + 1 <= 65) {         \
            constexpr int NZM = 65;          \
            CALL;                            \
        } else {                             \
            constexpr int NZM = OC_MAXNZ + 1; \
            CALL;                            \
        }                                    \
    } while (0)

static dim3 col_block() { return dim3(32, 4); }
static dim3 col_grid(const KP& P) { return dim3((P.nx + 31) / 32, (P.ny + 3) / 4); }

void launch_qsolve(const KP& P, const double* km, double* q, cudaStream_t s) {
    NZ_DISPATCH(P.nz, (k_qsolve<NZM><<<col_grid(P), col_block(), 0, s>>>(P, km, q)));
}

void launch_closure(const KP& P, const double* u, const double* v, const double* b, double* e,
                    double* km, double* kh, double* q, cudaStream_t s) {
    NZ_DISPATCH(P.nz, (k_closure<NZM><<<col_grid(P), col_block(), 0, s>>>(P, u, v, b, e, km, kh, q)));
}

void launch_kukv(const KP& P, const double* q, double* Ku, double* Kv, cudaStream_t s) {
    k_kukv<<<col_grid(P), col_block(), 0, s>>>(P, q, Ku, Kv);
}

void launch_wcol(const KP& P, const double* u, const double* v, double* w, cudaStream_t s) {
    k_wcol<<<col_grid(P), col_block(), 0, s>>>(P, u, v, w);
}

void launch_phi(const KP& P, const double* b, double* phi, cudaStream_t s) {
    k_phi<<<col_grid(P), col_block(), 0, s>>>(P, b, phi);
}

static dim3 cell_block() { return dim3(32, 8, 1); }
static dim3 cell_grid(const KP& P) { return dim3((P.nx + 31) / 32, (P.ny + 7) / 8, P.nz); }

void launch_mom_explicit(const KP& P, const double* u, const double* v, const double* b,
                         const double* phi, const double* w, const double* km, double* pgx,
                         double* pgy, double* avpv, double* avpu, double* dzu, double* dzv,
                         double* stu, double* stv, cudaStream_t s) {
    const dim3 grid((P.nx + MOM_TX - 1) / MOM_TX, (P.ny + MOM_TY - 1) / MOM_TY, (P.nz + P.mom_kl - 1) / P.mom_kl);
    k_mom_column<<<grid, dim3(MOM_TX, MOM_TY, 2), 0, s>>>(P, u, v, b, phi, w, km, pgx, pgy, avpv, avpu, dzu, dzv, stu,
                                             stv);
}

void launch_predictor_rhs(const KP& P, const double* u, const double* v, const double* u_it,
                          const double* v_it, const double* pgx, const double* pgy, const double* avpv,
                          const double* avpu, const double* dzu, const double* dzv, const double* stu,
                          const double* stv, const double* gx2, const double* gy2, double* ru, double* rv,
                          cudaStream_t s) {
    k_predictor_rhs<<<cell_grid(P), cell_block(), 0, s>>>(P, u, v, u_it, v_it, pgx, pgy, avpv, avpu, dzu,
                                                          dzv, stu, stv, gx2, gy2, ru, rv);
}

void launch_momentum_solve(const KP& P, const double* km, double* ghu, double* ghv, double* Ug, double* Vg,
                           cudaStream_t s) {
    NZ_DISPATCH(P.nz, (k_momentum_solve<NZM><<<col_grid(P), col_block(), 0, s>>>(P, km, ghu, ghv, Ug, Vg)));
}

void launch_backsub(const KP& P, const double* ghu, const double* ghv, const double* q,
                    const double* eta_new, double* u_out, double* v_out, cudaStream_t s) {
    k_backsub<<<col_grid(P), col_block(), 0, s>>>(P, ghu, ghv, q, eta_new, u_out, v_out);
}

void launch_tracer_rhs(const KP& P, const double* T, const double* S, const double* bold,
                       const double* u, const double* v, const double* w, const double* kh, double* rT,
                       double* rS, cudaStream_t s) {
    const dim3 grid((P.nx + TRX - 1) / TRX, (P.ny + TRY - 1) / TRY, (P.nz + P.tr_kl - 1) / P.tr_kl);
    k_tracer_rhs<<<grid, dim3(TRX, TRY), 0, s>>>(P, T, S, bold, u, v, w, kh, rT, rS);
}

void launch_tracer_solve(const KP& P, const double* rT, const double* rS, const double* kh,
                         double* T_out, double* S_out, double* b_out, cudaStream_t s) {
    NZ_DISPATCH(P.nz, (k_tracer_solve<NZM><<<col_grid(P), col_block(), 0, s>>>(P, rT, rS, kh, T_out,
                                                                             S_out, b_out)));
}

void launch_buoyancy_flat(const KP& P, const double* T, const double* S, const double* z, double* b,
                          int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    k_buoyancy<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P, T, S, z, b, n);
}

void launch_diag_buoyancy(const KP& P, const double* T, const double* S, double* b, cudaStream_t s) {
    k_diag_buoyancy<<<col_grid(P), col_block(), 0, s>>>(P, T, S, b);
}

void launch_transport(const KP& P, const double* u, const double* v, double* U, double* V,
                      cudaStream_t s) {
    k_transport<<<col_grid(P), col_block(), 0, s>>>(P, u, v, U, V);
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
