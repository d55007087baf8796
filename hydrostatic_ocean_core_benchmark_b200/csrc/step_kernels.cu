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

#include <atomic>

#include "oc_internal.cuh"
#include "step_common.cuh"
#include "step_kernels.cuh"

namespace oc {

// The floating type of the 3D fields: double for the fp64 path, float for the
// mixed-precision path (OC_MIXED builds this file a second time). The buoyancy
// b and the buoyancy potential phi stay fp64 on both paths (wide), and so do
// every 2D field and every depth-integrated sum.
#ifdef OC_MIXED
typedef float real;
#else
typedef double real;
#endif
typedef double wide;

// Minimum resident CTAs per SM the register allocation of the three largest
// stencil/column kernels is bounded for (__launch_bounds__): k_closure runs
// 128 threads, k_mom_column 512 and k_tracer_rhs 256 per CTA. The bits of the
// results do not depend on them.
#ifndef OC_MINB_CLOSURE
#ifdef OC_MIXED
#define OC_MINB_CLOSURE 4
#else
#define OC_MINB_CLOSURE 8
#endif
#endif
#ifndef OC_MINB_MOM
#define OC_MINB_MOM 2
#endif
#ifndef OC_MINB_TRACER
#ifdef OC_MIXED
#define OC_MINB_TRACER 6  // FP32: 0.56 against 0.59 ms per step at 512 x 512 x 50
#else
#define OC_MINB_TRACER 4
#endif
#endif
using KPR = KPT<real>;
using ColGeoR = ColGeoT<real>;

// ------------------------------------------------------------------ helpers



__device__ __forceinline__ real m3u_at(const KPR& P, const Nbr& n, int dj, int di, int k) {
    return col_m3u(P, n.at(dj, di), k);
}

__device__ __forceinline__ real m3v_at(const KPR& P, const Nbr& n, int dj, int di, int k) {
    return col_m3v(P, n.at(dj, di), k);
}

__device__ __forceinline__ real m3_at(const KPR& P, const Nbr& n, int dj, int di, int k) {
    return col_m3(P, n.at(dj, di), k);
}



// ------------------------------------------------------------------ q = A^-1 1 on a column
// interface spacing of the column (closure.py:43-62): dz[0] at the surface,
// dz[nz-1] at the bottom, the mean of the two levels elsewhere
__device__ __forceinline__ real col_dzi(const KPR& P, const ColGeoR& g, int k) {
    real m;
    if (k == 0) return g.dz(P, 0, m);
    if (k == P.nz) return g.dz(P, P.nz - 1, m);
    const real a = g.dz(P, k - 1, m);
    return real(0.5) * (a + g.dz(P, k, m));
}

// Momentum tridiagonal with a unit right-hand side for the column's interface
// viscosity Km(k), k = 0..nz (reference model3d_v05.py:147-153). The forward
// elimination keeps its coefficients in cs and its right-hand sides in q, which
// the back substitution then overwrites with the solution.
template <class KM>
__device__ __forceinline__ void column_q(const KPR& P, const ColGeoR& g, KM Km, real* cs,
                                         real* __restrict__ q, int c, size_t n2) {
    const int nz = P.nz;
    real m3_k, dz_k = g.dz(P, 0, m3_k);
    real dzi_k = dz_k;
    real km_k = Km(0);
    real ds = real(0.0), cp = real(0.0);
#pragma unroll 2
    for (int k = 0; k < nz; ++k) {
        real m3_k1 = real(0.0), dz_k1 = real(0.0);
        if (k + 1 < nz) dz_k1 = g.dz(P, k + 1, m3_k1);
        const real dzi_k1 = (k + 1 < nz) ? real(0.5) * (dz_k + dz_k1) : dz_k;
        const real km_k1 = Km(k + 1);
        real sub, diag, sup;
        implicit_row(P, k, dz_k, m3_k, m3_k1, dzi_k, dzi_k1, km_k, km_k1, P.thv_dt_drag, sub, diag, sup);
        if (k == 0) {
            cp = sup / diag;
            ds = real(1.0) / diag;
        } else {
            const real den = diag - sub * cp;
            cp = sup / den;
            ds = (real(1.0) - sub * ds) / den;
        }
        cs[k] = cp;
        if (k + 1 < nz) q[(size_t)k * n2 + c] = ds;
        km_k = km_k1;
        dz_k = dz_k1;
        m3_k = m3_k1;
        dzi_k = dzi_k1;
    }
    real x = ds;
    q[(size_t)(nz - 1) * n2 + c] = x;
#pragma unroll 4
    for (int k = nz - 2; k >= 0; --k) {
        const size_t o = (size_t)k * n2 + c;
        x = q[o] - cs[k] * x;
        q[o] = x;
    }
}

template <int NZM>
__global__ void __launch_bounds__(128) k_qsolve(KPR P, const real* __restrict__ km,
                                                real* __restrict__ q) {
    COLUMN_PROLOGUE
    const int c = nb.c;
    const ColGeoR g = ColGeoR::load(P, c);
    real cs[NZM];
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
__global__ void __launch_bounds__(128, OC_MINB_CLOSURE) k_closure(KPR P, const real* __restrict__ u,
                                                 const real* __restrict__ v,
                                                 const wide* __restrict__ b,
                                                 real* __restrict__ e, real* __restrict__ km,
                                                 real* __restrict__ kh, real* __restrict__ q) {
#ifdef OC_MIXED
    // FP32 build: N^2 of the column on its interfaces, which the Gaspar length
    // marches read O(nz) times per interface, lives in shared memory: interface k
    // of the CTA's thread t at [k * threads + t] (dynamic, (nz + 1) x threads
    // values). Measured at 512 x 512 x 50: 0.52 against 0.57 ms for the local
    // array; the fp64 build keeps the local array (0.81 against 1.07 ms).
    extern __shared__ __align__(16) unsigned char s_dyn[];
    const StridedCol<real> nn2{reinterpret_cast<real*>(s_dyn) + threadIdx.y * blockDim.x + threadIdx.x,
                               (int)(blockDim.x * blockDim.y)};
#endif
    COLUMN_PROLOGUE
    const int nz = P.nz;
    const int c = nb.c;
    const size_t cw = nb.at(0, -1), cs_ = nb.at(-1, 0);
    const ColGeoR g = ColGeoR::load(P, c);
#ifndef OC_MIXED
    real nn2[NZM + 1];
#endif
    real sh2[NZM + 1], lk[NZM + 1], le[NZM + 1], cst[NZM + 1];
    real depth = real(0.0);
    for (int k = 0; k < nz; ++k) {
        real m;
        const real dz = g.dz(P, k, m);
        depth = (k == 0) ? dz : depth + dz;
    }
    // shear^2 and N^2 on interfaces (closure.py:150-161)
    {
        real uc_prev = real(0.0), vc_prev = real(0.0), dz_prev = real(0.0), m3_prev = real(0.0);
        wide b_prev = 0.0;
#pragma unroll 2
        for (int k = 0; k < nz; ++k) {
            const size_t o = (size_t)k * n2;
            const real uc = real(0.5) * (u[o + c] + u[o + cw]);
            const real vc = real(0.5) * (v[o + c] + v[o + cs_]);
            const wide bk = b[o + c];
            real m3k;
            const real dzk = g.dz(P, k, m3k);
            if (k >= 1) {
                const real wk = m3_prev * m3k;
                const real idz = inv_pos(real(0.5) * (dz_prev + dzk));
                const real du = (uc_prev - uc) * idz;
                const real dv = (vc_prev - vc) * idz;
                // the difference of two fp64 buoyancies (their ~1e-2 relative
                // vertical contrast would lose digits in FP32)
                const real db = real((b_prev - bk) * idz);
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
    sh2[0] = real(0.0);
    nn2[0] = real(0.0);
    sh2[nz] = real(0.0);
    nn2[nz] = real(0.0);
    // recursive lengths (closure.py:106-129) need whole-column sweeps first
    if (P.mxl_recursive) {
        real zi = real(0.0);
        for (int k = 0; k <= nz; ++k) {
            real m;
            if (k >= 1) zi = (k == 1) ? g.dz(P, 0, m) : zi + g.dz(P, k - 1, m);
            const real zb = fmax(depth - zi, real(0.0));
            const real ek = fmax(e[(size_t)k * n2 + c], P.e_min);
            const real n2c = fmax(nn2[k], P.n2_min);
            const real ell = sqrt(real(2.0) * ek / n2c);
            le[k] = fmin(ell, fmin(zi + P.z_0, zb + P.z_0));
        }
        for (int k = 1; k <= nz; ++k) le[k] = fmin(le[k], le[k - 1] + col_dzi(P, g, k));
        for (int k = nz - 1; k >= 0; --k) le[k] = fmin(le[k], le[k + 1] + col_dzi(P, g, k + 1));
        for (int k = 0; k <= nz; ++k) {
            real m0, m1;
            g.dz(P, k >= 1 ? k - 1 : 0, m0);
            g.dz(P, k, m1);
            const real wk = (k >= 1 && k <= nz - 1) ? m0 * m1 : real(0.0);
            const real ell = le[k] * wk;
            lk[k] = fmax(P.l_min, sqrt(ell * ell));
            le[k] = fmax(P.l_min, fmin(ell, ell));
        }
    }
    // implicit TKE rows and forward sweep (closure.py:171-198)
    real rhs0 = real(0.0), ds = real(0.0), cp = real(0.0), zi = real(0.0);
    real km_prev = real(0.0), km_cur = km[c];
    real m3_km1 = real(0.0), dz_km1 = real(0.0);  // level k-1
    real m3_k, dz_k = g.dz(P, 0, m3_k);
    for (int k = 0; k <= nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        const real km_next = (k < nz) ? km[o + n2] : real(0.0);
        const real wk = (k >= 1 && k <= nz - 1) ? m3_km1 * m3_k : real(0.0);
        const real e_old = e[o];
        real le_k;
        if (!P.mxl_recursive) {
            // Gaspar lengths (closure.py:65-104): march away from interface k
            // until the energy budget is spent; once the budget is zero the
            // reference's remaining steps add exactly 0
            if (k >= 1) zi = (k == 1) ? dz_km1 : zi + dz_km1;
            const real zb = fmax(depth - zi, real(0.0));
            const real ek = fmax(e_old, P.e_min);
            real lu = real(0.0), bud = ek;
            for (int kk = k - 1; kk >= 0 && bud > real(0.0); --kk) {
                const real n2j = fmax(nn2[kk], real(0.0)), dzj = col_dzi(P, g, kk);
                const real cost = n2j * dzj * (lu + real(0.5) * dzj);
                const bool full = cost <= bud;
                real step = dzj;
                if (!full && n2j > real(0.0)) {
                    const real part = sqrt(fmax(lu * lu + real(2.0) * bud / n2j, real(0.0))) - lu;
                    step = fmin(fmax(part, real(0.0)), dzj);
                }
                lu = lu + step;
                bud = full ? bud - cost : real(0.0);
            }
            real ld = real(0.0);
            bud = ek;
            for (int kk = k + 1; kk <= nz && bud > real(0.0); ++kk) {
                const real n2j = fmax(nn2[kk], real(0.0)), dzj = col_dzi(P, g, kk);
                const real cost = n2j * dzj * (ld + real(0.5) * dzj);
                const bool full = cost <= bud;
                real step = dzj;
                if (!full && n2j > real(0.0)) {
                    const real part = sqrt(fmax(ld * ld + real(2.0) * bud / n2j, real(0.0))) - ld;
                    step = fmin(fmax(part, real(0.0)), dzj);
                }
                ld = ld + step;
                bud = full ? bud - cost : real(0.0);
            }
            lu = fmin(lu, zi + P.z_0) * wk;
            ld = fmin(ld, zb + P.z_0) * wk;
            lk[k] = fmax(P.l_min, sqrt(lu * ld));
            le_k = fmax(P.l_min, fmin(lu, ld));
        } else {
            le_k = le[k];
        }
        const real prod = (km_cur - P.nu) * sh2[k] - (kh[o] - P.kappa) * nn2[k];
        const real diss = P.c_eps * sqrt(fmax(e_old, P.e_min)) / le_k;
        real a_up = real(0.0), a_dn = real(0.0);
        if (k >= 1 && k <= nz - 1) {
            const real idzi = inv_pos(real(0.5) * (dz_km1 + dz_k));
            a_up = P.dt * (real(0.5) * (km_prev + km_cur)) * inv_pos(dz_km1) * idzi;
            a_dn = P.dt * (real(0.5) * (km_cur + km_next)) * inv_pos(dz_k) * idzi;
        }
        real sub = -a_up, sup = -a_dn;
        real diag = real(1.0) + a_up + a_dn + P.dt * diss;
        real rhs = e_old + P.dt * prod;
        if (wk <= real(0.0)) {
            diag = real(1.0);
            sub = real(0.0);
            sup = real(0.0);
            rhs = P.e_min;
        }
        if (k == 0) {
            rhs = (g.kb > 0) ? P.e_bb * P.ustar2[c] : P.e_min;
            rhs0 = rhs;
            cp = sup / diag;
            ds = rhs / diag;
        } else {
            const real den = diag - sub * cp;
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
            dz_k = real(0.0);
            m3_k = real(0.0);
        }
    }
    // back substitution, e/K update (closure.py:198-205)
    real x = real(0.0);
    for (int k = nz; k >= 0; --k) {
        const size_t o = (size_t)k * n2 + c;
        x = (k == nz) ? ds : e[o] - cst[k] * x;
        real m0, m1;
        g.dz(P, k >= 1 ? k - 1 : 0, m0);
        g.dz(P, k < nz ? k : 0, m1);
        const real wk = (k >= 1 && k <= nz - 1) ? m0 * m1 : real(0.0);
        real en = fmax(x, P.e_min);
        en = (wk > real(0.0)) ? en : P.e_min;
        if (k == 0) en = rhs0;
        const real kmn = P.c_k * lk[k] * sqrt(en) * wk + P.nu;
        const real khn = (kmn - P.nu) / P.pr_t + P.kappa;
        e[o] = en;
        km[o] = kmn;
        kh[o] = khn;
        lk[k] = kmn;
    }
    column_q(P, g, [&](int k) { return lk[k]; }, cst, q, c, n2);
}

// ------------------------------------------------------------------ Ku, Kv
// Ku = sum_k dz3u * min(q, q_east) * mask_u (model3d_v05.py:154-157)
__global__ void k_kukv(KPR P, const real* __restrict__ q, wide* __restrict__ Ku,
                       wide* __restrict__ Kv) {
    COLUMN_PROLOGUE
    const size_t c = nb.c;
    const size_t ce = nb.at(0, 1), cn = nb.at(1, 0);
    const ColGeoR gc = ColGeoR::load(P, (int)c), ge = ColGeoR::load(P, (int)ce), gn = ColGeoR::load(P, (int)cn);
    const int2 kf = P.kface[c];
    wide su = 0.0, sv = 0.0;  // depth sums in fp64 on both paths
#pragma unroll 4
    for (int k = 0; k < P.nz; ++k) {
        const size_t o = (size_t)k * n2;
        real m;
        const real dzc = gc.dz(P, k, m), dze = ge.dz(P, k, m), dzn = gn.dz(P, k, m);
        const real qc = q[o + c];
        const real tu = face_dz(P, kf.x, k, dzc, dze) * fmin(qc, q[o + ce]);
        const real tv = face_dz(P, kf.y, k, dzc, dzn) * fmin(qc, q[o + cn]);
        su = (k == 0) ? wide(tu) : su + wide(tu);
        sv = (k == 0) ? wide(tv) : sv + wide(tv);
    }
    Ku[c] = su * P.mask_u64[c];
    Kv[c] = sv * P.mask_v64[c];
}

// ------------------------------------------------------------------ w from transport divergence
// w[k] = -sum_{k'>=k} div(dz3u u, dz3v v)[k'], accumulated from the bottom
// (vertical_var.py:109-121); w[nz] = 0.
__global__ void __launch_bounds__(128, 8) k_wcol(KPR P, const real* __restrict__ u, const real* __restrict__ v,
                       real* __restrict__ w) {
    COLUMN_PROLOGUE
    const int nz = P.nz;
    const size_t c = nb.c, cw = nb.at(0, -1), cs_ = nb.at(-1, 0);
    const ColGeoR gc = ColGeoR::load(P, (int)c), ge = ColGeoR::load(P, nb.at(0, 1)),
                 gw = ColGeoR::load(P, (int)cw), gn = ColGeoR::load(P, nb.at(1, 0)), gs = ColGeoR::load(P, (int)cs_);
    const int2 kf = P.kface[c];
    const int kuw = P.kface[cw].x, kvs = P.kface[cs_].y;
    real acc = real(0.0);
    w[(size_t)nz * n2 + c] = real(0.0);
#pragma unroll 2
    for (int k = nz - 1; k >= 0; --k) {
        const size_t o = (size_t)k * n2;
        real m3, m;
        const real dzc = gc.dz(P, k, m3);
        const real dzu_c = face_dz(P, kf.x, k, dzc, ge.dz(P, k, m));
        const real dzu_w = face_dz(P, kuw, k, gw.dz(P, k, m), dzc);
        const real dzv_c = face_dz(P, kf.y, k, dzc, gn.dz(P, k, m));
        const real dzv_s = face_dz(P, kvs, k, gs.dz(P, k, m), dzc);
        const real td = m3 * ((dzu_c * u[o + c] - dzu_w * u[o + cw]) / P.dx +
                                (dzv_c * v[o + c] - dzv_s * v[o + cs_]) / P.dy);
        acc = (k == nz - 1) ? td : acc + td;
        w[o + c] = -acc;
    }
}

// ------------------------------------------------------------------ buoyancy potential
// phi[k] = 0.5 dz3 b + sum_{k'<k} dz3 b, optionally minus its thickness-weighted
// column mean (vertical_var.py:132-145).
__global__ void k_phi(KPR P, const wide* __restrict__ b, wide* __restrict__ phi) {
    // fp64 on both paths: neighbouring columns' potentials of ~1e3 m2 s-2 differ
    // by the baroclinic pressure signal, which FP32 would not resolve
    COLUMN_PROLOGUE
    const int nz = P.nz;
    const size_t c = nb.c;
    const ColGeo64 g = ColGeo64::load(P, (int)c);
    wide above = 0.0, total = 0.0;
#pragma unroll 4
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        const wide dz = g.dz(P, k);
        const wide bk = b[o];
        phi[o] = 0.5 * dz * bk + above;
        const wide t = dz * bk;
        above = (k == 0) ? t : above + t;
        total = (k == 0) ? dz : total + dz;
    }
    if (P.pgf_remove) {
        wide s = 0.0;
        for (int k = 0; k < nz; ++k) {
            const wide dz = g.dz(P, k);
            const wide t = dz * phi[(size_t)k * n2 + c];
            s = (k == 0) ? t : s + t;
        }
        const wide mean = s * inv_pos(total);
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
    const KPR& P;
    const Nbr& nb;
    const real* __restrict__ u;
    const real* __restrict__ v;
    size_t o;
    int k;
    __device__ __forceinline__ real U(int dj, int di) const { return u[o + nb.at(dj, di)]; }
    __device__ __forceinline__ real V(int dj, int di) const { return v[o + nb.at(dj, di)]; }
    __device__ __forceinline__ real MU(int dj, int di) const { return col_m3u(P, nb.at(dj, di), k); }
    __device__ __forceinline__ real MV(int dj, int di) const { return col_m3v(P, nb.at(dj, di), k); }
};

// ------------------------------------------------------------------ Coriolis averages
// v averaged onto u points over wet v faces (operators_masked.py:45-52)
template <class A>
__device__ __forceinline__ real v_on_u_at(const A& a) {
    const real f0 = a.V(0, 0), f1 = a.V(-1, 0), f2 = a.V(0, 1), f3 = a.V(-1, 1);
    const real w0 = a.MV(0, 0), w1 = a.MV(-1, 0), w2 = a.MV(0, 1), w3 = a.MV(-1, 1);
    real num = real(0.0) + w0 * f0;
    num = num + w1 * f1;
    num = num + w2 * f2;
    num = num + w3 * f3;
    real den = real(0.0) + w0;
    den = den + w1;
    den = den + w2;
    den = den + w3;
    const real avg = den > real(0.0) ? num / den : real(0.0);
    return avg * a.MU(0, 0);
}

// u averaged onto v points over wet u faces (operators_masked.py:55-61)
template <class A>
__device__ __forceinline__ real u_on_v_at(const A& a) {
    const real f0 = a.U(0, 0), f1 = a.U(0, -1), f2 = a.U(1, 0), f3 = a.U(1, -1);
    const real w0 = a.MU(0, 0), w1 = a.MU(0, -1), w2 = a.MU(1, 0), w3 = a.MU(1, -1);
    real num = real(0.0) + w0 * f0;
    num = num + w1 * f1;
    num = num + w2 * f2;
    num = num + w3 * f3;
    real den = real(0.0) + w0;
    den = den + w1;
    den = den + w2;
    den = den + w3;
    const real avg = den > real(0.0) ? num / den : real(0.0);
    return avg * a.MV(0, 0);
}

__device__ __forceinline__ real v_on_u(const KPR& P, const Nbr& nb, const real* __restrict__ v, size_t o,
                                         int k) {
    return v_on_u_at(GlobalLevel{P, nb, nullptr, v, o, k});
}

__device__ __forceinline__ real u_on_v(const KPR& P, const Nbr& nb, const real* __restrict__ u, size_t o,
                                         int k) {
    return u_on_v_at(GlobalLevel{P, nb, u, nullptr, o, k});
}

// horizontal Laplacian D o G with the given face masks (operators_masked.py:64-68);
// which = 0: u (x-mask m3u, y-mask m3v, cell mask m3u), 1: v (cell mask m3v),
// 2: tracer (cell mask m3)
__device__ real hlap(const KPR& P, const Nbr& nb, const real* __restrict__ f, int k, int which) {
    const size_t o = (size_t)k * P.n2;
    auto F = [&](int dj, int di) { return f[o + nb.at(dj, di)]; };
    const real gx0 = m3u_at(P, nb, 0, 0, k) * (F(0, 1) - F(0, 0)) / P.dx;
    const real gxw = m3u_at(P, nb, 0, -1, k) * (F(0, 0) - F(0, -1)) / P.dx;
    const real gy0 = m3v_at(P, nb, 0, 0, k) * (F(1, 0) - F(0, 0)) / P.dy;
    const real gys = m3v_at(P, nb, -1, 0, k) * (F(0, 0) - F(-1, 0)) / P.dy;
    const real m = which == 0 ? m3u_at(P, nb, 0, 0, k)
                                : (which == 1 ? m3v_at(P, nb, 0, 0, k) : m3_at(P, nb, 0, 0, k));
    return m * ((gx0 - gxw) / P.dx + (gy0 - gys) / P.dy);
}

// explicit vertical diffusion of a face velocity (vertical_var.py:80-106) with
// the column's interface viscosity, the face thickness table dzf[k-1..k+1], the
// cell mask's bottom rule and surface flux `surf`
__device__ __forceinline__ real explicit_dz(const KPR& P, int k, real fkm1, real fk, real fkp1,
                                              real Kk, real Kk1, real dzf_m1, real dzf_k,
                                              real dzf_p1, real m3k_m1_bottom,
                                              real m3k_bottom, real m3k, real surf,
                                              real drag) {
    const int nz = P.nz;
    real flux_k, flux_k1;
    if (k == 0) {
        flux_k = surf;
    } else {
        const real dzi = real(0.5) * (dzf_m1 + dzf_k);
        flux_k = Kk * (fkm1 - fk) * inv_pos(dzi);
        if (m3k_m1_bottom > real(0.0)) flux_k = real(0.0);
    }
    if (k == nz - 1) {
        flux_k1 = real(0.0);
    } else {
        const real dzi = real(0.5) * (dzf_k + dzf_p1);
        flux_k1 = Kk1 * (fk - fkp1) * inv_pos(dzi);
        if (m3k_bottom > real(0.0)) flux_k1 = real(0.0);
    }
    const real idz = inv_pos(dzf_k);
    const real out = (flux_k - flux_k1) * idz;
    const real dragc = drag * fk * m3k_bottom;
    return (out - dragc * idz) * (m3k > real(0.0) ? real(1.0) : real(0.0));
}

// ------------------------------------------------------------------ momentum advection
// x- and y-flux divergence of u at its east face (advection_v06.py:77-99 for the
// kappa/TVD scheme, advection.py:62-79 for the centred one); the reference forms
// ax + ay + az left to right, so (ax + ay) + az is its sum
template <class A>
__device__ __forceinline__ real mom_adv_u_xy(const KPR& P, const A& a) {
    if (P.advection >= 3) {
        const bool lim = P.advection == 4;
        const real ub_c0 = real(0.5) * (a.U(0, -1) + a.U(0, 0));
        const real ub_c1 = real(0.5) * (a.U(0, 0) + a.U(0, 1));
        const real uc0 = kappa_face(P, a.U(0, -2), a.U(0, -1), a.U(0, 0), a.U(0, 1), ub_c0, a.MU(0, -2),
                                      a.MU(0, 1), lim);
        const real uc1 = kappa_face(P, a.U(0, -1), a.U(0, 0), a.U(0, 1), a.U(0, 2), ub_c1, a.MU(0, -1),
                                      a.MU(0, 2), lim);
        const real ax = (ub_c1 * uc1 - ub_c0 * uc0) / P.dx;
        const real vb0 = real(0.5) * (a.V(0, 0) + a.V(0, 1));
        const real vbm = real(0.5) * (a.V(-1, 0) + a.V(-1, 1));
        const real fy0 = vb0 * kappa_face(P, a.U(-1, 0), a.U(0, 0), a.U(1, 0), a.U(2, 0), vb0, a.MU(-1, 0),
                                            a.MU(2, 0), lim);
        const real fym = vbm * kappa_face(P, a.U(-2, 0), a.U(-1, 0), a.U(0, 0), a.U(1, 0), vbm, a.MU(-2, 0),
                                            a.MU(1, 0), lim);
        return ax + (fy0 - fym) / P.dy;
    }
    const real ub_c0 = real(0.5) * (a.U(0, -1) + a.U(0, 0));
    const real ub_c1 = real(0.5) * (a.U(0, 0) + a.U(0, 1));
    const real ax = (ub_c1 * ub_c1 - ub_c0 * ub_c0) / P.dx;
    const real vb0 = real(0.5) * (a.V(0, 0) + a.V(0, 1));
    const real vbm = real(0.5) * (a.V(-1, 0) + a.V(-1, 1));
    const real fy0 = vb0 * (real(0.5) * (a.U(0, 0) + a.U(1, 0)));
    const real fym = vbm * (real(0.5) * (a.U(-1, 0) + a.U(0, 0)));
    return ax + (fy0 - fym) / P.dy;
}

// the same for v at its north face (advection_v06.py:100-108, advection.py:81-95):
// bx + by, formed in that order
template <class A>
__device__ __forceinline__ real mom_adv_v_xy(const KPR& P, const A& a) {
    if (P.advection >= 3) {
        const bool lim = P.advection == 4;
        const real vb_c0 = real(0.5) * (a.V(-1, 0) + a.V(0, 0));
        const real vb_c1 = real(0.5) * (a.V(0, 0) + a.V(1, 0));
        const real vc0 = kappa_face(P, a.V(-2, 0), a.V(-1, 0), a.V(0, 0), a.V(1, 0), vb_c0, a.MV(-2, 0),
                                      a.MV(1, 0), lim);
        const real vc1 = kappa_face(P, a.V(-1, 0), a.V(0, 0), a.V(1, 0), a.V(2, 0), vb_c1, a.MV(-1, 0),
                                      a.MV(2, 0), lim);
        const real by = (vb_c1 * vc1 - vb_c0 * vc0) / P.dy;
        const real ub0 = real(0.5) * (a.U(0, 0) + a.U(1, 0));
        const real ubm = real(0.5) * (a.U(0, -1) + a.U(1, -1));
        const real fx0 = ub0 * kappa_face(P, a.V(0, -1), a.V(0, 0), a.V(0, 1), a.V(0, 2), ub0, a.MV(0, -1),
                                            a.MV(0, 2), lim);
        const real fxm = ubm * kappa_face(P, a.V(0, -2), a.V(0, -1), a.V(0, 0), a.V(0, 1), ubm, a.MV(0, -2),
                                            a.MV(0, 1), lim);
        return (fx0 - fxm) / P.dx + by;
    }
    const real vb_c0 = real(0.5) * (a.V(-1, 0) + a.V(0, 0));
    const real vb_c1 = real(0.5) * (a.V(0, 0) + a.V(1, 0));
    const real by = (vb_c1 * vb_c1 - vb_c0 * vb_c0) / P.dy;
    const real ub0 = real(0.5) * (a.U(0, 0) + a.U(1, 0));
    const real ubm = real(0.5) * (a.U(0, -1) + a.U(1, -1));
    const real fx0 = ub0 * (real(0.5) * (a.V(0, 0) + a.V(0, 1)));
    const real fxm = ubm * (real(0.5) * (a.V(0, -1) + a.V(0, 0)));
    return (fx0 - fxm) / P.dx + by;
}

// advective flux of a face velocity through interface kk of its column (0 =
// surface), from the velocity at kk-2 .. kk+1, the interface w averaged over
// the two cells of the face, and the face's wet levels kf
// (advection_v06.py:50-74 and :86-99; advection.py:75-79)
__device__ __forceinline__ real mom_vflux(const KPR& P, int kk, int kf, real f_m2, real f_m1, real f_0,
                                            real f_p1, real wa, real wb_) {
    const int nz = P.nz;
    if (kk == 0 || kk == nz) return real(0.0);
    const real wb = real(0.5) * (wa + wb_);
    if (P.advection >= 3) {
        const real fu = (kk >= 2) ? f_m2 : real(0.0);
        const real fd = (kk + 1 <= nz - 1) ? f_p1 : real(0.0);
        const bool hu = (kk >= 2) && kk - 2 < kf;
        const bool hd = (kk + 1 <= nz - 1) && kk + 1 < kf;
        return wb * kappa_face_z(P, fu, f_m1, f_0, fd, wb, hu, hd, P.advection == 4);
    }
    return wb * real(0.5) * (f_m1 + f_0);
}

// the diffusive flux K (f_above - f_below) / dzi through interface k of a face
// velocity column (vertical_var.py:80-106), zero when the level above is the
// column's last wet one
__device__ __forceinline__ real diff_flux(real Kk, real f_above, real f_below, real dzf_above,
                                           real dzf_below, real bottom_above) {
    const real dzi = real(0.5) * (dzf_above + dzf_below);
    const real flux = Kk * (f_above - f_below) * inv_pos(dzi);
    return bottom_above > real(0.0) ? real(0.0) : flux;
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
    const real* su;
    const real* sv;
    const int* sku;
    const int* skv;
    int rc;  // the thread's column in the region
    int k;
    __device__ __forceinline__ real U(int dj, int di) const { return su[rc + dj * MOM_RX + di]; }
    __device__ __forceinline__ real V(int dj, int di) const { return sv[rc + dj * MOM_RX + di]; }
    __device__ __forceinline__ real MU(int dj, int di) const { return k < sku[rc + dj * MOM_RX + di] ? real(1.0) : real(0.0); }
    __device__ __forceinline__ real MV(int dj, int di) const { return k < skv[rc + dj * MOM_RX + di] ? real(1.0) : real(0.0); }
};

__global__ void __launch_bounds__(MOM_TX * MOM_TY * 2, OC_MINB_MOM) k_mom_column(
    KPR P, const real* __restrict__ u, const real* __restrict__ v, const wide* __restrict__ b,
    const wide* __restrict__ phi, const real* __restrict__ w, const real* __restrict__ km,
    real* __restrict__ pgx, real* __restrict__ pgy, real* __restrict__ avpv,
    real* __restrict__ avpu, real* __restrict__ dzu, real* __restrict__ dzv,
    real* __restrict__ stu, real* __restrict__ stv) {
    __shared__ int s_g[MOM_RN], s_ku[MOM_RN], s_kv[MOM_RN];
    __shared__ real s_u[2][MOM_RN], s_v[2][MOM_RN];  // level planes, double-buffered
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
    const ColGeoR gc = ColGeoR::load(P, c), gf = ColGeoR::load(P, cf);
#ifdef OC_MIXED
    // the pressure gradient's depths in fp64 (FP32 depths of ~4 km carry 2e-4 m errors)
    const ColGeo64 gc64 = ColGeo64::load(P, c), gf64 = ColGeo64::load(P, cf);
#endif
    const int kff = comp ? P.kface[c].y : P.kface[c].x;
    const real tau = comp ? P.tau_v[c] : P.tau_u[c];
    const real* __restrict__ X = comp ? v : u;
    // face thickness of the column's face at level kk (0 outside)
    auto dzf_at = [&](int kk) {
        if (kk < 0 || kk >= nz) return real(0.0);
        real m;
        return face_dz(P, kff, kk, gc.dz(P, kk, m), gf.dz(P, kk, m));
    };
    auto m3c_at = [&](int kk) { return (kk >= 0 && kk < gc.kb) ? real(1.0) : real(0.0); };
    auto Xc = [&](int kk) { return (kk >= 0 && kk < nz) ? X[(size_t)kk * n2 + c] : real(0.0); };
    // rolling values of the component at k-1, k, k+1 (and k+2 for advection)
    real x_m1 = real(0.0), x_0 = real(0.0), x_p1 = real(0.0), dz_0 = real(0.0);
    // fluxes through the top of level kbeg
    real fz = real(0.0), df = real(0.0);
    if (live) {
        x_m1 = Xc(kbeg - 1);
        x_0 = Xc(kbeg);
        x_p1 = Xc(kbeg + 1);
        const real dz_m1 = dzf_at(kbeg - 1);
        dz_0 = dzf_at(kbeg);
        const int kk = kbeg;
        if (P.advection != 0)
            fz = mom_vflux(P, kk, kff, Xc(kk - 2), x_m1, x_0, x_p1, w[(size_t)kk * n2 + c], w[(size_t)kk * n2 + cf]);
        if (kk == 0) {
            df = tau;
        } else {
            const real bot = (m3c_at(kk - 1) > real(0.0) && m3c_at(kk) == real(0.0)) ? real(1.0) : real(0.0);
            df = diff_flux(km[(size_t)kbeg * n2 + c], x_m1, x_0, dz_m1, dz_0, bot);
        }
    }
    // level k's u and v of the region go to buffer (k - kbeg) & 1; level k + 1's
    // copies are in flight while level k is computed (each thread copies the
    // region cells whose s_g it wrote itself)
    auto stage = [&](int k) {
        const size_t o = (size_t)k * n2;
        const int buf = (k - kbeg) & 1;
        for (int r = tid; r < MOM_RN; r += nthreads) {
            cp_async_elem(&s_u[buf][r], u + o + s_g[r]);
            cp_async_elem(&s_v[buf][r], v + o + s_g[r]);
        }
        cp_async_commit();
    };
    stage(kbeg);
    for (int k = kbeg; k < kend; ++k) {
        const size_t o = (size_t)k * n2;
        // every thread is done with the previous level, whose buffer level k + 1 takes
        __syncthreads();
        if (k + 1 < kend) {
            stage(k + 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        if (!live) continue;
        const int buf = (k - kbeg) & 1;
        const TileLevel lv{s_u[buf], s_v[buf], s_ku, s_kv, rc, k};
        const real x_p2 = Xc(k + 2);
        const real dz_p1 = dzf_at(k + 1);
        const real K_1 = km[o + n2 + c];
        real m3c, m3f;
        const real dz_c = gc.dz(P, k, m3c), dz_f = gf.dz(P, k, m3f);
        const real m3f_k = k < kff ? real(1.0) : real(0.0);
        const real bottom_k = (m3c > real(0.0) && m3c_at(k + 1) == real(0.0)) ? real(1.0) : real(0.0);
        // ---- pressure gradient at a common depth (model3d_v05.py:211-230), in
        // fp64 on both paths: it is a small difference of large potentials
        const wide phc = phi[o + c], phf = phi[o + cf];
        const wide bc = b[o + c], bf = b[o + cf];
        const wide dxy = comp ? P.dy64 : P.dx64;
        wide pg;
        if (P.pgf_correction) {
#ifdef OC_MIXED
            const wide zc_c = gc64.above(P, k) + 0.5 * gc64.dz(P, k);
            const wide zc_f = gf64.above(P, k) + 0.5 * gf64.dz(P, k);
#else
            const wide zc_c = gc.above(P, k) + 0.5 * dz_c;
            const wide zc_f = gf.above(P, k) + 0.5 * dz_f;
#endif
            const wide zf = 0.5 * (zc_c + zc_f);
            pg = m3f_k * ((phf + bf * (zf - zc_f)) - (phc + bc * (zf - zc_c))) / dxy;
        } else {
            pg = m3f_k * (phf - phc) / dxy * m3f_k;
        }
        (comp ? pgy : pgx)[o + c] = real(pg);
        // ---- Coriolis average of the old state (v at u points, u at v points)
        if (comp)
            avpu[o + c] = u_on_v_at(lv);
        else
            avpv[o + c] = v_on_u_at(lv);
        // ---- explicit vertical diffusion: top flux carried, bottom flux formed here
        const real db = (k < nz - 1) ? diff_flux(K_1, x_0, x_p1, dz_0, dz_p1, bottom_k) : real(0.0);
        {
            const real mk = m3c > real(0.0) ? real(1.0) : real(0.0);
            const real id = inv_pos(dz_0);
            const real out = (df - db) * id;
            const real drag = P.bottom_drag * x_0 * bottom_k;
            (comp ? dzv : dzu)[o + c] = (out - drag * id) * mk;
        }
        // ---- advection and horizontal viscosity, then the stress increment
        real ex = real(0.0), fb = real(0.0);
        if (P.advection != 0) {
            fb = mom_vflux(P, k + 1, kff, x_m1, x_0, x_p1, x_p2, w[o + n2 + c], w[o + n2 + cf]);
            const real a = (comp ? mom_adv_v_xy(P, lv) : mom_adv_u_xy(P, lv)) + (fz - fb) / P.dz_nom[k];
            ex = ex - a * m3f_k;
        }
        if (P.a_h > real(0.0)) {
            Nbr nb;
            nb.init(wi, wj, nx, ny);
            ex = ex + P.a_h * hlap(P, nb, X, k, comp);
        }
        (comp ? stv : stu)[o + c] = (k == 0) ? P.thv_dt * tau * inv_pos(dz_0) + P.dt * ex : real(0.0) + P.dt * ex;
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
    KPR P, const real* __restrict__ u, const real* __restrict__ v,
    const real* __restrict__ u_it, const real* __restrict__ v_it,
    const real* __restrict__ pgx, const real* __restrict__ pgy,
    const real* __restrict__ avpv, const real* __restrict__ avpu,
    const real* __restrict__ dzu, const real* __restrict__ dzv,
    const real* __restrict__ stu, const real* __restrict__ stv,
    const wide* __restrict__ gx2, const wide* __restrict__ gy2, real* __restrict__ ru,
    real* __restrict__ rv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= P.nx || j >= P.ny) return;
    const int c = j * P.nx + i;
    const size_t o = (size_t)k * P.n2;
    const real av_v = avpv[o + c], av_u = avpu[o + c];
    // the iterate's averages; in the first pass the iterate is the old state,
    // whose averages the explicit-terms kernel formed already by the same function
    real it_v = av_v, it_u = av_u;
    if (u_it != u || v_it != v) {
        Nbr nb;
        nb.init(i, j, P.nx, P.ny);
        it_v = v_on_u(P, nb, v_it, o, k);
        it_u = u_on_v(P, nb, u_it, o, k);
    }
    const real vcor = P.one_m_tc * av_v + P.theta_cor * it_v;
    const real ucor = P.one_m_tc * av_u + P.theta_cor * it_u;
    real gu, gv;
    if (P.scheme != 2) {
        const real m3u_k = col_m3u(P, c, k), m3v_k = col_m3v(P, c, k);
        gu = u[o + c] + P.dt * (P.f0 * vcor + pgx[o + c]) - P.c1 * (real(gx2[c]) * m3u_k) + P.c3 * dzu[o + c];
        gv = v[o + c] + P.dt * (P.neg_f0 * ucor + pgy[o + c]) - P.c1 * (real(gy2[c]) * m3v_k) + P.c3 * dzv[o + c];
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
__global__ void __launch_bounds__(128) k_momentum_solve(KPR P, const real* __restrict__ km,
                                                        real* __restrict__ ghu,
                                                        real* __restrict__ ghv,
                                                        wide* __restrict__ Ug,
                                                        wide* __restrict__ Vg) {
    COLUMN_PROLOGUE
    const int nz = P.nz;
    const int c = nb.c;
    const ColGeoR g = ColGeoR::load(P, c);
    real cs[NZM];
    real m3_k, dz_k = g.dz(P, 0, m3_k);
    real dzi_k = dz_k;
    real km_k = km[c];
    real du = real(0.0), dv = real(0.0), cp = real(0.0);
#pragma unroll 4
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        const real km_k1 = km[o + n2];
        const real ru = ghu[o], rv = ghv[o];
        real m3_k1 = real(0.0), dz_k1 = real(0.0);
        if (k + 1 < nz) dz_k1 = g.dz(P, k + 1, m3_k1);
        const real dzi_k1 = (k + 1 < nz) ? real(0.5) * (dz_k + dz_k1) : dz_k;
        real sub, diag, sup;
        implicit_row(P, k, dz_k, m3_k, m3_k1, dzi_k, dzi_k1, km_k, km_k1, P.thv_dt_drag, sub, diag, sup);
        if (k == 0) {
            cp = sup / diag;
            du = ru / diag;
            dv = rv / diag;
        } else {
            const real den = diag - sub * cp;
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
    real xu = du, xv = dv;
    {
        const size_t o = (size_t)(nz - 1) * n2 + c;
        const real m = (nz - 1 < g.kb) ? real(1.0) : real(0.0);
        ghu[o] = xu * m;
        ghv[o] = xv * m;
    }
#pragma unroll 4
    for (int k = nz - 2; k >= 0; --k) {
        const size_t o = (size_t)k * n2 + c;
        const real m = (k < g.kb) ? real(1.0) : real(0.0);
        xu = ghu[o] - cs[k] * xu;
        xv = ghv[o] - cs[k] * xv;
        ghu[o] = xu * m;
        ghv[o] = xv * m;
    }
    const ColGeoR ge = ColGeoR::load(P, nb.at(0, 1)), gn = ColGeoR::load(P, nb.at(1, 0));
    const int2 kfc = P.kface[c];
    wide su = 0.0, sv = 0.0;  // depth sums in fp64 on both paths
#pragma unroll 4
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        real m3c, m3e, m3n;
        const real dzc = g.dz(P, k, m3c);
        const real dze = ge.dz(P, k, m3e);
        const real dzn = gn.dz(P, k, m3n);
        const real tu = (k < kfc.x ? real(1.0) : real(0.0)) * face_combine(P, dzc, dze) * ghu[o];
        const real tv = (k < kfc.y ? real(1.0) : real(0.0)) * face_combine(P, dzc, dzn) * ghv[o];
        su = (k == 0) ? wide(tu) : su + wide(tu);
        sv = (k == 0) ? wide(tv) : sv + wide(tv);
    }
    Ug[c] = su;
    Vg[c] = sv;
}

// ------------------------------------------------------------------ back substitution
// u = (gh_u - g dt theta q dx(eta_new) m3u) m3   (model3d_v05.py:404-406)
__global__ void k_backsub(KPR P, const real* __restrict__ ghu, const real* __restrict__ ghv,
                          const real* __restrict__ q, const wide* __restrict__ eta_new,
                          real* __restrict__ u_out, real* __restrict__ v_out) {
    COLUMN_PROLOGUE
    const size_t c = nb.c, ce = nb.at(0, 1), cn = nb.at(1, 0);
    // the surface gradient in fp64 on both paths (a difference of neighbouring elevations)
    const real gx = real(P.mask_u64[c] * (eta_new[ce] - eta_new[c]) / P.dx64);
    const real gy = real(P.mask_v64[c] * (eta_new[cn] - eta_new[c]) / P.dy64);
    const int kb = P.kinfo[c].y;
    const int2 kf = P.kface[c];
#pragma unroll 4
    for (int k = 0; k < P.nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        const real m3 = k < kb ? real(1.0) : real(0.0);
        const real m3u_k = k < kf.x ? real(1.0) : real(0.0);
        const real m3v_k = k < kf.y ? real(1.0) : real(0.0);
        const real qk = q[o];
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
__device__ __forceinline__ real tracer_face(const KPR& P, const real* __restrict__ C, size_t o,
                                              const Stencil4& s, real vel, int k) {
    const real a = C[o + s.c0], b = C[o + s.c1];
    if (P.advection == 1) return real(0.5) * (a + b);
    if (P.advection >= 3)
        return kappa_face(P, C[o + s.cm], a, b, C[o + s.cp], vel, col_m3(P, s.cm, k), col_m3(P, s.cp, k),
                          P.advection == 4);
    return vel > real(0.0) ? a : b;
}

// flux through an east (ax = 0) or north (ax = 1) face: face thickness x
// normal velocity x face value (model3d_v05.py:498-501)
__device__ __forceinline__ real tracer_flux(const KPR& P, const real* __restrict__ C,
                                              const real* __restrict__ vel_f, size_t o,
                                              const Stencil4& s, int k, int ax) {
    const real vel = vel_f[o + s.c0];
    const int2 kf = P.kface[s.c0];
    real m;
    const real dzf = face_dz(P, ax == 0 ? kf.x : kf.y, k, col_dz(P, s.c0, k, m), col_dz(P, s.c1, k, m));
    return dzf * vel * tracer_face(P, C, o, s, vel, k);
}

// tracer value on interface kk of a column (0 = surface) from the column values
// at kk-2, kk-1, kk, kk+1 and w there (model3d_v05.py:502-510)
__device__ __forceinline__ real tracer_vface(const KPR& P, const ColGeoR& g, int kk, real f_m2, real f_m1,
                                               real f_0, real f_p1, real wv) {
    const int nz = P.nz;
    if (kk == 0) return f_0;
    if (kk == nz) return real(0.0);
    if (P.advection >= 3) {
        const real fu = (kk >= 2) ? f_m2 : real(0.0);
        const real fd = (kk + 1 <= nz - 1) ? f_p1 : real(0.0);
        const bool hu = (kk >= 2) && kk - 2 < g.kb;
        const bool hd = (kk + 1 <= nz - 1) && kk + 1 < g.kb;
        return kappa_face_z(P, fu, f_m1, f_0, fd, wv, hu, hd, P.advection == 4);
    }
    return real(0.5) * (f_m1 + f_0);
}

__global__ void __launch_bounds__(TRX * TRY, OC_MINB_TRACER) k_tracer_rhs(KPR P, const real* __restrict__ C0,
                                                             const real* __restrict__ S,
                                                             const real* __restrict__ u,
                                                             const real* __restrict__ v,
                                                             const real* __restrict__ w,
                                                             const real* __restrict__ kh,
                                                             real* __restrict__ rT,
                                                             real* __restrict__ rS) {
    // C0 is T with TS tracers, else the buoyancy (the fp64 path's only tracer).
    // The tile's columns plus a 2-column ring: flat 2D index and compact geometry
    // (once), then each level's tracers and face velocities (staged per level)
    constexpr int RX = TRX + 4, RY = TRY + 4, RNC = RX * RY;
    // level indices are at most 128: the column's (kf, kb) and its faces' wet
    // levels (ku, kv) fit one byte each
    __shared__ int s_g[RNC];
    __shared__ uchar4 s_k[RNC];
    __shared__ real s_d0[RNC], s_d1[RNC];
    // level planes, double-buffered: [buffer][field] tracers, [buffer] face velocities
    __shared__ real s_f[2][2][RNC], s_u[2][RNC], s_v[2][RNC];
    __shared__ real sfx[2][TRY][TRX + 1];  // [field][row][west face of column]
    __shared__ real sfy[2][TRY + 1][TRX];  // [field][south face of row][column]
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
    const ColGeoR g = ColGeoR::load(P, c);
    real* __restrict__ R0 = rT;
    for (int r = tid; r < RNC; r += TRX * TRY) {
        const int rj = r / RX, ri = r - rj * RX;
        const int gc = wrapi(j0 - 2 + rj, ny) * nx + wrapi(i0 - 2 + ri, nx);
        const int2 ki = P.kinfo[gc], kfc = P.kface[gc];
        const auto dx = P.dzx[gc];
        s_g[r] = gc;
        s_k[r] = make_uchar4((unsigned char)ki.x, (unsigned char)ki.y, (unsigned char)kfc.x, (unsigned char)kfc.y);
        s_d0[r] = dx.x;
        s_d1[r] = dx.y;
    }
    // thickness and wet flag of region column r at level k (col_dz from the staged geometry)
    auto sdz = [&](int r, int k, real& m3) {
        const uchar4 q = s_k[r];
        if (k >= q.y) {
            m3 = real(0.0);
            return real(0.0);
        }
        m3 = real(1.0);
        if (k < q.x) return P.dzr[k];
        return k == q.x ? s_d0[r] : s_d1[r];
    };
    // flux through a face with stencil cells (cm, c0, c1, cp) of the region,
    // normal velocity vel and face wet levels kfa (tracer_flux from shared memory)
    auto sflux = [&](const real* F, int cm, int c0, int c1, int cp, real vel, int kfa, int k) {
        real m;
        const real dzf = face_dz(P, kfa, k, sdz(c0, k, m), sdz(c1, k, m));
        const real a = F[c0], b = F[c1];
        real val;
        if (P.advection == 1)
            val = real(0.5) * (a + b);
        else if (P.advection >= 3)
            val = kappa_face(P, F[cm], a, b, F[cp], vel, k < s_k[cm].y ? real(1.0) : real(0.0),
                             k < s_k[cp].y ? real(1.0) : real(0.0), P.advection == 4);
        else
            val = vel > real(0.0) ? a : b;
        return dzf * vel * val;
    };
    const int rc = (ty + 2) * RX + tx + 2;                    // this thread's cell in the region
    const int rce = (tx + 2) * RX + TRX + 1;                  // east-column cell of row tx (x extras)
    const int rcn = (TRY + 1) * RX + tx + 2;                  // north-row cell of column tx (y extras)
    // rolling column values of each field at k-1, k, k+1 and the face at the top of level k
    real fm1[2] = {real(0.0), real(0.0)}, f0[2] = {real(0.0), real(0.0)}, fp1[2] = {real(0.0), real(0.0)}, ftop[2] = {real(0.0), real(0.0)};
    real w_k = real(0.0), kh_k = real(0.0);
    if (live) {
#pragma unroll
        for (int f = 0; f < 2; ++f) {
            if (f >= nf) break;
            const real* __restrict__ C = f == 0 ? C0 : S;
            const real fm2 = kbeg >= 2 ? C[(size_t)(kbeg - 2) * n2 + c] : real(0.0);
            fm1[f] = kbeg >= 1 ? C[(size_t)(kbeg - 1) * n2 + c] : real(0.0);
            f0[f] = C[(size_t)kbeg * n2 + c];
            fp1[f] = kbeg + 1 < nz ? C[(size_t)(kbeg + 1) * n2 + c] : real(0.0);
            if (adv) ftop[f] = tracer_vface(P, g, kbeg, fm2, fm1[f], f0[f], fp1[f], w[(size_t)kbeg * n2 + c]);
        }
        w_k = w[(size_t)kbeg * n2 + c];
        kh_k = kh[(size_t)kbeg * n2 + c];
    }
    // level k's planes go to buffer (k - kbeg) & 1; level k + 1's copies are in
    // flight while level k is computed (each thread copies the region cells
    // whose s_g it wrote itself)
    auto stage = [&](int k) {
        const size_t o = (size_t)k * n2;
        const int buf = (k - kbeg) & 1;
        for (int r = tid; r < RNC; r += TRX * TRY) {
            const size_t g = o + s_g[r];
            cp_async_elem(&s_f[buf][0][r], C0 + g);
            if (ts) cp_async_elem(&s_f[buf][1][r], S + g);
            cp_async_elem(&s_u[buf][r], u + g);
            cp_async_elem(&s_v[buf][r], v + g);
        }
        cp_async_commit();
    };
    if (adv) stage(kbeg);
    for (int k = kbeg; k < kend; ++k) {
        const size_t o = (size_t)k * n2;
        if (adv) {
            // every thread is done with the previous level, whose buffer level k + 1 takes
            __syncthreads();
            if (k + 1 < kend) {
                stage(k + 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
            const int buf = (k - kbeg) & 1;
            const real* su = s_u[buf];
            const real* sv = s_v[buf];
#pragma unroll 1
            for (int f = 0; f < nf; ++f) {
                const real* F = s_f[buf][f];
                // west face of this cell (cells rc-2 .. rc+1), south face (rc-2RX .. rc+RX)
                sfx[f][ty][tx] = sflux(F, rc - 2, rc - 1, rc, rc + 1, su[rc - 1], s_k[rc - 1].z, k);
                sfy[f][ty][tx] = sflux(F, rc - 2 * RX, rc - RX, rc, rc + RX, sv[rc - RX], s_k[rc - RX].w, k);
                if (xextra) sfx[f][tx][TRX] = sflux(F, rce - 1, rce, rce + 1, rce + 2, su[rce], s_k[rce].z, k);
                if (yextra)
                    sfy[f][TRY][tx] = sflux(F, rcn - RX, rcn, rcn + RX, rcn + 2 * RX, sv[rcn], s_k[rcn].w, k);
            }
            __syncthreads();
        }
        if (!live) continue;
        real m3k, m3_m1 = real(0.0), m3_p1 = real(0.0);
        const real dzk = g.dz(P, k, m3k);
        const real dz_m1 = (k > 0) ? g.dz(P, k - 1, m3_m1) : real(0.0);
        const real dz_p1 = (k + 1 < nz) ? g.dz(P, k + 1, m3_p1) : real(0.0);
        const real bottom_m1 = (k > 0 && m3_m1 > real(0.0) && m3k == real(0.0)) ? real(1.0) : real(0.0);
        const real bottom_k = (m3k > real(0.0) && m3_p1 == real(0.0)) ? real(1.0) : real(0.0);
        const real w_k1 = w[o + n2 + c];
        const real kh_k1 = kh[o + n2 + c];
        const real inv = inv_pos(dzk);
#pragma unroll
        for (int f = 0; f < 2; ++f) {
            if (f >= nf) break;
            const real* __restrict__ C = f == 0 ? C0 : S;
            const real fp2 = (k + 2 < nz) ? C[o + 2 * n2 + c] : real(0.0);
            const real surf = ts ? (f == 0 ? P.flux_t : P.flux_s) : real(0.0);
            real tend = ts ? real(0.0) : P.neg_n2 * (real(0.5) * (w_k + w_k1));
            real fbot = real(0.0);
            if (adv) {
                fbot = tracer_vface(P, g, k + 1, fm1[f], f0[f], fp1[f], fp2, w_k1);
                const real hdiv = ((sfx[f][ty][tx + 1] - sfx[f][ty][tx]) / P.dx +
                                     (sfy[f][ty + 1][tx] - sfy[f][ty][tx]) / P.dy) *
                                    inv;
                const real vdiv = (w_k * ftop[f] - w_k1 * fbot) * inv;
                tend = tend - (hdiv + vdiv) * m3k;
            }
            if (P.k_h > real(0.0)) {
                Nbr nb;
                nb.init(wrapi(i, nx), wrapi(j, ny), nx, ny);
                tend = tend + P.k_h * hlap(P, nb, C, k, 2);
            }
            // explicit vertical diffusion with zero drag (vertical_var.py:80-106)
            const real diff = explicit_dz(P, k, k > 0 ? fm1[f] : real(0.0), f0[f], k + 1 < nz ? fp1[f] : real(0.0), kh_k,
                                            kh_k1, dz_m1, dzk, dz_p1, bottom_m1, bottom_k, m3k, surf, real(0.0));
            real rhs = f0[f] + P.dt * tend + P.c3 * diff;
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
__global__ void __launch_bounds__(128) k_tracer_solve(KPR P, const real* __restrict__ rT,
                                                      const real* __restrict__ rS,
                                                      const real* __restrict__ kh,
                                                      real* __restrict__ T_out,
                                                      real* __restrict__ S_out,
                                                      wide* __restrict__ b_out) {
    COLUMN_PROLOGUE
    const int nz = P.nz;
    const int c = nb.c;
    const ColGeoR g = ColGeoR::load(P, c);
    real cs[NZM];
    const bool ts = P.tracers_ts;
#ifdef OC_MIXED
    real* __restrict__ o1 = T_out;  // the mixed path carries T and S (checked on the host)
    const ColGeo64 g64 = ColGeo64::load(P, c);
#else
    real* __restrict__ o1 = ts ? T_out : b_out;
#endif
    real m3_k, dz_k = g.dz(P, 0, m3_k);
    real dzi_k = dz_k;
    real kh_k = kh[c];
    real d1 = real(0.0), d2 = real(0.0), cp = real(0.0);
#pragma unroll 4
    for (int k = 0; k < nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        const real kh_k1 = kh[o + n2];
        real m3_k1 = real(0.0), dz_k1 = real(0.0);
        if (k + 1 < nz) dz_k1 = g.dz(P, k + 1, m3_k1);
        const real dzi_k1 = (k + 1 < nz) ? real(0.5) * (dz_k + dz_k1) : dz_k;
        const real r1 = rT[o];
        const real r2 = ts ? rS[o] : real(0.0);
        real sub, diag, sup;
        implicit_row(P, k, dz_k, m3_k, m3_k1, dzi_k, dzi_k1, kh_k, kh_k1, P.thv_dt_zero, sub, diag, sup);
        if (k == 0) {
            cp = sup / diag;
            d1 = r1 / diag;
            d2 = r2 / diag;
        } else {
            const real den = diag - sub * cp;
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
    real x1 = d1, x2 = d2;
#pragma unroll 4
    for (int k = nz - 1; k >= 0; --k) {
        const size_t o = (size_t)k * n2 + c;
        if (k < nz - 1) {
            x1 = o1[o] - cs[k] * x1;
            if (ts) x2 = S_out[o] - cs[k] * x2;
        }
        real m3;
        const real dz = g.dz(P, k, m3);
        if (ts) {
            const real Tn = x1 * m3;
            const real Sn = x2 * m3;
#ifdef OC_MIXED
            const wide zc = g64.above(P, k) + 0.5 * g64.dz(P, k);
#else
            const wide zc = col_above(P, c, k) + real(0.5) * dz;
#endif
            T_out[o] = Tn;
            S_out[o] = Sn;
            b_out[o] = buoyancy_of(P, wide(Tn), wide(Sn), zc) * wide(m3);  // EOS in fp64 on both paths
        } else {
            b_out[o] = wide(x1 * m3);
        }
    }
}


// diagnose b = EOS(T, S, zc) * m3 on the model grid (initial states)
__global__ void k_diag_buoyancy(KPR P, const real* __restrict__ T, const real* __restrict__ S,
                                wide* __restrict__ b) {
    COLUMN_PROLOGUE
    const size_t c = nb.c;
#ifdef OC_MIXED
    const ColGeo64 g64 = ColGeo64::load(P, (int)c);
    for (int k = 0; k < P.nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        const wide dz = g64.dz(P, k);
        const wide zc = g64.above(P, k) + 0.5 * dz;
        b[o] = buoyancy_of(P, wide(T[o]), wide(S[o]), zc) * (k < g64.kb ? 1.0 : 0.0);
    }
#else
    real above = real(0.0);
    for (int k = 0; k < P.nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        real m3;
        const real dz = col_dz(P, (int)c, k, m3);
        const real zc = above + real(0.5) * dz;
        above = (k == 0) ? dz : above + dz;
        b[o] = buoyancy_of(P, T[o], S[o], zc) * m3;
    }
#endif
}

// ------------------------------------------------------------------ transports
// depth-integrated transports sum_k dz3u u, sum_k dz3v v (fp64 sums on both paths)
__global__ void k_transport(KPR P, const real* __restrict__ u, const real* __restrict__ v,
                            wide* __restrict__ U, wide* __restrict__ V) {
    COLUMN_PROLOGUE
    const size_t c = nb.c;
    const ColGeoR gc = ColGeoR::load(P, (int)c), ge = ColGeoR::load(P, nb.at(0, 1)), gn = ColGeoR::load(P, nb.at(1, 0));
    const int2 kf = P.kface[c];
    wide su = 0.0, sv = 0.0;
#pragma unroll 4
    for (int k = 0; k < P.nz; ++k) {
        const size_t o = (size_t)k * n2 + c;
        real m;
        const real dzc = gc.dz(P, k, m);
        const real tu = face_dz(P, kf.x, k, dzc, ge.dz(P, k, m)) * u[o];
        const real tv = face_dz(P, kf.y, k, dzc, gn.dz(P, k, m)) * v[o];
        su = (k == 0) ? wide(tu) : su + wide(tu);
        sv = (k == 0) ? wide(tv) : sv + wide(tv);
    }
    U[c] = su;
    V[c] = sv;
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
void launch_qsolve(const KPR& P, const real* km, real* q, cudaStream_t s) {
    NZ_DISPATCH(P.nz, (k_qsolve<NZM><<<col_grid(P), col_block(), 0, s>>>(P, km, q)));
}
template <int NZM>
static void closure_nzm(const KPR& P, const real* u, const real* v, const wide* b, real* e, real* km, real* kh,
                        real* q, cudaStream_t s) {
    const dim3 blk = col_block();
#ifdef OC_MIXED
    const size_t smem = (size_t)(P.nz + 1) * blk.x * blk.y * sizeof(real);
    // above 48 KB a kernel's dynamic shared memory is opt-in, once per device
    static std::atomic<unsigned long long> opted{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ULL << (dev & 63);
    if (!(opted.load() & bit)) {
        cudaFuncSetAttribute(k_closure<NZM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)((size_t)(NZM + 1) * blk.x * blk.y * sizeof(real)));
        opted.fetch_or(bit);
    }
#else
    const size_t smem = 0;
#endif
    k_closure<NZM><<<col_grid(P), blk, smem, s>>>(P, u, v, b, e, km, kh, q);
}
void launch_closure(const KPR& P, const real* u, const real* v, const wide* b, real* e,
                    real* km, real* kh, real* q, cudaStream_t s) {
    NZ_DISPATCH(P.nz, (closure_nzm<NZM>(P, u, v, b, e, km, kh, q, s)));
}
void launch_kukv(const KPR& P, const real* q, wide* Ku, wide* Kv, cudaStream_t s) {
    k_kukv<<<col_grid(P), col_block(), 0, s>>>(P, q, Ku, Kv);
}
void launch_wcol(const KPR& P, const real* u, const real* v, real* w, cudaStream_t s) {
    k_wcol<<<col_grid(P), col_block(), 0, s>>>(P, u, v, w);
}
void launch_phi(const KPR& P, const wide* b, wide* phi, cudaStream_t s) {
    k_phi<<<col_grid(P), col_block(), 0, s>>>(P, b, phi);
}
static dim3 cell_block() { return dim3(32, 8, 1); }
static dim3 cell_grid(const KPR& P) { return dim3((P.nx + 31) / 32, (P.ny + 7) / 8, P.nz); }
void launch_mom_explicit(const KPR& P, const real* u, const real* v, const wide* b,
                         const wide* phi, const real* w, const real* km, real* pgx,
                         real* pgy, real* avpv, real* avpu, real* dzu, real* dzv,
                         real* stu, real* stv, cudaStream_t s) {
    const dim3 grid((P.nx + MOM_TX - 1) / MOM_TX, (P.ny + MOM_TY - 1) / MOM_TY, (P.nz + P.mom_kl - 1) / P.mom_kl);
    k_mom_column<<<grid, dim3(MOM_TX, MOM_TY, 2), 0, s>>>(P, u, v, b, phi, w, km, pgx, pgy, avpv, avpu, dzu, dzv, stu,
                                             stv);
}
void launch_predictor_rhs(const KPR& P, const real* u, const real* v, const real* u_it,
                          const real* v_it, const real* pgx, const real* pgy, const real* avpv,
                          const real* avpu, const real* dzu, const real* dzv, const real* stu,
                          const real* stv, const wide* gx2, const wide* gy2, real* ru, real* rv,
                          cudaStream_t s) {
    k_predictor_rhs<<<cell_grid(P), cell_block(), 0, s>>>(P, u, v, u_it, v_it, pgx, pgy, avpv, avpu, dzu,
                                                          dzv, stu, stv, gx2, gy2, ru, rv);
}
void launch_momentum_solve(const KPR& P, const real* km, real* ghu, real* ghv, wide* Ug, wide* Vg,
                           cudaStream_t s) {
    NZ_DISPATCH(P.nz, (k_momentum_solve<NZM><<<col_grid(P), col_block(), 0, s>>>(P, km, ghu, ghv, Ug, Vg)));
}
void launch_backsub(const KPR& P, const real* ghu, const real* ghv, const real* q,
                    const wide* eta_new, real* u_out, real* v_out, cudaStream_t s) {
    k_backsub<<<col_grid(P), col_block(), 0, s>>>(P, ghu, ghv, q, eta_new, u_out, v_out);
}
void launch_tracer_rhs(const KPR& P, const real* C0, const real* S, const real* u, const real* v,
                       const real* w, const real* kh, real* rT, real* rS, cudaStream_t s) {
    const dim3 grid((P.nx + TRX - 1) / TRX, (P.ny + TRY - 1) / TRY, (P.nz + P.tr_kl - 1) / P.tr_kl);
    k_tracer_rhs<<<grid, dim3(TRX, TRY), 0, s>>>(P, C0, S, u, v, w, kh, rT, rS);
}
void launch_tracer_solve(const KPR& P, const real* rT, const real* rS, const real* kh,
                         real* T_out, real* S_out, wide* b_out, cudaStream_t s) {
    NZ_DISPATCH(P.nz, (k_tracer_solve<NZM><<<col_grid(P), col_block(), 0, s>>>(P, rT, rS, kh, T_out,
                                                                             S_out, b_out)));
}
void launch_diag_buoyancy(const KPR& P, const real* T, const real* S, wide* b, cudaStream_t s) {
    k_diag_buoyancy<<<col_grid(P), col_block(), 0, s>>>(P, T, S, b);
}
void launch_transport(const KPR& P, const real* u, const real* v, wide* U, wide* V,
                      cudaStream_t s) {
    k_transport<<<col_grid(P), col_block(), 0, s>>>(P, u, v, U, V);
}

}  // namespace oc
