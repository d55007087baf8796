// Helpers shared by the step's 3D kernels (step_kernels.cu, compiled for the
// fp64 and the mixed-precision path) and its 2D kernels (step2d_kernels.cu).
#pragma once

#include "oc_internal.cuh"

namespace oc {

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

// asynchronous copy of one 4- or 8-byte element from global to shared memory
// (cp.async: no register round trip, so a level plane's staging runs while the
// previous level is computed); committed in groups, waited for by group
template <class T>
__device__ __forceinline__ void cp_async_elem(T* sdst, const T* gsrc) {
    static_assert(sizeof(T) == 4 || sizeof(T) == 8, "cp.async copies 4, 8 or 16 bytes");
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gsrc), "n"(sizeof(T)) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N of this thread's committed groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// a column's values strided across the threads of a CTA in shared memory
template <class T>
struct StridedCol {
    T* p;
    int stride;
    __device__ __forceinline__ T& operator[](int k) const { return p[k * stride]; }
};

#define COLUMN_PROLOGUE                                  \
    const int i = blockIdx.x * blockDim.x + threadIdx.x; \
    const int j = blockIdx.y * blockDim.y + threadIdx.y; \
    if (i >= P.nx || j >= P.ny) return;                  \
    Nbr nb;                                              \
    nb.init(i, j, P.nx, P.ny);                           \
    const size_t n2 = (size_t)P.n2;                      \
    (void)n2;

// face thickness at level k of a face whose wet levels are the top kf ones,
// between cells of thickness dza and dzb: mask3_face x face_combine(dza, dzb)
// (reference domain.py:93-96, 142-146)
template <class T>
__device__ __forceinline__ T face_dz(const KPT<T>& P, int kf, int k, T dza, T dzb) {
    return (k < kf ? T(1.0) : T(0.0)) * face_combine(P, dza, dzb);
}

// Row k of A = I - thv dt Dz for a column (reference vertical_var.py:35-77).
template <class real>
__device__ __forceinline__ void implicit_row(const KPT<real>& P, int k, real dzk, real m3k, real m3k1,
                                             real dzi_k, real dzi_k1, real Kk, real Kk1,
                                             real thv_dt_drag, real& sub, real& diag,
                                             real& sup) {
    const real inv_dz = inv_pos(dzk);
    const real fac = P.thv_dt * inv_dz;
    const real at = fac * Kk * inv_pos(dzi_k);
    const real ab = fac * Kk1 * inv_pos(dzi_k1);
    sub = -at;
    sup = -ab;
    diag = real(1.0) + at + ab;
    if (k == 0) {
        diag = real(1.0) + ab;
        sub = real(0.0);
    }
    if (m3k > real(0.0) && m3k1 == real(0.0)) {
        diag = real(1.0) + at + thv_dt_drag * inv_dz;
        sup = real(0.0);
    }
    if (m3k == real(0.0)) {
        diag = real(1.0);
        sub = real(0.0);
        sup = real(0.0);
    }
}

// one thread per column, 32 x 4 columns per CTA
static inline dim3 col_block() { return dim3(32, 4); }
template <class T>
static inline dim3 col_grid(const KPT<T>& P) { return dim3((P.nx + 31) / 32, (P.ny + 3) / 4); }

}  // namespace oc
