// fhd_vec.cuh -- Stokes-vector kernels: the fused saddle-point operator,
// preconditioner glue, deterministic reductions and the Gram-Schmidt steps
// of GMRES.
#pragma once
#include "fhd_kernels.cuh"

namespace fhd {

// A Stokes vector (u_0 .. u_{dim-1}, p): component pointers, p at [dim].
template <typename T>
struct SVec {
    T* c[4];
};
template <typename T>
struct CSVec {
    const T* c[4];
};

// ---------------------------------------------------------------------
// deterministic reductions: grid-stride partial sums, a warp-shuffle tree
// per block, one partial per block, and the last block to finish adds the
// partials in block order.  The result lands in device memory so that
// following kernels can consume it without a host round trip.
// ---------------------------------------------------------------------
constexpr int RED_THREADS = 256;
constexpr int RED_MAX_BLOCKS = 1184;  // 8 blocks per SM on 148 SMs

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double block_sum(double v, double* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    const int nw = blockDim.x >> 5;
    v = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
    if (wid == 0) v = warp_sum(v);
    __syncthreads();
    return v;  // valid in thread 0
}

struct RedSlot {
    double* partials;    // RED_MAX_BLOCKS entries
    unsigned* counter;   // zero between uses
    double* out;
};

__device__ __forceinline__ void red_finish(double v, RedSlot rs) {
    __shared__ double sh[32];
    __shared__ bool last;
    v = block_sum(v, sh);
    if (threadIdx.x == 0) {
        rs.partials[blockIdx.x] = v;
        __threadfence();
        const unsigned t = atomicAdd(rs.counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double s = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) s += ((volatile double*)rs.partials)[b];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) {
        *rs.out = s;
        *rs.counter = 0u;
    }
}

// sum_c w_c * sum_f a_c[f] b_c[f]; weights: 1 for velocity, wp for p
template <typename TA, typename TB>
static __global__ void __launch_bounds__(RED_THREADS) k_sdot(i64 n, int ncomp, CSVec<TA> a, CSVec<TB> b, double wlast,
                                                      RedSlot rs) {
    double s = 0.0;
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x) {
        double su = 0.0;
        for (int c = 0; c < ncomp - 1; c++) su += (double)a.c[c][f] * (double)b.c[c][f];
        const int c = ncomp - 1;
        su += wlast * ((double)a.c[c][f] * (double)b.c[c][f]);
        s += su;
    }
    red_finish(s, rs);
}

// sum_f a[f]
template <typename T>
static __global__ void __launch_bounds__(RED_THREADS) k_sum(i64 n, const T* a, RedSlot rs) {
    double s = 0.0;
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x) s += (double)a[f];
    red_finish(s, rs);
}

// Modified Gram-Schmidt step (gmres.f90:352-378), fused: w -= h*vprev with
// h read from device memory, then the weighted dot of the updated w with
// vnext (or with itself when vnext is null).
static __global__ void __launch_bounds__(RED_THREADS) k_mgs(i64 n, int ncomp, SVec<double> w, CSVec<double> vprev,
                                                     const double* hprev, CSVec<double> vnext, double wp2,
                                                     RedSlot rs) {
    const double h = hprev ? *hprev : 0.0;
    double s = 0.0;
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x) {
        double su = 0.0;
        for (int c = 0; c < ncomp; c++) {
            double x = w.c[c][f];
            if (hprev) {
                x = x - vprev.c[c][f] * h;
                w.c[c][f] = x;
            }
            const double y = vnext.c[0] ? vnext.c[c][f] : x;
            const double t = x * y;
            su += (c == ncomp - 1) ? wp2 * t : t;
        }
        s += su;
    }
    red_finish(s, rs);
}

// v = w / sqrt(nrm2)  (gmres.f90:380-389 with H(i+1,i) = sqrt(nrm2))
// (every component of an element is loaded before any is stored, so a
// thread keeps ncomp loads in flight although v and w may alias)
static __global__ void __launch_bounds__(256) k_scale_by_norm(i64 n, int ncomp, SVec<double> v, CSVec<double> w,
                                                       const double* nrm2) {
    const double h = sqrt(*nrm2);
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x) {
        double a[4];
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (c < ncomp) a[c] = w.c[c][f];
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (c < ncomp) v.c[c][f] = a[c] / h;
    }
}

// v = w / s (host scalar)
static __global__ void __launch_bounds__(256) k_scale_div(i64 n, int ncomp, SVec<double> v, CSVec<double> w, double s) {
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x) {
        double a[4];
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (c < ncomp) a[c] = w.c[c][f];
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (c < ncomp) v.c[c][f] = a[c] / s;
    }
}

// x += sum_{it < m} y[it] v_it (update_sol, gmres.f90:495-529; same order)
static __global__ void __launch_bounds__(256) k_update_sol(i64 n, int ncomp, SVec<double> x, const double* __restrict__ V,
                                                    i64 vstride, const double* y, int m) {
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x) {
        // all components advance together (each in the order of update_sol),
        // so the loads of every component are in flight at once
        double acc[4];
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (c < ncomp) acc[c] = x.c[c][f];
        for (int it = 0; it < m; it++) {
            const double yi = y[it];
#pragma unroll
            for (int c = 0; c < 4; c++)
                if (c < ncomp) acc[c] = acc[c] + V[it * vstride + (i64)c * n + f] * yi;
        }
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (c < ncomp) x.c[c][f] = acc[c];
    }
}

template <typename TO, typename TI>
static __global__ void __launch_bounds__(256) k_copy_conv(i64 n, TO* __restrict__ o, const TI* __restrict__ in, double s) {
    // four grid strides per pass: four loads in flight per thread
    const i64 st = (i64)gridDim.x * blockDim.x;
    i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    for (; f + 3 * st < n; f += 4 * st) {
        TI a[4];
#pragma unroll
        for (int u = 0; u < 4; u++) a[u] = in[f + u * st];
#pragma unroll
        for (int u = 0; u < 4; u++) o[f + u * st] = (TO)((double)a[u] * s);
    }
    for (; f < n; f += st) o[f] = (TO)((double)in[f] * s);
}

template <typename T>
static __global__ void __launch_bounds__(256) k_sub_mean(i64 n, T* a, const double* sum, double count) {
    const double m = (*sum) / count;
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x)
        a[f] = (T)((double)a[f] - m);
}

template <typename T>
static __global__ void __launch_bounds__(256) k_fill(i64 n, T* a, T v) {
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x) a[f] = v;
}

template <typename T>
static __global__ void __launch_bounds__(256) k_recip(i64 n, T* o, const double* a) {
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x)
        o[f] = (T)(1.0 / a[f]);
}

// ---------------------------------------------------------------------
// saddle-point operator, one pass (apply_matrix.f90:117-147):
//   b_u = (alpha_scale*alpha - L) x_u + G x_p ;  b_p = -D x_u
// mode 1 returns rhs - A x instead (the GMRES residual, gmres.f90:205-213).
// ---------------------------------------------------------------------
template <int DIM, int VISC>
static __global__ void __launch_bounds__(256) k_stokes_apply(Grid g, StagOp<double> A, CSVec<double> x, CSVec<double> rhs,
                                                      SVec<double> out, int mode, double dxinv) {
    CellF P;
    if (!cellf_of_thread(g, P)) return;
    const double* phi[3] = {x.c[0], x.c[1], DIM == 3 ? x.c[2] : nullptr};
    const double* p = x.c[DIM];
    const i64 f = P.id(0, 0, 0);
    const double pc = ld(p, f);
    double div = 0.0;
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        const int dx_ = (c == 0), dy_ = (c == 1), dz_ = (c == 2);
        double dg;
        double L = stag_lface_c<double, DIM, VISC>(c, A, phi, P, dg);
        const double gp = (pc - ld(p, P.id(-dx_, -dy_, -dz_))) * dxinv;
        L = L + gp;
        out.c[c][f] = mode ? ld(rhs.c[c], f) - L : L;
        div += (ld(phi[c], P.id(dx_, dy_, dz_)) - ld(phi[c], f)) * dxinv;
    }
    const double bp = div * -1.0;
    out.c[DIM][f] = mode ? ld(rhs.c[DIM], f) - bp : bp;
}

// the same with gmres_spatial_order = 4 (apply_matrix.f90:124-135): the
// visc_type 1 operator of stag_applyop_4o_2d/_3d (stag_applyop.f90:1262-1510,
// per direction +16 phi(+-1) - phi(+-2) over 12 dx^2, diagonal 30 dim over
// 12 dx^2) and the gradient of compute_grad_4o (div_and_grad.f90:804-880,
// (-p(+1) + 15 p - 15 p(-1) + p(-2)) / 12 dx); the divergence stays second
// order.  Terms summed in the order of those loops.  The constant viscosity
// is the first cell's (stag_applyop.f90:1306); t2 = 1/(12 dx^2),
// t1 = 1/(12 dx).
template <int DIM>
static __global__ void __launch_bounds__(256) k_stokes_apply4(Grid g, StagOp<double> A, CSVec<double> x,
                                                              CSVec<double> rhs, SVec<double> out, int mode,
                                                              double dxinv, double t1, double t2) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const double b = ld(A.beta, 0);
    const double* p = x.c[DIM];
    const i64 f = P.id(0, 0, 0);
    const double cdiag = DIM == 2 ? 60.0 : 90.0;
    double div = 0.0;
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        const double* u = x.c[c];
        double s = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
            const double t = 16.0 * ld(u, P.id(e0, e1, e2));
            s = d == 0 ? t : s + t;
            s = s + 16.0 * ld(u, P.id(-e0, -e1, -e2));
            s = s - 1.0 * ld(u, P.id(2 * e0, 2 * e1, 2 * e2));
            s = s - 1.0 * ld(u, P.id(-2 * e0, -2 * e1, -2 * e2));
        }
        const double a = A.alpha_scale * ld(A.alpha[c], f);
        double L = (a + cdiag * b * t2) * ld(u, f) - s * b * t2;
        const int e0 = c == 0, e1 = c == 1, e2 = c == 2;
        const double gp = (-ld(p, P.id(e0, e1, e2)) + 15.0 * ld(p, f) - 15.0 * ld(p, P.id(-e0, -e1, -e2)) +
                           ld(p, P.id(-2 * e0, -2 * e1, -2 * e2))) *
                          t1;
        L = L + gp;
        out.c[c][f] = mode ? ld(rhs.c[c], f) - L : L;
        div += (ld(u, P.id(e0, e1, e2)) - ld(u, f)) * dxinv;
    }
    const double bp = div * -1.0;
    out.c[DIM][f] = mode ? ld(rhs.c[DIM], f) - bp : bp;
}

// mac_rhs = D x_u + b_p  (apply_precon.f90:118-123)
template <typename T, int DIM>
static __global__ void __launch_bounds__(256) k_div_plus(Grid g, const T* u0, const T* u1, const T* u2, const double* bp,
                                                  T* out, T dxinv) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
    T s = (ld(u0, P.id(1, 0, 0)) - ld(u0, f)) * dxinv + (ld(u1, P.id(0, 1, 0)) - ld(u1, f)) * dxinv;
    if constexpr (DIM == 3) s += (ld(u2, P.id(0, 0, 1)) - ld(u2, f)) * dxinv;
    out[f] = bp ? s + (T)bp[f] : s;
}

// mu^-1 = 1 / diagonal of the viscous operator on the faces
// (inverse_diag_lap.f90:17-330), evaluated in FP64 in the summation order of
// its 2D and 3D loops; visc_type 1 / 2 take the first cell's beta
template <typename T, int DIM>
static __global__ void __launch_bounds__(256) k_inv_diag_lap(Grid g, int visc, const double* beta, const double* be0,
                                                      const double* be1, const double* be2, T* o0, T* o1, T* o2) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
    T* out[3] = {o0, o1, o2};
    if (visc == 1 || visc == 2) {
        const double m = (DIM == 2 ? (visc == 1 ? 4.0 : 6.0) : (visc == 1 ? 6.0 : 8.0)) * beta[0];
#pragma unroll
        for (int c = 0; c < DIM; c++) out[c][f] = (T)(1.0 / m);
        return;
    }
    const double cb = visc == -2 ? 2.0 : 1.0;
    const double* be[3] = {be0, be1, be2};
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        double s = cb * beta[f] + cb * beta[P.id(-(c == 0), -(c == 1), -(c == 2))];
        if constexpr (DIM == 2) {
            // x face: node (i, j+1) then (i, j); y face: (i+1, j) then (i, j)
            s = s + be0[c == 0 ? P.id(0, 1, 0) : P.id(1, 0, 0)];
            s = s + be0[f];
        } else {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                if (d == c) continue;
                const int e = (c + d == 1) ? 0 : (c + d == 2) ? 1 : 2;  // xy, xz, yz
                s = s + be[e][f];
                s = s + be[e][P.id(d == 0, d == 1, d == 2)];
            }
        }
        out[c][f] = (T)(1.0 / s);
    }
}

// out_d = (G Phi)_d * w_d on the faces (compute_grad, div_and_grad.f90:
// 417-703, then the face product of visc_schur_complement)
template <typename T, int DIM>
static __global__ void __launch_bounds__(256) k_grad_mul(Grid g, const T* Phi, const T* w0, const T* w1, const T* w2,
                                                  T* o0, T* o1, T* o2, T dxinv) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
    const T* w[3] = {w0, w1, w2};
    T* out[3] = {o0, o1, o2};
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        const T gp = (Phi[f] - Phi[P.id(-(d == 0), -(d == 1), -(d == 2))]) * dxinv;
        out[d][f] = gp * w[d][f];
    }
}

// a_c *= w_c on the faces
template <typename T>
static __global__ void __launch_bounds__(256) k_mul_faces(i64 n, int ncomp, T* a0, T* a1, T* a2, const T* w0,
                                                   const T* w1, const T* w2) {
    T* a[3] = {a0, a1, a2};
    const T* w[3] = {w0, w1, w2};
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x)
        for (int c = 0; c < ncomp; c++) a[c][f] = a[c][f] * w[c][f];
}

// x_p = Phi_mu (+ theta Phi when add), negated on request
// (visc_schur_complement's output, apply_precon.f90:664-683)
template <typename T>
static __global__ void __launch_bounds__(256) k_bfbt_out(i64 n, double* xp, const T* phimu, const T* phi,
                                                  double theta, int add, int negate) {
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x) {
        double v = (double)phimu[f];
        if (add) v = v + (double)phi[f] * theta;
        xp[f] = negate ? v * -1.0 : v;
    }
}

// x_u = phi - w * G Phi (subtract_weighted_gradp, macproject.f90:318-362),
// written to FP64 output (w = alphainv or 1 when null)
template <typename T, int DIM>
static __global__ void __launch_bounds__(256) k_sub_wgrad(Grid g, const T* phi0, const T* phi1, const T* phi2,
                                                   const T* w0, const T* w1, const T* w2, const T* Phi, double* o0,
                                                   double* o1, double* o2, T dxinv) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
    const T pc = ld(Phi, f);
    const T* ph[3] = {phi0, phi1, phi2};
    const T* w[3] = {w0, w1, w2};
    double* o[3] = {o0, o1, o2};
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        const int dx_ = (c == 0), dy_ = (c == 1), dz_ = (c == 2);
        T gp = (pc - ld(Phi, P.id(-dx_, -dy_, -dz_))) * dxinv;
        if (w[c]) gp = gp * ld(w[c], f);
        o[c][f] = (double)(ld(ph[c], f) + T(-1) * gp);
    }
}

// T-precision variant writing into T arrays (b_u - G x_p for precon 3/5)
template <typename T, int DIM>
static __global__ void __launch_bounds__(256) k_sub_grad_T(Grid g, const double* b0, const double* b1, const double* b2,
                                                    const double* xp, T* o0, T* o1, T* o2, double dxinv) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
    const double pc = xp[f];
    const double* b[3] = {b0, b1, b2};
    T* o[3] = {o0, o1, o2};
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        const int dx_ = (c == 0), dy_ = (c == 1), dz_ = (c == 2);
        const double gp = (pc - xp[P.id(-dx_, -dy_, -dz_)]) * dxinv;
        o[c][f] = (T)(b[c][f] + (-1.0) * gp);
    }
}

// Schur-complement pressure update (apply_precon.f90:140-195 and
// simple_schur_complement 479-534) into FP64 x_p.
//   kind 0: x_p = c*beta*(-mac_rhs) [+ gamma part] + theta*Phi
//   kind 1: precon_type = -1: -L_alpha Phi in place of -mac_rhs
// negate: multiply by -1 at the end (precon_type -2/-5)
template <typename T, int DIM>
static __global__ void __launch_bounds__(256) k_schur(Grid g, CCOp<T> A, const T* mac_rhs, const T* Phi, const double* beta,
                                               const double* gamma, double theta, int av, int kind, int add_phi,
                                               int negate, double* xp) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
    double v;
    if (kind == 1) {
        T dg;
        v = -(double)cc_lap<T, DIM>(A, Phi, P, dg);
    } else {
        v = (double)mac_rhs[f] * -1.0;
    }
    if (av == 1 || av == 2) {
        v = v * beta[f];
        if (av == 2) v = v * 2.0;
    } else {
        const double m = v * gamma[f];
        v = v * beta[f];
        v = v * (4.0 / 3.0);
        v = v + m;
    }
    if (add_phi) v = v + (double)Phi[f] * theta;
    if (negate) v = v * -1.0;
    xp[f] = v;
}

// block-diagonal pressure update (apply_precon.f90:378-416)
static __global__ void __launch_bounds__(256) k_schur_blockdiag(i64 n, const double* bp, const double* beta,
                                                         const double* gamma, const double* Phi, double theta,
                                                         int use_phi, int av, int pt, double* xp) {
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x) {
        double ph = use_phi ? Phi[f] * theta : 0.0;
        double v = bp[f] * beta[f];
        v = v - ph;
        if (av == 1 && pt == 4) v = v * -1.0;
        else if (av == 2 && pt == 4) v = v * -2.0;
        else if (av == 2 && pt == -4) v = v * 2.0;
        else if (av == 3 && pt == 4) { v = v * (-4.0 / 3.0); v = v + (bp[f] * gamma[f]) * -1.0; }
        else if (av == 3 && pt == -4) { v = v * (4.0 / 3.0); v = v + bp[f] * gamma[f]; }
        xp[f] = v;
    }
}

}  // namespace fhd
