// fhd_walls.cuh -- homogeneous domain walls (zero wall velocity) for the
// staggered Stokes solve with visc_type 1, 2 or 3 (constant coefficients): no-slip
// and slip walls in any direction, the other directions periodic.
//
// The reference imposes walls through ghost cells, refilled after every
// operation of the solve (multifab_physbc_domainvel / multifab_physbc_macvel,
// multifab_physbc_stag.f90:91-1116; stag_mg_solver.f90:360-440, 655-740):
//   * the velocity normal to a wall is zero on the wall face and behind it;
//   * the transverse velocity behind a wall is the first interior value,
//     negated at a no-slip wall and kept at a slip wall;
//   * Lphi, the smoother updates and the restricted residual are zero on the
//     wall faces; the pressure gradient there is zero (first-order
//     extrapolated pressure ghost, div_and_grad.f90:540-556).
// Here the arrays keep the periodic layout (n faces per direction): in a wall
// direction face 0 is the low wall face, held at zero, and the high wall face
// (index n) is not stored; reads of it give zero.  The ghost values come from
// wall_vel at the read.  The pressure multigrid sees walls as faces of zero
// coefficient (no flux), which its periodic index wrap then applies to both
// walls, so its kernels are unchanged.
#pragma once
#include "fhd_kernels.cuh"
#include "fhd_vec.cuh"

namespace fhd {

// per direction and side: 0 periodic; -1 no-slip wall, +1 slip wall (the
// sign of the transverse velocity behind the wall)
struct Walls {
    int lo[3], hi[3];
};

__device__ __forceinline__ bool on_wall(const Walls& W, int c, int i, int j, int k) {
    const int q[3] = {i, j, k};
    return W.lo[c] != 0 && q[c] == 0;
}

// component c at face (i, j, k), possibly one face past the domain
template <typename T, int DIM>
__device__ __forceinline__ T wall_vel(const Grid& g, const Walls& W, const T* u, int c, int i, int j, int k) {
    int q[3] = {i, j, k};
    T sg = T(1);
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        if (W.lo[d] == 0) {
            q[d] = wrapc(q[d], g.n[d]);
        } else if (q[d] < 0) {
            if (d == c) return T(0);
            if (W.lo[d] < 0) sg = -sg;
            q[d] = 0;
        } else if (q[d] >= g.n[d]) {
            if (d == c) return T(0);
            if (W.hi[d] < 0) sg = -sg;
            q[d] = g.n[d] - 1;
        }
    }
    return sg * ld(u, (i64)q[0] + (i64)g.n[0] * ((i64)q[1] + (i64)g.n[1] * (DIM == 3 ? q[2] : 0)));
}

// (theta alpha - L) phi of component C at face (i, j, k), constant
// coefficients, visc_type 1, 2 or 3: the expression of stag_lface_acc with every
// neighbour under the wall rules (visc_type 2 and 3 also read the other
// components around the face: their values on and behind a wall come from
// wall_vel as well, as the reference's ghost cells give them to the uniform
// stencil of stag_applyop_level)
template <typename T, int DIM, int VISC, int C>
__device__ __forceinline__ T stag_lface_w(const Grid& g, const Walls& W, const StagOp<T>& A, const T* const* phi,
                                          int i, int j, int k, T& dg) {
    static_assert(VISC >= 1 && VISC <= 3, "walls: visc_type 1, 2 or 3");
    CellF P;
    P.set(g, i, j, k);
    const T* pc = phi[C];
    return stag_lface_acc<T, DIM, VISC, C>(
        A, P,
        [&](int a, int b, int c) {
            return (a == 0 && b == 0 && c == 0) ? ld(pc, P.base) : wall_vel<T, DIM>(g, W, pc, C, i + a, j + b, k + c);
        },
        [&](int d, int a, int b, int c) { return wall_vel<T, DIM>(g, W, phi[d], d, i + a, j + b, k + c); },
        [&]() { return ld(A.alpha[C], P.base); }, dg);
}

template <typename T, int DIM, int VISC>
__device__ __forceinline__ T stag_lface_w_c(int c, const Grid& g, const Walls& W, const StagOp<T>& A,
                                            const T* const* phi, int i, int j, int k, T& dg) {
    if (c == 0) return stag_lface_w<T, DIM, VISC, 0>(g, W, A, phi, i, j, k, dg);
    if (DIM == 3 && c == 2) return stag_lface_w<T, DIM, VISC, (DIM == 3 ? 2 : 1)>(g, W, A, phi, i, j, k, dg);
    return stag_lface_w<T, DIM, VISC, 1>(g, W, A, phi, i, j, k, dg);
}

// first pass of a colour (stag_applyop_level(colour) of stag_mg_solver.f90:
// 360-396): Lphi and the diagonal of the colour's faces into Lo, Do.  A wall
// face gets Lo = rhs, Do = 1, so that k_stag_color_update leaves it at zero.
template <typename T, int DIM, int VISC>
__global__ void __launch_bounds__(256) k_stag_color_apply_w(Grid g, Walls W, StagOp<T> A, const T* p0, const T* p1,
                                                            const T* p2, const T* r0, const T* r1, const T* r2,
                                                            T* L0, T* L1, T* L2, T* D0, T* D1, T* D2, int color) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const T* ph[3] = {p0, p1, p2};
    const T* rh[3] = {r0, r1, r2};
    T* Lo[3] = {L0, L1, L2};
    T* Do[3] = {D0, D1, D2};
    const i64 f = P.id(0, 0, 0);
    const int par = (P.i + P.j + P.k) & 1;
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        if ((color - 1) / 2 != c || par != ((color + 1) & 1)) continue;
        if (on_wall(W, c, P.i, P.j, P.k)) {
            Lo[c][f] = rh[c][f];
            Do[c][f] = T(1);
            continue;
        }
        T dg;
        Lo[c][f] = stag_lface_w_c<T, DIM, VISC>(c, g, W, A, ph, P.i, P.j, P.k, dg);
        Do[c][f] = dg;
    }
}

// residual rhs - (theta alpha - L) phi (mode 1) or Lphi (mode 0), zero on
// the wall faces
template <typename T, int DIM, int VISC>
__global__ void __launch_bounds__(256) k_stag_apply_w(Grid g, Walls W, StagOp<T> A, const T* p0, const T* p1,
                                                      const T* p2, T* o0, T* o1, T* o2, const T* r0, const T* r1,
                                                      const T* r2, int mode) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const T* phi[3] = {p0, p1, p2};
    T* out[3] = {o0, o1, o2};
    const T* rhs[3] = {r0, r1, r2};
    const i64 f = P.id(0, 0, 0);
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        if (on_wall(W, c, P.i, P.j, P.k)) {
            out[c][f] = T(0);
            continue;
        }
        T dg;
        const T L = stag_lface_w_c<T, DIM, VISC>(c, g, W, A, phi, P.i, P.j, P.k, dg);
        out[c][f] = mode ? ld(rhs[c], f) - L : L;
    }
}

// fine += P coarse (stag_prolongation, stag_mg_solver.f90:1365-1628), thread
// per fine face, the coarse neighbours under the wall rules; the fine wall
// faces are set to zero
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_stag_prolong_w(Grid gf, Grid gc, Walls W, T* f0, T* f1, T* f2, const T* c0,
                                                        const T* c1, const T* c2) {
    Cell P;
    if (!cell_of_thread(gf, P)) return;
    T* fo[3] = {f0, f1, f2};
    const T* ci[3] = {c0, c1, c2};
    const int I[3] = {P.i, P.j, P.k};
    const int h[3] = {P.i >> 1, P.j >> 1, P.k >> 1};
    const i64 f = P.id(0, 0, 0);
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        if (on_wall(W, c, P.i, P.j, P.k)) {
            fo[c][f] = T(0);
            continue;
        }
        const int a = (c == 0) ? 1 : 0;
        const int b = (c == 2) ? 1 : 2;
        const int oa = (I[a] & 1) ? 1 : -1;
        const int ob = (DIM == 3) ? ((I[b] & 1) ? 1 : -1) : 0;
        const T v = stag_prolong_expr<T, DIM>((I[c] & 1) == 0, oa, ob, [&](int o, int pa, int pb) {
            int q[3] = {h[0], h[1], h[2]};
            q[c] += o;
            q[a] += pa;
            if (DIM == 3) q[b] += pb;
            return wall_vel<T, DIM>(gc, W, ci[c], c, q[0], q[1], q[2]);
        });
        fo[c][f] = fo[c][f] + v;
    }
}

// zero the wall faces of a face vector (any of u0..u2 may be null)
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_zero_walls(Grid g, Walls W, T* u0, T* u1, T* u2) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    T* u[3] = {u0, u1, u2};
    const i64 f = P.id(0, 0, 0);
#pragma unroll
    for (int c = 0; c < DIM; c++)
        if (u[c] && on_wall(W, c, P.i, P.j, P.k)) u[c][f] = T(0);
}

// apply_matrix (apply_matrix.f90:117-147) with walls: zero Lphi and pressure
// gradient on the wall faces; mode 1 returns rhs - A x
template <int DIM, int VISC>
static __global__ void __launch_bounds__(256) k_stokes_apply_w(Grid g, Walls W, StagOp<double> A, CSVec<double> x,
                                                               CSVec<double> rhs, SVec<double> out, int mode,
                                                               double dxinv) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const double* phi[3] = {x.c[0], x.c[1], DIM == 3 ? x.c[2] : nullptr};
    const double* p = x.c[DIM];
    const i64 f = P.id(0, 0, 0);
    const double pc = ld(p, f);
    double div = 0.0;
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        const int dx_ = (c == 0), dy_ = (c == 1), dz_ = (c == 2);
        double L = 0.0;
        if (!on_wall(W, c, P.i, P.j, P.k)) {
            double dg;
            L = stag_lface_w_c<double, DIM, VISC>(c, g, W, A, phi, P.i, P.j, P.k, dg);
            const double gp = (pc - ld(p, P.id(-dx_, -dy_, -dz_))) * dxinv;
            L = L + gp;
        }
        out.c[c][f] = mode ? ld(rhs.c[c], f) - L : L;
        div += (ld(phi[c], P.id(dx_, dy_, dz_)) - ld(phi[c], f)) * dxinv;
    }
    const double bp = div * -1.0;
    out.c[DIM][f] = mode ? ld(rhs.c[DIM], f) - bp : bp;
}

// host dispatch of the wall kernels on the context's visc_type (1, 2 or 3)
template <class F>
inline void with_wall_visc(int visc, F&& f) {
    if (visc == 2) f(std::integral_constant<int, 2>());
    else if (visc == 3) f(std::integral_constant<int, 3>());
    else f(std::integral_constant<int, 1>());
}

}  // namespace fhd
