// fhd_step.cu -- stochastic momentum flux divergence and the device-resident
// inertial predictor-corrector step of a single-species fluid.
//
// stochastic_m_fluxdiv.f90:42-778 (homogeneous walls through mflux_bc; the
// stress filter of filtering_width 1, 2, 4 on periodic boxes) and
// advance_timestep_inertial.f90:45-923 (nspecies = 1, centred advection,
// no gravity; periodic boxes or homogeneous walls).
#include <cmath>
#include <cstring>

#include "fhd_solver.cuh"

namespace fhd {

struct StochArgs {
    const double* Wcc[4 * 3];  // n_rngs * dim
    const double* Wed[4 * 6];  // n_rngs * 2 * nE
    double wts[4];
    int n_rngs;
    const double* eta;
    const double* eta_ed[3];
    const double* T;
    const double* T_ed[3];
    double variance;
    double dxinv;
};

// scaled random stress at a cell (component c) or on an edge (edge set e,
// component comp): variance * (sum_r w_r W_r) * sqrt(eta T)
// (stochastic_m_fluxdiv.f90:115-125, 137, 280-361)
template <typename T>
__device__ __forceinline__ T stoch_cc(const StochArgs& a, int dim, int c, i64 f) {
    T s = T(0);
    for (int r = 0; r < a.n_rngs; r++) s = s + (T)a.wts[r] * (T)ld(a.Wcc[r * dim + c], f);
    return ((T)a.variance * s) * (T)sqrt((T)ld(a.eta, f) * (T)ld(a.T, f));
}
template <typename T>
__device__ __forceinline__ T stoch_ed(const StochArgs& a, int nE, int e, int comp, i64 f) {
    T s = T(0);
    for (int r = 0; r < a.n_rngs; r++) s = s + (T)a.wts[r] * (T)ld(a.Wed[r * 2 * nE + 2 * e + comp], f);
    return ((T)a.variance * s) * (T)sqrt((T)ld(a.eta_ed[e], f) * (T)ld(a.T_ed[e], f));
}

// divergence of the scaled random stress onto the faces (stoch_m_force_2d /
// _3d, stochastic_m_fluxdiv.f90:453-600), overwrite or increment.
// T is the arithmetic precision (double, or float in the mixed mode).
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_stoch_m(Grid g, StochArgs a, double* o0, double* o1, double* o2,
                                                 int increment) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
    const T dxi = (T)a.dxinv;
    T dv[3];
    if constexpr (DIM == 2) {
        dv[0] = (stoch_cc<T>(a, 2, 0, f) - stoch_cc<T>(a, 2, 0, P.id(-1, 0, 0))) * dxi +
                (stoch_ed<T>(a, 1, 0, 0, P.id(0, 1, 0)) - stoch_ed<T>(a, 1, 0, 0, f)) * dxi;
        dv[1] = (stoch_ed<T>(a, 1, 0, 1, P.id(1, 0, 0)) - stoch_ed<T>(a, 1, 0, 1, f)) * dxi +
                (stoch_cc<T>(a, 2, 1, f) - stoch_cc<T>(a, 2, 1, P.id(0, -1, 0))) * dxi;
    } else {
        dv[0] = (stoch_cc<T>(a, 3, 0, f) - stoch_cc<T>(a, 3, 0, P.id(-1, 0, 0))) * dxi +
                (stoch_ed<T>(a, 3, 0, 0, P.id(0, 1, 0)) - stoch_ed<T>(a, 3, 0, 0, f)) * dxi +
                (stoch_ed<T>(a, 3, 1, 0, P.id(0, 0, 1)) - stoch_ed<T>(a, 3, 1, 0, f)) * dxi;
        dv[1] = (stoch_ed<T>(a, 3, 0, 1, P.id(1, 0, 0)) - stoch_ed<T>(a, 3, 0, 1, f)) * dxi +
                (stoch_cc<T>(a, 3, 1, f) - stoch_cc<T>(a, 3, 1, P.id(0, -1, 0))) * dxi +
                (stoch_ed<T>(a, 3, 2, 0, P.id(0, 0, 1)) - stoch_ed<T>(a, 3, 2, 0, f)) * dxi;
        dv[2] = (stoch_ed<T>(a, 3, 1, 1, P.id(1, 0, 0)) - stoch_ed<T>(a, 3, 1, 1, f)) * dxi +
                (stoch_ed<T>(a, 3, 2, 1, P.id(0, 1, 0)) - stoch_ed<T>(a, 3, 2, 1, f)) * dxi +
                (stoch_cc<T>(a, 3, 2, f) - stoch_cc<T>(a, 3, 2, P.id(0, 0, -1))) * dxi;
    }
    double* o[3] = {o0, o1, o2};
#pragma unroll
    for (int c = 0; c < DIM; c++) o[c][f] = increment ? o[c][f] + (double)dv[c] : (double)dv[c];
}

// Walls (fhd_walls.cuh): edge set e (2D the nodes; 3D xy, xz, yz) has one
// more plane in a wall direction of the set, holding the edges on the high
// wall; ext[e] are its extents.
struct EdgeExt {
    int ext[3][3];
};
__device__ __forceinline__ void edge_dirs_d(int dim, int e, int& a, int& b) {
    a = (dim == 3 && e == 2) ? 1 : 0;
    b = (dim == 3 && e != 0) ? 2 : 1;
}
// the scaled random stress on edge (i, j, k) of set e with the wall rules
// of mflux_bc_2d / _3d (stochastic_m_fluxdiv.f90:363-451): times sqrt(2) on
// a no-slip wall, zero on a slip wall, the boundaries of x, then y, then z
template <typename T, int DIM>
__device__ __forceinline__ T stoch_ed_w(const StochArgs& a, const Grid& g, const fhd::Walls& W, const EdgeExt& X,
                                        int e, int comp, int i, int j, int k) {
    constexpr int nE = DIM == 2 ? 1 : 3;
    int da, db;
    edge_dirs_d(DIM, e, da, db);
    int q[3] = {i, j, k};
#pragma unroll
    for (int d = 0; d < 3; d++)
        if (X.ext[e][d] == g.n[d]) q[d] = wrapc(q[d], g.n[d]);
    const i64 f = (i64)q[0] + (i64)X.ext[e][0] * ((i64)q[1] + (i64)X.ext[e][1] * q[2]);
    T v = stoch_ed<T>(a, nE, e, comp, f);
    const int ds[2] = {da, db};
#pragma unroll
    for (int t = 0; t < 2; t++) {
        const int d = ds[t];
        if (W.lo[d] == 0) continue;
        const int side = q[d] == 0 ? W.lo[d] : (q[d] == g.n[d] ? W.hi[d] : 0);
        if (side < 0) v = (T)1.4142135623730951 * v;
        else if (side > 0) v = T(0);
    }
    return v;
}

// k_stoch_m with walls: edges through stoch_ed_w, and the normal component
// on a wall face zero (multifab_physbc_domainvel), increment or not
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_stoch_m_w(Grid g, fhd::Walls W, EdgeExt X, StochArgs a, double* o0,
                                                   double* o1, double* o2, int increment) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
    const T dxi = (T)a.dxinv;
    const int i = P.i, j = P.j, k = P.k;
    auto E = [&](int e, int comp, int ii, int jj, int kk) { return stoch_ed_w<T, DIM>(a, g, W, X, e, comp, ii, jj, kk); };
    T dv[3];
    if constexpr (DIM == 2) {
        dv[0] = (stoch_cc<T>(a, 2, 0, f) - stoch_cc<T>(a, 2, 0, P.id(-1, 0, 0))) * dxi +
                (E(0, 0, i, j + 1, k) - E(0, 0, i, j, k)) * dxi;
        dv[1] = (E(0, 1, i + 1, j, k) - E(0, 1, i, j, k)) * dxi +
                (stoch_cc<T>(a, 2, 1, f) - stoch_cc<T>(a, 2, 1, P.id(0, -1, 0))) * dxi;
    } else {
        dv[0] = (stoch_cc<T>(a, 3, 0, f) - stoch_cc<T>(a, 3, 0, P.id(-1, 0, 0))) * dxi +
                (E(0, 0, i, j + 1, k) - E(0, 0, i, j, k)) * dxi + (E(1, 0, i, j, k + 1) - E(1, 0, i, j, k)) * dxi;
        dv[1] = (E(0, 1, i + 1, j, k) - E(0, 1, i, j, k)) * dxi +
                (stoch_cc<T>(a, 3, 1, f) - stoch_cc<T>(a, 3, 1, P.id(0, -1, 0))) * dxi +
                (E(2, 0, i, j, k + 1) - E(2, 0, i, j, k)) * dxi;
        dv[2] = (E(1, 1, i + 1, j, k) - E(1, 1, i, j, k)) * dxi + (E(2, 1, i, j + 1, k) - E(2, 1, i, j, k)) * dxi +
                (stoch_cc<T>(a, 3, 2, f) - stoch_cc<T>(a, 3, 2, P.id(0, 0, -1))) * dxi;
    }
    double* o[3] = {o0, o1, o2};
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        if (fhd::on_wall(W, c, i, j, k)) o[c][f] = 0.0;
        else o[c][f] = increment ? o[c][f] + (double)dv[c] : (double)dv[c];
    }
}

// ---------------------------------------------------------------------
// filtering_width 1, 2 or 4: the scaled stresses are written out, smoothed
// by the separable filter of filter_stoch_m_flux (x, then y, then z;
// stochastic_m_fluxdiv.f90:604-778) and then differenced
// (stochastic_m_fluxdiv.f90:172-174, 226-230).  Array q of the stress set
// s (q*nc + f): the dim cell stresses, then edge set e component comp at
// dim + 2e + comp.  Periodic boxes.
// ---------------------------------------------------------------------
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_stoch_stress(Grid g, StochArgs a, T* __restrict__ s) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    constexpr int nE = DIM == 2 ? 1 : 3;
    const i64 f = P.id(0, 0, 0), nc = g.nc;
#pragma unroll
    for (int c = 0; c < DIM; c++) s[c * nc + f] = stoch_cc<T>(a, DIM, c, f);
#pragma unroll
    for (int q = 0; q < 2 * nE; q++) s[(DIM + q) * nc + f] = stoch_ed<T>(a, nE, q / 2, q % 2, f);
}

// one filter pass along direction D over the nq arrays of the set; the
// terms in the order of filter_stoch_m_flux, each division by a power of
// two written as the exact product
template <typename T, int W, int D>
__global__ void __launch_bounds__(256) k_stoch_filter(Grid g, const T* __restrict__ in, T* __restrict__ out,
                                                      int nq) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 nc = g.nc, f = P.id(0, 0, 0);
    i64 o[2 * W + 1];
#pragma unroll
    for (int s = -W; s <= W; s++) o[s + W] = P.id(D == 0 ? s : 0, D == 1 ? s : 0, D == 2 ? s : 0);
    for (int q = 0; q < nq; q++) {
        const T* a = in + q * nc;
        auto at = [&](int s) { return ld(a, o[s + W]); };
        T v;
        if constexpr (W == 1) {
            v = at(0) * T(0.5) + at(-1) * T(0.25) + at(1) * T(0.25);
        } else if constexpr (W == 2) {
            v = (T(5) * at(0)) * T(0.125) - at(-2) * T(0.0625) + at(-1) * T(0.25) - at(2) * T(0.0625) +
                at(1) * T(0.25);
        } else {
            v = (T(93) * at(0)) * T(0.0078125) + (T(7) * at(-1)) * T(0.03125) - (T(7) * at(-2)) * T(0.015625) +
                at(-3) * T(0.03125) - at(-4) * T(0.00390625) + (T(7) * at(1)) * T(0.03125) -
                (T(7) * at(2)) * T(0.015625) + at(3) * T(0.03125) - at(4) * T(0.00390625);
        }
        out[q * nc + f] = v;
    }
}

// k_stoch_m with the stresses read from the (filtered) set s
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_stoch_div(Grid g, const T* __restrict__ s, double* o0, double* o1,
                                                   double* o2, int increment, double dxinv) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0), nc = g.nc;
    const T dxi = (T)dxinv;
    auto C = [&](int c, i64 q) { return ld(s + c * nc, q); };
    auto E = [&](int e, int comp, i64 q) { return ld(s + (DIM + 2 * e + comp) * nc, q); };
    T dv[3];
    if constexpr (DIM == 2) {
        dv[0] = (C(0, f) - C(0, P.id(-1, 0, 0))) * dxi + (E(0, 0, P.id(0, 1, 0)) - E(0, 0, f)) * dxi;
        dv[1] = (E(0, 1, P.id(1, 0, 0)) - E(0, 1, f)) * dxi + (C(1, f) - C(1, P.id(0, -1, 0))) * dxi;
    } else {
        dv[0] = (C(0, f) - C(0, P.id(-1, 0, 0))) * dxi + (E(0, 0, P.id(0, 1, 0)) - E(0, 0, f)) * dxi +
                (E(1, 0, P.id(0, 0, 1)) - E(1, 0, f)) * dxi;
        dv[1] = (E(0, 1, P.id(1, 0, 0)) - E(0, 1, f)) * dxi + (C(1, f) - C(1, P.id(0, -1, 0))) * dxi +
                (E(2, 0, P.id(0, 0, 1)) - E(2, 0, f)) * dxi;
        dv[2] = (E(1, 1, P.id(1, 0, 0)) - E(1, 1, f)) * dxi + (E(2, 1, P.id(0, 1, 0)) - E(2, 1, f)) * dxi +
                (C(2, f) - C(2, P.id(0, 0, -1))) * dxi;
    }
    double* o[3] = {o0, o1, o2};
#pragma unroll
    for (int c = 0; c < DIM; c++) o[c][f] = increment ? o[c][f] + (double)dv[c] : (double)dv[c];
}

template <typename T, int DIM>
static int stoch_filtered(fhd_ctx* ctx, const StochArgs& a, int width, double* const force[], int increment) {
    constexpr int nq = DIM + (DIM == 2 ? 2 : 6);
    const Grid g = ctx->g0;
    const i64 nc = g.nc;
    if (!ctx->stoch_filt) {
        ctx->stoch_filt = ctx->arena.alloc<T>(2 * (i64)nq * nc);
        if (!ctx->stoch_filt) {
            set_last_error("stochastic_m_fluxdiv: out of device memory for the filtered stresses");
            return FHD_ERR_OOM;
        }
    }
    T* s = (T*)ctx->stoch_filt;
    T* t = s + (i64)nq * nc;
    const dim3 gr = cell_grid(g), bl = cell_block();
    k_stoch_stress<T, DIM><<<gr, bl, 0, ctx->stream>>>(g, a, s);
    ctx->launches++;
    for (int d = 0; d < DIM; d++) {
        auto pass = [&](auto Wc) {
            constexpr int W = decltype(Wc)::value;
            if (d == 0) k_stoch_filter<T, W, 0><<<gr, bl, 0, ctx->stream>>>(g, s, t, nq);
            else if (d == 1) k_stoch_filter<T, W, 1><<<gr, bl, 0, ctx->stream>>>(g, s, t, nq);
            else k_stoch_filter<T, W, 2><<<gr, bl, 0, ctx->stream>>>(g, s, t, nq);
        };
        if (width == 1) pass(std::integral_constant<int, 1>());
        else if (width == 2) pass(std::integral_constant<int, 2>());
        else pass(std::integral_constant<int, 4>());
        ctx->launches++;
        T* x = s;
        s = t;
        t = x;
    }
    k_stoch_div<T, DIM><<<gr, bl, 0, ctx->stream>>>(g, s, force[0], force[1], DIM == 3 ? force[2] : nullptr,
                                                     increment, a.dxinv);
    ctx->launches++;
    FHD_CUDA_TRY(cudaPeekAtLastError());
    return 0;
}

int stoch_launch(fhd_ctx* ctx, const fhd_stoch_params* sp, double* const force[], int increment, const double* eta,
                 const double* const eta_ed[], const double* T, const double* const T_ed[], double dt,
                 const double* weights, int n_rngs, const double* const W_cc[], const double* const W_ed[]) {
    const int dim = ctx->dim, nE = dim == 2 ? 1 : 3;
    const int width = sp->filtering_width;
    if (n_rngs < 1 || n_rngs > 4) {
        set_last_error("stochastic_m_fluxdiv: n_rngs must be 1..4");
        return FHD_ERR_UNSUPPORTED;
    }
    if (width != 0 && width != 1 && width != 2 && width != 4) {
        set_last_error("stochastic_m_fluxdiv: filtering_width must be 0, 1, 2 or 4");
        return FHD_ERR_BAD_ARG;
    }
    if (width != 0) {
        if (ctx->has_walls) {
            set_last_error("stochastic_m_fluxdiv: filtering_width != 0 is built for periodic boxes only");
            return FHD_ERR_UNSUPPORTED;
        }
        for (int d = 0; d < dim; d++)
            if (ctx->g0.n[d] < width) {
                set_last_error("stochastic_m_fluxdiv: the filter is wider than the domain");
                return FHD_ERR_BAD_ARG;
            }
    }
    StochArgs a;
    memset(&a, 0, sizeof(a));
    for (int i = 0; i < n_rngs * dim; i++) a.Wcc[i] = W_cc[i];
    for (int i = 0; i < n_rngs * 2 * nE; i++) a.Wed[i] = W_ed[i];
    for (int r = 0; r < n_rngs; r++) a.wts[r] = weights[r];
    a.n_rngs = n_rngs;
    a.eta = eta;
    a.T = T;
    for (int e = 0; e < nE; e++) {
        a.eta_ed[e] = eta_ed[e];
        a.T_ed[e] = T_ed[e];
    }
    a.variance = sqrt(sp->variance_coef_mom * 2.0 * sp->k_B / (sp->dV * dt));
    a.dxinv = 1.0 / ctx->dx;
    const Grid g = ctx->g0;
    double* f2 = dim == 3 ? force[2] : nullptr;
    const bool mixed = ctx->prec == FHD_PREC_MIXED;
    if (width != 0) {
        int rc = 0;
        with_dim(dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            rc = mixed ? stoch_filtered<float, DIM>(ctx, a, width, force, increment)
                       : stoch_filtered<double, DIM>(ctx, a, width, force, increment);
        });
        return rc;
    }
    if (ctx->has_walls) {
        EdgeExt X;
        for (int e = 0; e < 3; e++) {
            const int da = (dim == 3 && e == 2) ? 1 : 0, db = (dim == 3 && e != 0) ? 2 : 1;
            for (int d = 0; d < 3; d++)
                X.ext[e][d] = g.n[d] + ((d == da || d == db) && d < dim && ctx->walls.lo[d] != 0 ? 1 : 0);
        }
        with_dim(dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            if (mixed)
                k_stoch_m_w<float, DIM><<<cell_grid(g), cell_block(), 0, ctx->stream>>>(g, ctx->walls, X, a, force[0],
                                                                                      force[1], f2, increment);
            else
                k_stoch_m_w<double, DIM><<<cell_grid(g), cell_block(), 0, ctx->stream>>>(g, ctx->walls, X, a, force[0],
                                                                                       force[1], f2, increment);
        });
        ctx->launches++;
        FHD_CUDA_TRY(cudaPeekAtLastError());
        return 0;
    }
    with_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        if (mixed)
            k_stoch_m<float, DIM><<<cell_grid(g), cell_block(), 0, ctx->stream>>>(g, a, force[0], force[1], f2,
                                                                                increment);
        else
            k_stoch_m<double, DIM><<<cell_grid(g), cell_block(), 0, ctx->stream>>>(g, a, force[0], force[1], f2,
                                                                                 increment);
    });
    ctx->launches++;
    FHD_CUDA_TRY(cudaPeekAtLastError());
    return 0;
}

// ---------------------------------------------------------------------
// step glue kernels
// ---------------------------------------------------------------------
// average_cc_to_face (convert_stag.f90:229-292): face = (cc(i)+cc(i-1))/2
template <int DIM>
__global__ void __launch_bounds__(256) k_avg_face(Grid g, const double* cc, double* o0, double* o1, double* o2) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
    const double v = ld(cc, f);
    o0[f] = 0.5 * (v + ld(cc, P.id(-1, 0, 0)));
    o1[f] = 0.5 * (v + ld(cc, P.id(0, -1, 0)));
    if constexpr (DIM == 3) o2[f] = 0.5 * (v + ld(cc, P.id(0, 0, -1)));
}

// centred scalar advection (mk_advective_s_fluxdiv.f90:138-220),
// upd = -div(s_fc u), folded into the scalar update; upd (nullable) is the
// rho_update array of the step, accumulated in place
//   mode 0: upd = -div;      s_out = s_a + dt*upd          (predictor)
//   mode 2: upd = upd - div; s_out = s_a + dt*upd          (predictor with F^n)
//   mode 1: upd = upd - div; s_out = ((s_out + s_a) + dt*upd)*0.5 (corrector)
template <int DIM>
__global__ void __launch_bounds__(256) k_adv_s_update(Grid g, CSVec<double> u, CSVec<double> sfc, const double* sa,
                                                      double* sout, double dt, double dxinv, int mode, double* upd) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
    double s = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        const i64 fp = P.id(d == 0, d == 1, d == 2);
        s += (ld(u.c[d], fp) * ld(sfc.c[d], fp) - ld(u.c[d], f) * ld(sfc.c[d], f)) * dxinv;
    }
    double up = (mode == 0) ? -s : upd[f] - s;
    if (upd) upd[f] = up;
    if (mode != 1) {
        sout[f] = sa[f] + dt * up;
    } else {
        double v = sout[f] + sa[f];
        v = v + dt * up;
        sout[f] = v * 0.5;
    }
}

// centred momentum advection (mk_advective_m_fluxdiv.f90:184-346):
// upd (+)= -div(m u); flux of m_c in direction d at q is
// 0.25*(m_c(q-e_d)+m_c(q))*(u_d(q-e_c)+u_d(q))
template <int DIM>
__global__ void __launch_bounds__(256) k_adv_m(Grid g, CSVec<double> u, CSVec<double> m, SVec<double> upd,
                                               int increment, double dxinv) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        const int cx = (c == 0), cy = (c == 1), cz = (c == 2);
        double s = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            const int ex = (d == 0), ey = (d == 1), ez = (d == 2);
            auto flux = [&](int qi, int qj, int qk) {
                const i64 q = P.id(qi, qj, qk);
                return 0.25 * (ld(m.c[c], P.id(qi - ex, qj - ey, qk - ez)) + ld(m.c[c], q)) *
                       (ld(u.c[d], P.id(qi - cx, qj - cy, qk - cz)) + ld(u.c[d], q));
            };
            s += (flux(ex, ey, ez) - flux(0, 0, 0)) * dxinv;
        }
        upd.c[c][f] = increment ? upd.c[c][f] - s : -s;
    }
}

template <int DIM>
__global__ void __launch_bounds__(256) k_grad(Grid g, const double* p, SVec<double> o, double dxinv) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
    const double v = ld(p, f);
#pragma unroll
    for (int d = 0; d < DIM; d++) o.c[d][f] = (v - ld(p, P.id(-(d == 0), -(d == 1), -(d == 2)))) * dxinv;
}

template <int DIM>
__global__ void __launch_bounds__(256) k_div_inc(Grid g, CSVec<double> u, double* out, double dxinv) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
    double s = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) s += (ld(u.c[d], P.id(d == 0, d == 1, d == 2)) - ld(u.c[d], f)) * dxinv;
    out[f] = out[f] + s;
}

// y = (keep ? y : 0) + a0*x0 + a1*x1 + ... (left to right), per component
struct Lin {
    const double* x[4][3];
    double a[4];
    int nt;
};
// (all components of an element advance together, each term in order, and
// are stored after every load of the element: ncomp * nt loads in flight)
__global__ void __launch_bounds__(256) k_lin(i64 n, int ncomp, SVec<double> y, Lin L, int keep) {
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x) {
        double v[3];  // ncomp <= 3 (Lin holds three components)
#pragma unroll
        for (int c = 0; c < 3; c++)
            if (c < ncomp) v[c] = keep ? y.c[c][f] : 0.0;
        for (int t = 0; t < L.nt; t++) {
            const double a = L.a[t];
#pragma unroll
            for (int c = 0; c < 3; c++)
                if (c < ncomp) v[c] = v[c] + a * L.x[t][c][f];
        }
#pragma unroll
        for (int c = 0; c < 3; c++)
            if (c < ncomp) y.c[c][f] = v[c];
    }
}

// y = s * u per component (convert_m_to_umac, m = rho_fc * umac)
__global__ void __launch_bounds__(256) k_mul(i64 n, int ncomp, SVec<double> y, CSVec<double> s, CSVec<double> u) {
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x)
        for (int c = 0; c < ncomp; c++) y.c[c][f] = s.c[c][f] * u.c[c][f];
}

// ---------------------------------------------------------------------
// inertial step (advance_timestep_inertial.f90:45-923) for ns species;
// ns = 1 without a mixture is a single fluid without mass fluxes
// ---------------------------------------------------------------------
enum {
    B_RFO = 0, B_RFN = 3, B_MOLD = 6, B_MTEMP = 9, B_ADV = 12, B_DIFF = 15, B_RHSV = 18, B_DU = 21, B_STOCH = 24,
    B_GPI = 27, B_RHOTOT = 30, B_RHSP = 31, B_DPI = 32, B_ETAH = 33, B_KAPH = 34, B_ETAEDH = 35, B_ZERO = 38,
    B_RHOOLD = 39, B_RUPD = 39 + FHD_MAX_SPECIES, B_SFC = 39 + 2 * FHD_MAX_SPECIES,
    B_COUNT = 39 + 5 * FHD_MAX_SPECIES
};
static_assert(B_COUNT <= 128, "step buffer table");

// work arrays of the steps: the shared ones once, the per-species ones for
// the species counts met so far
static int step_alloc(fhd_ctx* ctx, int ns) {
    const i64 nc = ctx->g0.nc;
    const int dim = ctx->dim;
    auto need = [&](int i) -> int {
        if (ctx->sb[i]) return 0;
        ctx->sb[i] = ctx->arena.alloc<double>(nc);
        return ctx->sb[i] ? 0 : FHD_ERR_OOM;
    };
    if (!ctx->step_ready) {
        for (int i = 0; i < B_RHOOLD; i++)
            if (need(i)) return FHD_ERR_OOM;
        FHD_CUDA_TRY(cudaMemsetAsync(ctx->sb[B_ZERO], 0, sizeof(double) * nc, ctx->stream));
        ctx->step_ready = true;
    }
    for (int s = 0; s < ns; s++) {
        if (need(B_RHOOLD + s) || need(B_RUPD + s)) return FHD_ERR_OOM;
        for (int c = 0; c < dim; c++)
            if (need(B_SFC + s * dim + c)) return FHD_ERR_OOM;
    }
    return 0;
}

static SVec<double> sv(fhd_ctx* ctx, int base) {
    SVec<double> v;
    for (int c = 0; c < 4; c++) v.c[c] = (c < ctx->dim) ? ctx->sb[base + c] : nullptr;
    return v;
}
static CSVec<double> cs(SVec<double> v) {
    CSVec<double> o;
    for (int c = 0; c < 4; c++) o.c[c] = v.c[c];
    return o;
}
static SVec<double> svp(double* const* a, int dim) {
    SVec<double> v;
    for (int c = 0; c < 4; c++) v.c[c] = (c < dim) ? a[c] : nullptr;
    return v;
}
static SVec<double> one(double* a) {
    SVec<double> v;
    for (int c = 0; c < 4; c++) v.c[c] = nullptr;
    v.c[0] = a;
    return v;
}

// Moving no-slip walls (fhd_ctx_set_wall_speed): behind such a wall the
// tangential ghost is 2 v_bc - u (physbc_macvel_2d_inhomogeneous /
// _3d_inhomogeneous, multifab_physbc_stag.f90:1118-1160) where the
// homogeneous operator has -u, so +L u (visc_type 1, beta of the first
// cell) gains 2 v_bc beta / dx^2 on the faces of the first row beside the
// wall.  Walls in direction order, the low side first, one addition each.
struct WallSpeed {
    double v[2][6];  // [side][t + 2 d]
};
template <int DIM>
__global__ void __launch_bounds__(256) k_wall_speed(Grid g, fhd::Walls W, WallSpeed S, const double* eta,
                                                    double* o0, double* o1, double* o2, double q) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
    const int at[3] = {P.i, P.j, P.k};
    const double b = ld(eta, 0);
    double* o[3] = {o0, o1, o2};
#pragma unroll
    for (int c = 0; c < DIM; c++) {
        if (fhd::on_wall(W, c, P.i, P.j, P.k)) continue;
        double v = 0.0;
        bool any = false;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            if (d == c) continue;
            const int t = c - (c > d ? 1 : 0);
            if (W.lo[d] < 0 && at[d] == 0 && S.v[0][t + 2 * d] != 0.0) {
                if (!any) v = o[c][f];
                v = v + ((2.0 * S.v[0][t + 2 * d]) * b) * q;
                any = true;
            }
            if (W.hi[d] < 0 && at[d] == g.n[d] - 1 && S.v[1][t + 2 * d] != 0.0) {
                if (!any) v = o[c][f];
                v = v + ((2.0 * S.v[1][t + 2 * d]) * b) * q;
                any = true;
            }
        }
        if (any) o[c][f] = v;
    }
}

// diffusive_m_fluxdiv (diffusive_m_fluxdiv.f90:25-...): -(stag_applyop with
// alpha = 0) applied to u, written to out; with moving walls the velocity's
// ghosts carry their speeds (every call here is on the step's velocity)
static int diff_m(fhd_ctx* ctx, SVec<double> out, CSVec<double> u, const double* eta, const double* const eta_ed[],
                  const double* kappa) {
    StagOp<double> A;
    const int nE = ctx->dim == 2 ? 1 : 3;
    for (int c = 0; c < 3; c++) {
        A.alpha[c] = ctx->sb[B_ZERO];
        A.bed[c] = c < nE ? eta_ed[c] : nullptr;
    }
    A.alpha_scale = 0.0;
    A.beta = eta;
    A.gamma = kappa;
    A.q = 1.0 / (ctx->dx * ctx->dx);
    const Grid g = ctx->g0;
    if (ctx->has_walls) {
        // visc_type 1 with the wall ghost rules; zero on the wall faces
        // (stag_applyop.f90:201-205)
        with_dim_wall_visc(ctx->dim, ctx->visc, [&](auto D, auto V) {
            constexpr int DIM = decltype(D)::value, VISC = decltype(V)::value;
            k_stag_apply_w<double, DIM, VISC><<<cell_grid(g), cell_block(), 0, ctx->stream>>>(
                g, ctx->walls, A, u.c[0], u.c[1], u.c[2], out.c[0], out.c[1], out.c[2], nullptr, nullptr, nullptr,
                0);
        });
    } else {
        with_dim_visc(ctx->dim, ctx->visc, [&](auto D, auto V) {
            constexpr int DIM = decltype(D)::value, VISC = decltype(V)::value;
            k_stag_apply<double, DIM, VISC><<<cell_grid(g), cell_block(), 0, ctx->stream>>>(
                g, A, u.c[0], u.c[1], u.c[2], out.c[0], out.c[1], out.c[2], nullptr, nullptr, nullptr, 0);
        });
    }
    ctx->launches++;
    FHD_CUDA_TRY(cudaPeekAtLastError());
    Lin L;
    memset(&L, 0, sizeof(L));
    L.nt = 1;
    L.a[0] = -1.0;
    for (int c = 0; c < ctx->dim; c++) L.x[0][c] = out.c[c];
    k_lin<<<flat_blocks(g.nc), 256, 0, ctx->stream>>>(g.nc, ctx->dim, out, L, 0);
    ctx->launches++;
    if (ctx->has_walls && ctx->moving_walls) {
        // after the sign flip: the term belongs to +L u
        WallSpeed S;
        memcpy(S.v, ctx->wall_speed, sizeof(S.v));
        with_dim(ctx->dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_wall_speed<DIM><<<cell_grid(g), cell_block(), 0, ctx->stream>>>(g, ctx->walls, S, eta, out.c[0],
                                                                             out.c[1], out.c[2], A.q);
        });
        ctx->launches++;
    }
    FHD_CUDA_TRY(cudaPeekAtLastError());
    return 0;
}

// y = (keep ? y : 0) + sum_t a_t x_t over the first ncomp components
static int lin_n(fhd_ctx* ctx, int ncomp, SVec<double> y, int keep,
                 std::initializer_list<std::pair<double, CSVec<double>>> terms) {
    Lin L;
    memset(&L, 0, sizeof(L));
    int t = 0;
    for (auto& pr : terms) {
        L.a[t] = pr.first;
        for (int c = 0; c < ncomp; c++) L.x[t][c] = pr.second.c[c];
        t++;
    }
    L.nt = t;
    k_lin<<<flat_blocks(ctx->g0.nc), 256, 0, ctx->stream>>>(ctx->g0.nc, ncomp, y, L, keep);
    ctx->launches++;
    FHD_CUDA_TRY(cudaPeekAtLastError());
    return 0;
}
static int lin(fhd_ctx* ctx, SVec<double> y, int keep, std::initializer_list<std::pair<double, CSVec<double>>> terms) {
    return lin_n(ctx, ctx->dim, y, keep, terms);
}

// out = sum over species (compute_rhotot)
__global__ void __launch_bounds__(256) k_sum_species(i64 n, int ns, const double* const* __restrict__ r, double* out) {
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x) {
        double v = 0.0;
        for (int s = 0; s < ns; s++) v = v + r[s][f];
        out[f] = v;
    }
}

int advance_inertial_ms(fhd_ctx* ctx, const fhd_stoch_params* sp, const fhd_mixture_params* mp, double dt,
                        double* const umac[], double* const rho[], double* pi, double* const fluxdiv[],
                        const double* eta, const double* const eta_ed[], const double* kappa,
                        const double* temperature, const double* const temperature_ed[], const double* const W_cc[],
                        const double* const W_ed[], const double* const W_mass[], fhd_solve_stats* stats2) {
    const int dim = ctx->dim, nE = dim == 2 ? 1 : 3;
    const int ns = mp ? mp->nspecies : 1;
    if (ns < 1 || ns > FHD_MAX_SPECIES) return FHD_ERR_BAD_ARG;
    int rc = step_alloc(ctx, ns);
    if (rc) return rc;
    const Grid g = ctx->g0;
    const i64 nc = g.nc;
    const int nb = flat_blocks(nc);
    cudaStream_t st = ctx->stream;
    const double dxinv = 1.0 / ctx->dx;
    const double theta = 1.0 / dt;
    SVec<double> u = svp(umac, dim);
    SVec<double> rfo = sv(ctx, B_RFO), rfn = sv(ctx, B_RFN), mold = sv(ctx, B_MOLD), mtemp = sv(ctx, B_MTEMP),
                 adv = sv(ctx, B_ADV), diff = sv(ctx, B_DIFF), rhs_v = sv(ctx, B_RHSV), du = sv(ctx, B_DU),
                 stoch = sv(ctx, B_STOCH), gpi = sv(ctx, B_GPI);
    double* rhotot = ctx->sb[B_RHOTOT];
    double* rhs_p = ctx->sb[B_RHSP];
    double* dpi = ctx->sb[B_DPI];
    double* eta_h = ctx->sb[B_ETAH];
    double* kap_h = ctx->sb[B_KAPH];
    const double* eta_ed_h[3] = {ctx->sb[B_ETAEDH], ctx->sb[B_ETAEDH + 1], ctx->sb[B_ETAEDH + 2]};
    double* rho_old[FHD_MAX_SPECIES];
    double* rupd[FHD_MAX_SPECIES];
    for (int s = 0; s < ns; s++) {
        rho_old[s] = ctx->sb[B_RHOOLD + s];
        rupd[s] = ctx->sb[B_RUPD + s];
    }
    auto sfc = [&](int s) { return sv(ctx, B_SFC + s * dim); };
    const double w1[1] = {1.0};
    // pointer tables for the species sums live in the zero-initialised
    // tail of the context's scalar block (slots 200..255)
    double** rtab = (double**)(ctx->dscal + 200);
    auto sum_species = [&](double* const* r, double* out) -> int {
        double* h[FHD_MAX_SPECIES];
        for (int s = 0; s < ns; s++) h[s] = r[s];
        FHD_CUDA_TRY(cudaMemcpyAsync(rtab, h, sizeof(double*) * ns, cudaMemcpyHostToDevice, st));
        k_sum_species<<<nb, 256, 0, st>>>(nc, ns, rtab, out);
        ctx->launches++;
        FHD_CUDA_TRY(cudaPeekAtLastError());
        // the host table is reused by the next call: wait for the copy
        FHD_CUDA_TRY(cudaStreamSynchronize(st));
        return 0;
    };
    auto species_fc = [&](double* const* r) {
        for (int s = 0; s < ns; s++) {
            SVec<double> o = sfc(s);
            with_dim(dim, [&](auto D) {
                constexpr int DIM = decltype(D)::value;
                k_avg_face<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, r[s], o.c[0], o.c[1], o.c[2]);
            });
            ctx->launches++;
        }
    };
    auto mass_fluxes = [&](const double* const* Wm) -> int {
        if (!mp) return 0;
        const double* cr[FHD_MAX_SPECIES];
        for (int s = 0; s < ns; s++) cr[s] = rho[s];
        return mass_fluxdiv(ctx, mp, sp, cr, dt, w1, 1, Wm, fluxdiv);
    };
    // -S = sum_i -F_i/rhobar_i into rhs_p (advance_timestep_inertial.f90:420-430)
    auto rhs_p_from_fluxes = [&]() -> int {
        if (!mp) {
            FHD_CUDA_TRY(cudaMemsetAsync(rhs_p, 0, sizeof(double) * nc, st));
            return 0;
        }
        // the species in order, up to four per pass, on a sum that starts
        // at zero (bitwise one pass per species after zeroing)
        for (int s0 = 0; s0 < ns; s0 += 4) {
            Lin Ls;
            memset(&Ls, 0, sizeof(Ls));
            Ls.nt = ns - s0 < 4 ? ns - s0 : 4;
            for (int t = 0; t < Ls.nt; t++) {
                Ls.a[t] = -1.0 / mp->rhobar[s0 + t];
                Ls.x[t][0] = fluxdiv[s0 + t];
            }
            k_lin<<<nb, 256, 0, st>>>(nc, 1, one(rhs_p), Ls, s0 > 0 ? 1 : 0);
            ctx->launches++;
            FHD_CUDA_TRY(cudaPeekAtLastError());
        }
        return 0;
    };
    auto launch_dim = [&](auto&& fn) {
        with_dim(dim, fn);
        ctx->launches++;
    };
    // walls: the pressure gradient (first-order extrapolated pressure,
    // div_and_grad.f90:540-556) and the advective update
    // (mk_advective_m_fluxdiv.f90:80-85) are zero on a wall face.  With u and
    // m zero on the wall faces the periodic stencils read no other value
    // across a wall: every flux through a wall carries the wall's zero normal
    // velocity, and the reads past the high wall wrap to the low wall face.
    auto zero_wall_faces = [&](SVec<double> v) {
        if (!ctx->has_walls) return;
        launch_dim([&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_zero_walls<double, DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, ctx->walls, v.c[0], v.c[1],
                                                                            DIM == 3 ? v.c[2] : nullptr);
        });
    };
    // eta/2, kappa/2 for the solves (advance_timestep_inertial.f90:467-474)
    k_copy_conv<double, double><<<nb, 256, 0, st>>>(nc, eta_h, eta, 0.5);
    k_copy_conv<double, double><<<nb, 256, 0, st>>>(nc, kap_h, kappa, 0.5);
    ctx->launches += 2;
    for (int e = 0; e < nE; e++) {
        k_copy_conv<double, double><<<nb, 256, 0, st>>>(nc, (double*)eta_ed_h[e], eta_ed[e], 0.5);
        ctx->launches++;
    }
    for (int s = 0; s < ns; s++)
        FHD_CUDA_TRY(cudaMemcpyAsync(rho_old[s], rho[s], sizeof(double) * nc, cudaMemcpyDeviceToDevice, st));
    // Step 2: predictor Euler step for the densities
    if ((rc = sum_species(rho_old, rhotot))) return rc;
    launch_dim([&](auto D) {
        constexpr int DIM = decltype(D)::value;
        k_avg_face<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, rhotot, rfo.c[0], rfo.c[1], rfo.c[2]);
    });
    species_fc(rho_old);
    for (int s = 0; s < ns; s++) {
        if (mp) FHD_CUDA_TRY(cudaMemcpyAsync(rupd[s], fluxdiv[s], sizeof(double) * nc, cudaMemcpyDeviceToDevice, st));
        // rho_new = rho_old + dt*(F^n - div(rho_fc u))
        const SVec<double> f3 = sfc(s);
        launch_dim([&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_adv_s_update<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, cs(u), cs(f3), rho_old[s], rho[s], dt, dxinv,
                                                                      mp ? 2 : 0, rupd[s]);
        });
    }
    if ((rc = sum_species(rho, rhotot))) return rc;
    launch_dim([&](auto D) {
        constexpr int DIM = decltype(D)::value;
        k_avg_face<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, rhotot, rfn.c[0], rfn.c[1], rfn.c[2]);
    });
    species_fc(rho);
    // Steps 3-4: predictor Crank-Nicolson right-hand side.  The terms are
    // formed first; two multi-term passes then add them in the order of
    // the reference's accumulation, each term in turn on the running sum,
    // which is bitwise the sum of one pass per term.  The explicit half of
    // the viscous term appears twice (0.5 L u of the right-hand side and of
    // -A u^n); both are the same L u.
    const bool with_stoch = sp->variance_coef_mom != 0.0;
    k_mul<<<nb, 256, 0, st>>>(nc, dim, mold, cs(rfo), cs(u));
    ctx->launches++;
    launch_dim([&](auto D) {
        constexpr int DIM = decltype(D)::value;
        k_grad<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, pi, gpi, dxinv);
    });
    launch_dim([&](auto D) {
        constexpr int DIM = decltype(D)::value;
        k_adv_m<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, cs(u), cs(mold), adv, 0, dxinv);
    });
    zero_wall_faces(gpi);
    zero_wall_faces(adv);
    if ((rc = diff_m(ctx, diff, cs(u), eta, eta_ed, kappa))) return rc;
    if ((rc = lin(ctx, rhs_v, 0, {{1.0 / dt, cs(mold)}, {-1.0, cs(gpi)}, {1.0, cs(adv)}, {0.5, cs(diff)}}))) return rc;
    if (with_stoch &&
        (rc = stoch_launch(ctx, sp, stoch.c, 0, eta, eta_ed, temperature, temperature_ed, dt, w1, 1, W_cc, W_ed)))
        return rc;
    if ((rc = mass_fluxes(W_mass))) return rc;
    if ((rc = rhs_p_from_fluxes())) return rc;
    k_mul<<<nb, 256, 0, st>>>(nc, dim, mtemp, cs(rfn), cs(u));
    ctx->launches++;
    if (with_stoch) rc = lin(ctx, rhs_v, 1, {{1.0, cs(stoch)}, {-1.0 / dt, cs(mtemp)}, {0.5, cs(diff)}});
    else rc = lin(ctx, rhs_v, 1, {{-1.0 / dt, cs(mtemp)}, {0.5, cs(diff)}});
    if (rc) return rc;
    for (int s = 0; s < ns; s++) {
        if (mp) FHD_CUDA_TRY(cudaMemcpyAsync(rupd[s], fluxdiv[s], sizeof(double) * nc, cudaMemcpyDeviceToDevice, st));
        else FHD_CUDA_TRY(cudaMemsetAsync(rupd[s], 0, sizeof(double) * nc, st));
    }
    launch_dim([&](auto D) {
        constexpr int DIM = decltype(D)::value;
        k_div_inc<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, cs(u), rhs_p, dxinv);
    });
    for (int c = 0; c < dim; c++) FHD_CUDA_TRY(cudaMemsetAsync(du.c[c], 0, sizeof(double) * nc, st));
    FHD_CUDA_TRY(cudaMemsetAsync(dpi, 0, sizeof(double) * nc, st));
    FHD_CUDA_TRY(cudaPeekAtLastError());
    const double abs_tol_in = ctx->p.gmres_abs_tol;
    double norm_pre_rhs = 0.0;
    const double* rfn_c[3] = {rfn.c[0], rfn.c[1], rfn.c[2]};
    auto solve = [&](fhd_solve_stats* s, double* npr) -> int {
        int r2 = prepare(ctx, rfn_c, eta_h, eta_ed_h, kap_h, theta);
        if (r2) return r2;
        CSVec<double> b;
        SVec<double> x;
        for (int c = 0; c < 4; c++) { b.c[c] = nullptr; x.c[c] = nullptr; }
        for (int c = 0; c < dim; c++) { b.c[c] = rhs_v.c[c]; x.c[c] = du.c[c]; }
        b.c[dim] = rhs_p;
        x.c[dim] = dpi;
        return gmres_dev(ctx, b, x, npr, s);
    };
    int st1 = solve(stats2 ? &stats2[0] : nullptr, &norm_pre_rhs);
    if (st1 < 0) return st1;
    // corrector stopping criterion (advance_timestep_inertial.f90:493-496)
    ctx->p.gmres_abs_tol = fmax(abs_tol_in, norm_pre_rhs * ctx->p.gmres_rel_tol);
    int rc2 = 0;
    do {
        if ((rc2 = lin(ctx, u, 1, {{1.0, cs(du)}}))) break;
        if ((rc2 = lin_n(ctx, 1, one(pi), 1, {{1.0, cs(one(dpi))}}))) break;
        k_mul<<<nb, 256, 0, st>>>(nc, dim, mtemp, cs(rfn), cs(u));
        ctx->launches++;
        // Step 5: trapezoidal scalar corrector
        for (int s = 0; s < ns; s++) {
            const SVec<double> f3 = sfc(s);
            launch_dim([&](auto D) {
                constexpr int DIM = decltype(D)::value;
                k_adv_s_update<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, cs(u), cs(f3), rho_old[s], rho[s], dt,
                                                                          dxinv, 1, rupd[s]);
            });
        }
        if ((rc2 = sum_species(rho, rhotot))) break;
        launch_dim([&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_avg_face<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, rhotot, rfn.c[0], rfn.c[1], rfn.c[2]);
        });
        // Steps 6-7: corrector Crank-Nicolson right-hand side, its terms
        // added in the reference's order by two multi-term passes (the
        // first with the predictor's L u^n, the second with L u*)
        launch_dim([&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_grad<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, pi, gpi, dxinv);
        });
        launch_dim([&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_adv_m<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, cs(u), cs(mtemp), adv, 1, dxinv);
        });
        zero_wall_faces(gpi);
        zero_wall_faces(adv);
        if ((rc2 = lin(ctx, rhs_v, 0, {{1.0 / dt, cs(mold)}, {-1.0, cs(gpi)}, {0.5, cs(adv)}, {0.5, cs(diff)}})))
            break;
        if (with_stoch && (rc2 = stoch_launch(ctx, sp, stoch.c, 1, eta, eta_ed, temperature, temperature_ed, dt, w1,
                                              1, W_cc, W_ed)))
            break;
        if ((rc2 = mass_fluxes(W_mass ? W_mass + dim * ns : nullptr))) break;
        if ((rc2 = rhs_p_from_fluxes())) break;
        k_mul<<<nb, 256, 0, st>>>(nc, dim, mtemp, cs(rfn), cs(u));
        ctx->launches++;
        if ((rc2 = diff_m(ctx, diff, cs(u), eta, eta_ed, kappa))) break;
        if (with_stoch) rc2 = lin(ctx, rhs_v, 1, {{0.5, cs(stoch)}, {-1.0 / dt, cs(mtemp)}, {0.5, cs(diff)}});
        else rc2 = lin(ctx, rhs_v, 1, {{-1.0 / dt, cs(mtemp)}, {0.5, cs(diff)}});
        if (rc2) break;
        launch_dim([&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_div_inc<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, cs(u), rhs_p, dxinv);
        });
        for (int c = 0; c < dim; c++) {
            if (cudaMemsetAsync(du.c[c], 0, sizeof(double) * nc, st) != cudaSuccess) rc2 = FHD_ERR_CUDA;
        }
        if (cudaMemsetAsync(dpi, 0, sizeof(double) * nc, st) != cudaSuccess) rc2 = FHD_ERR_CUDA;
    } while (0);
    if (rc2) {
        ctx->p.gmres_abs_tol = abs_tol_in;
        return rc2;
    }
    int st2 = solve(stats2 ? &stats2[1] : nullptr, nullptr);
    ctx->p.gmres_abs_tol = abs_tol_in;
    if (st2 < 0) return st2;
    if ((rc = lin(ctx, u, 1, {{1.0, cs(du)}}))) return rc;
    if ((rc = lin_n(ctx, 1, one(pi), 1, {{1.0, cs(one(dpi))}}))) return rc;
    FHD_CUDA_TRY(cudaPeekAtLastError());
    return st1 > st2 ? st1 : st2;
}

// ---------------------------------------------------------------------
// overdamped step (advance_timestep_overdamped.f90:135-734): periodic,
// centred advection, no gravity or reactions, barodiffusion off,
// midpoint_stoch_mass_flux_type = 1; theta_alpha = 0.  Two random stages:
// W_cc[r*dim+c], W_ed[r*2*nE+...], W_mass[(r*dim+d)*ns+i], r = 0, 1.
// ---------------------------------------------------------------------
int advance_overdamped(fhd_ctx* ctx, const fhd_stoch_params* sp, const fhd_mixture_params* mp, double dt,
                       double* const umac[], double* const rho[], double* pi, const double* eta,
                       const double* const eta_ed[], const double* kappa, const double* temperature,
                       const double* const temperature_ed[], const double* const W_cc[], const double* const W_ed[],
                       const double* const W_mass[], fhd_solve_stats* stats2) {
    const int dim = ctx->dim;
    const int ns = mp ? mp->nspecies : 1;
    if (ns < 1 || ns > FHD_MAX_SPECIES) return FHD_ERR_BAD_ARG;
    int rc = step_alloc(ctx, ns);
    if (rc) return rc;
    const Grid g = ctx->g0;
    const i64 nc = g.nc;
    const int nb = flat_blocks(nc);
    cudaStream_t st = ctx->stream;
    const double dxinv = 1.0 / ctx->dx;
    SVec<double> u = svp(umac, dim);
    SVec<double> rtf = sv(ctx, B_RFN), diff = sv(ctx, B_DIFF), rhs_v = sv(ctx, B_RHSV), du = sv(ctx, B_DU),
                 gpi = sv(ctx, B_GPI);
    double* rhotot = ctx->sb[B_RHOTOT];
    double* rhs_p = ctx->sb[B_RHSP];
    double* dpi = ctx->sb[B_DPI];
    double* rho_old[FHD_MAX_SPECIES];
    double* rupd[FHD_MAX_SPECIES];
    for (int s = 0; s < ns; s++) {
        rho_old[s] = ctx->sb[B_RHOOLD + s];
        rupd[s] = ctx->sb[B_RUPD + s];
    }
    auto sfc = [&](int s) { return sv(ctx, B_SFC + s * dim); };
    double** rtab = (double**)(ctx->dscal + 200);
    auto sum_species = [&](double* const* r, double* out) -> int {
        double* h[FHD_MAX_SPECIES];
        for (int s = 0; s < ns; s++) h[s] = r[s];
        FHD_CUDA_TRY(cudaMemcpyAsync(rtab, h, sizeof(double*) * ns, cudaMemcpyHostToDevice, st));
        k_sum_species<<<nb, 256, 0, st>>>(nc, ns, rtab, out);
        ctx->launches++;
        FHD_CUDA_TRY(cudaPeekAtLastError());
        FHD_CUDA_TRY(cudaStreamSynchronize(st));
        return 0;
    };
    auto launch_dim = [&](auto&& fn) {
        with_dim(dim, fn);
        ctx->launches++;
    };
    // faces of rho_tot and of every species (lines 181-183 / 410-411)
    auto faces = [&](double* const* r) -> int {
        int r2 = sum_species(r, rhotot);
        if (r2) return r2;
        launch_dim([&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_avg_face<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, rhotot, rtf.c[0], rtf.c[1], rtf.c[2]);
        });
        for (int s = 0; s < ns; s++) {
            SVec<double> o = sfc(s);
            launch_dim([&](auto D) {
                constexpr int DIM = decltype(D)::value;
                k_avg_face<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, r[s], o.c[0], o.c[1], o.c[2]);
            });
        }
        return 0;
    };
    // one half of the step over h with the stage weights: rhs, GMRES,
    // u += du, pi += dpi, rho = rho_old + h*(F - div(rho_fc u))
    auto stage = [&](const double* wts, double h, double* npr, fhd_solve_stats* sst) -> int {
        int r2;
        launch_dim([&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_grad<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, pi, gpi, dxinv);
            // at a wall the pressure ghost is the interior value (first-order
            // extrapolation): no gradient on a wall face (div_and_grad.f90:540-556)
            if (ctx->has_walls)
                k_zero_walls<double, DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, ctx->walls, gpi.c[0], gpi.c[1],
                                                                                DIM == 3 ? gpi.c[2] : nullptr);
        });
        if ((r2 = lin(ctx, rhs_v, 0, {{-1.0, cs(gpi)}}))) return r2;
        if (sp->variance_coef_mom != 0.0 &&
            (r2 = stoch_launch(ctx, sp, rhs_v.c, 1, eta, eta_ed, temperature, temperature_ed, h, wts, 2, W_cc, W_ed)))
            return r2;
        if (mp) {
            const double* cr[FHD_MAX_SPECIES];
            for (int s = 0; s < ns; s++) cr[s] = rho[s];
            if ((r2 = mass_fluxdiv(ctx, mp, sp, cr, h, wts, 2, W_mass, rupd))) return r2;
        } else {
            FHD_CUDA_TRY(cudaMemsetAsync(rupd[0], 0, sizeof(double) * nc, st));
        }
        FHD_CUDA_TRY(cudaMemsetAsync(rhs_p, 0, sizeof(double) * nc, st));
        if (mp)
            for (int s = 0; s < ns; s++)
                if ((r2 = lin_n(ctx, 1, one(rhs_p), 1, {{-1.0 / mp->rhobar[s], cs(one(rupd[s]))}}))) return r2;
        if ((r2 = diff_m(ctx, diff, cs(u), eta, eta_ed, kappa))) return r2;
        if ((r2 = lin(ctx, rhs_v, 1, {{1.0, cs(diff)}}))) return r2;
        launch_dim([&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_div_inc<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, cs(u), rhs_p, dxinv);
        });
        for (int c = 0; c < dim; c++) FHD_CUDA_TRY(cudaMemsetAsync(du.c[c], 0, sizeof(double) * nc, st));
        FHD_CUDA_TRY(cudaMemsetAsync(dpi, 0, sizeof(double) * nc, st));
        FHD_CUDA_TRY(cudaPeekAtLastError());
        const double* rtf_c[3] = {rtf.c[0], rtf.c[1], rtf.c[2]};
        if ((r2 = prepare(ctx, rtf_c, eta, eta_ed, kappa, 0.0))) return r2;
        CSVec<double> b;
        SVec<double> x;
        for (int c = 0; c < 4; c++) { b.c[c] = nullptr; x.c[c] = nullptr; }
        for (int c = 0; c < dim; c++) { b.c[c] = rhs_v.c[c]; x.c[c] = du.c[c]; }
        b.c[dim] = rhs_p;
        x.c[dim] = dpi;
        const int sg = gmres_dev(ctx, b, x, npr, sst);
        if (sg < 0) return sg;
        if ((r2 = lin(ctx, u, 1, {{1.0, cs(du)}}))) return r2;
        if ((r2 = lin_n(ctx, 1, one(pi), 1, {{1.0, cs(one(dpi))}}))) return r2;
        for (int s = 0; s < ns; s++) {
            const SVec<double> f3 = sfc(s);
            launch_dim([&](auto D) {
                constexpr int DIM = decltype(D)::value;
                k_adv_s_update<DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, cs(u), cs(f3), rho_old[s], rho[s], h,
                                                                          dxinv, 2, rupd[s]);
            });
        }
        FHD_CUDA_TRY(cudaPeekAtLastError());
        return sg;
    };
    for (int s = 0; s < ns; s++)
        FHD_CUDA_TRY(cudaMemcpyAsync(rho_old[s], rho[s], sizeof(double) * nc, cudaMemcpyDeviceToDevice, st));
    if ((rc = faces(rho_old))) return rc;
    const double w_pred[2] = {1.0, 0.0};
    const double w_corr[2] = {1.0 / std::sqrt(2.0), 1.0 / std::sqrt(2.0)};
    const double abs_tol_in = ctx->p.gmres_abs_tol;
    double norm_pre_rhs = 0.0;
    const int st1 = stage(w_pred, 0.5 * dt, &norm_pre_rhs, stats2 ? &stats2[0] : nullptr);
    if (st1 < 0) return st1;
    // the corrector stops at the predictor's preconditioned rhs (line 338);
    // the tolerance is restored after it (line 587)
    ctx->p.gmres_abs_tol = fmax(abs_tol_in, norm_pre_rhs * ctx->p.gmres_rel_tol);
    int st2 = faces(rho);
    if (!st2) st2 = stage(w_corr, dt, nullptr, stats2 ? &stats2[1] : nullptr);
    ctx->p.gmres_abs_tol = abs_tol_in;
    if (st2 < 0) return st2;
    return st1 > st2 ? st1 : st2;
}

}  // namespace fhd

using namespace fhd;

extern "C" {

int fhd_dev_advance_overdamped(fhd_ctx* ctx, const fhd_stoch_params* sp, const fhd_mixture_params* mp, double dt,
                               double* const umac[], double* const rho[], double* pi, const double* eta,
                               const double* const eta_ed[], const double* kappa, const double* temperature,
                               const double* const temperature_ed[], const double* const W_cc[],
                               const double* const W_ed[], const double* const W_mass[], fhd_solve_stats* stats2) {
    if (!ctx || !sp || !umac || !rho || !pi || !eta || !eta_ed || !kappa || !temperature || !temperature_ed ||
        !W_cc || !W_ed || (mp && !W_mass) || !(dt > 0.0))
        return FHD_ERR_BAD_ARG;
    if (mp)
        if (int r0 = fhd::refuse_reservoirs(ctx, "advance_timestep_overdamped (multispecies)")) return r0;
    int rc = advance_overdamped(ctx, sp, mp, dt, umac, rho, pi, eta, eta_ed, kappa, temperature, temperature_ed, W_cc,
                                W_ed, W_mass, stats2);
    if (rc < 0) return rc;
    FHD_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return rc;
}

int fhd_dev_stochastic_m_fluxdiv(fhd_ctx* ctx, const fhd_stoch_params* sp, double* const force[], int increment,
                                 const double* eta, const double* const eta_ed[], const double* temperature,
                                 const double* const temperature_ed[], double dt, const double* weights, int n_rngs,
                                 const double* const W_cc[], const double* const W_ed[]) {
    if (!ctx || !sp || !force || !eta || !eta_ed || !temperature || !temperature_ed || !weights || !W_cc || !W_ed)
        return FHD_ERR_BAD_ARG;
    int rc = stoch_launch(ctx, sp, force, increment, eta, eta_ed, temperature, temperature_ed, dt, weights, n_rngs,
                          W_cc, W_ed);
    if (rc) return rc;
    FHD_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int fhd_dev_advance_inertial(fhd_ctx* ctx, const fhd_stoch_params* sp, double dt, double* const umac[], double* rho,
                             double* pi, const double* eta, const double* const eta_ed[], const double* kappa,
                             const double* temperature, const double* const temperature_ed[],
                             const double* const W_cc[], const double* const W_ed[], fhd_solve_stats* stats2) {
    if (!ctx || !sp || !umac || !rho || !pi || !eta || !eta_ed || !kappa || !temperature || !temperature_ed ||
        !W_cc || !W_ed || !(dt > 0.0))
        return FHD_ERR_BAD_ARG;
    double* r[1] = {rho};
    int rc = advance_inertial_ms(ctx, sp, nullptr, dt, umac, r, pi, nullptr, eta, eta_ed, kappa, temperature,
                                 temperature_ed, W_cc, W_ed, nullptr, stats2);
    if (rc < 0) return rc;
    FHD_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return rc;
}

int fhd_dev_advance_inertial_multispecies(fhd_ctx* ctx, const fhd_stoch_params* sp, const fhd_mixture_params* mp,
                                          double dt, double* const umac[], double* const rho[], double* pi,
                                          double* const mass_fluxdiv[], const double* eta,
                                          const double* const eta_ed[], const double* kappa,
                                          const double* temperature, const double* const temperature_ed[],
                                          const double* const W_cc[], const double* const W_ed[],
                                          const double* const W_mass[], fhd_solve_stats* stats2) {
    if (!ctx || !sp || !mp || !umac || !rho || !pi || !mass_fluxdiv || !eta || !eta_ed || !kappa || !temperature ||
        !temperature_ed || !W_cc || !W_ed || !W_mass || !(dt > 0.0))
        return FHD_ERR_BAD_ARG;
    if (int r0 = fhd::refuse_reservoirs(ctx, "advance_timestep_inertial_multispecies")) return r0;
    int rc = advance_inertial_ms(ctx, sp, mp, dt, umac, rho, pi, mass_fluxdiv, eta, eta_ed, kappa, temperature,
                                 temperature_ed, W_cc, W_ed, W_mass, stats2);
    if (rc < 0) return rc;
    FHD_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return rc;
}

}  // extern "C"
