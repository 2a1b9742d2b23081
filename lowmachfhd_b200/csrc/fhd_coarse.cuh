// fhd_coarse.cuh -- the coarse end of both multigrid V-cycles in ONE
// thread block.
//
// Below a few thousand cells a multigrid level is pure latency: every
// smoother colour, residual, restriction and prolongation of the
// stag_mg_solver V-cycle (stag_mg_solver.f90:301-599) and of the pressure
// V-cycle behind macproject (macproject.f90:294-298) is a dependent launch
// that moves a few kilobytes.  These kernels run every level from the first
// one whose arrays fit in shared memory down to the bottom inside one CTA
// of 1024 threads: the unknowns, right-hand sides and residuals of all
// those levels live in shared memory, the read-only coefficients come
// through the L1 (non-coherent loads), and a __syncthreads() replaces each
// launch boundary.
//
// Arithmetic is the same as the per-level kernels: the operator, smoother
// update, restriction and prolongation are the shared expressions of
// fhd_kernels.cuh (stag_lface_acc, cc_lap_acc, stag_restrict_expr,
// stag_prolong_expr, cc_resid_avg) evaluated on shared-memory values, so in
// FP64 the result equals the multi-launch V-cycle bit for bit.  A colour of
// a level whose extents are all even is updated in place (its faces do not
// neighbour each other); odd extents and the Jacobi smoother take two
// passes (new values into the scratch array, then copied), as the
// two-pass kernels do.
#pragma once
#include "fhd_kernels.cuh"

namespace fhd {

constexpr int CS_MAXL = 12;      // levels handled by one coarse kernel
constexpr int CS_THREADS = 1024;

__device__ __forceinline__ bool cs_all_even(const Grid& g) {
    return !(g.n[0] & 1) && !(g.n[1] & 1) && (g.dim == 2 || !(g.n[2] & 1));
}

// linear cell index -> (i, j, k)
__device__ __forceinline__ void cs_ijk(const Grid& g, int f, int& i, int& j, int& k) {
    const int nx = g.n[0], ny = g.n[1];
    i = f % nx;
    const int r = f / nx;
    j = r % ny;
    k = r / ny;
}

// h-th cell of parity par on a level with even n[0]: the half-row index
// of the colour kernels (k_stag_gs, k_cc_gsrb)
__device__ __forceinline__ void cs_ijk_half(const Grid& g, int h, int par, int& i, int& j, int& k) {
    const int nxh = g.n[0] >> 1, ny = g.n[1];
    const int ih = h % nxh;
    const int r = h / nxh;
    j = r % ny;
    k = r / ny;
    i = 2 * ih + ((j + k + par) & 1);
}

// ---------------------------------------------------------------------
// staggered multigrid
// ---------------------------------------------------------------------
template <typename T>
struct StagCoarseArgs {
    int nlev;      // levels of this kernel; level 0 = the first coarse level
    int load_phi;  // level-0 unknowns from phi (else zero, the V-cycle's start)
    int n_down, n_up, n_bottom;
    int jacobi;    // stag_mg_smoother == 0
    T omega;
    T* phi[3];          // level-0 unknowns in global memory (in/out)
    const T* rhs[3];    // level-0 right-hand side
    Grid g[CS_MAXL];
    StagOp<T> A[CS_MAXL];
    int off[CS_MAXL];   // shared-memory element offset of each level
};

// shared-memory arrays of one level: phi, rhs and scratch, dim components
// each of nc elements, in that order from off
template <typename T>
struct CSStag {
    T* ph[3];
    T* rh[3];
    T* tm[3];
    __device__ __forceinline__ void set(T* S, int off, int dim, int nc) {
        for (int c = 0; c < 3; c++) {
            const int cc = c < dim ? c : 0;
            ph[c] = S + off + cc * nc;
            rh[c] = S + off + (dim + cc) * nc;
            tm[c] = S + off + (2 * dim + cc) * nc;
        }
    }
};

// (alpha - L) phi of component C at cell P on shared-memory unknowns, and
// the diagonal
template <typename T, int DIM, int VISC, int C>
__device__ __forceinline__ T cs_lface(const StagOp<T>& A, const CSStag<T>& V, const CellF& P, T& dg) {
    const T* pc = V.ph[C];
    const i64 f = P.base;
    return stag_lface_acc<T, DIM, VISC, C>(
        A, P, [&](int a, int b, int c) { return pc[P.id(a, b, c)]; },
        [&](int d, int a, int b, int c) { return V.ph[d][P.id(a, b, c)]; },
        [&]() { return ld(A.alpha[C], f); }, dg);
}

// new value of the face of component C at (i, j, k): the update of
// k_stag_gs / k_stag_color_update
template <typename T, int DIM, int VISC, int C>
__device__ __forceinline__ T cs_stag_new(const Grid& g, const StagOp<T>& A, const CSStag<T>& V, int i, int j, int k,
                                         T omega, i64& f) {
    CellF P;
    P.set(g, i, j, k);
    f = P.base;
    T dg;
    const T L = cs_lface<T, DIM, VISC, C>(A, V, P, dg);
    return V.ph[C][f] + sm_quot(omega * (V.rh[C][f] - L), dg);
}

// one colour of component C (1-based colour of stag_mg_smoother 1)
template <typename T, int DIM, int VISC, int C>
__device__ void cs_stag_colour(const Grid& g, const StagOp<T>& A, const CSStag<T>& V, int par, T omega) {
    const int nc = (int)g.nc;
    if (cs_all_even(g)) {
        for (int h = threadIdx.x; h < (nc >> 1); h += blockDim.x) {
            int i, j, k;
            cs_ijk_half(g, h, par, i, j, k);
            i64 f;
            const T v = cs_stag_new<T, DIM, VISC, C>(g, A, V, i, j, k, omega, f);
            V.ph[C][f] = v;
        }
        __syncthreads();
    } else {
        for (int f0 = threadIdx.x; f0 < nc; f0 += blockDim.x) {
            int i, j, k;
            cs_ijk(g, f0, i, j, k);
            if (((i + j + k) & 1) != par) continue;
            i64 f;
            const T v = cs_stag_new<T, DIM, VISC, C>(g, A, V, i, j, k, omega, f);
            V.tm[C][f] = v;
        }
        __syncthreads();
        for (int f0 = threadIdx.x; f0 < nc; f0 += blockDim.x) {
            int i, j, k;
            cs_ijk(g, f0, i, j, k);
            if (((i + j + k) & 1) == par) V.ph[C][f0] = V.tm[C][f0];
        }
        __syncthreads();
    }
}

// count smooths of one level (stag_mg_smooth: colours 1..2*dim, or the
// Jacobi sweep)
template <typename T, int DIM, int VISC>
__device__ void cs_stag_smooths(const Grid& g, const StagOp<T>& A, const CSStag<T>& V, int count, int jacobi,
                                T omega) {
    const int nc = (int)g.nc;
    for (int s = 0; s < count; s++) {
        if (jacobi) {
            for (int f0 = threadIdx.x; f0 < nc; f0 += blockDim.x) {
                int i, j, k;
                cs_ijk(g, f0, i, j, k);
                i64 f;
                V.tm[0][f0] = cs_stag_new<T, DIM, VISC, 0>(g, A, V, i, j, k, omega, f);
                V.tm[1][f0] = cs_stag_new<T, DIM, VISC, 1>(g, A, V, i, j, k, omega, f);
                if constexpr (DIM == 3) V.tm[2][f0] = cs_stag_new<T, DIM, VISC, (DIM == 3 ? 2 : 1)>(g, A, V, i, j, k, omega, f);
            }
            __syncthreads();
            for (int f0 = threadIdx.x; f0 < nc; f0 += blockDim.x)
                for (int c = 0; c < DIM; c++) V.ph[c][f0] = V.tm[c][f0];
            __syncthreads();
            continue;
        }
        // colour 2c + 1 is component c at parity 0, colour 2c + 2 the same
        // component at parity 1
        cs_stag_colour<T, DIM, VISC, 0>(g, A, V, 0, omega);
        cs_stag_colour<T, DIM, VISC, 0>(g, A, V, 1, omega);
        cs_stag_colour<T, DIM, VISC, 1>(g, A, V, 0, omega);
        cs_stag_colour<T, DIM, VISC, 1>(g, A, V, 1, omega);
        if constexpr (DIM == 3) {
            cs_stag_colour<T, DIM, VISC, (DIM == 3 ? 2 : 1)>(g, A, V, 0, omega);
            cs_stag_colour<T, DIM, VISC, (DIM == 3 ? 2 : 1)>(g, A, V, 1, omega);
        }
    }
}

// residual rhs - L phi of every component into the scratch arrays
template <typename T, int DIM, int VISC>
__device__ void cs_stag_residual(const Grid& g, const StagOp<T>& A, const CSStag<T>& V) {
    const int nc = (int)g.nc;
    for (int f0 = threadIdx.x; f0 < nc; f0 += blockDim.x) {
        int i, j, k;
        cs_ijk(g, f0, i, j, k);
        CellF P;
        P.set(g, i, j, k);
        T dg;
        V.tm[0][f0] = V.rh[0][f0] - cs_lface<T, DIM, VISC, 0>(A, V, P, dg);
        V.tm[1][f0] = V.rh[1][f0] - cs_lface<T, DIM, VISC, 1>(A, V, P, dg);
        if constexpr (DIM == 3) V.tm[2][f0] = V.rh[2][f0] - cs_lface<T, DIM, VISC, (DIM == 3 ? 2 : 1)>(A, V, P, dg);
    }
    __syncthreads();
}

// the operator of level m with a constant viscosity (visc_type > 0) loaded
// into a register once, rather than after every block barrier
template <typename T, int VISC>
__device__ __forceinline__ StagOp<T> cs_op(const StagCoarseArgs<T>& a, int m) {
    StagOp<T> A = a.A[m];
    if constexpr (VISC > 0) {
        if (!A.beta0_set) {
            A.beta0 = A.beta[0];
            A.beta0_set = 1;
        }
    }
    return A;
}

// the coarse end of one staggered V-cycle in the calling CTA (shared memory
// from the dynamic allocation); also run per box by the batched solver
template <typename T, int DIM, int VISC>
__device__ __forceinline__ void stag_coarse_run(const StagCoarseArgs<T>& a) {
    extern __shared__ __align__(16) unsigned char cs_smem[];
    T* S = reinterpret_cast<T*>(cs_smem);
    const int nt = blockDim.x;
    {
        CSStag<T> V;
        const int nc = (int)a.g[0].nc;
        V.set(S, a.off[0], DIM, nc);
        for (int f = threadIdx.x; f < nc; f += nt)
            for (int c = 0; c < DIM; c++) {
                V.ph[c][f] = a.load_phi ? a.phi[c][f] : T(0);
                V.rh[c][f] = a.rhs[c][f];
            }
    }
    __syncthreads();
    // down: smooth, residual, restrict (stag_mg_solver.f90:301-380)
    for (int m = 0; m + 1 < a.nlev; m++) {
        const Grid& g = a.g[m];
        const Grid& gc = a.g[m + 1];
        CSStag<T> V, W;
        V.set(S, a.off[m], DIM, (int)g.nc);
        W.set(S, a.off[m + 1], DIM, (int)gc.nc);
        const StagOp<T> A = cs_op<T, VISC>(a, m);
        cs_stag_smooths<T, DIM, VISC>(g, A, V, a.n_down, a.jacobi, a.omega);
        cs_stag_residual<T, DIM, VISC>(g, A, V);
        for (int q = threadIdx.x; q < (int)gc.nc; q += nt) {
            int qi, qj, qk;
            cs_ijk(gc, q, qi, qj, qk);
            Cell F;
            F.nx = g.n[0]; F.ny = g.n[1]; F.nz = g.n[2];
            F.i = 2 * qi; F.j = 2 * qj; F.k = (DIM == 3) ? 2 * qk : 0;
#pragma unroll
            for (int c = 0; c < DIM; c++) {
                const T* Fp = V.tm[c];
                W.rh[c][q] = stag_restrict_expr<T, DIM>(
                    0, [&](int o, int pa, int pb) { return Fp[comp_off_id<DIM>(F, c, o, pa, pb)]; });
                W.ph[c][q] = T(0);
            }
        }
        __syncthreads();
    }
    {
        const int m = a.nlev - 1;
        CSStag<T> V;
        V.set(S, a.off[m], DIM, (int)a.g[m].nc);
        cs_stag_smooths<T, DIM, VISC>(a.g[m], cs_op<T, VISC>(a, m), V, a.n_bottom, a.jacobi, a.omega);
    }
    // up: prolong, smooth (stag_mg_solver.f90:380-420)
    for (int m = a.nlev - 2; m >= 0; m--) {
        const Grid& g = a.g[m];
        const Grid& gc = a.g[m + 1];
        CSStag<T> V, W;
        V.set(S, a.off[m], DIM, (int)g.nc);
        W.set(S, a.off[m + 1], DIM, (int)gc.nc);
        for (int f0 = threadIdx.x; f0 < (int)g.nc; f0 += nt) {
            int I[3];
            cs_ijk(g, f0, I[0], I[1], I[2]);
            Cell H;
            H.nx = gc.n[0]; H.ny = gc.n[1]; H.nz = gc.n[2];
            H.i = I[0] >> 1; H.j = I[1] >> 1; H.k = I[2] >> 1;
#pragma unroll
            for (int c = 0; c < DIM; c++) {
                const T* Cp = W.ph[c];
                const int ca = (c == 0) ? 1 : 0;
                const int cb = (c == 2) ? 1 : 2;
                const int oa = (I[ca] & 1) ? 1 : -1;
                const int ob = (DIM == 3) ? ((I[cb] & 1) ? 1 : -1) : 0;
                const T v = stag_prolong_expr<T, DIM>((I[c] & 1) == 0, oa, ob, [&](int o, int pa, int pb) {
                    return Cp[comp_off_id<DIM>(H, c, o, pa, pb)];
                });
                V.ph[c][f0] = V.ph[c][f0] + v;
            }
        }
        __syncthreads();
        cs_stag_smooths<T, DIM, VISC>(g, cs_op<T, VISC>(a, m), V, a.n_up, a.jacobi, a.omega);
    }
    {
        CSStag<T> V;
        const int nc = (int)a.g[0].nc;
        V.set(S, a.off[0], DIM, nc);
        for (int f = threadIdx.x; f < nc; f += nt)
            for (int c = 0; c < DIM; c++) a.phi[c][f] = V.ph[c][f];
    }
}

template <typename T, int DIM, int VISC>
__global__ void __launch_bounds__(CS_THREADS) k_stag_coarse(const __grid_constant__ StagCoarseArgs<T> a) {
    stag_coarse_run<T, DIM, VISC>(a);
}

// ---------------------------------------------------------------------
// pressure multigrid
// ---------------------------------------------------------------------
template <typename T>
struct CCCoarseArgs {
    int nlev;
    int load_phi;
    int n_down, n_up, n_bottom;
    T* phi;          // level-0 unknowns in global memory (in/out)
    const T* rhs;
    Grid g[CS_MAXL];
    CCOp<T> A[CS_MAXL];
    int off[CS_MAXL];  // phi at off, rhs at off + nc, scratch at off + 2 nc
};

// count red-black smooths (k_cc_gsrb / the two-pass colour kernels)
template <typename T, int DIM>
__device__ void cs_cc_smooths(const Grid& g, const CCOp<T>& A, T* ph, const T* rh, T* tm, int count) {
    const int nc = (int)g.nc;
    const bool even = cs_all_even(g);
    for (int s = 0; s < count; s++)
        for (int par = 0; par < 2; par++) {
            if (even) {
                for (int h = threadIdx.x; h < (nc >> 1); h += blockDim.x) {
                    int i, j, k;
                    cs_ijk_half(g, h, par, i, j, k);
                    CellF P;
                    P.set(g, i, j, k);
                    T dg;
                    const T L = cc_lap_acc<T, DIM>(A, P, [&](int a, int b, int c) { return ph[P.id(a, b, c)]; }, dg);
                    const i64 f = P.base;
                    ph[f] = ph[f] + sm_quot(rh[f] - L, dg);
                }
                __syncthreads();
            } else {
                for (int f0 = threadIdx.x; f0 < nc; f0 += blockDim.x) {
                    int i, j, k;
                    cs_ijk(g, f0, i, j, k);
                    if (((i + j + k) & 1) != par) continue;
                    CellF P;
                    P.set(g, i, j, k);
                    T dg;
                    const T L = cc_lap_acc<T, DIM>(A, P, [&](int a, int b, int c) { return ph[P.id(a, b, c)]; }, dg);
                    tm[f0] = sm_quot(rh[f0] - L, dg);
                }
                __syncthreads();
                for (int f0 = threadIdx.x; f0 < nc; f0 += blockDim.x) {
                    int i, j, k;
                    cs_ijk(g, f0, i, j, k);
                    if (((i + j + k) & 1) == par) ph[f0] = ph[f0] + tm[f0];
                }
                __syncthreads();
            }
        }
}

// the coarse end of one pressure V-cycle in the calling CTA; also run per
// box by the batched solver
template <typename T, int DIM>
__device__ __forceinline__ void cc_coarse_run(const CCCoarseArgs<T>& a) {
    extern __shared__ __align__(16) unsigned char cs_smem[];
    T* S = reinterpret_cast<T*>(cs_smem);
    const int nt = blockDim.x;
    {
        const int nc = (int)a.g[0].nc;
        T* ph = S + a.off[0];
        T* rh = ph + nc;
        for (int f = threadIdx.x; f < nc; f += nt) {
            ph[f] = a.load_phi ? a.phi[f] : T(0);
            rh[f] = a.rhs[f];
        }
    }
    __syncthreads();
    for (int m = 0; m + 1 < a.nlev; m++) {
        const Grid& g = a.g[m];
        const Grid& gc = a.g[m + 1];
        const int nc = (int)g.nc, ncc = (int)gc.nc;
        T* ph = S + a.off[m];
        T* rh = ph + nc;
        T* tm = rh + nc;
        T* cph = S + a.off[m + 1];
        T* crh = cph + ncc;
        cs_cc_smooths<T, DIM>(g, a.A[m], ph, rh, tm, a.n_down);
        for (int q = threadIdx.x; q < ncc; q += nt) {
            int qi, qj, qk;
            cs_ijk(gc, q, qi, qj, qk);
            crh[q] = cc_resid_avg<T, DIM>(
                a.A[m], g, qi, qj, qk, [&](i64 i) { return ph[i]; }, [&](i64 i) { return rh[i]; });
            cph[q] = T(0);
        }
        __syncthreads();
    }
    {
        const int m = a.nlev - 1;
        const int nc = (int)a.g[m].nc;
        T* ph = S + a.off[m];
        cs_cc_smooths<T, DIM>(a.g[m], a.A[m], ph, ph + nc, ph + 2 * nc, a.n_bottom);
    }
    for (int m = a.nlev - 2; m >= 0; m--) {
        const Grid& g = a.g[m];
        const Grid& gc = a.g[m + 1];
        const int nc = (int)g.nc;
        T* ph = S + a.off[m];
        const T* cph = S + a.off[m + 1];
        for (int f0 = threadIdx.x; f0 < nc; f0 += nt) {
            int i, j, k;
            cs_ijk(g, f0, i, j, k);
            const i64 c = (i64)(i >> 1) + (i64)gc.n[0] * ((i64)(j >> 1) + (i64)gc.n[1] * (k >> 1));
            ph[f0] = ph[f0] + cph[c];
        }
        __syncthreads();
        cs_cc_smooths<T, DIM>(g, a.A[m], ph, ph + nc, ph + 2 * nc, a.n_up);
    }
    {
        const int nc = (int)a.g[0].nc;
        const T* ph = S + a.off[0];
        for (int f = threadIdx.x; f < nc; f += nt) a.phi[f] = ph[f];
    }
}

template <typename T, int DIM>
__global__ void __launch_bounds__(CS_THREADS) k_cc_coarse(const __grid_constant__ CCCoarseArgs<T> a) {
    cc_coarse_run<T, DIM>(a);
}

}  // namespace fhd
