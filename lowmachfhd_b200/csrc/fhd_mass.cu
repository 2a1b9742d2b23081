// fhd_mass.cu -- multispecies mass fluxes (compute_mass_fluxdiv of
// LowMachFHD src_multiSpec) for an ideal isothermal mixture: the diffusive
// flux rhoWchi * grad(x) and the stochastic flux sqrt(2 k_B var/(dV dt)) *
// chol(L(rho_av)) * W, each corrected to a zero species sum, and their
// divergence.
//
// Compute-bound per face (Dbar2chi_iterative: chi_iterations dense NS x NS
// products, a Cholesky factorisation, two matrix-vector products); the
// matrices live in registers, the species count is a template parameter.
// T = double, or float in the mixed-precision mode.
#include <cmath>
#include <cstring>

#include "fhd_solver.cuh"

namespace fhd {

struct MixDev {
    int ns;
    double molmass[FHD_MAX_SPECIES];
    double D[FHD_MAX_SPECIES][FHD_MAX_SPECIES];
    double var_mass;
    int chi_it;
    double frac_tol;
    int correct;
    int avg_type;
    double kB, dV;
    // FP32 mirrors for the mixed-precision kernels: the constants and the
    // reciprocals of the constant divisors (Dinv_f[i][i] = 0)
    float mm_f[FHD_MAX_SPECIES], imm_f[FHD_MAX_SPECIES];
    float Dinv_f[FHD_MAX_SPECIES][FHD_MAX_SPECIES];
    float ikB_f, dV_f, tol_f;
};

#ifndef FHD_MASS_F32_TU
MixDev make_mixdev(const fhd_mixture_params* mp, const fhd_stoch_params* sp) {
    MixDev m;
    memset(&m, 0, sizeof(m));
    m.ns = mp->nspecies;
    for (int i = 0; i < m.ns; i++) m.molmass[i] = mp->molmass[i];
    int k = 0;
    for (int r = 0; r < m.ns; r++) {
        for (int c = 0; c < r; c++) {
            m.D[r][c] = mp->Dbar[k];
            m.D[c][r] = mp->Dbar[k];
            k++;
        }
        m.D[r][r] = 0.0;
    }
    m.var_mass = mp->variance_coef_mass;
    m.chi_it = mp->chi_iterations;
    m.frac_tol = mp->fraction_tolerance;
    m.correct = mp->correct_flux;
    m.avg_type = mp->avg_type;
    m.kB = sp->k_B;
    m.dV = sp->dV;
    for (int i = 0; i < m.ns; i++) {
        m.mm_f[i] = (float)m.molmass[i];
        m.imm_f[i] = (float)(1.0 / m.molmass[i]);
        for (int j = 0; j < m.ns; j++) m.Dinv_f[i][j] = (i == j) ? 0.0f : (float)(1.0 / m.D[i][j]);
    }
    m.ikB_f = (float)(1.0 / m.kB);
    m.dV_f = (float)m.dV;
    m.tol_f = (float)m.frac_tol;
    return m;
}
#endif

// FP32 arithmetic of the mixed-precision kernels: fused multiply-adds,
// products with the host-computed reciprocals of the constant divisors
// (molar masses, Dbar, k_B), one fast reciprocal per repeated divisor, and
// the closed forms of two of Dbar2chi_iterative's products: P J = J - 1 (Y^T
// J) and P diag(Minv) P^T = diag(Minv) - Y Minv 1^T - 1 (Y Minv)^T +
// sum(Y^2 Minv), with P = I - 1 Y^T.  The FP64 kernels keep the
// restatement's operations and order (parity with the CPU oracle).
__device__ __forceinline__ float frcp(float x) { return __fdividef(1.0f, x); }

template <int NS>
__device__ __forceinline__ void d_molconc_f(const MixDev& m, const float* rho, float rhotot, float* x, float& mtot) {
    const float ri = frcp(rhotot);
    float W[NS];
    float s = 0.0f;
#pragma unroll
    for (int n = 0; n < NS; n++) {
        W[n] = rho[n] * ri;
        s = __fmaf_rn(W[n], m.imm_f[n], s);
    }
    mtot = frcp(s);
#pragma unroll
    for (int n = 0; n < NS; n++) x[n] = mtot * W[n] * m.imm_f[n];
}

// Dbar2chi_iterative (matrix_utilities.f90:19-158), NS >= 3, FP32
template <int NS>
__device__ __forceinline__ void d_chi_f(const MixDev& m, const float* Xk, int chi_it, float (&chi)[NS][NS]) {
    float mw = 0.0f;
#pragma unroll
    for (int i = 0; i < NS; i++) mw = __fmaf_rn(Xk[i], m.mm_f[i], mw);
    const float imw = frcp(mw);
    float Y[NS], Minv[NS], Mm[NS], t2[NS];
#pragma unroll
    for (int i = 0; i < NS; i++) {
        Y[i] = m.mm_f[i] * imw * Xk[i];
        float t = 0.0f;
#pragma unroll
        for (int j = 0; j < NS; j++) t = __fmaf_rn(Xk[j], m.Dinv_f[i][j], t);
        t2[i] = t;
        const float Di = __fdividef(1.0f - Y[i], t);
        Mm[i] = __fdividef(Xk[i], Di);
        Minv[i] = __fdividef(Di, Xk[i]);
    }
    // J = Minv (M - Delta): Delta_ii = X_i sum_k X_k / D_ik, Delta_ij = -X_i X_j / D_ij
    float J[NS][NS];
#pragma unroll
    for (int i = 0; i < NS; i++)
#pragma unroll
        for (int j = 0; j < NS; j++)
            J[i][j] = (i == j) ? Minv[i] * (Mm[i] - Xk[i] * t2[i]) : Minv[i] * (Xk[i] * Xk[j] * m.Dinv_f[i][j]);
    float cs[NS];
#pragma unroll
    for (int j = 0; j < NS; j++) {
        float a = 0.0f;
#pragma unroll
        for (int k = 0; k < NS; k++) a = __fmaf_rn(Y[k], J[k][j], a);
        cs[j] = a;
    }
    float sY = 0.0f, YM[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) {
        YM[k] = Y[k] * Minv[k];
        sY = __fmaf_rn(Y[k], YM[k], sY);
    }
    float PJ[NS][NS], m2[NS][NS];
#pragma unroll
    for (int i = 0; i < NS; i++)
#pragma unroll
        for (int j = 0; j < NS; j++) {
            PJ[i][j] = J[i][j] - cs[j];
            m2[i][j] = ((i == j) ? Minv[i] : 0.0f) - YM[i] - YM[j] + sY;
            chi[i][j] = m2[i][j];
        }
    for (int it = 0; it < chi_it; it++) {
        float m1[NS][NS];
#pragma unroll
        for (int i = 0; i < NS; i++)
#pragma unroll
            for (int j = 0; j < NS; j++) {
                float a = m2[i][j];
#pragma unroll
                for (int k = 0; k < NS; k++) a = __fmaf_rn(PJ[i][k], chi[k][j], a);
                m1[i][j] = a;
            }
#pragma unroll
        for (int i = 0; i < NS; i++)
#pragma unroll
            for (int j = 0; j < NS; j++) chi[i][j] = m1[i][j];
    }
}

// choldc (matrix_utilities.f90:162-241), FP32: 1/p from the fast
// reciprocal square root
template <int NS>
__device__ __forceinline__ void d_choldc_f(float (&a)[NS][NS]) {
    float p[NS];
#pragma unroll
    for (int i = 0; i < NS; i++) {
        int ising = 0;
        float r = 0.0f;
#pragma unroll
        for (int j = i; j < NS; j++) {
            float s = a[i][j];
#pragma unroll
            for (int k = i - 1; k >= 0; k--) s = __fmaf_rn(-a[i][k], a[j][k], s);
            if (i == j) {
                if (s <= 0.0f) {
                    p[i] = 0.0f;
                    ising = 1;
                } else {
                    r = rsqrtf(s);
                    p[i] = s * r;
                }
            } else {
                a[j][i] = (ising == 0) ? s * r : 0.0f;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < NS; i++) {
#pragma unroll
        for (int j = i + 1; j < NS; j++) a[i][j] = 0.0f;
        a[i][i] = p[i];
    }
}

// compute_molconc_molmtot_local (mass_flux_utilities.f90:159-186)
template <typename T, int NS>
__device__ __forceinline__ void d_molconc(const MixDev& m, const T* rho, T rhotot, T* x, T& mtot) {
    T W[NS];
    T s = T(0);
#pragma unroll
    for (int n = 0; n < NS; n++) {
        W[n] = rho[n] / rhotot;
        s = s + W[n] / (T)m.molmass[n];
    }
    mtot = T(1) / s;
#pragma unroll
    for (int n = 0; n < NS; n++) x[n] = mtot * W[n] / (T)m.molmass[n];
}

// compute_chi (mass_flux_utilities.f90:743-922): closed form for two
// species, Dbar2chi_iterative (matrix_utilities.f90:19-158) otherwise
template <typename T, int NS>
__device__ __forceinline__ void d_chi(const MixDev& m, const T* rho, T rhotot, const T* Xk, T (&chi)[NS][NS]) {
    if constexpr (NS == 2) {
        const T W0 = rho[0] / rhotot, W1 = rho[1] / rhotot;
        T t = (T)m.molmass[0] * W1 + (T)m.molmass[1] * W0;
        t = (T)m.D[0][1] * t * t / (T)m.molmass[0] / (T)m.molmass[1];
        chi[0][0] = t * W1 / W0;
        chi[0][1] = -t;
        chi[1][0] = -t;
        chi[1][1] = t * W0 / W1;
    } else {
        T mw = T(0), Y[NS], Minv[NS];
#pragma unroll
        for (int i = 0; i < NS; i++) mw = mw + Xk[i] * (T)m.molmass[i];
#pragma unroll
        for (int i = 0; i < NS; i++) Y[i] = (T)m.molmass[i] / mw * Xk[i];
        T Mm[NS];
#pragma unroll
        for (int i = 0; i < NS; i++) {
            T t2 = T(0);
#pragma unroll
            for (int j = 0; j < NS; j++)
                if (j != i) t2 = t2 + Xk[j] / (T)m.D[i][j];
            const T Di = (T(1) - Y[i]) / t2;
            Mm[i] = Xk[i] / Di;
            Minv[i] = Di / Xk[i];
        }
        // J = Minv * (M - Delta); PJ = P J with P = I - 1 Y^T
        T J[NS][NS];
#pragma unroll
        for (int i = 0; i < NS; i++) {
#pragma unroll
            for (int j = 0; j < NS; j++) {
                T dl;
                if (i == j) {
                    T t1 = T(0);
#pragma unroll
                    for (int k = 0; k < NS; k++)
                        if (k != i) t1 = t1 + Xk[i] * Xk[k] / (T)m.D[i][k];
                    dl = t1;
                } else {
                    dl = -Xk[i] * Xk[j] / (T)m.D[i][j];
                }
                T z = -dl;
                if (i == j) z = z + Mm[i];
                J[i][j] = Minv[i] * z;
            }
        }
        T PJ[NS][NS], m2[NS][NS];
#pragma unroll
        for (int i = 0; i < NS; i++)
#pragma unroll
            for (int j = 0; j < NS; j++) {
                T a = T(0);
#pragma unroll
                for (int k = 0; k < NS; k++) {
                    const T pik = (i == k ? T(1) : T(0)) - Y[k];
                    a = a + pik * J[k][j];
                }
                PJ[i][j] = a;
            }
#pragma unroll
        for (int i = 0; i < NS; i++)
#pragma unroll
            for (int j = 0; j < NS; j++) {
                T scr = T(0);
#pragma unroll
                for (int k = 0; k < NS; k++) {
                    const T pik = (i == k ? T(1) : T(0)) - Y[k];
                    const T pjk = (j == k ? T(1) : T(0)) - Y[k];
                    scr = scr + pik * Minv[k] * pjk;
                }
                m2[i][j] = scr;
                chi[i][j] = scr;
            }
        for (int it = 0; it < m.chi_it; it++) {
            T m1[NS][NS];
#pragma unroll
            for (int i = 0; i < NS; i++)
#pragma unroll
                for (int j = 0; j < NS; j++) {
                    T scr = T(0);
#pragma unroll
                    for (int k = 0; k < NS; k++) scr = scr + PJ[i][k] * chi[k][j];
                    m1[i][j] = scr + m2[i][j];
                }
#pragma unroll
            for (int i = 0; i < NS; i++)
#pragma unroll
                for (int j = 0; j < NS; j++) chi[i][j] = m1[i][j];
        }
    }
}

// trace species (mass fraction below fraction_tolerance): returns the
// mask of the non-trace species and their count in *nact
template <typename T, int NS>
__device__ __forceinline__ unsigned d_active(const MixDev& m, const T* rho, T rhotot, int* nact) {
    unsigned act = 0u;
    int na = 0;
    if constexpr (sizeof(T) == 4) {
        const float ri = frcp(rhotot);
#pragma unroll
        for (int i = 0; i < NS; i++)
            if (!(rho[i] * ri < m.tol_f)) {
                act |= 1u << i;
                na++;
            }
    } else {
#pragma unroll
        for (int i = 0; i < NS; i++)
            if (!(rho[i] / rhotot < (T)m.frac_tol)) {
                act |= 1u << i;
                na++;
            }
    }
    *nact = na;
    return act;
}

// ---------------------------------------------------------------------
// the subsystem of non-trace species (compute_chi_sub and
// compute_sqrtLonsager_sub, mass_flux_utilities.f90:654-739, 1425-1502),
// on the full NS-sized register arrays: a trace species' entries are
// skipped by the mask `act`, and every sum runs over the non-trace species
// in increasing order, which is the order of the reference's compacted
// subsystem arrays (dest).  A face or cell takes this branch only when some
// but not all-but-one species are trace.
// ---------------------------------------------------------------------
template <typename T, int NS>
struct SubSys {
    T rt, mt;          // subsystem total density, molar mass
    T x[NS];           // subsystem molar concentrations (0 for trace species)
    T chi[NS][NS];     // subsystem chi (0 on trace rows and columns)
};

template <typename T, int NS, class MX>
__device__ __forceinline__ void d_subsys(const MX& m, unsigned act, int nsub, const T* rho, SubSys<T, NS>& S) {
    const auto on = [&](int i) { return (act >> i) & 1u; };
    S.rt = T(0);
#pragma unroll
    for (int i = 0; i < NS; i++)
        if (on(i)) S.rt = S.rt + rho[i];
    // compute_molconc_molmtot_local on the subsystem
    T W[NS];
    T s = T(0);
#pragma unroll
    for (int i = 0; i < NS; i++) {
        W[i] = T(0);
        if (on(i)) {
            W[i] = rho[i] / S.rt;
            s = s + W[i] / (T)m.molmass[i];
        }
    }
    S.mt = T(1) / s;
#pragma unroll
    for (int i = 0; i < NS; i++) S.x[i] = on(i) ? S.mt * W[i] / (T)m.molmass[i] : T(0);
#pragma unroll
    for (int i = 0; i < NS; i++)
#pragma unroll
        for (int j = 0; j < NS; j++) S.chi[i][j] = T(0);
    if (nsub == 2) {
        // compute_chi's closed form for two species (mass_flux_utilities.f90:767-786)
        int a = -1, b = -1;
#pragma unroll
        for (int i = 0; i < NS; i++)
            if (on(i)) {
                if (a < 0) a = i;
                else b = i;
            }
        T ra = T(0), rb = T(0);
#pragma unroll
        for (int i = 0; i < NS; i++) {
            if (i == a) ra = rho[i];
            if (i == b) rb = rho[i];
        }
        const T W0 = ra / S.rt, W1 = rb / S.rt;
        const T ma = (T)m.molmass[a], mb = (T)m.molmass[b];
        T t = ma * W1 + mb * W0;
        t = (T)m.D[a][b] * t * t / ma / mb;
#pragma unroll
        for (int i = 0; i < NS; i++)
#pragma unroll
            for (int j = 0; j < NS; j++) {
                if (i == a && j == a) S.chi[i][j] = t * W1 / W0;
                if ((i == a && j == b) || (i == b && j == a)) S.chi[i][j] = -t;
                if (i == b && j == b) S.chi[i][j] = t * W0 / W1;
            }
        return;
    }
    // Dbar2chi_iterative (matrix_utilities.f90:19-158) on the subsystem
    const T* Xk = S.x;
    T mw = T(0), Y[NS], Minv[NS], Mm[NS];
#pragma unroll
    for (int i = 0; i < NS; i++)
        if (on(i)) mw = mw + Xk[i] * (T)m.molmass[i];
#pragma unroll
    for (int i = 0; i < NS; i++) {
        Y[i] = on(i) ? (T)m.molmass[i] / mw * Xk[i] : T(0);
        Mm[i] = T(0);
        Minv[i] = T(0);
        if (on(i)) {
            T t2 = T(0);
#pragma unroll
            for (int j = 0; j < NS; j++)
                if (j != i && on(j)) t2 = t2 + Xk[j] / (T)m.D[i][j];
            const T Di = (T(1) - Y[i]) / t2;
            Mm[i] = Xk[i] / Di;
            Minv[i] = Di / Xk[i];
        }
    }
    T J[NS][NS];
#pragma unroll
    for (int i = 0; i < NS; i++)
#pragma unroll
        for (int j = 0; j < NS; j++) {
            J[i][j] = T(0);
            if (!on(i) || !on(j)) continue;
            T dl;
            if (i == j) {
                T t1 = T(0);
#pragma unroll
                for (int k = 0; k < NS; k++)
                    if (k != i && on(k)) t1 = t1 + Xk[i] * Xk[k] / (T)m.D[i][k];
                dl = t1;
            } else {
                dl = -Xk[i] * Xk[j] / (T)m.D[i][j];
            }
            T z = -dl;
            if (i == j) z = z + Mm[i];
            J[i][j] = Minv[i] * z;
        }
    T PJ[NS][NS], m2[NS][NS];
#pragma unroll
    for (int i = 0; i < NS; i++)
#pragma unroll
        for (int j = 0; j < NS; j++) {
            T a = T(0), scr = T(0);
            if (on(i) && on(j)) {
#pragma unroll
                for (int k = 0; k < NS; k++) {
                    if (!on(k)) continue;
                    const T pik = (i == k ? T(1) : T(0)) - Y[k];
                    const T pjk = (j == k ? T(1) : T(0)) - Y[k];
                    a = a + pik * J[k][j];
                    scr = scr + pik * Minv[k] * pjk;
                }
            }
            PJ[i][j] = a;
            m2[i][j] = scr;
            S.chi[i][j] = scr;
        }
    for (int it = 0; it < m.chi_it; it++) {
        T m1[NS][NS];
#pragma unroll
        for (int i = 0; i < NS; i++)
#pragma unroll
            for (int j = 0; j < NS; j++) {
                T scr = T(0);
#pragma unroll
                for (int k = 0; k < NS; k++)
                    if (on(k)) scr = scr + PJ[i][k] * S.chi[k][j];
                m1[i][j] = (on(i) && on(j)) ? scr + m2[i][j] : T(0);
            }
#pragma unroll
        for (int i = 0; i < NS; i++)
#pragma unroll
            for (int j = 0; j < NS; j++) S.chi[i][j] = m1[i][j];
    }
}

// compute_chi_sub's rho W chi (mass_flux_utilities.f90:698-738): the
// subsystem's rho chi, and for a trace species' column its effective
// diffusion coefficient terms
template <typename T, int NS, class MX>
__device__ __forceinline__ void d_rhowchi_sub(const MX& m, unsigned act, int nsub, const T* rho, T (&out)[NS][NS]) {
    const auto on = [&](int i) { return (act >> i) & 1u; };
    SubSys<T, NS> S;
    d_subsys<T, NS, MX>(m, act, nsub, rho, S);
#pragma unroll
    for (int col = 0; col < NS; col++) {
        if (!on(col)) {
            T deff = T(0);
#pragma unroll
            for (int k = 0; k < NS; k++)
                if (on(k)) deff = deff + S.x[k] / (T)m.D[k][col];
            deff = T(1) / deff;
#pragma unroll
            for (int row = 0; row < NS; row++) {
                if (row == col) {
                    out[row][col] = S.rt * deff * (T)m.molmass[row] / S.mt;
                } else if (!on(row)) {
                    out[row][col] = T(0);
                } else {
                    T tmp = T(0);
#pragma unroll
                    for (int k = 0; k < NS; k++)
                        if (on(k)) tmp = tmp + S.chi[row][k] * S.x[k] / (T)m.D[k][col];
                    out[row][col] = deff * rho[row] * (tmp - (T)m.molmass[col] / S.mt);
                }
            }
        } else {
#pragma unroll
            for (int row = 0; row < NS; row++) out[row][col] = on(row) ? rho[row] * S.chi[row][col] : T(0);
        }
    }
}

// compute_sqrtLonsager_sub (mass_flux_utilities.f90:1440-1500): the
// Cholesky factor of the subsystem's Onsager matrix, expanded with zeros
template <typename T, int NS, class MX>
__device__ __forceinline__ void d_sqrtL_sub(const MX& m, unsigned act, int nsub, const T* rho, T (&L)[NS][NS]) {
    const auto on = [&](int i) { return (act >> i) & 1u; };
    SubSys<T, NS> S;
    d_subsys<T, NS, MX>(m, act, nsub, rho, S);
    T Ws[NS];
#pragma unroll
    for (int i = 0; i < NS; i++) Ws[i] = on(i) ? rho[i] / S.rt : T(0);
    const T kB = (T)m.kB;
#pragma unroll
    for (int c = 0; c < NS; c++)
#pragma unroll
        for (int r = 0; r < NS; r++)
            L[r][c] = (on(r) && on(c)) ? S.mt * S.rt * Ws[r] * S.chi[r][c] * Ws[c] / kB : T(0);
    // choldc (matrix_utilities.f90:162-241) over the non-trace rows; the
    // inner sums run downwards, as the reference's do
    T p[NS];
#pragma unroll
    for (int i = 0; i < NS; i++) {
        p[i] = T(0);
        if (!on(i)) continue;
        int ising = 0;
#pragma unroll
        for (int j = i; j < NS; j++) {
            if (!on(j)) continue;
            T s = L[i][j];
#pragma unroll
            for (int k = i - 1; k >= 0; k--)
                if (on(k)) s = s - L[i][k] * L[j][k];
            if (i == j) {
                if (s <= T(0)) {
                    p[i] = T(0);
                    ising = 1;
                } else {
                    p[i] = sqrt(s);
                }
            } else {
                L[j][i] = (ising == 0) ? s / p[i] : T(0);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < NS; i++) {
#pragma unroll
        for (int j = i + 1; j < NS; j++) L[i][j] = T(0);
        L[i][i] = p[i];
    }
}

// molar concentrations and chi in the arithmetic of T
template <typename T, int NS>
__device__ __forceinline__ void d_molconc_t(const MixDev& m, const T* rho, T rhotot, T* x, T& mtot) {
    if constexpr (sizeof(T) == 4) d_molconc_f<NS>(m, rho, rhotot, x, mtot);
    else d_molconc<T, NS>(m, rho, rhotot, x, mtot);
}

template <typename T, int NS>
__device__ __forceinline__ void d_chi_t(const MixDev& m, const T* rho, T rhotot, const T* Xk, T (&chi)[NS][NS]) {
    if constexpr (sizeof(T) == 4 && NS >= 3) d_chi_f<NS>(m, Xk, m.chi_it, chi);
    else d_chi<T, NS>(m, rho, rhotot, Xk, chi);
}

// choldc (matrix_utilities.f90:162-241)
template <typename T, int NS>
__device__ __forceinline__ void d_choldc(T (&a)[NS][NS]) {
    T p[NS];
#pragma unroll
    for (int i = 0; i < NS; i++) {
        int ising = 0;
#pragma unroll
        for (int j = i; j < NS; j++) {
            T s = a[i][j];
#pragma unroll
            for (int k = i - 1; k >= 0; k--) s = s - a[i][k] * a[j][k];
            if (i == j) {
                if (s <= T(0)) {
                    p[i] = T(0);
                    ising = 1;
                } else {
                    p[i] = sqrt(s);
                }
            } else {
                a[j][i] = (ising == 0) ? s / p[i] : T(0);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < NS; i++) {
#pragma unroll
        for (int j = i + 1; j < NS; j++) a[i][j] = T(0);
        a[i][i] = p[i];
    }
}

// Faces and cells with some but not all-but-one trace species take the
// subsystem branch.  It is rare, and its registers would lower the
// occupancy of the latency-bound main kernels, so those append the index to
// a list and skip it; a follow-up kernel finishes exactly the listed ones.
struct TraceList {
    int* idx;          // capacity: one entry per cell of the level
    unsigned* count;   // entries appended (cleared before each main kernel)
};

__device__ __forceinline__ void trace_push(const TraceList& tl, i64 f) {
    const unsigned q = atomicAdd(tl.count, 1u);
    tl.idx[q] = (int)f;
}

// ---------------------------------------------------------------------
// per cell: rhoWchi (compute_rhoWchi_local) and the molar concentrations
// ---------------------------------------------------------------------
template <typename T, int NS>
__global__ void __launch_bounds__(128, (sizeof(T) == 4 && NS <= 4) ? 8 : 1)
    k_rhowchi(Grid g, MixDev m, const double* const* __restrict__ rho, T* const* rwc, T* const* xo, TraceList tl) {
    const i64 n = g.nc;
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x) {
        T r[NS];
        T rt = T(0);
#pragma unroll
        for (int s = 0; s < NS; s++) {
            r[s] = (T)rho[s][f];
            rt = rt + r[s];
        }
        T x[NS], mt;
        d_molconc_t<T, NS>(m, r, rt, x, mt);
#pragma unroll
        for (int s = 0; s < NS; s++) xo[s][f] = x[s];
        int na;
        d_active<T, NS>(m, r, rt, &na);
        if (na == 1) {
#pragma unroll
            for (int q = 0; q < NS * NS; q++) rwc[q][f] = T(0);
            continue;
        }
        if (na != NS) {
            trace_push(tl, f);
            continue;
        }
        T chi[NS][NS];
        d_chi_t<T, NS>(m, r, rt, x, chi);
#pragma unroll
        for (int i = 0; i < NS; i++)
#pragma unroll
            for (int j = 0; j < NS; j++) rwc[i * NS + j][f] = r[i] * chi[i][j];
    }
}

// the listed cells of k_rhowchi: compute_chi_sub's rho W chi
template <typename T, int NS>
__global__ void __launch_bounds__(128) k_rhowchi_trace(MixDev m, const double* const* __restrict__ rho,
                                                       T* const* rwc, TraceList tl) {
    const unsigned cnt = *tl.count;
    for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt; q += gridDim.x * blockDim.x) {
        const i64 f = tl.idx[q];
        T r[NS];
        T rt = T(0);
#pragma unroll
        for (int s = 0; s < NS; s++) {
            r[s] = (T)rho[s][f];
            rt = rt + r[s];
        }
        int na;
        const unsigned act = d_active<T, NS>(m, r, rt, &na);
        T a[NS][NS];
        d_rhowchi_sub<T, NS>(m, act, na, r, a);
#pragma unroll
        for (int i = 0; i < NS; i++)
#pragma unroll
            for (int j = 0; j < NS; j++) rwc[i * NS + j][f] = a[i][j];
    }
}

// compute_nonnegative_rho_av (mass_flux_utilities.f90:1231-1328) on the face
// between cells fm and f, and the sum of the averages
template <typename T, int NS>
__device__ __forceinline__ void d_face_rho_av(const MixDev& m, const double* const* __restrict__ rho, i64 f, i64 fm,
                                              T (&ra)[NS], T& rt) {
    rt = T(0);
#pragma unroll
    for (int c = 0; c < NS; c++) {
        T mm, v1, v2;
        if constexpr (sizeof(T) == 4) {
            mm = m.mm_f[c];
            v1 = (float)ld(rho[c], fm) * m.imm_f[c];
            v2 = (float)ld(rho[c], f) * m.imm_f[c];
        } else {
            mm = (T)m.molmass[c];
            v1 = (T)ld(rho[c], fm) / mm;
            v2 = (T)ld(rho[c], f) / mm;
        }
        T o;
        if (m.avg_type == 2) {
            o = mm * sqrt(fmax(v1, T(0)) * fmax(v2, T(0)));
        } else if (m.avg_type == 3) {
            o = (v1 <= T(0) || v2 <= T(0)) ? T(0) : mm * T(2) / (T(1) / v1 + T(1) / v2);
        } else if (m.avg_type == 10) {
            o = (v1 <= T(0) || v2 <= T(0)) ? T(0) : mm * (v1 + v2) / T(2);
        } else {
            if (v1 <= T(0) || v2 <= T(0)) {
                o = T(0);
            } else {
                const T t1 = fmin((T)m.dV * v1, T(1)), t2 = fmin((T)m.dV * v2, T(1));
                o = mm * (v1 + v2) / T(2) * t1 * t2;
            }
        }
        ra[c] = o;
        rt = rt + o;
    }
}

// compute_sqrtLonsager_local (mass_flux_utilities.f90:1331-1522) without
// trace species: chol(mtot rhotot W chi W / k_B)
template <typename T, int NS>
__device__ __forceinline__ void d_sqrtL_full(const MixDev& m, const T (&ra)[NS], T rt, T (&L)[NS][NS]) {
    T Wf[NS], x[NS], mt;
    d_molconc_t<T, NS>(m, ra, rt, x, mt);
    T chi[NS][NS];
    d_chi_t<T, NS>(m, ra, rt, x, chi);
    if constexpr (sizeof(T) == 4) {
        const float ri = frcp(rt);
#pragma unroll
        for (int i = 0; i < NS; i++) Wf[i] = ra[i] * ri;
        const float fac = mt * rt * m.ikB_f;
#pragma unroll
        for (int c = 0; c < NS; c++)
#pragma unroll
            for (int r = 0; r < NS; r++) L[r][c] = fac * Wf[r] * chi[r][c] * Wf[c];
        d_choldc_f<NS>(L);
    } else {
#pragma unroll
        for (int i = 0; i < NS; i++) Wf[i] = ra[i] / rt;
        const T kB = (T)m.kB;
#pragma unroll
        for (int c = 0; c < NS; c++)
#pragma unroll
            for (int r = 0; r < NS; r++) L[r][c] = mt * rt * Wf[r] * chi[r][c] * Wf[c] / kB;
        d_choldc<T, NS>(L);
    }
}

// the subsystem's factor (compute_sqrtLonsager_sub).  Its Onsager matrix is
// singular (the rows sum to zero), so its last Cholesky pivot is a roundoff
// residue.  In the full system that pivot only reaches the last species,
// whose flux correction_flux replaces; in a subsystem it can belong to a
// kept species, and its square root would be sqrt(FP32 eps) ~ 2e-4 of the
// factor there.  So the subsystem factorises in FP64 in the
// mixed-precision mode too.
template <typename T, int NS>
__device__ __forceinline__ void d_sqrtL_trace(const MixDev& m, unsigned act, int na, const T (&ra)[NS],
                                              T (&L)[NS][NS]) {
    double rd[NS], Ld[NS][NS];
#pragma unroll
    for (int i = 0; i < NS; i++) rd[i] = (double)ra[i];
    d_sqrtL_sub<double, NS>(m, act, na, rd, Ld);
#pragma unroll
    for (int i = 0; i < NS; i++)
#pragma unroll
        for (int j = 0; j < NS; j++) L[i][j] = (T)Ld[i][j];
}

// every case of compute_sqrtLonsager_local on one face
template <typename T, int NS>
__device__ __forceinline__ void d_face_sqrtL(const MixDev& m, const double* const* __restrict__ rho, i64 f, i64 fm,
                                             T (&L)[NS][NS]) {
    T ra[NS], rt;
    d_face_rho_av<T, NS>(m, rho, f, fm, ra, rt);
    int na;
    const unsigned act = d_active<T, NS>(m, ra, rt, &na);
    if (na == 1) {
#pragma unroll
        for (int i = 0; i < NS; i++)
#pragma unroll
            for (int j = 0; j < NS; j++) L[i][j] = T(0);
    } else if (na != NS) {
        d_sqrtL_trace<T, NS>(m, act, na, ra, L);
    } else {
        d_sqrtL_full<T, NS>(m, ra, rt, L);
    }
}

// stochastic_mass_fluxdiv.f90:70-102 on one face: variance * sqrtL * sum_r
// w_r W_r, corrected (correction_flux.f90:17-226)
template <typename T, int NS, int DIM>
__device__ __forceinline__ void d_stoch_face(const MixDev& m, int d, i64 f, const T (&L)[NS][NS],
                                             const double* const* __restrict__ W, int n_rngs, const double* wts,
                                             T variance, T (&fs)[NS]) {
    T w[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) {
        T acc = T(0);
        for (int rr = 0; rr < n_rngs; rr++) acc = acc + (T)wts[rr] * (T)ld(W[(rr * DIM + d) * NS + s], f);
        w[s] = acc;
    }
#pragma unroll
    for (int r = 0; r < NS; r++) {
        T acc = T(0);
#pragma unroll
        for (int c = 0; c < NS; c++) {
            if constexpr (sizeof(T) == 4) acc = __fmaf_rn(L[r][c], w[c], acc);
            else acc = acc + L[r][c] * w[c];
        }
        fs[r] = acc * variance;
    }
    if (m.correct && NS > 1) {
        T sum = T(0);
#pragma unroll
        for (int s = 0; s < NS - 1; s++) sum = sum + fs[s];
        fs[NS - 1] = -sum;
    }
}

// ---------------------------------------------------------------------
// per face of direction D (the low face of each cell): diffusive +
// stochastic flux, corrected (correction_flux.f90:17-226)
// ---------------------------------------------------------------------
// (FP32 with up to 4 species: a 64-register cap for 8 CTAs = 32 warps per
// SM to hide the dependent chains)
template <typename T, int NS, int DIM>
__global__ void __launch_bounds__(128, (sizeof(T) == 4 && NS <= 4) ? 8 : 1)
    k_mass_flux(Grid g, MixDev m, int d, int wall, const double* const* __restrict__ rho,
                const T* const* __restrict__ rwc, const T* const* __restrict__ xc,
                const double* const* __restrict__ W, int n_rngs, const double* wts, T variance, T dxinv,
                T* const* flux, TraceList tl) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
    if (wall && (d == 0 ? P.i : (d == 1 ? P.j : P.k)) == 0) {
        // a wall face (wall: direction d has walls): the concentrations'
        // ghost cells are first-order extrapolated (scalar_bc,
        // inhomogeneous_bc_val.f90:21-54), so the diffusive flux vanishes,
        // and stoch_mass_bc zeroes the random field there
#pragma unroll
        for (int s = 0; s < NS; s++) flux[d * NS + s][f] = T(0);
        return;
    }
    const i64 fm = P.id(-(d == 0), -(d == 1), -(d == 2));
    T fd[NS];
    {
        T gx[NS];
#pragma unroll
        for (int s = 0; s < NS; s++) gx[s] = (ld(xc[s], f) - ld(xc[s], fm)) * dxinv;
#pragma unroll
        for (int r = 0; r < NS; r++) {
            T acc = T(0);
#pragma unroll
            for (int c = 0; c < NS; c++) {
                if constexpr (sizeof(T) == 4)
                    acc = __fmaf_rn(0.5f * (ld(rwc[r * NS + c], fm) + ld(rwc[r * NS + c], f)), gx[c], acc);
                else
                    acc = acc + T(0.5) * (ld(rwc[r * NS + c], fm) + ld(rwc[r * NS + c], f)) * gx[c];
            }
            fd[r] = acc;
        }
        if (m.correct && NS > 1) {
            T sum = T(0);
#pragma unroll
            for (int s = 0; s < NS - 1; s++) sum = sum + fd[s];
            fd[NS - 1] = -sum;
        }
    }
    T fs[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) fs[s] = T(0);
    if (m.var_mass != 0.0) {
        T ra[NS], rt;
        d_face_rho_av<T, NS>(m, rho, f, fm, ra, rt);
        int na;
        d_active<T, NS>(m, ra, rt, &na);
        if (na == NS) {
            T L[NS][NS];
            d_sqrtL_full<T, NS>(m, ra, rt, L);
            d_stoch_face<T, NS, DIM>(m, d, f, L, W, n_rngs, wts, variance, fs);
        } else if (na != 1) {
            // finished by k_mass_flux_trace, which adds the stochastic flux
            trace_push(tl, f);
        }
        // na == 1: zero factor, no stochastic flux
    }
#pragma unroll
    for (int s = 0; s < NS; s++) flux[d * NS + s][f] = fd[s] + fs[s];
}

// the listed faces of k_mass_flux: the stochastic flux through the
// subsystem of non-trace species, added to the stored diffusive flux
template <typename T, int NS, int DIM>
__global__ void __launch_bounds__(128) k_mass_flux_trace(Grid g, MixDev m, int d, const double* const* __restrict__ rho,
                                                         const double* const* __restrict__ W, int n_rngs,
                                                         const double* wts, T variance, T* const* flux,
                                                         TraceList tl) {
    const unsigned cnt = *tl.count;
    for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt; q += gridDim.x * blockDim.x) {
        const i64 f = tl.idx[q];
        const int i = (int)(f % g.n[0]), j = (int)((f / g.n[0]) % g.n[1]), k = (int)(f / ((i64)g.n[0] * g.n[1]));
        const int im = d == 0 ? (i == 0 ? g.n[0] - 1 : i - 1) : i;
        const int jm = d == 1 ? (j == 0 ? g.n[1] - 1 : j - 1) : j;
        const int km = d == 2 ? (k == 0 ? g.n[2] - 1 : k - 1) : k;
        const i64 fm = (i64)im + (i64)g.n[0] * ((i64)jm + (i64)g.n[1] * km);
        T ra[NS], rt;
        d_face_rho_av<T, NS>(m, rho, f, fm, ra, rt);
        int na;
        const unsigned act = d_active<T, NS>(m, ra, rt, &na);
        T L[NS][NS], fs[NS];
        d_sqrtL_trace<T, NS>(m, act, na, ra, L);
        d_stoch_face<T, NS, DIM>(m, d, f, L, W, n_rngs, wts, variance, fs);
#pragma unroll
        for (int s = 0; s < NS; s++) flux[d * NS + s][f] = flux[d * NS + s][f] + fs[s];
    }
}

// ---------------------------------------------------------------------
// the split form of the drop-in boundary: compute_sqrtLonsager_fc and
// stochastic_mass_fluxdiv with the face factors materialised (FP64; the
// pointer tables travel as kernel parameters)
// ---------------------------------------------------------------------
struct SqrtLArgs {
    const double* rho[FHD_MAX_SPECIES];
    double* out[FHD_MAX_SPECIES * FHD_MAX_SPECIES];  // this direction, entry (r, c) at r + ns*c
};

// compute_sqrtLonsager_fc (mass_flux_utilities.f90:1096-1229): every face
// of direction d
template <int NS>
// (wall: direction d has walls; on a wall face the ghost cell is the
// first-order extrapolation of the interior cell, scalar_bc,
// inhomogeneous_bc_val.f90:21-54)
__global__ void __launch_bounds__(128) k_sqrtL_fc(Grid g, MixDev m, int d, int wall, SqrtLArgs a) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
    const bool wf = wall && (d == 0 ? P.i : (d == 1 ? P.j : P.k)) == 0;
    const i64 fm = wf ? f : P.id(-(d == 0), -(d == 1), -(d == 2));
    double L[NS][NS];
    d_face_sqrtL<double, NS>(m, a.rho, f, fm, L);
#pragma unroll
    for (int r = 0; r < NS; r++)
#pragma unroll
        for (int c = 0; c < NS; c++) a.out[r + NS * c][f] = L[r][c];
}

struct StochMassArgs {
    const double* L[FHD_MAX_SPECIES * FHD_MAX_SPECIES];  // this direction's factors, (r, c) at r + ns*c
    const double* W[4 * FHD_MAX_SPECIES];                 // this direction's fields, [rr*ns + s]
    double wts[4];
    double* flux[FHD_MAX_SPECIES];                        // this direction's flux
};

// stochastic_mass_fluxdiv.f90:70-102: flux = variance * sqrtL (sum_r w_r W_r)
// (setval, saxpy per stage, matvec_mul, scaling), then correction_flux
template <int NS>
__global__ void __launch_bounds__(256) k_stoch_mass_flux(Grid g, MixDev m, int n_rngs, double variance,
                                                         StochMassArgs a) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
    double w[NS], fs[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) {
        double acc = 0.0;
        for (int rr = 0; rr < n_rngs; rr++) acc = acc + a.wts[rr] * ld(a.W[rr * NS + s], f);
        w[s] = acc;
    }
#pragma unroll
    for (int r = 0; r < NS; r++) {
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < NS; c++) acc = acc + ld(a.L[r + NS * c], f) * w[c];
        fs[r] = acc * variance;
    }
    if (m.correct && NS > 1) {
        double sum = 0.0;
#pragma unroll
        for (int s = 0; s < NS - 1; s++) sum = sum + fs[s];
        fs[NS - 1] = -sum;
    }
#pragma unroll
    for (int s = 0; s < NS; s++) a.flux[s][f] = fs[s];
}

struct DivArgs {
    const double* flux[3 * FHD_MAX_SPECIES];  // [d*ns + s]
    double* out[FHD_MAX_SPECIES];
};

// compute_div (div_and_grad.f90:884-1035) of every species' face flux,
// overwriting or (increment) adding to out in the reference's order
template <int NS, int DIM>
__global__ void __launch_bounds__(256) k_species_div(Grid g, double dxinv, int increment, DivArgs a) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const double x = (ld(a.flux[0 * NS + s], P.id(1, 0, 0)) - ld(a.flux[0 * NS + s], f)) * dxinv;
        const double y = (ld(a.flux[1 * NS + s], P.id(0, 1, 0)) - ld(a.flux[1 * NS + s], f)) * dxinv;
        double v = increment ? a.out[s][f] + x + y : x + y;
        if constexpr (DIM == 3) v = v + (ld(a.flux[2 * NS + s], P.id(0, 0, 1)) - ld(a.flux[2 * NS + s], f)) * dxinv;
        a.out[s][f] = v;
    }
}

// fluxdiv_s = div(flux_s)  (compute_div, div_and_grad.f90:884-1035)
template <typename T, int NS, int DIM>
__global__ void __launch_bounds__(256) k_mass_div(Grid g, const T* const* __restrict__ flux, double* const* out,
                                                  T dxinv) {
    Cell P;
    if (!cell_of_thread(g, P)) return;
    const i64 f = P.id(0, 0, 0);
#pragma unroll
    for (int s = 0; s < NS; s++) {
        T v = (ld(flux[0 * NS + s], P.id(1, 0, 0)) - ld(flux[0 * NS + s], f)) * dxinv +
              (ld(flux[1 * NS + s], P.id(0, 1, 0)) - ld(flux[1 * NS + s], f)) * dxinv;
        if constexpr (DIM == 3) v += (ld(flux[2 * NS + s], P.id(0, 0, 1)) - ld(flux[2 * NS + s], f)) * dxinv;
        out[s][f] = (double)v;
    }
}

// ---------------------------------------------------------------------
// host driver: device work arrays in the context, pointer tables in a
// small device block
// ---------------------------------------------------------------------
struct MassBufs {
    bool ready = false;
    int ns = 0;
    void* rwc = nullptr;   // ns*ns arrays of T
    void* xc = nullptr;    // ns arrays of T
    void* flux = nullptr;  // dim*ns arrays of T
    void** tab = nullptr;  // device pointer tables
    double* wts = nullptr;
    TraceList tl{nullptr, nullptr};  // deferred trace cells / faces
};

template <typename T>
static int mass_alloc(fhd_ctx* ctx, MassBufs& B, int ns) {
    if (B.ready && B.ns == ns) return 0;
    if (B.ready) {
        set_last_error("mass fluxes: the species count of a context cannot change");
        return FHD_ERR_BAD_ARG;
    }
    const i64 nc = ctx->g0.nc;
    const int dim = ctx->dim;
    T* rw = ctx->arena.alloc<T>((i64)ns * ns * nc);
    T* xc = ctx->arena.alloc<T>((i64)ns * nc);
    T* fl = ctx->arena.alloc<T>((i64)dim * ns * nc);
    void** tab = (void**)ctx->arena.alloc<double>(4 * 128);
    double* wts = ctx->arena.alloc<double>(8);
    int* tidx = (int*)ctx->arena.alloc<float>(nc);
    unsigned* tcnt = (unsigned*)ctx->arena.alloc<double>(1);
    if (!rw || !xc || !fl || !tab || !wts || !tidx || !tcnt) return FHD_ERR_OOM;
    B.tl = TraceList{tidx, tcnt};
    B.rwc = rw;
    B.xc = xc;
    B.flux = fl;
    B.tab = tab;
    B.wts = wts;
    B.ns = ns;
    B.ready = true;
    return 0;
}

template <typename T, int NS>
static int mass_fluxdiv_T(fhd_ctx* ctx, MassBufs& B, const MixDev& m, const double* const rho[], double dt,
                          const double* weights, int n_rngs, const double* const W[], double* const fluxdiv[]) {
    const int dim = ctx->dim;
    const i64 nc = ctx->g0.nc;
    const Grid g = ctx->g0;
    cudaStream_t st = ctx->stream;
    // pointer tables: [0,128) rho, [128,256) rwc, [256,384) xc/flux, [384,512) W/out
    void* h[512];
    memset(h, 0, sizeof(h));
    for (int s = 0; s < NS; s++) h[s] = (void*)rho[s];
    for (int q = 0; q < NS * NS; q++) h[128 + q] = (T*)B.rwc + (i64)q * nc;
    for (int s = 0; s < NS; s++) h[256 + s] = (T*)B.xc + (i64)s * nc;
    for (int q = 0; q < dim * NS; q++) h[256 + 16 + q] = (T*)B.flux + (i64)q * nc;
    for (int q = 0; q < n_rngs * dim * NS; q++) h[384 + q] = (void*)W[q];
    for (int s = 0; s < NS; s++) h[384 + 96 + s] = (void*)fluxdiv[s];
    FHD_CUDA_TRY(cudaMemcpyAsync(B.tab, h, sizeof(h), cudaMemcpyHostToDevice, st));
    double hw[8] = {0};
    for (int r = 0; r < n_rngs; r++) hw[r] = weights[r];
    FHD_CUDA_TRY(cudaMemcpyAsync(B.wts, hw, sizeof(hw), cudaMemcpyHostToDevice, st));
    const double* const* d_rho = (const double* const*)(B.tab);
    T* const* d_rwc = (T* const*)(B.tab + 128);
    T* const* d_xc = (T* const*)(B.tab + 256);
    T* const* d_flux = (T* const*)(B.tab + 256 + 16);
    const double* const* d_W = (const double* const*)(B.tab + 384);
    double* const* d_out = (double* const*)(B.tab + 384 + 96);
    const int nb = flat_blocks(nc);
    // the follow-up kernels of the deferred trace cells and faces: a few
    // blocks, which leave at once when the list is empty
    const int nbt = 2 * ctx->sms;
    FHD_CUDA_TRY(cudaMemsetAsync(B.tl.count, 0, sizeof(unsigned), st));
    k_rhowchi<T, NS><<<nb, 128, 0, st>>>(g, m, d_rho, d_rwc, d_xc, B.tl);
    ctx->launches++;
    FHD_CUDA_TRY(cudaPeekAtLastError());
    k_rhowchi_trace<T, NS><<<nbt, 128, 0, st>>>(m, d_rho, d_rwc, B.tl);
    ctx->launches++;
    FHD_CUDA_TRY(cudaPeekAtLastError());
    const T variance = (T)sqrt(2.0 * m.kB * m.var_mass / (m.dV * dt));
    const T dxinv = (T)(1.0 / ctx->dx);
    for (int d = 0; d < dim; d++) {
        FHD_CUDA_TRY(cudaMemsetAsync(B.tl.count, 0, sizeof(unsigned), st));
        with_dim(dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_mass_flux<T, NS, DIM><<<dim3((g.n[0] + 31) / 32, (g.n[1] + 3) / 4, g.n[2]), dim3(32, 4, 1), 0, st>>>(
                g, m, d, ctx->has_walls && ctx->walls.lo[d] != 0, d_rho, (const T* const*)d_rwc, (const T* const*)d_xc,
                d_W, n_rngs, B.wts, variance, dxinv, d_flux, B.tl);
            k_mass_flux_trace<T, NS, DIM><<<nbt, 128, 0, st>>>(g, m, d, d_rho, d_W, n_rngs, B.wts, variance, d_flux,
                                                               B.tl);
        });
        ctx->launches += 2;
        FHD_CUDA_TRY(cudaPeekAtLastError());
    }
    with_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        k_mass_div<T, NS, DIM><<<cell_grid(g), cell_block(), 0, st>>>(g, (const T* const*)d_flux, d_out, dxinv);
    });
    ctx->launches++;
    FHD_CUDA_TRY(cudaPeekAtLastError());
    return 0;
}

template <typename T>
static int mass_fluxdiv_dispatch(fhd_ctx* ctx, MassBufs& B, const MixDev& m, const double* const rho[], double dt,
                                 const double* weights, int n_rngs, const double* const W[],
                                 double* const fluxdiv[]) {
    switch (m.ns) {
        case 2: return mass_fluxdiv_T<T, 2>(ctx, B, m, rho, dt, weights, n_rngs, W, fluxdiv);
        case 3: return mass_fluxdiv_T<T, 3>(ctx, B, m, rho, dt, weights, n_rngs, W, fluxdiv);
        case 4: return mass_fluxdiv_T<T, 4>(ctx, B, m, rho, dt, weights, n_rngs, W, fluxdiv);
        case 5: return mass_fluxdiv_T<T, 5>(ctx, B, m, rho, dt, weights, n_rngs, W, fluxdiv);
        default:
            set_last_error("mass fluxes: nspecies must be 2..5");
            return FHD_ERR_UNSUPPORTED;
    }
}

// the FP32 instantiation lives in its own translation unit, compiled with
// FMA contraction (fhd_mass_f32.cu); FP64 stays uncontracted for parity
int mass_fluxdiv_f32(fhd_ctx* ctx, MassBufs& B, const MixDev& m, const double* const rho[], double dt,
                     const double* weights, int n_rngs, const double* const W[], double* const fluxdiv[]);

}  // namespace fhd

#ifdef FHD_MASS_F32_TU
namespace fhd {
int mass_fluxdiv_f32(fhd_ctx* ctx, MassBufs& B, const MixDev& m, const double* const rho[], double dt,
                     const double* weights, int n_rngs, const double* const W[], double* const fluxdiv[]) {
    if (int rc = mass_alloc<float>(ctx, B, m.ns)) return rc;
    return mass_fluxdiv_dispatch<float>(ctx, B, m, rho, dt, weights, n_rngs, W, fluxdiv);
}
}  // namespace fhd
#else

using namespace fhd;

#include <map>
#include <mutex>
static std::mutex g_mass_mu;
static std::map<fhd_ctx*, MassBufs*> g_mass;

extern "C" void fhd_mass_release(fhd_ctx* ctx) {
    std::lock_guard<std::mutex> lk(g_mass_mu);
    auto it = g_mass.find(ctx);
    if (it == g_mass.end()) return;
    delete it->second;
    g_mass.erase(it);
}

namespace fhd {
static MassBufs& mass_bufs(fhd_ctx* ctx) {
    std::lock_guard<std::mutex> lk(g_mass_mu);
    auto it = g_mass.find(ctx);
    if (it != g_mass.end()) return *it->second;
    MassBufs* b = new MassBufs();
    g_mass[ctx] = b;
    return *b;
}

// compute_mass_fluxdiv on the context's stream (trace species are handled
// per face and cell by the non-trace subsystem)
int mass_fluxdiv(fhd_ctx* ctx, const fhd_mixture_params* mp, const fhd_stoch_params* sp, const double* const rho[],
                 double dt, const double* weights, int n_rngs, const double* const W[], double* const fluxdiv[]) {
    if (!mp || mp->nspecies < 2 || mp->nspecies > 5 || n_rngs < 1 || n_rngs > 4) {
        set_last_error("mass fluxes: nspecies must be 2..5 and n_rngs 1..4");
        return FHD_ERR_UNSUPPORTED;
    }
    if (ctx->dim * mp->nspecies * n_rngs > 96) return FHD_ERR_UNSUPPORTED;
    MassBufs& B = mass_bufs(ctx);
    const MixDev m = make_mixdev(mp, sp);
    int rc;
    if (ctx->prec == FHD_PREC_MIXED) return mass_fluxdiv_f32(ctx, B, m, rho, dt, weights, n_rngs, W, fluxdiv);
    if ((rc = mass_alloc<double>(ctx, B, mp->nspecies))) return rc;
    return mass_fluxdiv_dispatch<double>(ctx, B, m, rho, dt, weights, n_rngs, W, fluxdiv);
}

}  // namespace fhd

namespace fhd {
template <int NS>
static int sqrtL_fc_T(fhd_ctx* ctx, const MixDev& m, const double* const rho[], double* const sqrtL[]) {
    const Grid g = ctx->g0;
    for (int d = 0; d < ctx->dim; d++) {
        SqrtLArgs a;
        memset(&a, 0, sizeof(a));
        for (int s = 0; s < NS; s++) a.rho[s] = rho[s];
        for (int q = 0; q < NS * NS; q++) a.out[q] = sqrtL[d * NS * NS + q];
        k_sqrtL_fc<NS><<<dim3((g.n[0] + 31) / 32, (g.n[1] + 3) / 4, g.n[2]), dim3(32, 4, 1), 0, ctx->stream>>>(
            g, m, d, ctx->has_walls && ctx->walls.lo[d] != 0, a);
        ctx->launches++;
        FHD_CUDA_TRY(cudaPeekAtLastError());
    }
    return 0;
}

// plane 0 of direction d of up to FHD_MAX_SPECIES face arrays set to zero
struct WallPlane {
    double* a[FHD_MAX_SPECIES];
};
__global__ void k_zero_plane(Grid g, int d, int n, WallPlane w) {
    const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const int u = d == 0 ? 1 : 0, v = d == 2 ? 1 : 2;  // the other two directions
    const i64 nu = g.n[u];
    if (t >= nu * g.n[v]) return;
    int q[3] = {0, 0, 0};
    q[u] = (int)(t % nu);
    q[v] = (int)(t / nu);
    const i64 f = (i64)q[0] + (i64)g.n[0] * ((i64)q[1] + (i64)g.n[1] * q[2]);
    for (int s = 0; s < n; s++) w.a[s][f] = 0.0;
}

template <int NS>
static int stoch_mass_T(fhd_ctx* ctx, const MixDev& m, const double* const sqrtL[], double dt, const double* weights,
                        int n_rngs, const double* const W[], int increment, double* const div[],
                        double* const flux[]) {
    const Grid g = ctx->g0;
    const int dim = ctx->dim;
    const double variance = sqrt(2.0 * m.kB * m.var_mass / (m.dV * dt));
    for (int d = 0; d < dim; d++) {
        StochMassArgs a;
        memset(&a, 0, sizeof(a));
        for (int q = 0; q < NS * NS; q++) a.L[q] = sqrtL[d * NS * NS + q];
        for (int rr = 0; rr < n_rngs; rr++)
            for (int sp = 0; sp < NS; sp++) a.W[rr * NS + sp] = W[(rr * dim + d) * NS + sp];
        for (int rr = 0; rr < n_rngs; rr++) a.wts[rr] = weights[rr];
        for (int sp = 0; sp < NS; sp++) a.flux[sp] = flux[d * NS + sp];
        k_stoch_mass_flux<NS><<<cell_grid(g), cell_block(), 0, ctx->stream>>>(g, m, n_rngs, variance, a);
        ctx->launches++;
        FHD_CUDA_TRY(cudaPeekAtLastError());
        if (ctx->has_walls && ctx->walls.lo[d] != 0) {
            // stoch_mass_bc (stochastic_mass_fluxdiv.f90:216-368): no flux
            // through a wall face (the high wall face, not stored, reads as
            // face 0 in the divergence's periodic wrap)
            WallPlane wp;
            for (int sp = 0; sp < NS; sp++) wp.a[sp] = flux[d * NS + sp];
            k_zero_plane<<<dim3((ctx->g0.nc / g.n[d] + 255) / 256), 256, 0, ctx->stream>>>(g, d, NS, wp);
            ctx->launches++;
            FHD_CUDA_TRY(cudaPeekAtLastError());
        }
    }
    DivArgs a;
    memset(&a, 0, sizeof(a));
    for (int q = 0; q < dim * NS; q++) a.flux[q] = flux[q];
    for (int sp = 0; sp < NS; sp++) a.out[sp] = div[sp];
    const double dxinv = 1.0 / ctx->dx;
    with_dim(dim, [&](auto D) {
        constexpr int DIM = decltype(D)::value;
        k_species_div<NS, DIM><<<cell_grid(g), cell_block(), 0, ctx->stream>>>(g, dxinv, increment, a);
    });
    ctx->launches++;
    FHD_CUDA_TRY(cudaPeekAtLastError());
    return 0;
}

static int check_mix(const fhd_mixture_params* mp) {
    if (!mp || mp->nspecies < 2 || mp->nspecies > 5) {
        set_last_error("mass fluxes: nspecies must be 2..5");
        return FHD_ERR_UNSUPPORTED;
    }
    return 0;
}
}  // namespace fhd

namespace fhd {
// the factors on the high wall face of direction d (not stored in the
// periodic layout): the last cell layer i_d = n_d - 1 with its extrapolated
// ghost (scalar_bc, inhomogeneous_bc_val.f90:21-54), one value per cell of
// the layer, in-plane index u + n_u v over the two other directions u < v
template <int NS>
__global__ void __launch_bounds__(128) k_sqrtL_hi_plane(Grid g, MixDev m, int d, SqrtLArgs a) {
    const int u = d == 0 ? 1 : 0, v = d == 2 ? 1 : 2;
    const i64 nu = g.n[u], np = nu * g.n[v];
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < np; t += (i64)gridDim.x * blockDim.x) {
        int q[3] = {0, 0, 0};
        q[d] = g.n[d] - 1;
        q[u] = (int)(t % nu);
        q[v] = (int)(t / nu);
        const i64 f = (i64)q[0] + (i64)g.n[0] * ((i64)q[1] + (i64)g.n[1] * q[2]);
        double L[NS][NS];
        d_face_sqrtL<double, NS>(m, a.rho, f, f, L);
#pragma unroll
        for (int r = 0; r < NS; r++)
#pragma unroll
            for (int c = 0; c < NS; c++) a.out[r + NS * c][t] = L[r][c];
    }
}

int sqrtL_high_wall_plane(fhd_ctx* ctx, const fhd_mixture_params* mp, const fhd_stoch_params* sp,
                          const double* const rho[], int d, double* const plane[]) {
    if (int rc = check_mix(mp)) return rc;
    const MixDev m = make_mixdev(mp, sp);
    SqrtLArgs a;
    memset(&a, 0, sizeof(a));
    for (int s = 0; s < m.ns; s++) a.rho[s] = rho[s];
    for (int q = 0; q < m.ns * m.ns; q++) a.out[q] = plane[q];
    const Grid g = ctx->g0;
    const i64 np = g.nc / g.n[d];
    const int nb = (int)((np + 127) / 128);
    switch (m.ns) {
        case 2: k_sqrtL_hi_plane<2><<<nb, 128, 0, ctx->stream>>>(g, m, d, a); break;
        case 3: k_sqrtL_hi_plane<3><<<nb, 128, 0, ctx->stream>>>(g, m, d, a); break;
        case 4: k_sqrtL_hi_plane<4><<<nb, 128, 0, ctx->stream>>>(g, m, d, a); break;
        default: k_sqrtL_hi_plane<5><<<nb, 128, 0, ctx->stream>>>(g, m, d, a); break;
    }
    ctx->launches++;
    FHD_CUDA_TRY(cudaPeekAtLastError());
    FHD_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return 0;
}
}  // namespace fhd

extern "C" int fhd_dev_compute_sqrtLonsager_fc(fhd_ctx* ctx, const fhd_mixture_params* mp,
                                               const fhd_stoch_params* sp, const double* const rho[],
                                               double* const sqrtLonsager_fc[]) {
    if (!ctx || !mp || !sp || !rho || !sqrtLonsager_fc) return FHD_ERR_BAD_ARG;
    if (int rc = fhd::refuse_reservoirs(ctx, "compute_sqrtLonsager_fc")) return rc;
    if (int rc = check_mix(mp)) return rc;
    const MixDev m = make_mixdev(mp, sp);
    int rc;
    switch (m.ns) {
        case 2: rc = sqrtL_fc_T<2>(ctx, m, rho, sqrtLonsager_fc); break;
        case 3: rc = sqrtL_fc_T<3>(ctx, m, rho, sqrtLonsager_fc); break;
        case 4: rc = sqrtL_fc_T<4>(ctx, m, rho, sqrtLonsager_fc); break;
        default: rc = sqrtL_fc_T<5>(ctx, m, rho, sqrtLonsager_fc); break;
    }
    if (rc < 0) return rc;
    FHD_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return 0;
}

extern "C" int fhd_dev_stochastic_mass_fluxdiv(fhd_ctx* ctx, const fhd_mixture_params* mp,
                                               const fhd_stoch_params* sp, const double* const sqrtLonsager_fc[],
                                               double dt, const double* weights, int n_rngs,
                                               const double* const W_fc[], int increment,
                                               double* const stoch_mass_fluxdiv[],
                                               double* const stoch_mass_flux[]) {
    if (!ctx || !mp || !sp || !sqrtLonsager_fc || !weights || !W_fc || !stoch_mass_fluxdiv || !(dt > 0.0))
        return FHD_ERR_BAD_ARG;
    if (int rc = fhd::refuse_reservoirs(ctx, "stochastic_mass_fluxdiv")) return rc;
    if (n_rngs < 1 || n_rngs > 4) {
        set_last_error("stochastic_mass_fluxdiv: n_rngs must be 1..4");
        return FHD_ERR_UNSUPPORTED;
    }
    if (int rc = check_mix(mp)) return rc;
    const MixDev m = make_mixdev(mp, sp);
    const int ns = m.ns, dim = ctx->dim;
    // the face flux: the caller's arrays, or stream-ordered scratch
    double* own = nullptr;
    double* fl[3 * FHD_MAX_SPECIES];
    if (stoch_mass_flux) {
        for (int q = 0; q < dim * ns; q++) fl[q] = stoch_mass_flux[q];
    } else {
        FHD_CUDA_TRY(cudaMallocAsync((void**)&own, sizeof(double) * (size_t)ctx->g0.nc * dim * ns, ctx->stream));
        for (int q = 0; q < dim * ns; q++) fl[q] = own + (i64)q * ctx->g0.nc;
    }
    int rc;
    switch (ns) {
        case 2: rc = stoch_mass_T<2>(ctx, m, sqrtLonsager_fc, dt, weights, n_rngs, W_fc, increment, stoch_mass_fluxdiv, fl); break;
        case 3: rc = stoch_mass_T<3>(ctx, m, sqrtLonsager_fc, dt, weights, n_rngs, W_fc, increment, stoch_mass_fluxdiv, fl); break;
        case 4: rc = stoch_mass_T<4>(ctx, m, sqrtLonsager_fc, dt, weights, n_rngs, W_fc, increment, stoch_mass_fluxdiv, fl); break;
        default: rc = stoch_mass_T<5>(ctx, m, sqrtLonsager_fc, dt, weights, n_rngs, W_fc, increment, stoch_mass_fluxdiv, fl); break;
    }
    if (own) cudaFreeAsync(own, ctx->stream);
    if (rc < 0) return rc;
    FHD_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return 0;
}

extern "C" int fhd_dev_compute_mass_fluxdiv(fhd_ctx* ctx, const fhd_mixture_params* mp, const fhd_stoch_params* sp,
                                            const double* const rho[], double dt, const double* weights, int n_rngs,
                                            const double* const W_fc[], double* const out[]) {
    if (!ctx || !mp || !sp || !rho || !weights || !W_fc || !out) return FHD_ERR_BAD_ARG;
    if (int r0 = fhd::refuse_reservoirs(ctx, "compute_mass_fluxdiv")) return r0;
    const int rc = fhd::mass_fluxdiv(ctx, mp, sp, rho, dt, weights, n_rngs, W_fc, out);
    if (rc < 0) return rc;
    // like every device entry point, the call returns with its work done
    FHD_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return rc;
}
#endif  // FHD_MASS_F32_TU
