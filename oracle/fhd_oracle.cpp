/*
 * fhd_oracle.cpp -- TEST INFRASTRUCTURE ONLY (parity checker and CPU
 * baseline).  A plain C++ FP64 restatement of the LowMachFHD hot path for
 * one periodic box, following the reference Fortran routine by routine.
 * Citations are to files under staggered_grid/ of the reference.
 *
 * Layout: unique periodic degrees of freedom (see include/fhd_b200.h); the
 * reference stores the periodic face twice and keeps both copies equal
 * (multifab_internal_sync), which is the same discrete problem.
 *
 * Reductions are deterministic: per-row partial sums added in row order.
 */
#include "fhd_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef std::vector<double> Vec;

// Domain walls of the grids built from here on (or_set_walls): per direction
// and side 0 = periodic, -1 = no-slip wall, +1 = slip wall (the sign the
// transverse velocity takes in the ghost cell behind the wall).
static int g_wl[3] = {0, 0, 0}, g_wh[3] = {0, 0, 0};
// Tangential speeds of moving no-slip walls (or_set_wall_speed), the
// namelist arrays wallspeed_lo / wallspeed_hi of probin_common in their
// Fortran layout: speed (t, d) of the t-th tangential component (the
// components other than d, ascending) on the wall normal to d at [t + 2 d];
// the constant values of inhomogeneous_bc_val_2d / _3d
// (src_lowMach/inhomogeneous_bc_val.f90:84-145, 274-372).
static double g_ws[2][6] = {{0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0}};

struct Geo {
    int dim = 2;
    int n[3] = {1, 1, 1};
    long nc = 1;
    double dx = 1.0;
    int wl[3] = {0, 0, 0}, wh[3] = {0, 0, 0};
    Geo() {}
    Geo(int d, const int nn[3], double h) : dim(d), dx(h) {
        n[0] = nn[0];
        n[1] = nn[1];
        n[2] = (d == 3) ? nn[2] : 1;
        nc = (long)n[0] * n[1] * n[2];
        for (int q = 0; q < 3; q++) {
            wl[q] = q < d ? g_wl[q] : 0;
            wh[q] = q < d ? g_wh[q] : 0;
        }
    }
    bool wall(int d) const { return wl[d] != 0; }
    bool any_wall() const { return wall(0) || wall(1) || wall(2); }
    inline long id(int i, int j, int k) const {
        if (i < 0) i += n[0]; else if (i >= n[0]) i -= n[0];
        if (j < 0) j += n[1]; else if (j >= n[1]) j -= n[1];
        if (k < 0) k += n[2]; else if (k >= n[2]) k -= n[2];
        return i + (long)n[0] * (j + (long)n[1] * k);
    }
    Geo coarsen() const {
        int nn[3] = {n[0] / 2, n[1] / 2, dim == 3 ? n[2] / 2 : 1};
        return Geo(dim, nn, dx * 2.0);
    }
};

// Extents of edge set e (edge_dirs): n[d], plus one in a wall direction d
// of the set, whose last plane holds the edges on the high wall (the
// reference's nodal multifab has hi+1 there and draws independent values
// for it).
inline void edge_ext(const Geo& g, int e, long m[3]) {
    int a = 0, b = 1;
    if (g.dim == 3) { a = e == 2 ? 1 : 0; b = e == 0 ? 1 : 2; }
    for (int d = 0; d < 3; d++) m[d] = g.n[d] + ((d == a || d == b) && g.wall(d) ? 1 : 0);
}
inline long edge_count(const Geo& g, int e) {
    long m[3];
    edge_ext(g, e, m);
    return m[0] * m[1] * m[2];
}
// index of edge (i, j, k) of set e: periodic directions wrap, wall
// directions of the set take 0 .. n[d]
inline long edge_id(const Geo& g, int e, int i, int j, int k) {
    long m[3];
    edge_ext(g, e, m);
    int q[3] = {i, j, k};
    for (int d = 0; d < 3; d++) {
        if (m[d] != g.n[d]) continue;
        if (q[d] < 0) q[d] += g.n[d]; else if (q[d] >= g.n[d]) q[d] -= g.n[d];
    }
    return q[0] + m[0] * (q[1] + m[1] * (long)q[2]);
}

// Velocity component c at face (i, j, k), which may lie one face beyond the
// domain: the ghost-cell rules of multifab_physbc_domainvel and
// multifab_physbc_macvel (multifab_physbc_stag.f90:91-173, 957-1116), homogeneous.
// Across a wall the normal component is zero (the high wall face, index n,
// included: it is not stored), the transverse one is the first interior
// value times the wall's sign (-1 no-slip, +1 slip); periodic directions wrap.
inline double vel(const Geo& g, const double* u, int c, int i, int j, int k) {
    int q[3] = {i, j, k};
    double sg = 1.0;
    for (int d = 0; d < g.dim; d++) {
        if (!g.wall(d)) continue;
        if (q[d] < 0) {
            if (d == c) return 0.0;
            sg *= g.wl[d];
            q[d] = 0;
        } else if (q[d] >= g.n[d]) {
            if (d == c) return 0.0;
            sg *= g.wh[d];
            q[d] = g.n[d] - 1;
        }
    }
    return sg * u[g.id(q[0], q[1], q[2])];
}

// the face of component c at cell (i, j, k) lies on a wall (index 0 in a
// wall direction c; the high wall face is not stored)
inline bool wall_face(const Geo& g, int c, int i, int j, int k) {
    const int q[3] = {i, j, k};
    return g.wall(c) && q[c] == 0;
}

// zero the wall faces of a face vector (multifab_physbc_domainvel)
inline void zero_wall_faces(const Geo& g, double* const u[]) {
    for (int c = 0; c < g.dim; c++) {
        if (!g.wall(c)) continue;
        for (int k = 0; k < g.n[2]; k++)
            for (int j = 0; j < g.n[1]; j++)
                for (int i = 0; i < g.n[0]; i++)
                    if (wall_face(g, c, i, j, k)) u[c][g.id(i, j, k)] = 0.0;
    }
}

inline int edge_of(int dim, int c, int d) {
    if (dim == 2) return 0;
    int a = std::min(c, d), b = std::max(c, d);
    if (a == 0 && b == 1) return 0;  // xy
    if (a == 0 && b == 2) return 1;  // xz
    return 2;                        // yz
}

inline int n_edge(int dim) { return dim == 2 ? 1 : 3; }

// Edge set e of a dim-D grid: its two nodal directions a < b (2D: the
// nodes, x and y; 3D: xy, xz, yz).
inline void edge_dirs(int dim, int e, int& a, int& b) {
    if (dim == 2) { a = 0; b = 1; }
    else { a = e == 2 ? 1 : 0; b = e == 0 ? 1 : 2; }
}

template <class F>
inline void forall(const Geo& g, F f) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < g.n[2]; k++)
        for (int j = 0; j < g.n[1]; j++)
            for (int i = 0; i < g.n[0]; i++) f(i, j, k);
}

// deterministic sum of f(i,j,k) over all cells
template <class F>
inline double reduce_sum(const Geo& g, F f) {
    long rows = (long)g.n[1] * g.n[2];
    std::vector<double> part(rows, 0.0);
#pragma omp parallel for schedule(static)
    for (long r = 0; r < rows; r++) {
        int j = (int)(r % g.n[1]), k = (int)(r / g.n[1]);
        double s = 0.0;
        for (int i = 0; i < g.n[0]; i++) s += f(i, j, k);
        part[r] = s;
    }
    double s = 0.0;
    for (long r = 0; r < rows; r++) s += part[r];
    return s;
}

template <class F>
inline double reduce_max(const Geo& g, F f) {
    long rows = (long)g.n[1] * g.n[2];
    std::vector<double> part(rows, 0.0);
#pragma omp parallel for schedule(static)
    for (long r = 0; r < rows; r++) {
        int j = (int)(r % g.n[1]), k = (int)(r / g.n[1]);
        double s = 0.0;
        for (int i = 0; i < g.n[0]; i++) s = std::max(s, f(i, j, k));
        part[r] = s;
    }
    double s = 0.0;
    for (long r = 0; r < rows; r++) s = std::max(s, part[r]);
    return s;
}

// ---------------------------------------------------------------------
// staggered multigrid level: coefficients and work arrays
// ---------------------------------------------------------------------
struct SLevel {
    Geo g;
    Vec alpha[3];  // theta_alpha * alpha on faces
    Vec beta, gamma;
    Vec bed[3];    // 2D: node; 3D: xy, xz, yz edges
    Vec phi[3], rhs[3], Lphi[3];
};

// (theta*alpha - L) phi on one face of component c; returns the value and
// the diagonal coefficient.  Restates stag_applyop_2d/_3d
// (stag_applyop.f90:212-1075) for all visc_type, with the periodic wrap
// standing in for the ghost-cell fill; the diagonal is the 'fac' of
// stag_mg_update (stag_mg_solver.f90:1764-2458).
inline double lface(const Geo& g, int visc, const Vec* alpha, const Vec& beta,
                    const Vec& gamma, const Vec* bed, const double* const* phi,
                    int c, int i, int j, int k, double* diag_out) {
    const int dim = g.dim;
    const double q = 1.0 / (g.dx * g.dx);
    int ec[3] = {0, 0, 0};
    ec[c] = 1;
    const long f = g.id(i, j, k);
    const long fpc = g.id(i + ec[0], j + ec[1], k + ec[2]);
    const long fmc = g.id(i - ec[0], j - ec[1], k - ec[2]);
    const double ph = phi[c][f];
    const double a = alpha[c][f];
    if (visc < 0) {
        const double bp = beta[f], bm = beta[fmc];
        double kp, km;
        if (visc == -1) {
            kp = bp; km = bm;
        } else if (visc == -2) {
            kp = 2.0 * bp; km = 2.0 * bm;
        } else {
            kp = (4.0 / 3.0) * bp + gamma[f];
            km = (4.0 / 3.0) * bm + gamma[fmc];
        }
        double s = kp + km;
        double nb = phi[c][fpc] * kp + phi[c][fmc] * km;
        double cross = 0.0;
        for (int d = 0; d < dim; d++) {
            if (d == c) continue;
            int ed[3] = {0, 0, 0};
            ed[d] = 1;
            const long fpd = g.id(i + ed[0], j + ed[1], k + ed[2]);
            const long fmd = g.id(i - ed[0], j - ed[1], k - ed[2]);
            const Vec& E = bed[edge_of(dim, c, d)];
            const double elo = E[f], ehi = E[fpd];
            s += elo + ehi;
            nb += phi[c][fpd] * ehi + phi[c][fmd] * elo;
            if (visc != -1) {
                const long fmcpd = g.id(i - ec[0] + ed[0], j - ec[1] + ed[1], k - ec[2] + ed[2]);
                double tp = 0.0, tm = 0.0;
                if (visc == -3) {
                    tp = -(2.0 / 3.0) * bp + gamma[f];
                    tm = -(2.0 / 3.0) * bm + gamma[fmc];
                }
                cross += phi[d][fpd] * (ehi + tp) - phi[d][f] * (elo + tp)
                       - phi[d][fmcpd] * (ehi + tm) + phi[d][fmc] * (elo + tm);
            }
        }
        const double diag = a + s * q;
        if (diag_out) *diag_out = diag;
        return ph * diag - (nb + cross) * q;
    }
    // constant coefficients: beta, gamma taken from the first cell
    // (stag_applyop.f90:654-656 'b = beta(xlo(1),xlo(2),xlo(3))')
    const double b = beta[0], cg = gamma[0];
    if (g.any_wall()) {
        // walls (visc_type 1, 2, 3): every neighbour through the ghost rules,
        // the uniform stencil of stag_applyop_level on ghost cells filled by
        // multifab_physbc_macvel / _domainvel
        const double own = vel(g, phi[c], c, i + ec[0], j + ec[1], k + ec[2]) +
                           vel(g, phi[c], c, i - ec[0], j - ec[1], k - ec[2]);
        double oth = 0.0, cross = 0.0;
        for (int d = 0; d < dim; d++) {
            if (d == c) continue;
            int ed[3] = {0, 0, 0};
            ed[d] = 1;
            oth += vel(g, phi[c], c, i + ed[0], j + ed[1], k + ed[2]) +
                   vel(g, phi[c], c, i - ed[0], j - ed[1], k - ed[2]);
            if (visc != 1)
                cross += vel(g, phi[d], d, i + ed[0], j + ed[1], k + ed[2]) - vel(g, phi[d], d, i, j, k) -
                         vel(g, phi[d], d, i - ec[0] + ed[0], j - ec[1] + ed[1], k - ec[2] + ed[2]) +
                         vel(g, phi[d], d, i - ec[0], j - ec[1], k - ec[2]);
        }
        if (visc == 2) {
            const double diag = a + (2.0 * dim + 2.0) * b * q;
            if (diag_out) *diag_out = diag;
            return ph * diag - (2.0 * own + oth + cross) * b * q;
        }
        if (visc == 3) {
            const double diag = a + ((8.0 / 3.0 + 2.0 * (dim - 1)) * b + 2.0 * cg) * q;
            if (diag_out) *diag_out = diag;
            return ph * diag - (own * ((4.0 / 3.0) * b + cg) + oth * b + cross * ((1.0 / 3.0) * b + cg)) * q;
        }
        const double diag = a + (2.0 * dim) * b * q;
        if (diag_out) *diag_out = diag;
        return ph * diag - (own + oth) * b * q;
    }
    const double own = phi[c][fpc] + phi[c][fmc];
    double oth = 0.0, cross = 0.0;
    for (int d = 0; d < dim; d++) {
        if (d == c) continue;
        int ed[3] = {0, 0, 0};
        ed[d] = 1;
        const long fpd = g.id(i + ed[0], j + ed[1], k + ed[2]);
        const long fmd = g.id(i - ed[0], j - ed[1], k - ed[2]);
        oth += phi[c][fpd] + phi[c][fmd];
        if (visc != 1) {
            const long fmcpd = g.id(i - ec[0] + ed[0], j - ec[1] + ed[1], k - ec[2] + ed[2]);
            cross += phi[d][fpd] - phi[d][f] - phi[d][fmcpd] + phi[d][fmc];
        }
    }
    double diag, L;
    if (visc == 1) {
        diag = a + (2.0 * dim) * b * q;
        L = ph * diag - (own + oth) * b * q;
    } else if (visc == 2) {
        diag = a + (2.0 * dim + 2.0) * b * q;
        L = ph * diag - (2.0 * own + oth + cross) * b * q;
    } else {
        diag = a + ((8.0 / 3.0 + 2.0 * (dim - 1)) * b + 2.0 * cg) * q;
        L = ph * diag - (own * ((4.0 / 3.0) * b + cg) + oth * b + cross * ((1.0 / 3.0) * b + cg)) * q;
    }
    if (diag_out) *diag_out = diag;
    return L;
}

inline bool in_color(int color, int c, int i, int j, int k) {
    if (color == 0) return true;
    if ((color - 1) / 2 != c) return false;
    return ((i + j + k) & 1) == ((color + 1) & 1);
}

// stag_applyop_level (stag_applyop.f90:70-210)
void s_applyop(SLevel& L, int visc, int color) {
    const Geo& g = L.g;
    const double* ph[3] = {L.phi[0].data(), L.phi[1].data(), g.dim == 3 ? L.phi[2].data() : nullptr};
    for (int c = 0; c < g.dim; c++) {
        if (color != 0 && (color - 1) / 2 != c) continue;
        double* out = L.Lphi[c].data();
        forall(g, [&](int i, int j, int k) {
            if (!in_color(color, c, i, j, k)) return;
            // Lphi on physical domain boundaries is zero (stag_applyop.f90:201-205)
            out[g.id(i, j, k)] = wall_face(g, c, i, j, k)
                                     ? 0.0
                                     : lface(g, visc, L.alpha, L.beta, L.gamma, L.bed, ph, c, i, j, k, nullptr);
        });
    }
}

// A wall speed is taken on no-slip walls only: on a slip wall the reference
// reads the value as a traction (DIR_TRACT, multifab_physbc_stag.f90:
// 1151-1160), which is not built.  A speed on a periodic side is ignored, as
// there.
int wall_speed_check(const Geo& g) {
    for (int d = 0; d < g.dim; d++)
        for (int side = 0; side < 2; side++)
            for (int t = 0; t < g.dim - 1; t++)
                if (g_ws[side][t + 2 * d] != 0.0 && (side ? g.wh[d] : g.wl[d]) > 0) return FHD_ERR_UNSUPPORTED;
    return 0;
}

// The part of diffusive_m_fluxdiv that moving no-slip walls add.  Behind
// such a wall the tangential ghost is 2 v_bc - u
// (physbc_macvel_2d_inhomogeneous / _3d_inhomogeneous,
// multifab_physbc_stag.f90:1118-1160) where the homogeneous rule has -u, so
// +L u (visc_type 1, beta of the first cell) gains 2 v_bc beta / dx^2 on the
// faces of the first row beside the wall.  The steps take every
// diffusive_m_fluxdiv of the velocity with those ghosts: that is how they put
// the solve in delta form with homogeneous walls
// (advance_timestep_overdamped.f90:310-333, advance_timestep_inertial.f90:
// 408-440).  Walls in direction order, the low side first, one addition each.
void wall_speed_term(const Geo& g, double beta0, double* const out[]) {
    const int dim = g.dim;
    const double q = 1.0 / (g.dx * g.dx);
    for (int d = 0; d < dim; d++)
        for (int side = 0; side < 2; side++) {
            if ((side ? g.wh[d] : g.wl[d]) >= 0) continue;
            const int row = side ? g.n[d] - 1 : 0;
            int t = 0;
            for (int c = 0; c < dim; c++) {
                if (c == d) continue;
                const double v = g_ws[side][t + 2 * d];
                t++;
                if (v == 0.0) continue;
                forall(g, [&](int i, int j, int k) {
                    const int at[3] = {i, j, k};
                    if (at[d] != row || wall_face(g, c, i, j, k)) return;
                    const long f = g.id(i, j, k);
                    out[c][f] = out[c][f] + ((2.0 * v) * beta0) * q;
                });
            }
        }
}

// one colour of the smoother: applyop(colour) then stag_mg_update(colour)
// (stag_mg_solver.f90:360-396, 1632-2458).  Two passes, so the update of a
// colour never sees another update of the same colour.
void s_smooth(SLevel& L, int visc, double omega, int color) {
    const Geo& g = L.g;
    const double* ph[3] = {L.phi[0].data(), L.phi[1].data(), g.dim == 3 ? L.phi[2].data() : nullptr};
    std::vector<Vec> diag(g.dim);
    for (int c = 0; c < g.dim; c++) {
        if (color != 0 && (color - 1) / 2 != c) continue;
        diag[c].assign(g.nc, 0.0);
        double* out = L.Lphi[c].data();
        double* dg = diag[c].data();
        forall(g, [&](int i, int j, int k) {
            if (!in_color(color, c, i, j, k)) return;
            long f = g.id(i, j, k);
            out[f] = lface(g, visc, L.alpha, L.beta, L.gamma, L.bed, ph, c, i, j, k, &dg[f]);
        });
    }
    for (int c = 0; c < g.dim; c++) {
        if (color != 0 && (color - 1) / 2 != c) continue;
        double* p = L.phi[c].data();
        const double* r = L.rhs[c].data();
        const double* lp = L.Lphi[c].data();
        const double* dg = diag[c].data();
        forall(g, [&](int i, int j, int k) {
            if (!in_color(color, c, i, j, k)) return;
            long f = g.id(i, j, k);
            // wall faces stay zero (multifab_physbc_domainvel after each colour)
            p[f] = wall_face(g, c, i, j, k) ? 0.0 : p[f] + omega * (r[f] - lp[f]) / dg[f];
        });
    }
}

// stag_restriction (stag_mg_solver.f90:966-1170): full 6/12-point stencil,
// or the 2/4-point 'simple' stencil used to coarsen alpha.
void s_restrict(const Geo& gf, const Geo& gc, const Vec* fine, Vec* coarse, bool simple) {
    const int dim = gf.dim;
    for (int c = 0; c < dim; c++) {
        const double* F = fine[c].data();
        double* C = coarse[c].data();
        int a = (c == 0) ? 1 : 0;
        int b = (dim == 3) ? ((c == 2) ? 1 : 2) : -1;
        forall(gc, [&](int i, int j, int k) {
            int I[3] = {2 * i, 2 * j, 2 * k};
            auto at = [&](int o, int pa, int pb) {
                int q[3] = {I[0], I[1], I[2]};
                q[c] += o;
                q[a] += pa;
                if (b >= 0) q[b] += pb;
                return F[gf.id(q[0], q[1], q[2])];
            };
            double v;
            if (dim == 2) {
                if (simple) v = 0.5 * (at(0, 0, 0) + at(0, 1, 0));
                else v = 0.25 * (at(0, 0, 0) + at(0, 1, 0))
                       + 0.125 * (at(1, 0, 0) + at(1, 1, 0) + at(-1, 0, 0) + at(-1, 1, 0));
            } else {
                if (simple) v = 0.25 * (at(0, 0, 0) + at(0, 1, 0) + at(0, 0, 1) + at(0, 1, 1));
                else v = 0.125 * (at(0, 0, 0) + at(0, 1, 0) + at(0, 0, 1) + at(0, 1, 1))
                       + 0.0625 * (at(1, 0, 0) + at(1, 1, 0) + at(1, 0, 1) + at(1, 1, 1))
                       + 0.0625 * (at(-1, 0, 0) + at(-1, 1, 0) + at(-1, 0, 1) + at(-1, 1, 1));
            }
            C[gc.id(i, j, k)] = v;
        });
    }
}

// cc_restriction (stag_mg_solver.f90:868-963): average of the 2^dim children
void cc_average(const Geo& gf, const Geo& gc, const Vec& F, Vec& C) {
    forall(gc, [&](int i, int j, int k) {
        double v;
        if (gf.dim == 2) {
            v = 0.25 * (F[gf.id(2 * i, 2 * j, 0)] + F[gf.id(2 * i + 1, 2 * j, 0)]
                      + F[gf.id(2 * i, 2 * j + 1, 0)] + F[gf.id(2 * i + 1, 2 * j + 1, 0)]);
        } else {
            v = 0.125 * (F[gf.id(2 * i, 2 * j, 2 * k)] + F[gf.id(2 * i + 1, 2 * j, 2 * k)]
                       + F[gf.id(2 * i, 2 * j + 1, 2 * k)] + F[gf.id(2 * i + 1, 2 * j + 1, 2 * k)]
                       + F[gf.id(2 * i, 2 * j, 2 * k + 1)] + F[gf.id(2 * i + 1, 2 * j, 2 * k + 1)]
                       + F[gf.id(2 * i, 2 * j + 1, 2 * k + 1)] + F[gf.id(2 * i + 1, 2 * j + 1, 2 * k + 1)]);
        }
        C[gc.id(i, j, k)] = v;
    });
}

// nodal_restriction (2D injection, stag_mg_solver.f90:1224-1239) and
// edge_restriction (3D 2-point, stag_mg_solver.f90:1321-1362)
void edge_coarsen(const Geo& gf, const Geo& gc, const Vec* F, Vec* C) {
    if (gf.dim == 2) {
        forall(gc, [&](int i, int j, int k) { C[0][gc.id(i, j, k)] = F[0][gf.id(2 * i, 2 * j, 0)]; });
        return;
    }
    forall(gc, [&](int i, int j, int k) {
        long c = gc.id(i, j, k);
        C[0][c] = 0.5 * (F[0][gf.id(2 * i, 2 * j, 2 * k)] + F[0][gf.id(2 * i, 2 * j, 2 * k + 1)]);
        C[1][c] = 0.5 * (F[1][gf.id(2 * i, 2 * j, 2 * k)] + F[1][gf.id(2 * i, 2 * j + 1, 2 * k)]);
        C[2][c] = 0.5 * (F[2][gf.id(2 * i, 2 * j, 2 * k)] + F[2][gf.id(2 * i + 1, 2 * j, 2 * k)]);
    });
}

// stag_prolongation (stag_mg_solver.f90:1365-1628): fine += P coarse
void s_prolong_add(const Geo& gf, const Geo& gc, Vec* fine, const Vec* coarse) {
    const int dim = gf.dim;
    for (int c = 0; c < dim; c++) {
        double* F = fine[c].data();
        const double* C = coarse[c].data();
        int a = (c == 0) ? 1 : 0;
        int b = (dim == 3) ? ((c == 2) ? 1 : 2) : -1;
        forall(gf, [&](int i, int j, int k) {
            int I[3] = {i, j, k};
            int h[3] = {i / 2, j / 2, k / 2};
            int oa = (I[a] % 2 == 0) ? -1 : 1;
            int ob = (b >= 0) ? ((I[b] % 2 == 0) ? -1 : 1) : 0;
            auto at = [&](int o, int pa, int pb) {
                int q[3] = {h[0], h[1], h[2]};
                q[c] += o;
                q[a] += pa;
                if (b >= 0) q[b] += pb;
                // the coarse ghost cells: multifab_physbc_macvel after the coarse smooths
                return gc.any_wall() ? vel(gc, C, c, q[0], q[1], q[2]) : C[gc.id(q[0], q[1], q[2])];
            };
            long f = gf.id(i, j, k);
            bool even = (I[c] % 2 == 0);
            double v;
            if (dim == 2) {
                if (even) v = 0.75 * at(0, 0, 0) + 0.25 * at(0, oa, 0);
                else v = 0.375 * at(0, 0, 0) + 0.125 * at(0, oa, 0) + 0.375 * at(1, 0, 0) + 0.125 * at(1, oa, 0);
            } else {
                const double n16 = 9.0 / 16.0, t16 = 3.0 / 16.0, o16 = 1.0 / 16.0;
                const double n32 = 9.0 / 32.0, t32 = 3.0 / 32.0, o32 = 1.0 / 32.0;
                if (even) v = n16 * at(0, 0, 0) + t16 * at(0, oa, 0) + t16 * at(0, 0, ob) + o16 * at(0, oa, ob);
                else v = n32 * at(0, 0, 0) + t32 * at(0, oa, 0) + t32 * at(0, 0, ob) + o32 * at(0, oa, ob)
                       + n32 * at(1, 0, 0) + t32 * at(1, oa, 0) + t32 * at(1, 0, ob) + o32 * at(1, oa, ob);
            }
            F[f] = F[f] + v;
        });
    }
    if (gf.any_wall()) {
        double* fp[3] = {fine[0].data(), fine[1].data(), dim == 3 ? fine[2].data() : nullptr};
        zero_wall_faces(gf, fp);
    }
}

int nlevs_mg(const Geo& g, int minwidth) {
    // compute_nlevs_mg (stag_mg_layout.f90:179-222), one box
    int nl = -1;
    for (int d = 0; d < g.dim; d++) {
        int t = g.n[d], r = 1;
        while (t % 2 == 0 && t / minwidth != 1) {
            t /= 2;
            r++;
        }
        nl = (nl < 0) ? r : std::min(nl, r);
    }
    return nl;
}

// The box layout of the level (probin_common max_grid_size), module state as
// in the reference: boxes of max_grid_size cells per direction (which must
// divide n_cells); 0 = one box covering the domain.
int g_max_grid_size[3] = {0, 0, 0};

// levels of the multi-box hierarchy (compute_nlevs_mg over boxes of
// max_grid_size) and whether its bottom is the "fancy" nested solve
// (stag_mg_solver.f90:97-101, 447): on when stag_mg_bottom_solver = 4 and
// n_cells / max_grid_size >= 2 in every direction
void box_layout(const Geo& g0, const fhd_gmres_params* p, int nl_domain, int* nl_box, bool* fancy) {
    *nl_box = nl_domain;
    *fancy = false;
    bool multi = true, any = false;
    int nb[3] = {g0.n[0], g0.n[1], g0.n[2]};
    for (int d = 0; d < g0.dim; d++) {
        const int m = g_max_grid_size[d];
        if (m <= 0 || m >= g0.n[d]) {
            multi = false;
            continue;
        }
        nb[d] = m;
        any = true;
    }
    if (!any) return;
    Geo gb(g0.dim, nb, g0.dx);
    *nl_box = nlevs_mg(gb, p->stag_mg_minwidth);
    *fancy = (p->stag_mg_bottom_solver == 4) && multi;
}

// stag_mg_solver (stag_mg_solver.f90:37-863).  With one box the hierarchy
// has compute_nlevs_mg(domain) levels.  With several boxes it has
// compute_nlevs_mg(box) levels; its bottom is either nsmooths_bottom smooths
// or, "fancy" (stag_mg_solver.f90:447-555), a nested stag_mg_solver on the
// bottom grid re-boxed as one box (stag_mg_layout.f90:96-107), whose own
// levels are the deeper levels of the domain hierarchy.
int stag_mg(const Geo& g0, int visc, const fhd_gmres_params* p, const double* const alpha_fc[],
            const double* beta, const double* const beta_ed[], const double* gamma, double theta,
            double* const phi[], const double* const rhs[], double* hist = nullptr) {
    const int dim = g0.dim;
    if (g0.any_wall() && visc < 1) return FHD_ERR_UNSUPPORTED;  // walls: visc_type 1, 2 or 3
    const int nl_domain = nlevs_mg(g0, p->stag_mg_minwidth);
    int nl_box;
    bool fancy;
    box_layout(g0, p, nl_domain, &nl_box, &fancy);
    // levels built: the whole domain hierarchy when the fancy bottom may
    // descend it, else the box hierarchy
    const int nl = fancy ? nl_domain : nl_box;
    std::vector<SLevel> L(nl);
    for (int l = 0; l < nl; l++) {
        L[l].g = (l == 0) ? g0 : L[l - 1].g.coarsen();
        const long nc = L[l].g.nc;
        for (int c = 0; c < dim; c++) {
            L[l].alpha[c].assign(nc, 0.0);
            L[l].phi[c].assign(nc, 0.0);
            L[l].rhs[c].assign(nc, 0.0);
            L[l].Lphi[c].assign(nc, 0.0);
        }
        L[l].beta.assign(nc, 0.0);
        L[l].gamma.assign(nc, 0.0);
        for (int e = 0; e < n_edge(dim); e++) L[l].bed[e].assign(nc, 0.0);
    }
    const long nc0 = g0.nc;
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc0; f++) L[0].alpha[c][f] = alpha_fc[c][f] * theta;
    std::copy(beta, beta + nc0, L[0].beta.begin());
    std::copy(gamma, gamma + nc0, L[0].gamma.begin());
    for (int e = 0; e < n_edge(dim); e++) std::copy(beta_ed[e], beta_ed[e] + nc0, L[0].bed[e].begin());
    for (int l = 1; l < nl; l++) {
        cc_average(L[l - 1].g, L[l].g, L[l - 1].beta, L[l].beta);
        cc_average(L[l - 1].g, L[l].g, L[l - 1].gamma, L[l].gamma);
        s_restrict(L[l - 1].g, L[l].g, L[l - 1].alpha, L[l].alpha, true);
        edge_coarsen(L[l - 1].g, L[l].g, L[l - 1].bed, L[l].bed);
    }
    for (int c = 0; c < dim; c++) {
        std::copy(phi[c], phi[c] + nc0, L[0].phi[c].begin());
        std::copy(rhs[c], rhs[c] + nc0, L[0].rhs[c].begin());
    }
    std::vector<int> colors;
    if (p->stag_mg_smoother == 0) colors.push_back(0);
    else for (int c = 1; c <= 2 * dim; c++) colors.push_back(c);
    const double omega = p->stag_mg_omega;

    // V-cycles on levels l0 .. lend-1 with level l0's phi and rhs as the
    // problem (one stag_mg_solver call); nest: the level whose bottom solve
    // is a nested call on levels nest .. nl-1 (the fancy bottom), or -1
    std::function<void(int, int, int, double*)> solve = [&](int l0, int lend, int nest, double* hst) {
        const Geo& gl = L[l0].g;
        // initial residual (stag_mg_solver.f90:259-313)
        double resid0[3] = {0, 0, 0};
        s_applyop(L[l0], visc, 0);
        for (int c = 0; c < dim; c++) {
            const double* lp = L[l0].Lphi[c].data();
            const double* r = L[l0].rhs[c].data();
            resid0[c] = reduce_max(gl, [&](int i, int j, int k) { long f = gl.id(i, j, k); return std::fabs(lp[f] - r[f]); });
        }
        // L2 norm of the initial residual, for the per-V-cycle history that
        // stag_mg_verbosity >= 1 prints (stag_mg_solver.f90:782-785)
        double r0l2 = 0.0;
        if (hst) {
            for (int c = 0; c < dim; c++) {
                const double* lp = L[l0].Lphi[c].data();
                const double* r = L[l0].rhs[c].data();
                r0l2 += reduce_sum(gl, [&](int i, int j, int k) { long f = gl.id(i, j, k); double d = lp[f] - r[f]; return d * d; });
            }
        }
        bool allzero = true, anyzero = false;
        double rmax = 0.0;
        for (int c = 0; c < dim; c++) {
            allzero = allzero && (resid0[c] == 0.0);
            anyzero = anyzero || (resid0[c] == 0.0);
            rmax = std::max(rmax, resid0[c]);
        }
        if (allzero) return;
        if (anyzero)
            for (int c = 0; c < dim; c++) resid0[c] = rmax;
        const int bottom = nest >= 0 ? nest : lend - 1;
        for (int vc = 1; vc <= p->stag_mg_max_vcycles; vc++) {
            for (int l = l0 + 1; l < lend; l++)
                for (int c = 0; c < dim; c++) std::fill(L[l].phi[c].begin(), L[l].phi[c].end(), 0.0);
            for (int l = l0; l < bottom; l++) {
                for (int m = 0; m < p->stag_mg_nsmooths_down; m++)
                    for (int col : colors) s_smooth(L[l], visc, omega, col);
                s_applyop(L[l], visc, 0);
                for (int c = 0; c < dim; c++) {
                    double* lp = L[l].Lphi[c].data();
                    const double* r = L[l].rhs[c].data();
                    for (long f = 0; f < L[l].g.nc; f++) lp[f] = -(lp[f] - r[f]);
                }
                if (L[l].g.any_wall()) {
                    // residual and restricted rhs zero on walls (stag_mg_solver.f90:420-440)
                    double* lp[3] = {L[l].Lphi[0].data(), L[l].Lphi[1].data(), dim == 3 ? L[l].Lphi[2].data() : nullptr};
                    zero_wall_faces(L[l].g, lp);
                }
                s_restrict(L[l].g, L[l + 1].g, L[l].Lphi, L[l + 1].rhs, false);
                if (L[l + 1].g.any_wall()) {
                    double* cr[3] = {L[l + 1].rhs[0].data(), L[l + 1].rhs[1].data(),
                                     dim == 3 ? L[l + 1].rhs[2].data() : nullptr};
                    zero_wall_faces(L[l + 1].g, cr);
                }
            }
            if (nest >= 0) {
                solve(nest, lend, -1, nullptr);  // theta_alpha = 1: the level's alpha carries it
            } else {
                for (int m = 0; m < p->stag_mg_nsmooths_bottom; m++)
                    for (int col : colors) s_smooth(L[bottom], visc, omega, col);
            }
            for (int l = bottom - 1; l >= l0; l--) {
                s_prolong_add(L[l].g, L[l + 1].g, L[l].phi, L[l + 1].phi);
                for (int m = 0; m < p->stag_mg_nsmooths_up; m++)
                    for (int col : colors) s_smooth(L[l], visc, omega, col);
            }
            if (vc == p->stag_mg_max_vcycles && !hst) break;  // the final residual decides nothing
            s_applyop(L[l0], visc, 0);
            bool done = true;
            double rl2 = 0.0;
            for (int c = 0; c < dim; c++) {
                const double* lp = L[l0].Lphi[c].data();
                const double* r = L[l0].rhs[c].data();
                double rr = reduce_max(gl, [&](int i, int j, int k) { long f = gl.id(i, j, k); return std::fabs(lp[f] - r[f]); });
                done = done && (rr / resid0[c] < p->stag_mg_rel_tol);
                if (hst) rl2 += reduce_sum(gl, [&](int i, int j, int k) { long f = gl.id(i, j, k); double d = lp[f] - r[f]; return d * d; });
            }
            if (hst) hst[vc - 1] = std::sqrt(rl2) / std::sqrt(r0l2);
            if (done || vc == p->stag_mg_max_vcycles) break;
        }
    };
    solve(0, nl, fancy && nl_box < nl ? nl_box - 1 : -1, hist);
    for (int c = 0; c < dim; c++) std::copy(L[0].phi[c].begin(), L[0].phi[c].end(), phi[c]);
    return 0;
}

// ---------------------------------------------------------------------
// cell-centred pressure multigrid (macproject.f90:34-316 calling FBoxLib
// ml_cc_solve).  Semantics restated from PreconditionerNotes.tex:484-575:
// red-black Gauss-Seidel (omega = 1), restriction by averaging the 2^dim
// children, piecewise-constant prolongation, nu1/nu2 smooths per level,
// mg_nsmooths_bottom smooths on the coarsest level, mg_max_vcycles cycles.
// ---------------------------------------------------------------------
struct CLevel {
    Geo g;
    Vec a[3];  // face coefficient (alphainv), low side of each cell
    Vec phi, rhs, res;
};

inline double c_lap(const Geo& g, const Vec* a, const double* phi, int i, int j, int k, double* diag) {
    const double q = 1.0 / (g.dx * g.dx);
    const long f = g.id(i, j, k);
    const double pc = phi[f];
    double s = 0.0, dg = 0.0;
    for (int d = 0; d < g.dim; d++) {
        int e[3] = {0, 0, 0};
        e[d] = 1;
        const long fp = g.id(i + e[0], j + e[1], k + e[2]);
        const long fm = g.id(i - e[0], j - e[1], k - e[2]);
        const double ahi = a[d][fp], alo = a[d][f];
        s += ahi * (phi[fp] - pc) - alo * (pc - phi[fm]);
        dg += ahi + alo;
    }
    if (diag) *diag = -dg * q;
    return s * q;
}

void c_gsrb(CLevel& L) {
    const Geo& g = L.g;
    for (int color = 0; color < 2; color++) {
        double* r = L.res.data();
        const double* ph = L.phi.data();
        forall(g, [&](int i, int j, int k) {
            if (((i + j + k) & 1) != color) return;
            long f = g.id(i, j, k);
            double dg;
            double lp = c_lap(g, L.a, ph, i, j, k, &dg);
            r[f] = (L.rhs[f] - lp) / dg;
        });
        double* p = L.phi.data();
        forall(g, [&](int i, int j, int k) {
            if (((i + j + k) & 1) != color) return;
            long f = g.id(i, j, k);
            p[f] = p[f] + r[f];
        });
    }
}

void c_vcycle(std::vector<CLevel>& L, int l, const fhd_gmres_params* p) {
    CLevel& C = L[l];
    const int nl = (int)L.size();
    if (l == nl - 1) {
        for (int m = 0; m < p->mg_nsmooths_bottom; m++) c_gsrb(C);
        return;
    }
    for (int m = 0; m < p->mg_nsmooths_down; m++) c_gsrb(C);
    const Geo& g = C.g;
    forall(g, [&](int i, int j, int k) {
        long f = g.id(i, j, k);
        C.res[f] = C.rhs[f] - c_lap(g, C.a, C.phi.data(), i, j, k, nullptr);
    });
    CLevel& D = L[l + 1];
    cc_average(g, D.g, C.res, D.rhs);
    std::fill(D.phi.begin(), D.phi.end(), 0.0);
    c_vcycle(L, l + 1, p);
    forall(g, [&](int i, int j, int k) {
        long f = g.id(i, j, k);
        C.phi[f] = C.phi[f] + D.phi[D.g.id(i / 2, j / 2, k / 2)];
    });
    for (int m = 0; m < p->mg_nsmooths_up; m++) c_gsrb(C);
}

int macproject_impl(const Geo& g0, const fhd_gmres_params* p, double* phi, const double* const ainv[],
                    const double* rhs, double* hist = nullptr) {
    const int dim = g0.dim;
    const int nl = nlevs_mg(g0, p->mg_minwidth);
    std::vector<CLevel> L(nl);
    for (int l = 0; l < nl; l++) {
        L[l].g = (l == 0) ? g0 : L[l - 1].g.coarsen();
        long nc = L[l].g.nc;
        for (int d = 0; d < dim; d++) L[l].a[d].assign(nc, 0.0);
        L[l].phi.assign(nc, 0.0);
        L[l].rhs.assign(nc, 0.0);
        L[l].res.assign(nc, 0.0);
    }
    for (int d = 0; d < dim; d++) std::copy(ainv[d], ainv[d] + g0.nc, L[0].a[d].begin());
    for (int l = 1; l < nl; l++) s_restrict(L[l - 1].g, L[l].g, L[l - 1].a, L[l].a, true);
    // walls: homogeneous Neumann, no flux through a wall face (with the
    // periodic index wrap the high wall face is face 0 as well)
    for (int l = 0; l < nl && g0.any_wall(); l++) {
        double* ap[3] = {L[l].a[0].data(), L[l].a[1].data(), dim == 3 ? L[l].a[2].data() : nullptr};
        zero_wall_faces(L[l].g, ap);
    }
    std::copy(rhs, rhs + g0.nc, L[0].rhs.begin());
    const double r0 = reduce_max(g0, [&](int i, int j, int k) { return std::fabs(rhs[g0.id(i, j, k)]); });
    if (hist) {
        // the L2 residual after each of mg_max_vcycles V-cycles over the
        // initial one, without the stopping test (the reference's multigrid
        // residual histories, run_result/Mg_StagMg_performance)
        auto l2 = [&](bool with_phi) {
            CLevel& C = L[0];
            return std::sqrt(reduce_sum(g0, [&](int i, int j, int k) {
                const double r = C.rhs[g0.id(i, j, k)] - (with_phi ? c_lap(g0, C.a, C.phi.data(), i, j, k, nullptr) : 0.0);
                return r * r;
            }));
        };
        const double n0 = l2(false);
        for (int vc = 0; vc < p->mg_max_vcycles; vc++) {
            c_vcycle(L, 0, p);
            hist[vc] = n0 > 0.0 ? l2(true) / n0 : 0.0;
        }
    } else if (r0 > 0.0) {
        for (int vc = 1; vc <= p->mg_max_vcycles; vc++) {
            c_vcycle(L, 0, p);
            if (vc == p->mg_max_vcycles) break;
            CLevel& C = L[0];
            double rr = reduce_max(g0, [&](int i, int j, int k) {
                return std::fabs(C.rhs[g0.id(i, j, k)] - c_lap(g0, C.a, C.phi.data(), i, j, k, nullptr));
            });
            if (rr <= std::max(p->mg_rel_tol * r0, p->mg_abs_tol)) break;
        }
    }
    std::copy(L[0].phi.begin(), L[0].phi.end(), phi);
    return 0;
}

// ---------------------------------------------------------------------
// div / grad / norms (div_and_grad.f90:417-703, 884-1035;
// norm_inner_product.f90)
// ---------------------------------------------------------------------
void c_div(const Geo& g, const double* const u[], double* div, bool increment) {
    const double dxinv = 1.0 / g.dx;
    forall(g, [&](int i, int j, int k) {
        long f = g.id(i, j, k);
        double s = (u[0][g.id(i + 1, j, k)] - u[0][f]) * dxinv + (u[1][g.id(i, j + 1, k)] - u[1][f]) * dxinv;
        if (g.dim == 3) s += (u[2][g.id(i, j, k + 1)] - u[2][f]) * dxinv;
        div[f] = increment ? div[f] + s : s;
    });
}

void c_grad(const Geo& g, const double* p, double* const gp[]) {
    const double dxinv = 1.0 / g.dx;
    for (int d = 0; d < g.dim; d++) {
        int e[3] = {0, 0, 0};
        e[d] = 1;
        forall(g, [&](int i, int j, int k) {
            long f = g.id(i, j, k);
            // at a wall the pressure ghost is the interior value (first-order
            // extrapolation), so the gradient there is zero (div_and_grad.f90:540-556)
            gp[d][f] = wall_face(g, d, i, j, k) ? 0.0 : (p[f] - p[g.id(i - e[0], j - e[1], k - e[2])]) * dxinv;
        });
    }
}

double dot(const Geo& g, const double* a, const double* b) {
    return reduce_sum(g, [&](int i, int j, int k) { long f = g.id(i, j, k); return a[f] * b[f]; });
}

double sum(const Geo& g, const double* a) {
    return reduce_sum(g, [&](int i, int j, int k) { return a[g.id(i, j, k)]; });
}

// a Stokes vector (u_0..u_{dim-1}, p), each of nc entries
struct SV {
    Vec c[4];
    int dim = 2;
    void init(int d, long nc) {
        dim = d;
        for (int i = 0; i <= d; i++) c[i].assign(nc, 0.0);
    }
    double* u(int d) { return c[d].data(); }
    double* p() { return c[dim].data(); }
};

void up_ptrs(SV& v, double** u, double*& p) {
    for (int d = 0; d < v.dim; d++) u[d] = v.u(d);
    p = v.p();
}

double stag_l2(const Geo& g, const double* const u[]) {
    double s = 0.0;
    for (int d = 0; d < g.dim; d++) s += dot(g, u[d], u[d]);
    return std::sqrt(s);
}

// gmres_spatial_order = 4 (apply_matrix.f90:54-67, 124-135): the viscous
// operator of stag_applyop_4o_2d/_3d (stag_applyop.f90:1262-1510, visc_type
// 1 only) and the gradient of compute_grad_4o_2d/_3d (div_and_grad.f90:
// 804-880); the divergence stays second order (apply_matrix.f90:143-147).
// Summation order as in those loops: for each direction x, y, z the terms
// +16 phi(+1), +16 phi(-1), -1 phi(+2), -1 phi(-2).
static void apply_matrix_4o(const Geo& g, double* const b_u[], const double* const x_u[], const double* x_p,
                            const Vec alpha[], double b) {
    const int dim = g.dim;
    const double t2 = 1.0 / (12.0 * g.dx * g.dx);
    const double t1 = 1.0 / (12.0 * g.dx);
    const double cdiag = dim == 2 ? 60.0 : 90.0;
    for (int c = 0; c < dim; c++) {
        const double* u = x_u[c];
        double* out = b_u[c];
        forall(g, [&](int i, int j, int k) {
            const long f = g.id(i, j, k);
            double s = 0.0;
            for (int d = 0; d < dim; d++) {
                const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
                const double t = 16.0 * u[g.id(i + e0, j + e1, k + e2)];
                s = d == 0 ? t : s + t;
                s = s + 16.0 * u[g.id(i - e0, j - e1, k - e2)];
                s = s - 1.0 * u[g.id(i + 2 * e0, j + 2 * e1, k + 2 * e2)];
                s = s - 1.0 * u[g.id(i - 2 * e0, j - 2 * e1, k - 2 * e2)];
            }
            const double L = (alpha[c][f] + cdiag * b * t2) * u[f] - s * b * t2;
            // compute_grad_4o: (-p(+1) + 15 p(0) - 15 p(-1) + p(-2)) / (12 dx)
            const int e0 = c == 0, e1 = c == 1, e2 = c == 2;
            const double gp = (-x_p[g.id(i + e0, j + e1, k + e2)] + 15.0 * x_p[f] -
                               15.0 * x_p[g.id(i - e0, j - e1, k - e2)] +
                               x_p[g.id(i - 2 * e0, j - 2 * e1, k - 2 * e2)]) *
                              t1;
            out[f] = L + gp;
        });
    }
}

int apply_matrix_impl(const Geo& g, int visc, double* const b_u[], double* b_p, const double* const x_u[],
                      const double* x_p, const double* const alpha_fc[], const double* beta,
                      const double* const beta_ed[], const double* gamma, double theta, int order) {
    const int dim = g.dim;
    // stag_applyop_4o supports visc_type 1 only (stag_applyop.f90:1355, 1506)
    if (order != 2 && (order != 4 || visc != 1)) return -5;
    // walls: visc_type 1, 2 or 3, second order
    if (g.any_wall() && (visc < 1 || order != 2)) return -5;
    Vec alpha[3], bed[3];
    Vec vb(beta, beta + g.nc), vg(gamma, gamma + g.nc);
    for (int c = 0; c < dim; c++) {
        alpha[c].resize(g.nc);
        for (long f = 0; f < g.nc; f++) alpha[c][f] = alpha_fc[c][f] * theta;
    }
    for (int e = 0; e < n_edge(dim); e++) bed[e].assign(beta_ed[e], beta_ed[e] + g.nc);
    if (order == 4) {
        apply_matrix_4o(g, b_u, x_u, x_p, alpha, beta[0]);
    } else {
        const double* ph[3] = {x_u[0], x_u[1], dim == 3 ? x_u[2] : nullptr};
        for (int c = 0; c < dim; c++) {
            double* out = b_u[c];
            forall(g, [&](int i, int j, int k) {
                out[g.id(i, j, k)] =
                    wall_face(g, c, i, j, k) ? 0.0 : lface(g, visc, alpha, vb, vg, bed, ph, c, i, j, k, nullptr);
            });
        }
        std::vector<Vec> gp(dim, Vec(g.nc));
        double* gpp[3] = {gp[0].data(), gp[1].data(), dim == 3 ? gp[2].data() : nullptr};
        c_grad(g, x_p, gpp);
        for (int c = 0; c < dim; c++)
            for (long f = 0; f < g.nc; f++) b_u[c][f] = b_u[c][f] + gp[c][f];
    }
    c_div(g, x_u, b_p, false);
    for (long f = 0; f < g.nc; f++) b_p[f] = b_p[f] * -1.0;
    return 0;
}

// 1 / diagonal of the viscous operator on faces (inverse_diag_lap.f90:
// 17-330); the same summation order as the 2D and 3D loops there
static void inverse_diag_lap(const Geo& g, int visc, const double* beta, const double* const beta_ed[],
                             double* const minv[]) {
    const int dim = g.dim;
    if (visc == 1 || visc == 2) {
        const double b = beta[0];
        const double m = (dim == 2 ? (visc == 1 ? 4.0 : 6.0) : (visc == 1 ? 6.0 : 8.0)) * b;
        for (int c = 0; c < dim; c++) std::fill(minv[c], minv[c] + g.nc, 1.0 / m);
        return;
    }
    const double cb = visc == -2 ? 2.0 : 1.0;
    for (int c = 0; c < dim; c++) {
        int e[3] = {0, 0, 0};
        e[c] = 1;
        forall(g, [&](int i, int j, int k) {
            const long f = g.id(i, j, k);
            double s = cb * beta[f] + cb * beta[g.id(i - e[0], j - e[1], k - e[2])];
            if (dim == 2) {
                // x face: node (i, j+1) then (i, j); y face: node (i+1, j) then (i, j)
                s = s + beta_ed[0][c == 0 ? g.id(i, j + 1, 0) : g.id(i + 1, j, 0)];
                s = s + beta_ed[0][f];
            } else {
                for (int d = 0; d < 3; d++) {
                    if (d == c) continue;
                    const double* be = beta_ed[edge_of(3, c, d)];
                    s = s + be[f];
                    s = s + be[g.id(i + (d == 0), j + (d == 1), k + (d == 2))];
                }
            }
            minv[c][f] = 1.0 / s;
        });
    }
}

// visc_schur_complement (apply_precon.f90:538-685): the BFBt
// approximation of the Schur complement, x_p = L_mu^-1 D mu^-1 L mu^-1 G
// L_mu^-1 rhs (+ theta phi), L_mu the pressure Laplacian with face
// coefficients mu^-1 = 1/diag(viscous operator); rhs is overwritten
static int visc_schur(const Geo& g, int visc, const fhd_gmres_params* p, double* rhs, double* x_out,
                      const double* beta, const double* const beta_ed[], double theta, const double* phi) {
    const int dim = g.dim;
    const long nc = g.nc;
    std::vector<Vec> mu(dim, Vec(nc)), gp(dim, Vec(nc)), lg(dim, Vec(nc));
    double* mup[3] = {mu[0].data(), mu[1].data(), dim == 3 ? mu[2].data() : nullptr};
    double* gpp[3] = {gp[0].data(), gp[1].data(), dim == 3 ? gp[2].data() : nullptr};
    double* lgp[3] = {lg[0].data(), lg[1].data(), dim == 3 ? lg[2].data() : nullptr};
    inverse_diag_lap(g, visc, beta, beta_ed, mup);
    const double* muc[3] = {mup[0], mup[1], mup[2]};
    Vec phi_mu(nc, 0.0);
    macproject_impl(g, p, phi_mu.data(), muc, rhs);
    c_grad(g, phi_mu.data(), gpp);
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) gp[c][f] = gp[c][f] * mu[c][f];
    // stag_applyop with zero alpha: theta*0*u - L u
    Vec zero(nc, 0.0), vb(beta, beta + nc);
    Vec alpha0[3], bed[3];
    for (int c = 0; c < dim; c++) alpha0[c] = zero;
    for (int e = 0; e < n_edge(dim); e++) bed[e].assign(beta_ed[e], beta_ed[e] + nc);
    const double* ph[3] = {gpp[0], gpp[1], gpp[2]};
    for (int c = 0; c < dim; c++)
        forall(g, [&](int i, int j, int k) {
            lg[c][g.id(i, j, k)] = lface(g, visc, alpha0, vb, zero, bed, ph, c, i, j, k, nullptr);
        });
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) lg[c][f] = lg[c][f] * mu[c][f];
    c_div(g, lgp, rhs, false);
    std::fill(phi_mu.begin(), phi_mu.end(), 0.0);
    macproject_impl(g, p, phi_mu.data(), muc, rhs);
    for (long f = 0; f < nc; f++) x_out[f] = phi_mu[f];
    if (std::fabs(theta) > 0.0)
        for (long f = 0; f < nc; f++) x_out[f] = x_out[f] + phi[f] * theta;
    return 0;
}

// apply_precon (apply_precon.f90:29-475); visc_schur_approx 0 (the simple
// Schur complements) or 1 (visc_schur_complement, |visc_type| 1 and 2)
int apply_precon_impl(const Geo& g, int visc, const fhd_gmres_params* p, const double* const b_u[],
                      const double* b_p, double* const x_u[], double* x_p, const double* const alpha_fc[],
                      const double* beta, const double* const beta_ed[], const double* gamma, double theta) {
    const int dim = g.dim;
    const long nc = g.nc;
    const int pt = p->precon_type;
    const int apt = std::abs(pt);
    const int av = std::abs(visc);
    const bool bfbt = p->visc_schur_approx != 0;
    if (bfbt && av == 3) return FHD_ERR_UNSUPPORTED;  // inverse_diag_lap.f90: no |visc_type| = 3
    if (apt < 1 || apt > 5) return FHD_ERR_UNSUPPORTED;
    Vec phi(nc, 0.0), mac_rhs(nc, 0.0);
    std::vector<Vec> ainv(dim, Vec(nc));
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) ainv[c][f] = 1.0 / alpha_fc[c][f];
    const double* ainvp[3] = {ainv[0].data(), ainv[1].data(), dim == 3 ? ainv[2].data() : nullptr};
    for (int c = 0; c < dim; c++) std::fill(x_u[c], x_u[c] + nc, 0.0);

    auto stagmg = [&](double* const ph[], const double* const rh[]) {
        return stag_mg(g, visc, p, alpha_fc, beta, beta_ed, gamma, theta, ph, rh);
    };
    auto subtract_weighted_gradp = [&](double* const u[], const double* w[], const double* ph) {
        std::vector<Vec> gp(dim, Vec(nc));
        double* gpp[3] = {gp[0].data(), gp[1].data(), dim == 3 ? gp[2].data() : nullptr};
        c_grad(g, ph, gpp);
        for (int c = 0; c < dim; c++)
            for (long f = 0; f < nc; f++) u[c][f] = u[c][f] + (-1.0) * (gp[c][f] * (w ? w[c][f] : 1.0));
    };
    // x_p = theta*Phi - c*beta*mac_rhs  (simple_schur_complement,
    // apply_precon.f90:479-534); also case 1 with +precon_type
    auto simple_schur = [&]() {
        for (long f = 0; f < nc; f++) {
            double v;
            if (av == 1 || av == 2) {
                v = mac_rhs[f] * -1.0;
                v = v * beta[f];
                if (av == 2) v = v * 2.0;
            } else {
                v = mac_rhs[f] * (-4.0 / 3.0);
                v = v * beta[f];
                double m = (mac_rhs[f] * -1.0) * gamma[f];
                v = v + m;
            }
            if (std::fabs(theta) > 0.0) v = v + phi[f] * theta;
            x_p[f] = v;
        }
    };

    if (apt == 1) {
        stagmg(x_u, b_u);
        c_div(g, x_u, mac_rhs.data(), false);
        for (long f = 0; f < nc; f++) mac_rhs[f] = mac_rhs[f] + b_p[f];
        macproject_impl(g, p, phi.data(), ainvp, mac_rhs.data());
        subtract_weighted_gradp(x_u, ainvp, phi.data());
        Vec xp(nc);
        if (bfbt) {
            visc_schur(g, visc, p, mac_rhs.data(), x_p, beta, beta_ed, theta, phi.data());
        } else if (pt == 1 || theta == 0.0) {
            for (long f = 0; f < nc; f++) xp[f] = mac_rhs[f] * -1.0;
        } else {
            // x_p = -L_alpha Phi (cc_applyop with zero cell coefficient)
            CLevel C;
            C.g = g;
            for (int d = 0; d < dim; d++) C.a[d] = ainv[d];
            forall(g, [&](int i, int j, int k) {
                xp[g.id(i, j, k)] = -c_lap(g, C.a, phi.data(), i, j, k, nullptr);
            });
        }
        for (long f = 0; f < nc && !bfbt; f++) {
            double v = xp[f];
            if (av == 1 || av == 2) {
                v = v * beta[f];
                if (av == 2) v = v * 2.0;
            } else {
                double m = v * gamma[f];
                v = v * beta[f];
                v = v * (4.0 / 3.0);
                v = v + m;
            }
            v = v + phi[f] * theta;
            x_p[f] = v;
        }
    } else if (apt == 2 || apt == 5) {
        stagmg(x_u, b_u);
        c_div(g, x_u, mac_rhs.data(), false);
        for (long f = 0; f < nc; f++) mac_rhs[f] = mac_rhs[f] + b_p[f];
        if (std::fabs(theta) > 0.0) macproject_impl(g, p, phi.data(), ainvp, mac_rhs.data());
        if (bfbt) visc_schur(g, visc, p, mac_rhs.data(), x_p, beta, beta_ed, theta, phi.data());
        else simple_schur();
        if (pt == -2 || pt == -5)
            for (long f = 0; f < nc; f++) x_p[f] = x_p[f] * -1.0;
        if (apt == 5) {
            std::vector<Vec> bt(dim);
            for (int c = 0; c < dim; c++) bt[c].assign(b_u[c], b_u[c] + nc);
            double* btp[3] = {bt[0].data(), bt[1].data(), dim == 3 ? bt[2].data() : nullptr};
            subtract_weighted_gradp(btp, nullptr, x_p);
            stagmg(x_u, btp);
        }
    } else if (apt == 3) {
        for (long f = 0; f < nc; f++) mac_rhs[f] = (pt == -3) ? b_p[f] * -1.0 : b_p[f];
        if (std::fabs(theta) > 0.0) macproject_impl(g, p, phi.data(), ainvp, mac_rhs.data());
        if (bfbt) visc_schur(g, visc, p, mac_rhs.data(), x_p, beta, beta_ed, theta, phi.data());
        else simple_schur();
        std::vector<Vec> bt(dim);
        for (int c = 0; c < dim; c++) bt[c].assign(b_u[c], b_u[c] + nc);
        double* btp[3] = {bt[0].data(), bt[1].data(), dim == 3 ? bt[2].data() : nullptr};
        subtract_weighted_gradp(btp, nullptr, x_p);
        stagmg(x_u, btp);
    } else {  // 4: block diagonal
        stagmg(x_u, b_u);
        if (std::fabs(theta) > 0.0) {
            for (long f = 0; f < nc; f++) mac_rhs[f] = b_p[f];
            macproject_impl(g, p, phi.data(), ainvp, mac_rhs.data());
        }
        if (bfbt) visc_schur(g, visc, p, mac_rhs.data(), x_p, beta, beta_ed, theta, phi.data());
        for (long f = 0; f < nc && !bfbt; f++) {
            double ph = phi[f];
            if (std::fabs(theta) > 0.0) ph = ph * theta;
            double v = b_p[f] * beta[f];
            v = v - ph;
            if (av == 1 && pt == 4) v = v * -1.0;
            else if (av == 2 && pt == 4) v = v * -2.0;
            else if (av == 2 && pt == -4) v = v * 2.0;
            else if (av == 3 && pt == 4) { v = v * (-4.0 / 3.0); v = v + (b_p[f] * gamma[f]) * -1.0; }
            else if (av == 3 && pt == -4) { v = v * (4.0 / 3.0); v = v + b_p[f] * gamma[f]; }
            x_p[f] = v;
        }
    }
    // null space (apply_precon.f90:429-460)
    const double mean_p = sum(g, x_p) / (double)nc;
    for (long f = 0; f < nc; f++) x_p[f] = x_p[f] - mean_p;
    // the velocity problem is singular too when theta = 0 and no wall is
    // no-slip; then the mean of each periodic direction's component goes
    bool no_slip = false;
    for (int d = 0; d < dim; d++) no_slip = no_slip || g.wl[d] == -1 || g.wh[d] == -1;
    if (theta == 0.0 && !no_slip) {
        for (int c = 0; c < dim; c++) {
            if (g.wall(c)) continue;
            const double mu = sum(g, x_u[c]) / (double)nc;
            for (long f = 0; f < nc; f++) x_u[c][f] = x_u[c][f] - mu;
        }
    }
    return 0;
}

// gmres (gmres.f90:32-619)
int gmres_impl(const Geo& g, int visc, const fhd_gmres_params* p, const double* const b_u_in[],
               const double* b_p, double* const x_u[], double* x_p, const double* const alpha_fc[],
               const double* beta_in, const double* const beta_ed_in[], const double* gamma_in,
               double theta_in, double* norm_pre_rhs, fhd_solve_stats* st) {
    const int dim = g.dim;
    const long nc = g.nc;
    const int m = p->gmres_max_inner;
    const double w = p->p_norm_weight;
    const double sf = p->scale_factor;
    // scaling (gmres.f90:118-135) is applied to private copies
    std::vector<Vec> bu(dim), bed(n_edge(dim));
    Vec beta(beta_in, beta_in + nc), gamma(gamma_in, gamma_in + nc);
    for (int c = 0; c < dim; c++) bu[c].assign(b_u_in[c], b_u_in[c] + nc);
    for (int e = 0; e < n_edge(dim); e++) bed[e].assign(beta_ed_in[e], beta_ed_in[e] + nc);
    double theta = theta_in;
    if (sf != 1.0) {
        theta = theta * sf;
        for (long f = 0; f < nc; f++) x_p[f] = x_p[f] * sf;
        for (int c = 0; c < dim; c++)
            for (long f = 0; f < nc; f++) bu[c][f] = bu[c][f] * sf;
        for (long f = 0; f < nc; f++) { beta[f] = beta[f] * sf; gamma[f] = gamma[f] * sf; }
        for (int e = 0; e < n_edge(dim); e++)
            for (long f = 0; f < nc; f++) bed[e][f] = bed[e][f] * sf;
    }
    const double* bup[3] = {bu[0].data(), bu[1].data(), dim == 3 ? bu[2].data() : nullptr};
    const double* bedp[3] = {bed[0].data(), dim == 3 ? bed[1].data() : nullptr, dim == 3 ? bed[2].data() : nullptr};

    SV r, wv, tmp;
    r.init(dim, nc); wv.init(dim, nc); tmp.init(dim, nc);
    std::vector<SV> V(m + 1);
    for (auto& v : V) v.init(dim, nc);
    double* ru[3]; double* rp; up_ptrs(r, ru, rp);
    double* wu[3]; double* wp; up_ptrs(wv, wu, wp);
    double* tu[3]; double* tp; up_ptrs(tmp, tu, tp);

    auto precon = [&](const double* const in_u[], const double* in_p, double* const out_u[], double* out_p) {
        return apply_precon_impl(g, visc, p, in_u, in_p, out_u, out_p, alpha_fc, beta.data(), bedp,
                                 gamma.data(), theta);
    };
    auto matrix = [&](double* const out_u[], double* out_p, const double* const in_u[], const double* in_p) {
        return apply_matrix_impl(g, visc, out_u, out_p, in_u, in_p, alpha_fc, beta.data(), bedp, gamma.data(),
                                 theta, p->gmres_spatial_order);
    };
    auto snorm = [&](const double* const u[], const double* pp) {
        double nu = stag_l2(g, u);
        double np = std::sqrt(dot(g, pp, pp)) * w;
        return std::sqrt(nu * nu + np * np);
    };

    std::vector<double> cs(m + 1), sn(m + 1), y(m + 1), s(m + 2);
    std::vector<double> H((m + 2) * (m + 1), 0.0);
    auto Hh = [&](int i, int j) -> double& { return H[i * (m + 1) + j]; };  // 1-based i,j

    precon(bup, b_p, tu, tp);
    const double norm_pre_b = snorm(tu, tp);
    if (norm_pre_rhs) *norm_pre_rhs = norm_pre_b;
    const double norm_b = snorm(bup, b_p);
    int status = 0;
    if (st) { std::memset(st, 0, sizeof(*st)); st->norm_b = norm_b; st->norm_pre_b = norm_pre_b; }
    if (norm_b <= p->gmres_abs_tol) {
        for (int c = 0; c < dim; c++) std::fill(x_u[c], x_u[c] + nc, 0.0);
        std::fill(x_p, x_p + nc, 0.0);
        if (sf != 1.0)
            for (long f = 0; f < nc; f++) x_p[f] = x_p[f] * (1.0 / sf);
        return 0;
    }
    int total_iter = 0, iter = 0, i_copy = 0;
    double norm_resid = 0, norm_init_resid = 0, norm_resid_Stokes = 0, norm_init_Stokes = 0, norm_resid_est = 0;
    for (;;) {
        matrix(tu, tp, x_u, x_p);
        for (int c = 0; c < dim; c++)
            for (long f = 0; f < nc; f++) tu[c][f] = (tu[c][f] - bu[c][f]) * -1.0;
        for (long f = 0; f < nc; f++) tp[f] = (tp[f] - b_p[f]) * -1.0;
        norm_resid_Stokes = snorm(tu, tp);
        if (iter == 0) norm_init_Stokes = norm_resid_Stokes;
        precon(tu, tp, ru, rp);
        norm_resid = snorm(ru, rp);
        if (iter == 0) { norm_init_resid = norm_resid; norm_resid_est = norm_resid; }
        if (total_iter >= p->gmres_max_iter) { status = FHD_WARN_NOT_CONVERGED_MAXITER; break; }
        else if (total_iter >= p->gmres_min_iter) {
            if (norm_resid <= p->gmres_rel_tol * std::min(norm_pre_b, norm_init_resid)) {
                if (norm_resid_Stokes >= 10 * p->gmres_rel_tol * std::min(norm_b, norm_init_Stokes))
                    status = FHD_WARN_TRUE_RESID;
                break;
            } else if (norm_resid <= p->gmres_abs_tol) {
                break;
            }
        }
        if (iter >= p->gmres_max_outer) { status = FHD_WARN_NOT_CONVERGED_OUTER; break; }
        iter++;
        for (int c = 0; c <= dim; c++)
            for (long f = 0; f < nc; f++) V[0].c[c][f] = r.c[c][f] / norm_resid;
        std::fill(s.begin(), s.end(), 0.0);
        s[1] = norm_resid;
        int i;
        for (i = 1; i <= m; i++) {
            total_iter++;
            i_copy = i;
            double* vu[3]; double* vp; up_ptrs(V[i - 1], vu, vp);
            matrix(tu, tp, vu, vp);
            precon(tu, tp, wu, wp);
            for (int k = 1; k <= i; k++) {
                double ip = 0.0;
                for (int c = 0; c < dim; c++) ip += dot(g, wu[c], V[k - 1].c[c].data());
                double pp = dot(g, wp, V[k - 1].c[dim].data());
                Hh(k, i) = ip + (w * w) * pp;
                for (int c = 0; c <= dim; c++) {
                    double* wc = wv.c[c].data();
                    const double* vc = V[k - 1].c[c].data();
                    for (long f = 0; f < nc; f++) wc[f] = wc[f] - vc[f] * Hh(k, i);
                }
            }
            Hh(i + 1, i) = snorm(wu, wp);
            if (Hh(i + 1, i) != 0.0) {
                for (int c = 0; c <= dim; c++)
                    for (long f = 0; f < nc; f++) V[i].c[c][f] = wv.c[c][f] / Hh(i + 1, i);
            } else {
                status = FHD_ERR_ORTHO_BREAKDOWN;
                goto done;
            }
            // least_squares (gmres.f90:531-566)
            for (int k = 1; k <= i - 1; k++) {
                double t = cs[k] * Hh(k, i) + sn[k] * Hh(k + 1, i);
                Hh(k + 1, i) = -sn[k] * Hh(k, i) + cs[k] * Hh(k + 1, i);
                Hh(k, i) = t;
            }
            {   // rotmat (gmres.f90:568-597)
                double a = Hh(i, i), b = Hh(i + 1, i);
                if (b == 0.0) { cs[i] = 1.0; sn[i] = 0.0; }
                else if (std::fabs(b) > std::fabs(a)) { double t = a / b; sn[i] = 1.0 / std::sqrt(1.0 + t * t); cs[i] = t * sn[i]; }
                else { double t = b / a; cs[i] = 1.0 / std::sqrt(1.0 + t * t); sn[i] = t * cs[i]; }
            }
            {
                double t = cs[i] * s[i];
                s[i + 1] = -sn[i] * s[i];
                s[i] = t;
                Hh(i, i) = cs[i] * Hh(i, i) + sn[i] * Hh(i + 1, i);
                Hh(i + 1, i) = 0.0;
            }
            norm_resid_est = std::fabs(s[i + 1]);
            if (total_iter >= p->gmres_max_iter) break;
            else if (total_iter >= p->gmres_min_iter) {
                if (norm_resid_est <= p->gmres_rel_tol * std::min(norm_pre_b, norm_init_resid) ||
                    norm_resid_est <= p->gmres_abs_tol)
                    break;
            }
        }
        {   // SolveUTriangular (gmres.f90:599-619) with k = i_copy-1
            int k = i_copy - 1;
            y[k + 1] = s[k + 1] / Hh(k + 1, k + 1);
            for (int ii = k; ii >= 1; ii--) {
                double acc = 0.0;
                for (int jj = ii + 1; jj <= k + 1; jj++) acc += Hh(ii, jj) * y[jj];
                y[ii] = (s[ii] - acc) / Hh(ii, ii);
            }
            // update_sol (gmres.f90:495-529)
            for (int it = 1; it <= i_copy; it++) {
                for (long f = 0; f < nc; f++) x_p[f] = x_p[f] + V[it - 1].c[dim][f] * y[it];
                for (int c = 0; c < dim; c++)
                    for (long f = 0; f < nc; f++) x_u[c][f] = x_u[c][f] + V[it - 1].c[c][f] * y[it];
            }
        }
    }
done:
    if (sf != 1.0)
        for (long f = 0; f < nc; f++) x_p[f] = x_p[f] * (1.0 / sf);
    if (st) {
        st->outer_iters = iter;
        st->total_iters = total_iter;
        st->status = status;
        st->norm_init_resid = norm_init_resid;
        st->norm_resid = norm_resid;
        st->norm_resid_Stokes = norm_resid_Stokes;
        st->norm_init_Stokes = norm_init_Stokes;
        st->norm_resid_est = norm_resid_est;
    }
    return status;
}

// One pass of filter_stoch_m_flux (stochastic_m_fluxdiv.f90:604-778) along
// direction d over a periodic array: the symmetric smoothing stencil of
// width 1, 2 or 4 taps a side, the terms summed in the order written there.
// The ghosts it reads are the periodic images of the previous pass
// (multifab_fill_boundary between the passes); n[d] >= width.
static void filter_pass(const Geo& g, Vec& a, int d, int width) {
    Vec out(a.size());
    const int e[3] = {d == 0, d == 1, d == 2};
    forall(g, [&](int i, int j, int k) {
        auto at = [&](int s) { return a[g.id(i + s * e[0], j + s * e[1], k + s * e[2])]; };
        double v;
        if (width == 1)
            v = at(0) / 2 + at(-1) / 4 + at(1) / 4;
        else if (width == 2)
            v = 5 * at(0) / 8 - at(-2) / 16 + at(-1) / 4 - at(2) / 16 + at(1) / 4;
        else
            v = 93 * at(0) / 128 + 7 * at(-1) / 32 - 7 * at(-2) / 64 + at(-3) / 32 - at(-4) / 256 +
                7 * at(1) / 32 - 7 * at(2) / 64 + at(3) / 32 - at(4) / 256;
        out[g.id(i, j, k)] = v;
    });
    a.swap(out);
}

// stochastic_m_fluxdiv (stochastic_m_fluxdiv.f90:42-602); filtering_width
// 1, 2 or 4 filters the scaled stresses (x, then y, then z) before the
// divergence (:172-174, :226-230), periodic boxes only
int stoch_m_impl(const Geo& g, const fhd_stoch_params* sp, double* const force[], int increment,
                 const double* eta, const double* const eta_ed[], const double* T, const double* const T_ed[],
                 double dt, const double* weights, int n_rngs, const double* const W_cc[],
                 const double* const W_ed[]) {
    const int dim = g.dim, nE = n_edge(dim);
    const long nc = g.nc;
    const int width = sp->filtering_width;
    if (width != 0) {
        if (width != 1 && width != 2 && width != 4) return FHD_ERR_BAD_ARG;
        if (g.any_wall()) return FHD_ERR_UNSUPPORTED;
        for (int d = 0; d < dim; d++)
            if (g.n[d] < width) return FHD_ERR_BAD_ARG;
    }
    long ne[3] = {0, 0, 0};
    for (int e = 0; e < nE; e++) ne[e] = edge_count(g, e);
    std::vector<Vec> fcc(dim, Vec(nc, 0.0)), fed(2 * nE);
    for (int e = 0; e < 2 * nE; e++) fed[e].assign(ne[e / 2], 0.0);
    for (int r = 0; r < n_rngs; r++) {
        for (int c = 0; c < dim; c++)
            for (long f = 0; f < nc; f++) fcc[c][f] = fcc[c][f] + weights[r] * W_cc[r * dim + c][f];
        for (int e = 0; e < 2 * nE; e++)
            for (long f = 0; f < ne[e / 2]; f++) fed[e][f] = fed[e][f] + weights[r] * W_ed[r * 2 * nE + e][f];
    }
    const double variance = std::sqrt(sp->variance_coef_mom * 2.0 * sp->k_B / (sp->dV * dt));
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) fcc[c][f] = (variance * fcc[c][f]) * std::sqrt(eta[f] * T[f]);
    for (int e = 0; e < nE; e++)
        for (int comp = 0; comp < 2; comp++)
            for (long f = 0; f < ne[e]; f++)
                fed[2 * e + comp][f] = (variance * fed[2 * e + comp][f]) * std::sqrt(eta_ed[e][f] * T_ed[e][f]);
    if (g.any_wall()) {
        // mflux_bc_2d / _3d (stochastic_m_fluxdiv.f90:363-451): the edges on a
        // no-slip wall times sqrt(2), on a slip wall zero; the boundaries of
        // x, then y, then z, each low side before its high side
        for (int e = 0; e < nE; e++) {
            int a, b;
            edge_dirs(dim, e, a, b);
            long m[3];
            edge_ext(g, e, m);
            for (long f = 0; f < ne[e]; f++) {
                const int q[3] = {(int)(f % m[0]), (int)((f / m[0]) % m[1]), (int)(f / (m[0] * m[1]))};
                for (int d : {a, b}) {
                    if (!g.wall(d)) continue;
                    int side = 0;
                    if (q[d] == 0) side = g.wl[d];
                    else if (q[d] == g.n[d]) side = g.wh[d];
                    if (side == 0) continue;
                    for (int comp = 0; comp < 2; comp++) {
                        double& v = fed[2 * e + comp][f];
                        v = side < 0 ? std::sqrt(2.0) * v : 0.0;
                    }
                }
            }
        }
    }
    if (width != 0) {
        for (auto& a : fed)
            for (int d = 0; d < dim; d++) filter_pass(g, a, d, width);
        for (auto& a : fcc)
            for (int d = 0; d < dim; d++) filter_pass(g, a, d, width);
    }
    const double dxinv = 1.0 / g.dx;
    auto E = [&](int e, int comp, int i, int j, int k) { return fed[2 * e + comp][edge_id(g, e, i, j, k)]; };
    forall(g, [&](int i, int j, int k) {
        long f = g.id(i, j, k);
        double dv[3];
        if (dim == 2) {
            // stoch_m_force_2d (stochastic_m_fluxdiv.f90:453-506)
            dv[0] = (fcc[0][f] - fcc[0][g.id(i - 1, j, k)]) * dxinv + (E(0, 0, i, j + 1, k) - E(0, 0, i, j, k)) * dxinv;
            dv[1] = (E(0, 1, i + 1, j, k) - E(0, 1, i, j, k)) * dxinv + (fcc[1][f] - fcc[1][g.id(i, j - 1, k)]) * dxinv;
        } else {
            // stoch_m_force_3d (stochastic_m_fluxdiv.f90:508-600); edge
            // arrays fed[2e+comp] for e = xy, xz, yz
            dv[0] = (fcc[0][f] - fcc[0][g.id(i - 1, j, k)]) * dxinv + (E(0, 0, i, j + 1, k) - E(0, 0, i, j, k)) * dxinv
                  + (E(1, 0, i, j, k + 1) - E(1, 0, i, j, k)) * dxinv;
            dv[1] = (E(0, 1, i + 1, j, k) - E(0, 1, i, j, k)) * dxinv + (fcc[1][f] - fcc[1][g.id(i, j - 1, k)]) * dxinv
                  + (E(2, 0, i, j, k + 1) - E(2, 0, i, j, k)) * dxinv;
            dv[2] = (E(1, 1, i + 1, j, k) - E(1, 1, i, j, k)) * dxinv + (E(2, 1, i, j + 1, k) - E(2, 1, i, j, k)) * dxinv
                  + (fcc[2][f] - fcc[2][g.id(i, j, k - 1)]) * dxinv;
        }
        const int q[3] = {i, j, k};
        for (int c = 0; c < dim; c++) {
            // multifab_physbc_domainvel: the normal component on a wall face is zero
            if (g.wall(c) && q[c] == 0) force[c][f] = 0.0;
            else force[c][f] = increment ? force[c][f] + dv[c] : dv[c];
        }
    });
    return 0;
}

void avg_face(const Geo& g, const double* cc, double* const fc[]) {
    for (int d = 0; d < g.dim; d++) {
        int e[3] = {0, 0, 0};
        e[d] = 1;
        forall(g, [&](int i, int j, int k) {
            long f = g.id(i, j, k);
            fc[d][f] = 0.5 * (cc[f] + cc[g.id(i - e[0], j - e[1], k - e[2])]);
        });
    }
}

void avg_edge(const Geo& g, const double* cc, double* const ed[]) {
    if (g.dim == 2) {
        forall(g, [&](int i, int j, int k) {
            ed[0][g.id(i, j, k)] = 0.25 * (cc[g.id(i, j, k)] + cc[g.id(i - 1, j, k)] + cc[g.id(i, j - 1, k)] +
                                           cc[g.id(i - 1, j - 1, k)]);
        });
        return;
    }
    forall(g, [&](int i, int j, int k) {
        long f = g.id(i, j, k);
        ed[0][f] = 0.25 * (cc[f] + cc[g.id(i - 1, j, k)] + cc[g.id(i, j - 1, k)] + cc[g.id(i - 1, j - 1, k)]);
        ed[1][f] = 0.25 * (cc[f] + cc[g.id(i - 1, j, k)] + cc[g.id(i, j, k - 1)] + cc[g.id(i - 1, j, k - 1)]);
        ed[2][f] = 0.25 * (cc[f] + cc[g.id(i, j - 1, k)] + cc[g.id(i, j, k - 1)] + cc[g.id(i, j - 1, k - 1)]);
    });
}

// mk_advective_m_fluxdiv, centred (mk_advective_m_fluxdiv.f90:184-346):
// m_update (+)= -div(m u) with face-to-edge averages
void adv_m(const Geo& g, const double* const u[], const double* const m[], double* const upd[], bool increment) {
    const int dim = g.dim;
    const double dxinv = 1.0 / g.dx;
    for (int c = 0; c < dim; c++) {
        int ec[3] = {0, 0, 0};
        ec[c] = 1;
        forall(g, [&](int i, int j, int k) {
            long f = g.id(i, j, k);
            double s = 0.0;
            for (int d = 0; d < dim; d++) {
                int ed[3] = {0, 0, 0};
                ed[d] = 1;
                // flux of m_c in direction d at position q:
                // 0.25*(m_c(q-e_d)+m_c(q))*(u_d(q-e_c)+u_d(q))
                auto flux = [&](int qi, int qj, int qk) {
                    long q = g.id(qi, qj, qk);
                    return 0.25 * (m[c][g.id(qi - ed[0], qj - ed[1], qk - ed[2])] + m[c][q]) *
                           (u[d][g.id(qi - ec[0], qj - ec[1], qk - ec[2])] + u[d][q]);
                };
                s += (flux(i + ed[0], j + ed[1], k + ed[2]) - flux(i, j, k)) * dxinv;
            }
            upd[c][f] = increment ? upd[c][f] - s : -s;
            // the advective update on a wall face is zero (multifab_physbc_domainvel,
            // mk_advective_m_fluxdiv.f90:80-85); the stencil above reads past a
            // wall only in fluxes that carry the wall's zero normal velocity
            if (wall_face(g, c, i, j, k)) upd[c][f] = 0.0;
        });
    }
}

// mk_advective_s_fluxdiv, centred (mk_advective_s_fluxdiv.f90:138-220):
// s_update (+)= -div(s_fc u)
void adv_s(const Geo& g, const double* const u[], const double* const s_fc[], double* upd, bool increment) {
    const double dxinv = 1.0 / g.dx;
    forall(g, [&](int i, int j, int k) {
        long f = g.id(i, j, k);
        double s = 0.0;
        for (int d = 0; d < g.dim; d++) {
            int e[3] = {0, 0, 0};
            e[d] = 1;
            long fp = g.id(i + e[0], j + e[1], k + e[2]);
            s += (u[d][fp] * s_fc[d][fp] - u[d][f] * s_fc[d][f]) * dxinv;
        }
        upd[f] = increment ? upd[f] - s : -s;
    });
}


// ---------------------------------------------------------------------
// multispecies mass fluxes (src_multiSpec of LowMachFHD), ideal mixture,
// isothermal, no barodiffusion, periodic
// ---------------------------------------------------------------------
struct Mix {
    int ns;
    double molmass[FHD_MAX_SPECIES];
    double D[FHD_MAX_SPECIES][FHD_MAX_SPECIES];  // D_bar, zero diagonal
    double rhobar[FHD_MAX_SPECIES];
    double var_mass;
    int chi_it;
    double frac_tol;
    int correct;
    int avg_type;
};

Mix make_mix(const fhd_mixture_params* mp) {
    Mix m;
    m.ns = mp->nspecies;
    for (int i = 0; i < m.ns; i++) {
        m.molmass[i] = mp->molmass[i];
        m.rhobar[i] = mp->rhobar[i];
    }
    // compute_D_bar_local (compute_mixture_properties.f90:217-273): the
    // off-diagonal entries in the order (2,1),(3,1),(3,2),(4,1),...
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
    return m;
}

// compute_molconc_molmtot_local (mass_flux_utilities.f90:159-186)
void molconc(int ns, const double* molmass, const double* rho, double rhotot, double* x, double* mtot) {
    double W[FHD_MAX_SPECIES];
    double s = 0.0;
    for (int n = 0; n < ns; n++) {
        W[n] = rho[n] / rhotot;
        s = s + W[n] / molmass[n];
    }
    *mtot = 1.0 / s;
    for (int n = 0; n < ns; n++) x[n] = *mtot * W[n] / molmass[n];
}

// Dbar2chi_iterative (matrix_utilities.f90:19-158)
void dbar2chi(int ns, int iters, const double D[][FHD_MAX_SPECIES], const double* Xk, const double* molmass,
              double chi[][FHD_MAX_SPECIES]) {
    double mw = 0.0, Y[FHD_MAX_SPECIES], Di[FHD_MAX_SPECIES], M[FHD_MAX_SPECIES], Minv[FHD_MAX_SPECIES];
    double Pm[FHD_MAX_SPECIES][FHD_MAX_SPECIES], Dl[FHD_MAX_SPECIES][FHD_MAX_SPECIES];
    double Z[FHD_MAX_SPECIES][FHD_MAX_SPECIES], J[FHD_MAX_SPECIES][FHD_MAX_SPECIES];
    double PJ[FHD_MAX_SPECIES][FHD_MAX_SPECIES], m2[FHD_MAX_SPECIES][FHD_MAX_SPECIES];
    double m1[FHD_MAX_SPECIES][FHD_MAX_SPECIES];
    for (int i = 0; i < ns; i++) mw = mw + Xk[i] * molmass[i];
    for (int i = 0; i < ns; i++) Y[i] = molmass[i] / mw * Xk[i];
    for (int i = 0; i < ns; i++) {
        double t2 = 0.0;
        for (int j = 0; j < ns; j++)
            if (j != i) t2 = t2 + Xk[j] / D[i][j];
        Di[i] = (1.0 - Y[i]) / t2;
    }
    for (int i = 0; i < ns; i++) {
        M[i] = Xk[i] / Di[i];
        Minv[i] = Di[i] / Xk[i];
    }
    for (int i = 0; i < ns; i++)
        for (int j = 0; j < ns; j++) {
            Pm[i][j] = -Y[j];
            if (i == j) Pm[i][j] = Pm[i][j] + 1.0;
        }
    for (int i = 0; i < ns; i++)
        for (int j = 0; j < ns; j++) {
            if (i == j) {
                double t1 = 0.0;
                for (int k = 0; k < ns; k++)
                    if (k != i) t1 = t1 + Xk[i] * Xk[k] / D[i][k];
                Dl[i][i] = t1;
            } else {
                Dl[i][j] = -Xk[i] * Xk[j] / D[i][j];
            }
            Z[i][j] = -Dl[i][j];
        }
    for (int i = 0; i < ns; i++) Z[i][i] = Z[i][i] + M[i];
    for (int i = 0; i < ns; i++)
        for (int j = 0; j < ns; j++) J[i][j] = Minv[i] * Z[i][j];
    for (int i = 0; i < ns; i++)
        for (int j = 0; j < ns; j++) {
            double a = 0.0;
            for (int k = 0; k < ns; k++) a = a + Pm[i][k] * J[k][j];
            PJ[i][j] = a;
        }
    for (int i = 0; i < ns; i++)
        for (int j = 0; j < ns; j++) {
            double scr = 0.0;
            for (int k = 0; k < ns; k++) scr = scr + Pm[i][k] * Minv[k] * Pm[j][k];
            m2[i][j] = scr;
            chi[i][j] = scr;
        }
    for (int it = 0; it < iters; it++) {
        for (int i = 0; i < ns; i++)
            for (int j = 0; j < ns; j++) {
                double scr = 0.0;
                for (int k = 0; k < ns; k++) scr = scr + PJ[i][k] * chi[k][j];
                m1[i][j] = scr + m2[i][j];
            }
        for (int i = 0; i < ns; i++)
            for (int j = 0; j < ns; j++) chi[i][j] = m1[i][j];
    }
}

// compute_chi (mass_flux_utilities.f90:743-922) without LAPACK, for a
// system of n species with molar masses mm and Maxwell-Stefan matrix D:
// the closed form for two species (767-786), Dbar2chi_iterative otherwise
void chi_n(int n, int iters, const double* mm, const double D[][FHD_MAX_SPECIES], const double* rho, double rhotot,
           const double* x, double chi[][FHD_MAX_SPECIES]) {
    if (n == 2) {
        double W0 = rho[0] / rhotot, W1 = rho[1] / rhotot;
        double t = mm[0] * W1 + mm[1] * W0;
        t = D[0][1] * t * t / mm[0] / mm[1];
        chi[0][0] = t * W1 / W0;
        chi[0][1] = -t;
        chi[1][0] = -t;
        chi[1][1] = t * W0 / W1;
        return;
    }
    dbar2chi(n, iters, D, x, mm, chi);
}

void chi_of(const Mix& m, const double* rho, double rhotot, const double* x, double chi[][FHD_MAX_SPECIES]) {
    chi_n(m.ns, m.chi_it, m.molmass, m.D, rho, rhotot, x, chi);
}

// number of trace species (w < fraction_tolerance) and the map dest of
// mass_flux_utilities.f90:583-594 (0-based here: dest[i] = index of species
// i in the subsystem of non-trace species, or -1 for a trace species)
int n_trace(const Mix& m, const double* rho, double rhotot, int* dest = nullptr) {
    int nt = 0;
    for (int i = 0; i < m.ns; i++) {
        if (rho[i] / rhotot < m.frac_tol) {
            nt++;
            if (dest) dest[i] = -1;
        } else if (dest) {
            dest[i] = i - nt;
        }
    }
    return nt;
}

// the subsystem of non-trace species (compute_chi_sub and
// compute_sqrtLonsager_sub, mass_flux_utilities.f90:654-688 and 1440-1482):
// densities, molar masses and D_bar restricted through dest, the subsystem
// total density, molar concentrations and chi
struct SubMix {
    int n;
    double rho[FHD_MAX_SPECIES], mm[FHD_MAX_SPECIES], D[FHD_MAX_SPECIES][FHD_MAX_SPECIES];
    double rt, x[FHD_MAX_SPECIES], mt, chi[FHD_MAX_SPECIES][FHD_MAX_SPECIES];
};

void sub_mix(const Mix& m, const double* rho, const int* dest, int nsub, SubMix& S) {
    S.n = nsub;
    for (int r = 0; r < m.ns; r++)
        if (dest[r] >= 0) {
            S.mm[dest[r]] = m.molmass[r];
            S.rho[dest[r]] = rho[r];
        }
    S.rt = 0.0;
    for (int r = 0; r < nsub; r++) S.rt = S.rt + S.rho[r];
    for (int r = 0; r < m.ns; r++) {
        if (dest[r] < 0) continue;
        for (int c = 0; c < m.ns; c++)
            if (dest[c] >= 0) S.D[dest[r]][dest[c]] = m.D[r][c];
    }
    molconc(nsub, S.mm, S.rho, S.rt, S.x, &S.mt);
    chi_n(nsub, m.chi_it, S.mm, S.D, S.rho, S.rt, S.x, S.chi);
}

// compute_rhoWchi_local (mass_flux_utilities.f90:529-741): rho W chi of
// the full system, of the non-trace subsystem expanded with the effective
// diffusion coefficients of the trace species (compute_chi_sub, 654-739), or
// zero when every species but one is trace
void rhowchi_local(const Mix& m, const double* rho, double out[][FHD_MAX_SPECIES]) {
    const int ns = m.ns;
    double rt = 0.0;
    for (int i = 0; i < ns; i++) rt = rt + rho[i];
    int dest[FHD_MAX_SPECIES];
    const int nt = n_trace(m, rho, rt, dest);
    if (nt == ns - 1) {
        for (int i = 0; i < ns; i++)
            for (int j = 0; j < ns; j++) out[i][j] = 0.0;
        return;
    }
    if (nt == 0) {
        double x[FHD_MAX_SPECIES], mt, chi[FHD_MAX_SPECIES][FHD_MAX_SPECIES];
        molconc(ns, m.molmass, rho, rt, x, &mt);
        chi_of(m, rho, rt, x, chi);
        for (int i = 0; i < ns; i++)
            for (int j = 0; j < ns; j++) out[i][j] = rho[i] * chi[i][j];
        return;
    }
    SubMix S;
    sub_mix(m, rho, dest, ns - nt, S);
    for (int col = 0; col < ns; col++) {
        if (dest[col] < 0) {
            // a trace species' column: its effective diffusion coefficient
            double deff = 0.0;
            for (int k = 0; k < ns; k++)
                if (dest[k] >= 0) deff = deff + S.x[dest[k]] / m.D[k][col];
            deff = 1.0 / deff;
            for (int row = 0; row < ns; row++) {
                if (row == col) {
                    out[row][col] = S.rt * deff * m.molmass[row] / S.mt;
                } else if (dest[row] < 0) {
                    out[row][col] = 0.0;
                } else {
                    double tmp = 0.0;
                    for (int k = 0; k < ns; k++)
                        if (dest[k] >= 0) tmp = tmp + S.chi[dest[row]][dest[k]] * S.x[dest[k]] / m.D[k][col];
                    out[row][col] = deff * S.rho[dest[row]] * (tmp - m.molmass[col] / S.mt);
                }
            }
        } else {
            for (int row = 0; row < ns; row++)
                out[row][col] = (dest[row] < 0) ? 0.0 : S.rho[dest[row]] * S.chi[dest[row]][dest[col]];
        }
    }
}

// choldc (matrix_utilities.f90:162-241): lower Cholesky factor in place,
// zero rows after a non-positive pivot
void choldc(int np, double a[][FHD_MAX_SPECIES]) {
    double p[FHD_MAX_SPECIES];
    for (int i = 0; i < np; i++) {
        int ising = 0;
        for (int j = i; j < np; j++) {
            double s = a[i][j];
            for (int k = i - 1; k >= 0; k--) s = s - a[i][k] * a[j][k];
            if (i == j) {
                if (s <= 0.0) {
                    p[i] = 0.0;
                    ising = 1;
                } else {
                    p[i] = std::sqrt(s);
                }
            } else {
                a[j][i] = (ising == 0) ? s / p[i] : 0.0;
            }
        }
    }
    for (int i = 0; i < np; i++) {
        for (int j = i + 1; j < np; j++) a[i][j] = 0.0;
        a[i][i] = p[i];
    }
}

// compute_nonnegative_rho_av (mass_flux_utilities.f90:1231-1328)
void rho_av(const Mix& m, const double* r1, const double* r2, double dv, double* out) {
    for (int c = 0; c < m.ns; c++) {
        const double v1 = r1[c] / m.molmass[c], v2 = r2[c] / m.molmass[c];
        double o;
        switch (m.avg_type) {
            case 2:
                o = m.molmass[c] * std::sqrt(std::max(v1, 0.0) * std::max(v2, 0.0));
                break;
            case 3:
                o = (v1 <= 10.0 * 2.2250738585072014e-308 || v2 <= 10.0 * 2.2250738585072014e-308)
                        ? 0.0 : m.molmass[c] * 2.0 / (1.0 / v1 + 1.0 / v2);
                break;
            case 10:
                o = (v1 <= 0.0 || v2 <= 0.0) ? 0.0 : m.molmass[c] * (v1 + v2) / 2.0;
                break;
            default: {  // 1: arithmetic with a C0-smoothed Heaviside
                if (v1 <= 0.0 || v2 <= 0.0) {
                    o = 0.0;
                } else {
                    const double t1 = std::min(dv * v1, 1.0), t2 = std::min(dv * v2, 1.0);
                    o = m.molmass[c] * (v1 + v2) / 2.0 * t1 * t2;
                }
            }
        }
        out[c] = o;
    }
}

// compute_sqrtLonsager_local (mass_flux_utilities.f90:1331-1522), k_B: the
// Cholesky factor of L = mtot rhotot W chi W / k_B of the full system, of the
// non-trace subsystem expanded with zeros (compute_sqrtLonsager_sub,
// 1425-1502), or zero when every species but one is trace
void sqrtL_local(const Mix& m, const double* rho, double kB, double out[][FHD_MAX_SPECIES]) {
    const int ns = m.ns;
    double rt = 0.0;
    for (int i = 0; i < ns; i++) rt = rt + rho[i];
    int dest[FHD_MAX_SPECIES];
    const int nt = n_trace(m, rho, rt, dest);
    if (nt == ns - 1) {
        for (int i = 0; i < ns; i++)
            for (int j = 0; j < ns; j++) out[i][j] = 0.0;
        return;
    }
    if (nt == 0) {
        double W[FHD_MAX_SPECIES], x[FHD_MAX_SPECIES], mt, chi[FHD_MAX_SPECIES][FHD_MAX_SPECIES];
        for (int i = 0; i < ns; i++) W[i] = rho[i] / rt;
        molconc(ns, m.molmass, rho, rt, x, &mt);
        chi_of(m, rho, rt, x, chi);
        for (int c = 0; c < ns; c++)
            for (int r = 0; r < ns; r++) out[r][c] = mt * rt * W[r] * chi[r][c] * W[c] / kB;
        choldc(ns, out);
        return;
    }
    SubMix S;
    const int nsub = ns - nt;
    sub_mix(m, rho, dest, nsub, S);
    double Ws[FHD_MAX_SPECIES], Ls[FHD_MAX_SPECIES][FHD_MAX_SPECIES];
    for (int r = 0; r < nsub; r++) Ws[r] = S.rho[r] / S.rt;
    for (int c = 0; c < nsub; c++)
        for (int r = 0; r < nsub; r++) Ls[r][c] = S.mt * S.rt * Ws[r] * S.chi[r][c] * Ws[c] / kB;
    choldc(nsub, Ls);
    for (int r = 0; r < ns; r++)
        for (int c = 0; c < ns; c++) out[r][c] = (dest[r] >= 0 && dest[c] >= 0) ? Ls[dest[r]][dest[c]] : 0.0;
}

// compute_mass_fluxdiv (compute_mass_fluxdiv.f90:29-183) for an ideal
// isothermal mixture: flux = rhoWchi_face * grad(x) + variance *
// sqrtL_face * sum_r w_r W_r, each corrected to zero species sum
// (correction_flux.f90:17-226), and its divergence.  Returns the faces'
// total flux in flux[d*ns+i] (nullable) and div into fluxdiv[i].
int mass_fluxdiv_impl(const Geo& g, const Mix& m, const fhd_stoch_params* sp, const double* const rho[], double dt,
                      const double* weights, int n_rngs, const double* const W_fc[], double* const fluxdiv[],
                      double* const flux_out[]) {
    const int dim = g.dim, ns = m.ns;
    const long nc = g.nc;
    std::vector<Vec> rwc(ns * ns, Vec(nc)), xcc(ns, Vec(nc));
#pragma omp parallel for
    for (long f = 0; f < nc; f++) {
        double r[FHD_MAX_SPECIES], a[FHD_MAX_SPECIES][FHD_MAX_SPECIES], x[FHD_MAX_SPECIES], mt;
        double rt = 0.0;
        for (int i = 0; i < ns; i++) {
            r[i] = rho[i][f];
            rt = rt + r[i];
        }
        rhowchi_local(m, r, a);
        molconc(ns, m.molmass, r, rt, x, &mt);
        for (int i = 0; i < ns; i++) {
            xcc[i][f] = x[i];
            for (int j = 0; j < ns; j++) rwc[i * ns + j][f] = a[i][j];
        }
    }
    const double variance = std::sqrt(2.0 * sp->k_B * m.var_mass / (sp->dV * dt));
    const double dxinv = 1.0 / g.dx;
    std::vector<Vec> flux(dim * ns, Vec(nc));
    for (int d = 0; d < dim; d++) {
        int e[3] = {0, 0, 0};
        e[d] = 1;
        forall(g, [&](int i, int j, int k) {
            const long f = g.id(i, j, k), fm = g.id(i - e[0], j - e[1], k - e[2]);
            const int q[3] = {i, j, k};
            if (g.wall(d) && q[d] == 0) {
                // a wall face: the concentrations' ghost cells are first-order
                // extrapolated (scalar_bc, inhomogeneous_bc_val.f90:21-54), so
                // grad x and the diffusive flux vanish, and stoch_mass_bc
                // zeroes the random field there
                for (int s = 0; s < ns; s++) flux[d * ns + s][f] = 0.0;
                return;
            }
            // diffusive: rhoWchi face average times grad(molar concentration)
            double gx[FHD_MAX_SPECIES], fd[FHD_MAX_SPECIES], fs[FHD_MAX_SPECIES];
            for (int s = 0; s < ns; s++) gx[s] = (xcc[s][f] - xcc[s][fm]) * dxinv;
            for (int r = 0; r < ns; r++) {
                double acc = 0.0;
                for (int c = 0; c < ns; c++) acc = acc + 0.5 * (rwc[r * ns + c][fm] + rwc[r * ns + c][f]) * gx[c];
                fd[r] = acc;
            }
            if (m.correct && ns > 1) {
                double sum = 0.0;
                for (int s = 0; s < ns - 1; s++) sum = sum + fd[s];
                fd[ns - 1] = -sum;
            }
            // stochastic: sqrtL(rho_av) times the weighted random vector
            for (int s = 0; s < ns; s++) fs[s] = 0.0;
            if (m.var_mass != 0.0) {
                double r1[FHD_MAX_SPECIES], r2[FHD_MAX_SPECIES], ra[FHD_MAX_SPECIES];
                double L[FHD_MAX_SPECIES][FHD_MAX_SPECIES], w[FHD_MAX_SPECIES];
                for (int s = 0; s < ns; s++) {
                    r1[s] = rho[s][fm];
                    r2[s] = rho[s][f];
                }
                rho_av(m, r1, r2, sp->dV, ra);
                sqrtL_local(m, ra, sp->k_B, L);
                for (int s = 0; s < ns; s++) {
                    double acc = 0.0;
                    for (int rr = 0; rr < n_rngs; rr++) acc = acc + weights[rr] * W_fc[(rr * dim + d) * ns + s][f];
                    w[s] = acc;
                }
                for (int r = 0; r < ns; r++) {
                    double acc = 0.0;
                    for (int c = 0; c < ns; c++) acc = acc + L[r][c] * w[c];
                    fs[r] = acc * variance;
                }
                if (m.correct && ns > 1) {
                    double sum = 0.0;
                    for (int s = 0; s < ns - 1; s++) sum = sum + fs[s];
                    fs[ns - 1] = -sum;
                }
            }
            for (int s = 0; s < ns; s++) flux[d * ns + s][f] = fd[s] + fs[s];
        });
    }
    forall(g, [&](int i, int j, int k) {
        const long f = g.id(i, j, k);
        for (int s = 0; s < ns; s++) {
            double v = (flux[0 * ns + s][g.id(i + 1, j, k)] - flux[0 * ns + s][f]) * dxinv +
                       (flux[1 * ns + s][g.id(i, j + 1, k)] - flux[1 * ns + s][f]) * dxinv;
            if (dim == 3) v += (flux[2 * ns + s][g.id(i, j, k + 1)] - flux[2 * ns + s][f]) * dxinv;
            fluxdiv[s][f] = v;
        }
    });
    if (flux_out)
        for (int q = 0; q < dim * ns; q++) std::copy(flux[q].begin(), flux[q].end(), flux_out[q]);
    return 0;
}

}  // namespace

// =====================================================================
// extern "C" API
// =====================================================================
extern "C" {

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// probin_common max_grid_size for the staggered multigrid's box layout
// (module state, as in the reference); 0 or >= n_cells: one box
void or_set_max_grid_size(const int mgs[3]) {
    for (int d = 0; d < 3; d++) g_max_grid_size[d] = mgs ? mgs[d] : 0;
}

int or_set_walls(const int bc_lo[3], const int bc_hi[3]) {
    auto code = [](int b, int& w) {
        if (b == -1) w = 0;
        else if (b == 100) w = -1;
        else if (b == 200) w = 1;
        else return false;
        return true;
    };
    int lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
        if (!code(bc_lo[d], lo[d]) || !code(bc_hi[d], hi[d])) return FHD_ERR_UNSUPPORTED;
        if ((lo[d] == 0) != (hi[d] == 0)) return FHD_ERR_BAD_ARG;  // periodic on both sides or neither
    }
    for (int d = 0; d < 3; d++) {
        g_wl[d] = lo[d];
        g_wh[d] = hi[d];
    }
    return 0;
}

void or_set_wall_speed(const double lo[6], const double hi[6]) {
    for (int q = 0; q < 6; q++) {
        g_ws[0][q] = lo ? lo[q] : 0.0;
        g_ws[1][q] = hi ? hi[q] : 0.0;
    }
}

int or_compute_nlevs_mg(int dim, const int n[3], int minwidth) {
    Geo g(dim, n, 1.0);
    return nlevs_mg(g, minwidth);
}

void or_stag_applyop(int dim, const int n[3], double dx, int visc_type, const double* const phi[],
                     double* const Lphi[], const double* const alpha_fc[], const double* beta,
                     const double* const beta_ed[], const double* gamma, int color) {
    Geo g(dim, n, dx);
    SLevel L;
    L.g = g;
    for (int c = 0; c < dim; c++) {
        L.alpha[c].assign(alpha_fc[c], alpha_fc[c] + g.nc);
        L.phi[c].assign(phi[c], phi[c] + g.nc);
        L.Lphi[c].assign(Lphi[c], Lphi[c] + g.nc);
    }
    L.beta.assign(beta, beta + g.nc);
    L.gamma.assign(gamma, gamma + g.nc);
    for (int e = 0; e < n_edge(dim); e++) L.bed[e].assign(beta_ed[e], beta_ed[e] + g.nc);
    s_applyop(L, visc_type, color);
    for (int c = 0; c < dim; c++) std::copy(L.Lphi[c].begin(), L.Lphi[c].end(), Lphi[c]);
}

int or_stag_mg_solver(int dim, const int n[3], double dx, int visc_type, const fhd_gmres_params* p,
                      const double* const alpha_fc[], const double* beta, const double* const beta_ed[],
                      const double* gamma, double theta_alpha, double* const phi[], const double* const rhs[]) {
    Geo g(dim, n, dx);
    return stag_mg(g, visc_type, p, alpha_fc, beta, beta_ed, gamma, theta_alpha, phi, rhs);
}

int or_stag_mg_history(int dim, const int n[3], double dx, int visc_type, const fhd_gmres_params* p,
                       const double* const alpha_fc[], const double* beta, const double* const beta_ed[],
                       const double* gamma, double theta_alpha, double* const phi[], const double* const rhs[],
                       double* hist) {
    Geo g(dim, n, dx);
    return stag_mg(g, visc_type, p, alpha_fc, beta, beta_ed, gamma, theta_alpha, phi, rhs, hist);
}

int or_macproject(int dim, const int n[3], double dx, const fhd_gmres_params* p, double* phi,
                  const double* const alphainv_fc[], const double* rhs) {
    Geo g(dim, n, dx);
    return macproject_impl(g, p, phi, alphainv_fc, rhs);
}

int or_macproject_history(int dim, const int n[3], double dx, const fhd_gmres_params* p, double* phi,
                          const double* const alphainv_fc[], const double* rhs, double* hist) {
    Geo g(dim, n, dx);
    return macproject_impl(g, p, phi, alphainv_fc, rhs, hist);
}

int or_apply_matrix(int dim, const int n[3], double dx, int visc_type, double* const b_u[], double* b_p,
                    const double* const x_u[], const double* x_p, const double* const alpha_fc[],
                    const double* beta, const double* const beta_ed[], const double* gamma, double theta_alpha) {
    Geo g(dim, n, dx);
    return apply_matrix_impl(g, visc_type, b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha, 2);
}

int or_apply_matrix_order(int dim, const int n[3], double dx, int visc_type, double* const b_u[], double* b_p,
                          const double* const x_u[], const double* x_p, const double* const alpha_fc[],
                          const double* beta, const double* const beta_ed[], const double* gamma,
                          double theta_alpha, int order) {
    Geo g(dim, n, dx);
    return apply_matrix_impl(g, visc_type, b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha,
                             order);
}

int or_apply_precon(int dim, const int n[3], double dx, int visc_type, const fhd_gmres_params* p,
                    const double* const b_u[], const double* b_p, double* const x_u[], double* x_p,
                    const double* const alpha_fc[], const double* beta, const double* const beta_ed[],
                    const double* gamma, double theta_alpha) {
    Geo g(dim, n, dx);
    return apply_precon_impl(g, visc_type, p, b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha);
}

int or_gmres(int dim, const int n[3], double dx, int visc_type, const fhd_gmres_params* p,
             const double* const b_u[], const double* b_p, double* const x_u[], double* x_p,
             const double* const alpha_fc[], const double* beta, const double* const beta_ed[],
             const double* gamma, double theta_alpha, double* norm_pre_rhs, fhd_solve_stats* stats) {
    Geo g(dim, n, dx);
    return gmres_impl(g, visc_type, p, b_u, b_p, x_u, x_p, alpha_fc, beta, beta_ed, gamma, theta_alpha,
                      norm_pre_rhs, stats);
}

int or_stochastic_m_fluxdiv(int dim, const int n[3], double dx, const fhd_stoch_params* sp, double* const force[],
                            int increment, const double* eta, const double* const eta_ed[],
                            const double* temperature, const double* const temperature_ed[], double dt,
                            const double* weights, int n_rngs, const double* const W_cc[],
                            const double* const W_ed[]) {
    Geo g(dim, n, dx);
    return stoch_m_impl(g, sp, force, increment, eta, eta_ed, temperature, temperature_ed, dt, weights, n_rngs,
                        W_cc, W_ed);
}

void or_average_cc_to_edge(int dim, const int n[3], const double* cc, double* const ed[]) {
    Geo g(dim, n, 1.0);
    avg_edge(g, cc, ed);
}

void or_average_cc_to_face(int dim, const int n[3], const double* cc, double* const fc[]) {
    Geo g(dim, n, 1.0);
    avg_face(g, cc, fc);
}

}  // extern "C" (reopened below)

namespace {
// advance_timestep_inertial (advance_timestep_inertial.f90:45-923),
// periodic, centred advection, no gravity; ns species (ns = 1 with no
// mixture: a single fluid without mass fluxes).  fluxdiv (ns arrays) holds
// F^n = div(diffusive + stochastic mass flux) on entry and F^{n+1} on exit;
// W_mass[0 .. dim*ns) are the mass-flux random fields of the previous
// corrector (used again by this predictor), W_mass[dim*ns .. 2*dim*ns) the
// new fields drawn for this corrector.
int step_impl(const Geo& g, int visc_type, const fhd_gmres_params* p_in, const fhd_stoch_params* sp, const Mix* mix,
              double dt, double* const umac[], double* const rho[], double* pi, double* const fluxdiv[],
              const double* eta, const double* const eta_ed[], const double* kappa, const double* temperature,
              const double* const temperature_ed[], const double* const W_cc[], const double* const W_ed[],
              const double* const W_mass[], fhd_solve_stats* stats2) {
    const int dim = g.dim;
    const long nc = g.nc;
    const int nE = n_edge(dim);
    const int ns = mix ? mix->ns : 1;
    if (int rc = wall_speed_check(g)) return rc;
    fhd_gmres_params p = *p_in;
    const double theta = 1.0 / dt;
    auto fvec = [&](std::vector<Vec>& v) { v.assign(dim, Vec(nc, 0.0)); };
    auto ptrs = [&](std::vector<Vec>& v, double** out) { for (int c = 0; c < dim; c++) out[c] = v[c].data(); };
    std::vector<Vec> rho_fc_old, rho_fc_new, mold, mtemp, adv, diff, rhs_v, dumac, stoch, gradpi;
    fvec(rho_fc_old); fvec(rho_fc_new); fvec(mold); fvec(mtemp); fvec(adv); fvec(diff); fvec(rhs_v);
    fvec(dumac); fvec(stoch); fvec(gradpi);
    double *rfo[3], *rfn[3], *mo[3], *mt[3], *ad[3], *df[3], *rv[3], *du[3], *sto[3], *gpi[3];
    ptrs(rho_fc_old, rfo); ptrs(rho_fc_new, rfn); ptrs(mold, mo); ptrs(mtemp, mt); ptrs(adv, ad); ptrs(diff, df);
    ptrs(rhs_v, rv); ptrs(dumac, du); ptrs(stoch, sto); ptrs(gradpi, gpi);
    std::vector<Vec> rho_old(ns), rho_update(ns, Vec(nc)), sfc(ns * dim, Vec(nc));
    for (int s = 0; s < ns; s++) rho_old[s].assign(rho[s], rho[s] + nc);
    Vec rhotot(nc), rhs_p(nc), dpi(nc), eta_h(nc), kappa_h(nc);
    std::vector<Vec> eta_ed_h(nE, Vec(nc));
    for (long f = 0; f < nc; f++) { eta_h[f] = eta[f] * 0.5; kappa_h[f] = kappa[f] * 0.5; }
    for (int e = 0; e < nE; e++)
        for (long f = 0; f < nc; f++) eta_ed_h[e][f] = eta_ed[e][f] * 0.5;
    const double* eh_ed[3] = {eta_ed_h[0].data(), nE == 3 ? eta_ed_h[1].data() : nullptr,
                              nE == 3 ? eta_ed_h[2].data() : nullptr};
    const double* um[3] = {umac[0], umac[1], dim == 3 ? umac[2] : nullptr};
    const double w1[1] = {1.0};
    auto diff_m = [&](double* const out[], const double* const u[]) {
        SLevel L;
        L.g = g;
        for (int c = 0; c < dim; c++) { L.alpha[c].assign(nc, 0.0); L.phi[c].assign(u[c], u[c] + nc); L.Lphi[c].assign(nc, 0.0); }
        L.beta.assign(eta, eta + nc);
        L.gamma.assign(kappa, kappa + nc);
        for (int e = 0; e < nE; e++) L.bed[e].assign(eta_ed[e], eta_ed[e] + nc);
        s_applyop(L, visc_type, 0);
        for (int c = 0; c < dim; c++)
            for (long f = 0; f < nc; f++) out[c][f] = L.Lphi[c][f] * -1.0;
        wall_speed_term(g, eta[0], out);
    };
    auto sum_species = [&](double* const* r, double* out) {
        for (long f = 0; f < nc; f++) {
            double v = 0.0;
            for (int s = 0; s < ns; s++) v = v + r[s][f];
            out[f] = v;
        }
    };
    auto species_fc = [&](double* const* r) {
        for (int s = 0; s < ns; s++) {
            double* o[3] = {sfc[s * dim].data(), sfc[s * dim + 1].data(), dim == 3 ? sfc[s * dim + 2].data() : nullptr};
            avg_face(g, r[s], o);
        }
    };
    // -S = sum_i -F_i/rhobar_i (advance_timestep_inertial.f90:420-430)
    auto rhs_p_from_fluxes = [&]() {
        std::fill(rhs_p.begin(), rhs_p.end(), 0.0);
        if (!mix) return;
        for (int s = 0; s < ns; s++)
            for (long f = 0; f < nc; f++) rhs_p[f] = rhs_p[f] + (-1.0 / mix->rhobar[s]) * fluxdiv[s][f];
    };
    auto mass_fluxes = [&](const double* const* Wm) -> int {
        if (!mix) return 0;
        const double* cr[FHD_MAX_SPECIES];
        for (int s = 0; s < ns; s++) cr[s] = rho[s];
        return mass_fluxdiv_impl(g, *mix, sp, cr, dt, w1, 1, Wm, fluxdiv, nullptr);
    };
    int st = 0, rc;
    double norm_pre_rhs = 0.0;
    // Step 2: predictor Euler step for the densities
    double* ro[FHD_MAX_SPECIES];
    for (int s = 0; s < ns; s++) ro[s] = rho_old[s].data();
    sum_species(ro, rhotot.data());
    avg_face(g, rhotot.data(), rfo);
    species_fc(ro);
    for (int s = 0; s < ns; s++) {
        if (mix) std::copy(fluxdiv[s], fluxdiv[s] + nc, rho_update[s].begin());
        const double* sp3[3] = {sfc[s * dim].data(), sfc[s * dim + 1].data(), dim == 3 ? sfc[s * dim + 2].data() : nullptr};
        adv_s(g, um, sp3, rho_update[s].data(), mix != nullptr);
        for (long f = 0; f < nc; f++) rho[s][f] = rho_old[s][f] + dt * rho_update[s][f];
    }
    sum_species(rho, rhotot.data());
    avg_face(g, rhotot.data(), rfn);
    species_fc(rho);
    // Steps 3-4: predictor Crank-Nicolson
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) mold[c][f] = rho_fc_old[c][f] * umac[c][f];
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) rhs_v[c][f] = (1.0 / dt) * mold[c][f];
    c_grad(g, pi, gpi);
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) rhs_v[c][f] = rhs_v[c][f] - gradpi[c][f];
    {
        const double* mop[3] = {mo[0], mo[1], dim == 3 ? mo[2] : nullptr};
        adv_m(g, um, mop, ad, false);
    }
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) rhs_v[c][f] = rhs_v[c][f] + adv[c][f];
    diff_m(df, um);
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) rhs_v[c][f] = rhs_v[c][f] + 0.5 * diff[c][f];
    if (sp->variance_coef_mom != 0.0) {
        stoch_m_impl(g, sp, sto, 0, eta, eta_ed, temperature, temperature_ed, dt, w1, 1, W_cc, W_ed);
        for (int c = 0; c < dim; c++)
            for (long f = 0; f < nc; f++) rhs_v[c][f] = rhs_v[c][f] + stoch[c][f];
    }
    if ((rc = mass_fluxes(W_mass))) return rc;
    rhs_p_from_fluxes();
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) mtemp[c][f] = rho_fc_new[c][f] * umac[c][f];
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) rhs_v[c][f] = rhs_v[c][f] + (-1.0 / dt) * mtemp[c][f];
    diff_m(mt, um);
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) rhs_v[c][f] = rhs_v[c][f] + 0.5 * mtemp[c][f];
    for (int s = 0; s < ns; s++) {
        if (mix) std::copy(fluxdiv[s], fluxdiv[s] + nc, rho_update[s].begin());
        else std::fill(rho_update[s].begin(), rho_update[s].end(), 0.0);
    }
    c_div(g, um, rhs_p.data(), true);
    for (int c = 0; c < dim; c++) std::fill(dumac[c].begin(), dumac[c].end(), 0.0);
    std::fill(dpi.begin(), dpi.end(), 0.0);
    const double gmres_abs_tol_in = p.gmres_abs_tol;
    {
        const double* rvp[3] = {rv[0], rv[1], dim == 3 ? rv[2] : nullptr};
        const double* rfnp[3] = {rfn[0], rfn[1], dim == 3 ? rfn[2] : nullptr};
        int s1 = gmres_impl(g, visc_type, &p, rvp, rhs_p.data(), du, dpi.data(), rfnp, eta_h.data(), eh_ed,
                            kappa_h.data(), theta, &norm_pre_rhs, stats2 ? &stats2[0] : nullptr);
        if (s1 < 0) return s1;
        st = std::max(st, s1);
    }
    p.gmres_abs_tol = std::max(gmres_abs_tol_in, norm_pre_rhs * p.gmres_rel_tol);
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) umac[c][f] = umac[c][f] + dumac[c][f];
    for (long f = 0; f < nc; f++) pi[f] = pi[f] + dpi[f];
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) mtemp[c][f] = rho_fc_new[c][f] * umac[c][f];
    // Step 5: trapezoidal scalar corrector
    for (int s = 0; s < ns; s++) {
        const double* sp3[3] = {sfc[s * dim].data(), sfc[s * dim + 1].data(), dim == 3 ? sfc[s * dim + 2].data() : nullptr};
        adv_s(g, um, sp3, rho_update[s].data(), true);
        for (long f = 0; f < nc; f++) {
            double v = rho[s][f] + rho_old[s][f];
            v = v + dt * rho_update[s][f];
            rho[s][f] = v * 0.5;
        }
    }
    sum_species(rho, rhotot.data());
    avg_face(g, rhotot.data(), rfn);
    // Steps 6-7: corrector Crank-Nicolson
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) rhs_v[c][f] = (1.0 / dt) * mold[c][f];
    c_grad(g, pi, gpi);
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) rhs_v[c][f] = rhs_v[c][f] - gradpi[c][f];
    {
        const double* mtp[3] = {mt[0], mt[1], dim == 3 ? mt[2] : nullptr};
        adv_m(g, um, mtp, ad, true);
    }
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) rhs_v[c][f] = rhs_v[c][f] + 0.5 * adv[c][f];
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) rhs_v[c][f] = rhs_v[c][f] + 0.5 * diff[c][f];
    if (sp->variance_coef_mom != 0.0) {
        stoch_m_impl(g, sp, sto, 1, eta, eta_ed, temperature, temperature_ed, dt, w1, 1, W_cc, W_ed);
        for (int c = 0; c < dim; c++)
            for (long f = 0; f < nc; f++) rhs_v[c][f] = rhs_v[c][f] + 0.5 * stoch[c][f];
    }
    if ((rc = mass_fluxes(W_mass ? W_mass + dim * ns : nullptr))) return rc;
    rhs_p_from_fluxes();
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) mtemp[c][f] = rho_fc_new[c][f] * umac[c][f];
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) rhs_v[c][f] = rhs_v[c][f] + (-1.0 / dt) * mtemp[c][f];
    diff_m(df, um);
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) rhs_v[c][f] = rhs_v[c][f] + 0.5 * diff[c][f];
    c_div(g, um, rhs_p.data(), true);
    for (int c = 0; c < dim; c++) std::fill(dumac[c].begin(), dumac[c].end(), 0.0);
    std::fill(dpi.begin(), dpi.end(), 0.0);
    {
        const double* rvp[3] = {rv[0], rv[1], dim == 3 ? rv[2] : nullptr};
        const double* rfnp[3] = {rfn[0], rfn[1], dim == 3 ? rfn[2] : nullptr};
        int s2 = gmres_impl(g, visc_type, &p, rvp, rhs_p.data(), du, dpi.data(), rfnp, eta_h.data(), eh_ed,
                            kappa_h.data(), theta, nullptr, stats2 ? &stats2[1] : nullptr);
        if (s2 < 0) return s2;
        st = std::max(st, s2);
    }
    for (int c = 0; c < dim; c++)
        for (long f = 0; f < nc; f++) umac[c][f] = umac[c][f] + dumac[c][f];
    for (long f = 0; f < nc; f++) pi[f] = pi[f] + dpi[f];
    return st;
}

// advance_timestep_overdamped (advance_timestep_overdamped.f90:135-734),
// periodic, centred advection, no gravity, no reactions, barodiffusion off,
// midpoint_stoch_mass_flux_type = 1.  theta_alpha = 0 (line 135).  Two
// random stages per step (n_rngs = 2 for this algorithm, main_driver.f90:
// 534-536), drawn once at the predictor: W_cc[r*dim+c], W_ed[r*2*nE+...]
// and W_mass[(r*dim+d)*ns+i] for r = 0, 1.  The predictor uses the weights
// (1, 0) over dt/2 (lines 187-188, 228-229, 246-249), the corrector
// (1/sqrt2, 1/sqrt2) over dt (lines 466-469, 485-490).
int overdamped_impl(const Geo& g, int visc_type, const fhd_gmres_params* p_in, const fhd_stoch_params* sp,
                    const Mix* mix, double dt, double* const umac[], double* const rho[], double* pi,
                    const double* eta, const double* const eta_ed[], const double* kappa, const double* temperature,
                    const double* const temperature_ed[], const double* const W_cc[], const double* const W_ed[],
                    const double* const W_mass[], fhd_solve_stats* stats2) {
    const int dim = g.dim;
    const long nc = g.nc;
    const int nE = n_edge(dim);
    const int ns = mix ? mix->ns : 1;
    if (int rc = wall_speed_check(g)) return rc;
    fhd_gmres_params p = *p_in;
    auto fvec = [&](std::vector<Vec>& v) { v.assign(dim, Vec(nc, 0.0)); };
    auto ptrs = [&](std::vector<Vec>& v, double** out) { for (int c = 0; c < dim; c++) out[c] = v[c].data(); };
    std::vector<Vec> rhotot_fc, rhs_v, dumac, gradpi, diff;
    fvec(rhotot_fc); fvec(rhs_v); fvec(dumac); fvec(gradpi); fvec(diff);
    double *rtf[3], *rv[3], *du[3], *gpi[3], *df[3];
    ptrs(rhotot_fc, rtf); ptrs(rhs_v, rv); ptrs(dumac, du); ptrs(gradpi, gpi); ptrs(diff, df);
    std::vector<Vec> rho_old(ns), rho_update(ns, Vec(nc)), sfc(ns * dim, Vec(nc)), fdiv(ns, Vec(nc, 0.0));
    for (int s = 0; s < ns; s++) rho_old[s].assign(rho[s], rho[s] + nc);
    Vec rhotot(nc), rhs_p(nc), dpi(nc);
    const double* um[3] = {umac[0], umac[1], dim == 3 ? umac[2] : nullptr};
    // diffusive_m_fluxdiv with the full viscosity (stag_applyop with alpha = 0,
    // sign flipped): out = +L u
    auto diff_m = [&](double* const out[]) {
        SLevel L;
        L.g = g;
        for (int c = 0; c < dim; c++) { L.alpha[c].assign(nc, 0.0); L.phi[c].assign(um[c], um[c] + nc); L.Lphi[c].assign(nc, 0.0); }
        L.beta.assign(eta, eta + nc);
        L.gamma.assign(kappa, kappa + nc);
        for (int e = 0; e < nE; e++) L.bed[e].assign(eta_ed[e], eta_ed[e] + nc);
        s_applyop(L, visc_type, 0);
        for (int c = 0; c < dim; c++)
            for (long f = 0; f < nc; f++) out[c][f] = L.Lphi[c][f] * -1.0;
        wall_speed_term(g, eta[0], out);
    };
    auto sum_species = [&](double* const* r, double* out) {
        for (long f = 0; f < nc; f++) {
            double v = 0.0;
            for (int s = 0; s < ns; s++) v = v + r[s][f];
            out[f] = v;
        }
    };
    auto species_fc = [&](double* const* r) {
        for (int s = 0; s < ns; s++) {
            double* o[3] = {sfc[s * dim].data(), sfc[s * dim + 1].data(), dim == 3 ? sfc[s * dim + 2].data() : nullptr};
            avg_face(g, r[s], o);
        }
    };
    double* fd[FHD_MAX_SPECIES];
    for (int s = 0; s < ns; s++) fd[s] = fdiv[s].data();
    // one half of the step: mass fluxes at rho, rhs, GMRES, velocity and
    // density update rho = rho_old + h * (F + advection)
    auto stage = [&](const double* weights, double h, double* norm_pre_rhs, fhd_solve_stats* sst) -> int {
        // -grad pi (lines 207-212 / 437-442)
        c_grad(g, pi, gpi);
        for (int c = 0; c < dim; c++)
            for (long f = 0; f < nc; f++) rhs_v[c][f] = -1.0 * gradpi[c][f];
        // += div(Sigma) with the stage weights over h (lines 214-220 / 444-449)
        if (sp->variance_coef_mom != 0.0) {
            int rc = stoch_m_impl(g, sp, rv, 1, eta, eta_ed, temperature, temperature_ed, h, weights, 2, W_cc, W_ed);
            if (rc) return rc;
        }
        // mass fluxes at the current densities (lines 233-236 / 464-469)
        if (mix) {
            const double* cr[FHD_MAX_SPECIES];
            for (int s = 0; s < ns; s++) cr[s] = rho[s];
            int rc = mass_fluxdiv_impl(g, *mix, sp, cr, h, weights, 2, W_mass, fd, nullptr);
            if (rc) return rc;
        }
        // rhs_p = sum_i -F_i/rhobar_i (lines 284-297 / 530-543)
        std::fill(rhs_p.begin(), rhs_p.end(), 0.0);
        if (mix)
            for (int s = 0; s < ns; s++)
                for (long f = 0; f < nc; f++) rhs_p[f] = rhs_p[f] + (-1.0 / mix->rhobar[s]) * fdiv[s][f];
        for (int s = 0; s < ns; s++) {
            if (mix) std::copy(fdiv[s].begin(), fdiv[s].end(), rho_update[s].begin());
            else std::fill(rho_update[s].begin(), rho_update[s].end(), 0.0);
        }
        // += A_0 u^n, rhs_p += div u (lines 322-327 / 569-574)
        diff_m(df);
        for (int c = 0; c < dim; c++)
            for (long f = 0; f < nc; f++) rhs_v[c][f] = rhs_v[c][f] + diff[c][f];
        c_div(g, um, rhs_p.data(), true);
        for (int c = 0; c < dim; c++) std::fill(dumac[c].begin(), dumac[c].end(), 0.0);
        std::fill(dpi.begin(), dpi.end(), 0.0);
        {
            const double* rvp[3] = {rv[0], rv[1], dim == 3 ? rv[2] : nullptr};
            const double* rtp[3] = {rtf[0], rtf[1], dim == 3 ? rtf[2] : nullptr};
            int s1 = gmres_impl(g, visc_type, &p, rvp, rhs_p.data(), du, dpi.data(), rtp, eta, eta_ed, kappa, 0.0,
                                norm_pre_rhs, sst);
            if (s1 < 0) return s1;
            for (int c = 0; c < dim; c++)
                for (long f = 0; f < nc; f++) umac[c][f] = umac[c][f] + dumac[c][f];
            for (long f = 0; f < nc; f++) pi[f] = pi[f] + dpi[f];
            // rho_update += -div(rho_fc u); rho = rho_old + h rho_update
            // (lines 390-391, 401-403 / 644-645, 651-653)
            for (int s = 0; s < ns; s++) {
                const double* sp3[3] = {sfc[s * dim].data(), sfc[s * dim + 1].data(),
                                        dim == 3 ? sfc[s * dim + 2].data() : nullptr};
                adv_s(g, um, sp3, rho_update[s].data(), true);
                for (long f = 0; f < nc; f++) rho[s][f] = rho_old[s][f] + h * rho_update[s][f];
            }
            return s1;
        }
    };
    // faces of rho^n and rho_tot^n (lines 181-183)
    double* ro[FHD_MAX_SPECIES];
    for (int s = 0; s < ns; s++) ro[s] = rho_old[s].data();
    sum_species(ro, rhotot.data());
    avg_face(g, rhotot.data(), rtf);
    species_fc(ro);
    const double w_pred[2] = {1.0, 0.0};
    const double w_corr[2] = {1.0 / std::sqrt(2.0), 1.0 / std::sqrt(2.0)};
    double norm_pre_rhs = 0.0;
    const double gmres_abs_tol_in = p.gmres_abs_tol;
    int st = stage(w_pred, 0.5 * dt, &norm_pre_rhs, stats2 ? &stats2[0] : nullptr);
    if (st < 0) return st;
    // the corrector's GMRES stops at the predictor's preconditioned rhs
    // (line 338) and the tolerance is restored afterwards (line 587)
    p.gmres_abs_tol = std::max(gmres_abs_tol_in, norm_pre_rhs * p.gmres_rel_tol);
    // faces of the predicted densities (lines 410-411)
    sum_species(rho, rhotot.data());
    avg_face(g, rhotot.data(), rtf);
    species_fc(rho);
    const int s2 = stage(w_corr, dt, nullptr, stats2 ? &stats2[1] : nullptr);
    if (s2 < 0) return s2;
    return std::max(st, s2);
}
}  // namespace

extern "C" {

int or_advance_inertial(int dim, const int n[3], double dx, int visc_type, const fhd_gmres_params* p_in,
                        const fhd_stoch_params* sp, double dt, double* const umac[], double* rho, double* pi,
                        const double* eta, const double* const eta_ed[], const double* kappa,
                        const double* temperature, const double* const temperature_ed[],
                        const double* const W_cc[], const double* const W_ed[], fhd_solve_stats* stats2) {
    Geo g(dim, n, dx);
    double* r[1] = {rho};
    return step_impl(g, visc_type, p_in, sp, nullptr, dt, umac, r, pi, nullptr, eta, eta_ed, kappa, temperature,
                     temperature_ed, W_cc, W_ed, nullptr, stats2);
}

int or_advance_inertial_ms(int dim, const int n[3], double dx, int visc_type, const fhd_gmres_params* p_in,
                           const fhd_stoch_params* sp, const fhd_mixture_params* mp, double dt,
                           double* const umac[], double* const rho[], double* pi, double* const fluxdiv[],
                           const double* eta, const double* const eta_ed[], const double* kappa,
                           const double* temperature, const double* const temperature_ed[],
                           const double* const W_cc[], const double* const W_ed[], const double* const W_mass[],
                           fhd_solve_stats* stats2) {
    Geo g(dim, n, dx);
    Mix m = make_mix(mp);
    return step_impl(g, visc_type, p_in, sp, &m, dt, umac, rho, pi, fluxdiv, eta, eta_ed, kappa, temperature,
                     temperature_ed, W_cc, W_ed, W_mass, stats2);
}

int or_advance_overdamped(int dim, const int n[3], double dx, int visc_type, const fhd_gmres_params* p_in,
                          const fhd_stoch_params* sp, const fhd_mixture_params* mp, double dt,
                          double* const umac[], double* const rho[], double* pi, const double* eta,
                          const double* const eta_ed[], const double* kappa, const double* temperature,
                          const double* const temperature_ed[], const double* const W_cc[],
                          const double* const W_ed[], const double* const W_mass[], fhd_solve_stats* stats2) {
    Geo g(dim, n, dx);
    if (mp) {
        Mix m = make_mix(mp);
        return overdamped_impl(g, visc_type, p_in, sp, &m, dt, umac, rho, pi, eta, eta_ed, kappa, temperature,
                               temperature_ed, W_cc, W_ed, W_mass, stats2);
    }
    return overdamped_impl(g, visc_type, p_in, sp, nullptr, dt, umac, rho, pi, eta, eta_ed, kappa, temperature,
                           temperature_ed, W_cc, W_ed, nullptr, stats2);
}

int or_mass_fluxdiv(int dim, const int n[3], double dx, const fhd_stoch_params* sp, const fhd_mixture_params* mp,
                    const double* const rho[], double dt, const double* weights, int n_rngs,
                    const double* const W_fc[], double* const fluxdiv[], double* const flux[]) {
    Geo g(dim, n, dx);
    Mix m = make_mix(mp);
    return mass_fluxdiv_impl(g, m, sp, rho, dt, weights, n_rngs, W_fc, fluxdiv, flux);
}

// chi and the Cholesky factor of the Onsager matrix at one state (test hook)
int or_mixture_local(const fhd_mixture_params* mp, double k_B, const double* rho, double* chi_out,
                     double* sqrtL_out) {
    Mix m = make_mix(mp);
    double rt = 0.0;
    for (int i = 0; i < m.ns; i++) rt = rt + rho[i];
    double x[FHD_MAX_SPECIES], mt, chi[FHD_MAX_SPECIES][FHD_MAX_SPECIES], L[FHD_MAX_SPECIES][FHD_MAX_SPECIES];
    molconc(m.ns, m.molmass, rho, rt, x, &mt);
    chi_of(m, rho, rt, x, chi);
    sqrtL_local(m, rho, k_B, L);
    for (int i = 0; i < m.ns; i++)
        for (int j = 0; j < m.ns; j++) {
            chi_out[i * m.ns + j] = chi[i][j];
            sqrtL_out[i * m.ns + j] = L[i][j];
        }
    return 0;
}

// compute_sqrtLonsager_fc (mass_flux_utilities.f90:1096-1229): on every
// face of direction d, the Cholesky factor of the Onsager matrix at the
// face-averaged density (compute_nonnegative_rho_av, then
// compute_sqrtLonsager_local with rhotot = sum of the averages).  Entry (r,
// c) of face f in direction d goes to sqrtL[d*ns*ns + r + ns*c][f], the
// column-major component order of the reference's ns^2-component multifab.
void or_sqrtLonsager_fc(int dim, const int n[3], const fhd_stoch_params* sp, const fhd_mixture_params* mp,
                        const double* const rho[], double* const sqrtL[]) {
    Geo g(dim, n, 1.0);
    Mix m = make_mix(mp);
    const int ns = m.ns;
    for (int d = 0; d < dim; d++) {
        int e[3] = {0, 0, 0};
        e[d] = 1;
        forall(g, [&](int i, int j, int k) {
            const int q[3] = {i, j, k};
            // on a wall face the ghost cell is the first-order extrapolation of
            // the interior cell (scalar_bc, inhomogeneous_bc_val.f90:21-54)
            const long f = g.id(i, j, k),
                       fm = (g.wall(d) && q[d] == 0) ? f : g.id(i - e[0], j - e[1], k - e[2]);
            double r1[FHD_MAX_SPECIES], r2[FHD_MAX_SPECIES], ra[FHD_MAX_SPECIES], L[FHD_MAX_SPECIES][FHD_MAX_SPECIES];
            for (int s = 0; s < ns; s++) {
                r1[s] = rho[s][fm];
                r2[s] = rho[s][f];
            }
            rho_av(m, r1, r2, sp->dV, ra);
            sqrtL_local(m, ra, sp->k_B, L);
            for (int r = 0; r < ns; r++)
                for (int c = 0; c < ns; c++) sqrtL[d * ns * ns + r + ns * c][f] = L[r][c];
        });
    }
}

// stochastic_mass_fluxdiv (stochastic_mass_fluxdiv.f90:37-116) with the
// face factors given: flux = variance * sqrtL_face * sum_r w_r W_r (setval,
// saxpy per random stage, matvec_mul, mult by the variance), corrected to a
// zero species sum (correction_flux.f90:17-226), and its divergence
// (compute_div, div_and_grad.f90:884-1035), added to div when increment.
// W_fc[(r*dim + d)*ns + s]; flux (nullable) receives flux[d*ns + s].
void or_stochastic_mass_fluxdiv(int dim, const int n[3], double dx, const fhd_stoch_params* sp,
                                const fhd_mixture_params* mp, const double* const sqrtL[], double dt,
                                const double* weights, int n_rngs, const double* const W_fc[], int increment,
                                double* const div[], double* const flux_out[]) {
    Geo g(dim, n, dx);
    Mix m = make_mix(mp);
    const int ns = m.ns;
    const double variance = std::sqrt(2.0 * sp->k_B * m.var_mass / (sp->dV * dt));
    std::vector<Vec> flux(dim * ns, Vec(g.nc));
    for (int d = 0; d < dim; d++) {
        forall(g, [&](int i, int j, int k) {
            const long f = g.id(i, j, k);
            double w[FHD_MAX_SPECIES], fs[FHD_MAX_SPECIES];
            // stoch_mass_bc (stochastic_mass_fluxdiv.f90:216-368): the random
            // field is zero on a wall face (no-slip or slip)
            const int q[3] = {i, j, k};
            const bool on_wall = g.wall(d) && q[d] == 0;
            for (int s = 0; s < ns; s++) {
                double acc = 0.0;
                for (int rr = 0; rr < n_rngs; rr++) acc = acc + weights[rr] * W_fc[(rr * dim + d) * ns + s][f];
                w[s] = on_wall ? 0.0 : acc;
            }
            for (int r = 0; r < ns; r++) {
                double acc = 0.0;
                for (int c = 0; c < ns; c++) acc = acc + sqrtL[d * ns * ns + r + ns * c][f] * w[c];
                fs[r] = acc * variance;
            }
            if (m.correct && ns > 1) {
                double sum = 0.0;
                for (int s = 0; s < ns - 1; s++) sum = sum + fs[s];
                fs[ns - 1] = -sum;
            }
            for (int s = 0; s < ns; s++) flux[d * ns + s][f] = fs[s];
        });
    }
    const double dxinv = 1.0 / dx;
    forall(g, [&](int i, int j, int k) {
        const long f = g.id(i, j, k);
        for (int s = 0; s < ns; s++) {
            const double a = (flux[0 * ns + s][g.id(i + 1, j, k)] - flux[0 * ns + s][f]) * dxinv;
            const double b = (flux[1 * ns + s][g.id(i, j + 1, k)] - flux[1 * ns + s][f]) * dxinv;
            double v;
            if (increment) {
                v = div[s][f] + a + b;
                if (dim == 3) v = v + (flux[2 * ns + s][g.id(i, j, k + 1)] - flux[2 * ns + s][f]) * dxinv;
            } else {
                v = a + b;
                if (dim == 3) v = v + (flux[2 * ns + s][g.id(i, j, k + 1)] - flux[2 * ns + s][f]) * dxinv;
            }
            div[s][f] = v;
        }
    });
    if (flux_out)
        for (int q = 0; q < dim * ns; q++) std::copy(flux[q].begin(), flux[q].end(), flux_out[q]);
}

// rho W chi and the Onsager Cholesky factor at one state, trace species
// included (test hook for compute_rhoWchi_local and
// compute_sqrtLonsager_local)
void or_mixture_trace_local(const fhd_mixture_params* mp, double k_B, const double* rho, double* rhowchi_out,
                            double* sqrtL_out) {
    Mix m = make_mix(mp);
    double a[FHD_MAX_SPECIES][FHD_MAX_SPECIES], L[FHD_MAX_SPECIES][FHD_MAX_SPECIES];
    rhowchi_local(m, rho, a);
    sqrtL_local(m, rho, k_B, L);
    for (int i = 0; i < m.ns; i++)
        for (int j = 0; j < m.ns; j++) {
            rhowchi_out[i * m.ns + j] = a[i][j];
            sqrtL_out[i * m.ns + j] = L[i][j];
        }
}

// ---------------------------------------------------------------------
// discretisation-accuracy harness (exec/stokes_preconditioner
// main_driver.f90:354-387).  The exact fields are those of init.f90
// (prob_sol = 1 Taylor vortex at time 0; prob_sol = 31); the forcing is
// the continuous operator applied to them, evaluated here from the
// analytic derivatives.
// ---------------------------------------------------------------------
namespace {
const double PI = 3.14159265358979323846;

struct Exact {
    int dim, sol, coeff, visc;
    double k = 2.0 * PI;
    // velocity component c and its derivatives at x
    void u(int c, const double* x, double& v, double* d1, double d2[3][3]) const {
        double s[3], co[3];
        for (int d = 0; d < 3; d++) { s[d] = std::sin(k * x[d]); co[d] = std::cos(k * x[d]); }
        for (int a = 0; a < 3; a++) { d1[a] = 0; for (int b = 0; b < 3; b++) d2[a][b] = 0; }
        if (dim == 2) {
            // f = A * X(x) * Y(y) with X, Y in {sin, cos}
            double A = 1.0, off = 0.0;
            int fx, fy;  // 0 sin, 1 cos
            if (sol == 1) {
                if (c == 0) { A = -2.0; off = 1.0; fx = 1; fy = 0; } else { A = 2.0; off = 1.0; fx = 0; fy = 1; }
            } else {
                if (c == 0) { fx = 0; fy = 0; } else { fx = 1; fy = 0; }
            }
            double X = fx ? co[0] : s[0], Xp = fx ? -k * s[0] : k * co[0], Xpp = -k * k * X;
            double Y = fy ? co[1] : s[1], Yp = fy ? -k * s[1] : k * co[1], Ypp = -k * k * Y;
            v = off + A * X * Y;
            d1[0] = A * Xp * Y; d1[1] = A * X * Yp;
            d2[0][0] = A * Xpp * Y; d2[1][1] = A * X * Ypp; d2[0][1] = d2[1][0] = A * Xp * Yp;
        } else {
            int f[3];
            if (c == 0) { f[0] = 0; f[1] = 0; f[2] = 0; }
            else if (c == 1) { f[0] = 1; f[1] = 0; f[2] = 0; }
            else { f[0] = 0; f[1] = 0; f[2] = 1; }
            double F[3], Fp[3], Fpp[3];
            for (int d = 0; d < 3; d++) {
                F[d] = f[d] ? co[d] : s[d];
                Fp[d] = f[d] ? -k * s[d] : k * co[d];
                Fpp[d] = -k * k * F[d];
            }
            v = F[0] * F[1] * F[2];
            d1[0] = Fp[0] * F[1] * F[2]; d1[1] = F[0] * Fp[1] * F[2]; d1[2] = F[0] * F[1] * Fp[2];
            d2[0][0] = Fpp[0] * F[1] * F[2]; d2[1][1] = F[0] * Fpp[1] * F[2]; d2[2][2] = F[0] * F[1] * Fpp[2];
            d2[0][1] = d2[1][0] = Fp[0] * Fp[1] * F[2];
            d2[0][2] = d2[2][0] = Fp[0] * F[1] * Fp[2];
            d2[1][2] = d2[2][1] = F[0] * Fp[1] * Fp[2];
        }
    }
    double p(const double* x, double* gp) const {
        double v = 0;
        for (int d = 0; d < dim; d++) {
            if (sol == 1) { v += -std::cos(2 * k * x[d]); gp[d] = 2 * k * std::sin(2 * k * x[d]); }
            else { v += std::cos(2 * k * x[d]); gp[d] = -2 * k * std::sin(2 * k * x[d]); }
        }
        return v;
    }
    // beta, gamma and gradients (init.f90 mat_val_2d/_3d): prob_coeff 1:
    // constant 1; 5: beta = 1 + 0.5 cos(kx) sin(ky) [sin(kz)],
    // gamma = sin(kx) sin(ky) [sin(kz)]
    double beta(const double* x, double* gb) const {
        if (coeff == 1) { gb[0] = gb[1] = gb[2] = 0; return 1.0; }
        double sz = dim == 3 ? std::sin(k * x[2]) : 1.0, cz = dim == 3 ? std::cos(k * x[2]) : 0.0;
        gb[0] = -0.5 * k * std::sin(k * x[0]) * std::sin(k * x[1]) * sz;
        gb[1] = 0.5 * k * std::cos(k * x[0]) * std::cos(k * x[1]) * sz;
        gb[2] = dim == 3 ? 0.5 * k * std::cos(k * x[0]) * std::sin(k * x[1]) * cz : 0.0;
        return 1.0 + 0.5 * std::cos(k * x[0]) * std::sin(k * x[1]) * sz;
    }
    double gam(const double* x, double* gg) const {
        if (coeff == 1) { gg[0] = gg[1] = gg[2] = 0; return 1.0; }
        double sz = dim == 3 ? std::sin(k * x[2]) : 1.0, cz = dim == 3 ? std::cos(k * x[2]) : 0.0;
        gg[0] = k * std::cos(k * x[0]) * std::sin(k * x[1]) * sz;
        gg[1] = k * std::sin(k * x[0]) * std::cos(k * x[1]) * sz;
        gg[2] = dim == 3 ? k * std::sin(k * x[0]) * std::sin(k * x[1]) * cz : 0.0;
        return std::sin(k * x[0]) * std::sin(k * x[1]) * sz;
    }
    // forcing of the velocity row c: -div(tau) + dp/dx_c
    double fu(int c, const double* x) const {
        double vu[3], d1[3][3], d2[3][3][3];
        for (int a = 0; a < dim; a++) u(a, x, vu[a], d1[a], d2[a]);
        double gb[3], gg[3], gp[3];
        double b = beta(x, gb), gm = gam(x, gg);
        p(x, gp);
        int av = std::abs(visc);
        double lap = 0, gdiv = 0, div = 0, gbdu = 0, gbdut = 0;
        for (int d = 0; d < dim; d++) {
            lap += d2[c][d][d];
            gdiv += d2[d][c][d];  // d/dx_c (du_d/dx_d)
            div += d1[d][d];
            gbdu += gb[d] * d1[c][d];
            gbdut += gb[d] * d1[d][c];
        }
        double val = -(b * lap + gbdu);  // -div(beta grad u_c)
        if (av >= 2) val += -(b * gdiv + gbdut);
        if (av == 3) {
            double lam = gm - (2.0 / 3.0) * b;
            double glam = gg[c] - (2.0 / 3.0) * gb[c];
            val += -(lam * gdiv + glam * div);
        }
        return val + gp[c];
    }
    double fp(const double* x) const {
        double div = 0, vu, d1[3], d2[3][3];
        for (int d = 0; d < dim; d++) { u(d, x, vu, d1, d2); div += d1[d]; }
        return -div;
    }
};
}  // namespace

int or_accuracy_test_order(int dim, int n, int prob_coeff, int prob_sol, int visc_type, int order, double* err) {
    int nn[3] = {n, n, dim == 3 ? n : 1};
    const double dx = 1.0 / n;
    Geo g(dim, nn, dx);
    const long nc = g.nc;
    Exact ex{dim, prob_sol, prob_coeff, visc_type};
    std::vector<Vec> xu(dim, Vec(nc)), bu(dim, Vec(nc)), fu(dim, Vec(nc)), alpha(dim, Vec(nc, 1.0));
    Vec xp(nc), bp(nc), fpv(nc), beta(nc), gamma(nc);
    std::vector<Vec> bed(n_edge(dim), Vec(nc));
    forall(g, [&](int i, int j, int k) {
        long f = g.id(i, j, k);
        int I[3] = {i, j, k};
        for (int c = 0; c < dim; c++) {
            double x[3] = {0, 0, 0};
            for (int d = 0; d < dim; d++) x[d] = (d == c) ? I[d] * dx : (I[d] + 0.5) * dx;
            double v, d1[3], d2[3][3];
            ex.u(c, x, v, d1, d2);
            xu[c][f] = v;
            fu[c][f] = ex.fu(c, x);
        }
        double x[3] = {0, 0, 0}, gd[3];
        for (int d = 0; d < dim; d++) x[d] = (I[d] + 0.5) * dx;
        xp[f] = ex.p(x, gd);
        fpv[f] = ex.fp(x);
        beta[f] = ex.beta(x, gd);
        gamma[f] = ex.gam(x, gd);
    });
    double* bedp[3] = {bed[0].data(), dim == 3 ? bed[1].data() : nullptr, dim == 3 ? bed[2].data() : nullptr};
    avg_edge(g, beta.data(), bedp);
    const double* xup[3] = {xu[0].data(), xu[1].data(), dim == 3 ? xu[2].data() : nullptr};
    double* bup[3] = {bu[0].data(), bu[1].data(), dim == 3 ? bu[2].data() : nullptr};
    const double* ap[3] = {alpha[0].data(), alpha[1].data(), dim == 3 ? alpha[2].data() : nullptr};
    const double* cbed[3] = {bedp[0], bedp[1], bedp[2]};
    if (int rc = apply_matrix_impl(g, visc_type, bup, bp.data(), xup, xp.data(), ap, beta.data(), cbed,
                                   gamma.data(), 0.0, order))
        return rc;
    for (int c = 0; c < dim; c++) {
        const Vec& F = fu[c];
        const Vec& B = bu[c];
        err[c] = reduce_max(g, [&](int i, int j, int k) { long f = g.id(i, j, k); return std::fabs(F[f] - B[f]); });
    }
    err[dim] = reduce_max(g, [&](int i, int j, int k) { long f = g.id(i, j, k); return std::fabs(fpv[f] - bp[f]); });
    return 0;
}

int or_accuracy_test(int dim, int n, int prob_coeff, int prob_sol, int visc_type, double* err) {
    return or_accuracy_test_order(dim, n, prob_coeff, prob_sol, visc_type, 2, err);
}

}  // extern "C"
