// fhd_noalloc.cu -- the staggered multigrid solve for callers that cannot
// allocate device memory.
//
// Some callers cannot call cudaMalloc: a Fortran or C host whose device
// memory is handed out by another runtime (an OpenACC or CUDA Fortran data
// region, a fixed pool of a job scheduler), or code running where an
// allocation would synchronise the device or fail outright.  For them
// fhd_dev_stag_mg_solver_noalloc runs the same V-cycles as
// fhd_dev_stag_mg_solver, with every work array (residuals, coarse-level
// coefficients, coarse unknowns and right-hand sides, reduction partials)
// carved from one file-scope __device__ array instead of a context's
// allocations.  That array is FHD_NOALLOC_SCRATCH_BYTES large; every device
// that loads this library holds it until the process exits.
//
// In host code the array's name is only a host-side handle: its device
// address is looked up on every call, with the caller's device current,
// through cudaGetSymbolAddress, and passed to the kernels.
//
// All calls share the one array and it keeps the contents of the last call:
// each call clears what must start at zero, and calls whose work overlaps on
// the GPU (on different streams, or from different host threads) race on it.
#include "fhd_solver.cuh"

namespace fhd {
namespace {

constexpr long long NA_DOUBLES = (long long)FHD_NOALLOC_SCRATCH_BYTES / 8;
constexpr int NA_MAX_LEVELS = 32;
constexpr long long NA_RED = 2048;  // reduction partials, counter, results

__device__ __align__(256) double g_noalloc_scratch[NA_DOUBLES];

// device address of the scratch array on the current device.  It is looked
// up on every call, with the caller's device current: the lookup is cheap,
// and an address kept from an earlier call would be stale after the host
// reset the device (cudaDeviceReset) and the module was loaded again.
int scratch_address(double** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
        set_last_error(std::string("cudaGetSymbolAddress(noalloc scratch): ") + cudaGetErrorString(e));
        return FHD_ERR_CUDA;
    }
    *out = (double*)p;
    return 0;
}

// max |a| of one array into *out: per-block maxima, the last block to
// finish combines them (counter cleared by the caller before first use)
__global__ void __launch_bounds__(RED_THREADS) k_na_maxabs(i64 n, const double* a, double* partials,
                                                           unsigned* counter, double* out) {
    __shared__ double sh[RED_THREADS];
    __shared__ bool last;
    double s = 0.0;
    for (i64 f = blockIdx.x * (i64)blockDim.x + threadIdx.x; f < n; f += (i64)gridDim.x * blockDim.x)
        s = fmax(s, fabs(a[f]));
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = sh[0];
        __threadfence();
        last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int b = 0; b < (int)gridDim.x; b++) m = fmax(m, ((volatile double*)partials)[b]);
        *out = m;
        *counter = 0u;
    }
}

struct NA {
    int dim, visc, nE;
    fhd_gmres_params p;
    cudaStream_t st;
    StagLevel<double> L[NA_MAX_LEVELS];
    int nl;
    double* partials;
    unsigned* counter;
    double* results;
};

#define NA_TRY_LAUNCH()                                                              \
    do {                                                                             \
        cudaError_t e_ = cudaPeekAtLastError();                                      \
        if (e_ != cudaSuccess) {                                                     \
            set_last_error(std::string("noalloc launch: ") + cudaGetErrorString(e_)); \
            return FHD_ERR_CUDA;                                                     \
        }                                                                            \
    } while (0)

int na_smooth(NA& S, StagLevel<double>& L, int color) {
    const StagOp<double> A = L.op();
    const double omega = S.p.stag_mg_omega;
    if (color != 0 && all_even(L.g)) {
        const int c = (color - 1) / 2, par = (color + 1) & 1;
        with_dim_visc(S.dim, S.visc, [&](auto D, auto V) {
            constexpr int DIM = decltype(D)::value, VISC = decltype(V)::value;
            if (c == 0)
                k_stag_gs<double, DIM, VISC, 0><<<half_grid(L.g), cell_block(), 0, S.st>>>(
                    L.g, A, L.phi[0], L.phi[1], L.phi[2], L.rhs[0], par, omega);
            else if (c == 1)
                k_stag_gs<double, DIM, VISC, 1><<<half_grid(L.g), cell_block(), 0, S.st>>>(
                    L.g, A, L.phi[0], L.phi[1], L.phi[2], L.rhs[1], par, omega);
            else
                k_stag_gs<double, DIM, VISC, (DIM == 3 ? 2 : 1)><<<half_grid(L.g), cell_block(), 0, S.st>>>(
                    L.g, A, L.phi[0], L.phi[1], L.phi[2], L.rhs[DIM == 3 ? 2 : 1], par, omega);
        });
        NA_TRY_LAUNCH();
        return 0;
    }
    with_dim_visc(S.dim, S.visc, [&](auto D, auto V) {
        constexpr int DIM = decltype(D)::value, VISC = decltype(V)::value;
        k_stag_color_apply<double, DIM, VISC><<<cell_grid(L.g), cell_block(), 0, S.st>>>(
            L.g, A, L.phi[0], L.phi[1], L.phi[2], L.tmp[0], L.tmp[1], L.tmp[2], L.diag[0], L.diag[1], L.diag[2],
            color);
        k_stag_color_update<double, DIM><<<cell_grid(L.g), cell_block(), 0, S.st>>>(
            L.g, L.phi[0], L.phi[1], L.phi[2], L.rhs[0], L.rhs[1], L.rhs[2], L.tmp[0], L.tmp[1], L.tmp[2],
            L.diag[0], L.diag[1], L.diag[2], color, omega);
    });
    NA_TRY_LAUNCH();
    return 0;
}

int na_smooths(NA& S, StagLevel<double>& L, int count) {
    for (int m = 0; m < count; m++) {
        if (S.p.stag_mg_smoother == 0) {
            if (int rc = na_smooth(S, L, 0)) return rc;
        } else {
            for (int color = 1; color <= 2 * S.dim; color++)
                if (int rc = na_smooth(S, L, color)) return rc;
        }
    }
    return 0;
}

int na_residual(NA& S, StagLevel<double>& L) {
    const StagOp<double> A = L.op();
    with_dim_visc(S.dim, S.visc, [&](auto D, auto V) {
        constexpr int DIM = decltype(D)::value, VISC = decltype(V)::value;
        k_stag_apply<double, DIM, VISC><<<cell_grid(L.g), cell_block(), 0, S.st>>>(
            L.g, A, L.phi[0], L.phi[1], L.phi[2], L.tmp[0], L.tmp[1], L.tmp[2], L.rhs[0], L.rhs[1], L.rhs[2], 1);
    });
    NA_TRY_LAUNCH();
    return 0;
}

// max-norm of the finest residual per component into host r[]
int na_resid_norms(NA& S, double* r) {
    StagLevel<double>& L0 = S.L[0];
    if (int rc = na_residual(S, L0)) return rc;
    const i64 nc = L0.g.nc;
    for (int c = 0; c < S.dim; c++) {
        k_na_maxabs<<<flat_blocks(nc), RED_THREADS, 0, S.st>>>(nc, L0.tmp[c], S.partials, S.counter, S.results + c);
        NA_TRY_LAUNCH();
    }
    FHD_CUDA_TRY(cudaMemcpyAsync(r, S.results, sizeof(double) * S.dim, cudaMemcpyDeviceToHost, S.st));
    FHD_CUDA_TRY(cudaStreamSynchronize(S.st));
    return 0;
}

int na_vcycle(NA& S) {
    const int nl = S.nl, dim = S.dim;
    for (int l = 1; l < nl; l++)
        for (int c = 0; c < dim; c++)
            FHD_CUDA_TRY(cudaMemsetAsync(S.L[l].phi[c], 0, sizeof(double) * S.L[l].g.nc, S.st));
    for (int l = 0; l < nl - 1; l++) {
        StagLevel<double>& F = S.L[l];
        StagLevel<double>& C = S.L[l + 1];
        if (int rc = na_smooths(S, F, S.p.stag_mg_nsmooths_down)) return rc;
        if (int rc = na_residual(S, F)) return rc;
        with_dim(dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_stag_restrict<double, DIM><<<cell_grid(C.g), cell_block(), 0, S.st>>>(
                F.g, C.g, F.tmp[0], F.tmp[1], F.tmp[2], C.rhs[0], C.rhs[1], C.rhs[2], 0);
        });
        NA_TRY_LAUNCH();
    }
    if (int rc = na_smooths(S, S.L[nl - 1], S.p.stag_mg_nsmooths_bottom)) return rc;
    for (int l = nl - 2; l >= 0; l--) {
        StagLevel<double>& F = S.L[l];
        StagLevel<double>& C = S.L[l + 1];
        with_dim(dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_stag_prolong<double, DIM><<<cell_grid(C.g), cell_block(), 0, S.st>>>(
                F.g, C.g, F.phi[0], F.phi[1], F.phi[2], C.phi[0], C.phi[1], C.phi[2], pair_aligned(dim, F.phi));
        });
        NA_TRY_LAUNCH();
        if (int rc = na_smooths(S, F, S.p.stag_mg_nsmooths_up)) return rc;
    }
    return 0;
}

}  // namespace
}  // namespace fhd

using namespace fhd;

extern "C" int fhd_dev_stag_mg_solver_noalloc(int dim, const int n_cells[3], double dx, int visc_type,
                                              const fhd_gmres_params* params, const double* const alpha_fc[],
                                              const double* beta, const double* const beta_ed[],
                                              const double* gamma, double theta_alpha, double* const phi[],
                                              const double* const rhs[], void* stream) {
    if ((dim != 2 && dim != 3) || !n_cells || !params || !alpha_fc || !beta || !beta_ed || !gamma || !phi || !rhs)
        return FHD_ERR_BAD_ARG;
    if (visc_type == 0 || visc_type < -3 || visc_type > 3) return FHD_ERR_BAD_ARG;
    const int nE = dim == 2 ? 1 : 3;
    for (int d = 0; d < dim; d++)
        if (n_cells[d] < 2 || !phi[d] || !rhs[d] || !alpha_fc[d]) return FHD_ERR_BAD_ARG;
    for (int e = 0; e < nE; e++)
        if (!beta_ed[e]) return FHD_ERR_BAD_ARG;
    NA S;
    S.dim = dim;
    S.visc = visc_type;
    S.nE = nE;
    S.p = *params;
    S.st = (cudaStream_t)stream;
    int n[3] = {n_cells[0], n_cells[1], dim == 3 ? n_cells[2] : 1};
    Grid g0 = make_grid(dim, n, dx);
    S.nl = nlevs_mg(g0, S.p.stag_mg_minwidth);
    if (S.nl < 1 || S.nl > NA_MAX_LEVELS) return FHD_ERR_BAD_ARG;
    // carve the levels out of the scratch array, after the reduction area
    long long need = NA_RED;
    for (int l = 0; l < S.nl; l++) {
        StagLevel<double>& L = S.L[l];
        L = StagLevel<double>();
        L.g = (l == 0) ? g0 : coarsen(S.L[l - 1].g);
        const bool two_pass = !all_even(L.g) || S.p.stag_mg_smoother == 0;
        long long arrays = dim + (two_pass ? dim : 0);  // tmp (+ diag)
        if (l > 0) arrays += dim /*alpha*/ + 2 /*beta, gamma*/ + nE + 2 * dim /*phi, rhs*/;
        need += arrays * L.g.nc;
    }
    if (need > NA_DOUBLES) {
        set_last_error("stag_mg_solver_noalloc: grid needs " + std::to_string(need * 8) +
                       " bytes of work arrays, more than the " + std::to_string((long long)NA_DOUBLES * 8) +
                       "-byte static scratch");
        return FHD_ERR_BAD_ARG;
    }
    double* base = nullptr;
    if (int rc = scratch_address(&base)) return rc;
    S.partials = base;
    S.results = base + RED_MAX_BLOCKS;
    S.counter = (unsigned*)(base + RED_MAX_BLOCKS + 8);
    double* cur = base + NA_RED;
    auto take = [&](i64 nc) {
        double* p = cur;
        cur += nc;
        return p;
    };
    for (int l = 0; l < S.nl; l++) {
        StagLevel<double>& L = S.L[l];
        const i64 nc = L.g.nc;
        const bool two_pass = !all_even(L.g) || S.p.stag_mg_smoother == 0;
        for (int c = 0; c < dim; c++) {
            L.tmp[c] = take(nc);
            if (two_pass) L.diag[c] = take(nc);
        }
        if (l == 0) {
            for (int c = 0; c < dim; c++) {
                L.alpha[c] = (double*)alpha_fc[c];
                L.phi[c] = phi[c];
                L.rhs[c] = (double*)rhs[c];
            }
            L.alpha_scale = theta_alpha;
            L.beta = beta;
            L.gamma = gamma;
            for (int e = 0; e < nE; e++) L.bed[e] = beta_ed[e];
        } else {
            for (int c = 0; c < dim; c++) L.alpha[c] = take(nc);
            L.own_beta = take(nc);
            L.own_gamma = take(nc);
            L.beta = L.own_beta;
            L.gamma = L.own_gamma;
            for (int e = 0; e < nE; e++) {
                L.own_bed[e] = take(nc);
                L.bed[e] = L.own_bed[e];
            }
            for (int c = 0; c < dim; c++) {
                L.phi[c] = take(nc);
                L.rhs[c] = take(nc);
            }
            L.alpha_scale = 1.0;
        }
    }
    // the reduction counter starts at zero in every call
    FHD_CUDA_TRY(cudaMemsetAsync(S.counter, 0, sizeof(unsigned), S.st));
    // coefficient hierarchy (stag_mg_solver.f90:200-230)
    for (int l = 1; l < S.nl; l++) {
        StagLevel<double>& F = S.L[l - 1];
        StagLevel<double>& C = S.L[l];
        const double* a0 = F.alpha[0];
        const double* a1 = F.alpha[1];
        const double* a2 = dim == 3 ? F.alpha[2] : nullptr;
        if (l == 1 && F.alpha_scale != 1.0) {
            const int nb = flat_blocks(F.g.nc);
            for (int c = 0; c < dim; c++) {
                k_copy_conv<double, double><<<nb, 256, 0, S.st>>>(F.g.nc, F.tmp[c], F.alpha[c], F.alpha_scale);
                NA_TRY_LAUNCH();
            }
            a0 = F.tmp[0];
            a1 = F.tmp[1];
            a2 = dim == 3 ? F.tmp[2] : nullptr;
        }
        with_dim(dim, [&](auto D) {
            constexpr int DIM = decltype(D)::value;
            k_cc_average<double, DIM><<<cell_grid(C.g), cell_block(), 0, S.st>>>(F.g, C.g, F.beta, C.own_beta);
            k_cc_average<double, DIM><<<cell_grid(C.g), cell_block(), 0, S.st>>>(F.g, C.g, F.gamma, C.own_gamma);
            k_edge_coarsen<double, DIM><<<cell_grid(C.g), cell_block(), 0, S.st>>>(
                F.g, C.g, F.bed[0], F.bed[1], F.bed[2], C.own_bed[0], C.own_bed[1], C.own_bed[2]);
            k_stag_restrict<double, DIM><<<cell_grid(C.g), cell_block(), 0, S.st>>>(
                F.g, C.g, a0, a1, a2, C.alpha[0], C.alpha[1], C.alpha[2], 1);
        });
        NA_TRY_LAUNCH();
    }
    // V-cycles with the stopping rule of stag_mg_solver.f90:259-313, 761-806
    const int maxv = S.p.stag_mg_max_vcycles;
    double resid0[3] = {0, 0, 0};
    if (maxv > 1) {
        if (int rc = na_resid_norms(S, resid0)) return rc;
        bool allzero = true, anyzero = false;
        double rmax = 0.0;
        for (int c = 0; c < dim; c++) {
            allzero = allzero && resid0[c] == 0.0;
            anyzero = anyzero || resid0[c] == 0.0;
            rmax = fmax(rmax, resid0[c]);
        }
        if (allzero) return FHD_OK;
        if (anyzero)
            for (int c = 0; c < dim; c++) resid0[c] = rmax;
    }
    for (int vc = 1; vc <= maxv; vc++) {
        if (int rc = na_vcycle(S)) return rc;
        if (vc == maxv) break;
        double r[3] = {0, 0, 0};
        if (int rc = na_resid_norms(S, r)) return rc;
        bool done = true;
        for (int c = 0; c < dim; c++) done = done && (r[c] / resid0[c] < S.p.stag_mg_rel_tol);
        if (done) break;
    }
    FHD_CUDA_TRY(cudaStreamSynchronize(S.st));
    return FHD_OK;
}
