// fhd_solver.cuh -- host-side objects of the solver: the context, the
// multigrid hierarchies and the launch helpers shared by the .cu files.
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/fhd_b200.h"
#include "fhd_vec.cuh"
#include "fhd_rb.cuh"
#include "fhd_walls.cuh"

namespace fhd {

#define FHD_CUDA_TRY(x)                                                                       \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess) {                                                              \
            fhd::set_last_error(std::string(#x) + ": " + cudaGetErrorString(e_));              \
            return FHD_ERR_CUDA;                                                              \
        }                                                                                     \
    } while (0)

void set_last_error(const std::string& s);

inline dim3 cell_block() { return dim3(32, 8, 1); }
inline dim3 cell_grid(const Grid& g) { return dim3((g.n[0] + 31) / 32, (g.n[1] + 7) / 8, g.n[2]); }
inline dim3 half_grid(const Grid& g) { return dim3(((g.n[0] + 1) / 2 + 31) / 32, (g.n[1] + 7) / 8, g.n[2]); }
inline int flat_blocks(i64 n) {
    i64 b = (n + 255) / 256;
    return (int)(b < RED_MAX_BLOCKS ? (b < 1 ? 1 : b) : RED_MAX_BLOCKS);
}

inline Grid make_grid(int dim, const int n[3], double dx) {
    Grid g;
    g.dim = dim;
    g.n[0] = n[0];
    g.n[1] = n[1];
    g.n[2] = dim == 3 ? n[2] : 1;
    g.nc = (i64)g.n[0] * g.n[1] * g.n[2];
    g.dx = dx;
    return g;
}

inline Grid coarsen(const Grid& g) {
    int n[3] = {g.n[0] / 2, g.n[1] / 2, g.dim == 3 ? g.n[2] / 2 : 1};
    return make_grid(g.dim, n, g.dx * 2.0);
}

inline bool all_even(const Grid& g) {
    for (int d = 0; d < g.dim; d++)
        if (g.n[d] & 1) return false;
    return true;
}

int nlevs_mg(const Grid& g, int minwidth);

// compile-time dispatch on (dim, visc_type)
template <class F>
inline void with_dim_visc(int dim, int visc, F&& f) {
    using std::integral_constant;
#define FHD_V(D, V) f(integral_constant<int, D>(), integral_constant<int, V>())
    if (dim == 2) {
        switch (visc) {
            case -3: FHD_V(2, -3); break;
            case -2: FHD_V(2, -2); break;
            case -1: FHD_V(2, -1); break;
            case 1: FHD_V(2, 1); break;
            case 2: FHD_V(2, 2); break;
            default: FHD_V(2, 3); break;
        }
    } else {
        switch (visc) {
            case -3: FHD_V(3, -3); break;
            case -2: FHD_V(3, -2); break;
            case -1: FHD_V(3, -1); break;
            case 1: FHD_V(3, 1); break;
            case 2: FHD_V(3, 2); break;
            default: FHD_V(3, 3); break;
        }
    }
#undef FHD_V
}

// 3D only (the fused smoothers)
template <class F>
inline void with_visc3(int visc, F&& f) {
    using std::integral_constant;
    switch (visc) {
        case -3: f(integral_constant<int, -3>()); break;
        case -2: f(integral_constant<int, -2>()); break;
        case -1: f(integral_constant<int, -1>()); break;
        case 1: f(integral_constant<int, 1>()); break;
        case 2: f(integral_constant<int, 2>()); break;
        default: f(integral_constant<int, 3>()); break;
    }
}

template <class F>
inline void with_dim(int dim, F&& f) {
    if (dim == 2) f(std::integral_constant<int, 2>());
    else f(std::integral_constant<int, 3>());
}

// (dim, visc_type 1, 2 or 3) for the wall kernels
template <class F>
inline void with_dim_wall_visc(int dim, int visc, F&& f) {
    with_dim(dim, [&](auto D) { with_wall_visc(visc, [&](auto V) { f(D, V); }); });
}



struct fhd_ctx_impl;

// device allocation owned by a context (freed at destroy).  Stream-ordered
// (cudaMallocAsync on the context's current stream, *stream): a plain
// cudaMalloc / cudaFree would serialise every other stream of the device,
// which would stall the concurrent contexts of a serving process.
struct Arena {
    std::vector<void*> blocks;
    size_t bytes = 0;
    cudaStream_t* stream = nullptr;
    template <typename T>
    T* alloc(i64 n) {
        void* p = nullptr;
        if (n <= 0) n = 1;
        if (cudaMallocAsync(&p, (size_t)n * sizeof(T), *stream) != cudaSuccess) return nullptr;
        blocks.push_back(p);
        bytes += (size_t)n * sizeof(T);
        return (T*)p;
    }
    void release() {
        for (void* p : blocks) cudaFreeAsync(p, *stream);
        if (!blocks.empty()) cudaStreamSynchronize(*stream);
        blocks.clear();
        bytes = 0;
    }
};

// pinned host blocks of NSCAL doubles, reused across contexts (a pinned
// allocation or free also serialises the device's streams)
double* pinned_scalars_acquire();
void pinned_scalars_release(double* p);

// how one multigrid level smooths, as the autotuner picked it (kind -1:
// not tuned, the fixed size rules choose).  Every plan evaluates the same
// update expression on the same operands in the same colour order.
struct SmoothPlan {
    int kind = -1;        // 0 colour launches, 1 tiled fused smooth, 2 row-tile smooth (FP32 visc_type 1)
    int bx = 32, by = 8;  // colour launches: thread block (bx * by = 256)
    RBGeom rb;            // kind 1
    RBXGeom rbx;          // kind 2
    float us = 0.f;       // measured time of one smooth pair
    int ncand = 0;        // candidates the tuner considered
    int index = -1;       // position of this plan in the level's candidate list
};

template <typename T>
struct StagLevel {
    Grid g;
    SmoothPlan plan;
    T* alpha[3] = {nullptr, nullptr, nullptr};  // owned on coarse levels
    T alpha_scale = T(1);
    const T* beta = nullptr;
    const T* gamma = nullptr;
    const T* bed[3] = {nullptr, nullptr, nullptr};
    T* own_beta = nullptr;
    T* own_gamma = nullptr;
    T* own_bed[3] = {nullptr, nullptr, nullptr};
    T* own_alpha0[3] = {nullptr, nullptr, nullptr};  // FP32 copy on level 0
    T* phi[3] = {nullptr, nullptr, nullptr};
    T* rhs[3] = {nullptr, nullptr, nullptr};
    T* tmp[3] = {nullptr, nullptr, nullptr};   // residual / L phi
    T* diag[3] = {nullptr, nullptr, nullptr};  // two-pass smoother
    // the visc_type 1 diagonal alpha_scale alpha + 2 dim beta q, staged by the
    // row-tile smoother in place of alpha (FP32 3D levels 64 to 256 wide)
    T* rbx_diag[3] = {nullptr, nullptr, nullptr};
    StagOp<T> op() const {
        StagOp<T> A;
        for (int c = 0; c < 3; c++) { A.alpha[c] = alpha[c]; A.bed[c] = bed[c]; }
        A.alpha_scale = alpha_scale;
        A.beta = beta;
        A.gamma = gamma;
        A.q = T(1.0 / (g.dx * g.dx));
        return A;
    }
};

template <typename T>
struct CCLevel {
    Grid g;
    SmoothPlan plan;
    T* a[3] = {nullptr, nullptr, nullptr};
    T* amu[3] = {nullptr, nullptr, nullptr};  // mu^-1 faces (visc_schur_approx != 0)
    T* phi = nullptr;
    T* rhs = nullptr;
    T* tmp = nullptr;
    CCOp<T> op() const {
        CCOp<T> A;
        for (int c = 0; c < 3; c++) A.a[c] = a[c];
        A.q = T(1.0 / (g.dx * g.dx));
        return A;
    }
};

template <typename T>
struct Multigrid {
    std::vector<StagLevel<T>> s;
    std::vector<CCLevel<T>> c;
    // preconditioner work arrays at the finest level, precision T
    T* x_u[3] = {nullptr, nullptr, nullptr};
    T* b_u[3] = {nullptr, nullptr, nullptr};
    T* mac_rhs = nullptr;
    T* bf_g[3] = {nullptr, nullptr, nullptr};  // mu^-1 G Phi_mu (visc_schur_approx != 0)
    T* bf_phi = nullptr;                       // Phi of the alpha^-1 solve, kept across the mu solves
};

}  // namespace fhd

struct fhd_ctx {
    int dim = 2;
    int n[3] = {1, 1, 1};
    // box layout of the level (probin_common max_grid_size; 0 = one box):
    // the staggered multigrid of several boxes stops at the boxes' depth,
    // or (stag_mg_bottom_solver 4, n/max_grid_size >= 2) solves its bottom
    // by a nested solve over the deeper levels of the domain ("fancy")
    int mgs[3] = {0, 0, 0};
    // domain walls (fhd_ctx_create_bc bc codes 100 no-slip, 200 slip): the
    // ghost sign per direction and side, 0 where periodic
    fhd::Walls walls = {{0, 0, 0}, {0, 0, 0}};
    bool has_walls = false;
    bool noslip = false;  // some wall is no-slip
    bool reservoirs = false;  // some wall is a reservoir (bc codes 101, 201)
    // tangential speeds of moving no-slip walls (fhd_ctx_set_wall_speed):
    // [side][t + 2 d], zero on periodic sides
    double wall_speed[2][6] = {{0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0}};
    bool moving_walls = false;
    int stag_nl_box = 0;      // levels of the box hierarchy (0: the domain's)
    bool stag_fancy = false;  // nested bottom solve from level stag_nl_box - 1
    double dx = 1.0;
    int visc = 1;
    int prec = FHD_PREC_FP64;
    fhd_gmres_params p;
    fhd::Grid g0;
    cudaStream_t stream = nullptr;  // stream the context launches on
    cudaStream_t own = nullptr;     // stream created by the context
    long long launches = 0;
    int vcycles = 0;
    fhd::Arena arena;
    fhd::Multigrid<double> mg64;
    fhd::Multigrid<float> mg32;
    // prepared coefficients (per gmres / per standalone call)
    const double* alpha_fc[3] = {nullptr, nullptr, nullptr};
    const double* beta = nullptr;
    const double* beta_ed[3] = {nullptr, nullptr, nullptr};
    const double* gamma = nullptr;
    double theta = 0.0;
    // FP64 Stokes work vectors (contiguous: dim velocity comps then p)
    double* V = nullptr;  // (m+1) vectors
    double* r = nullptr;
    double* w = nullptr;
    double* tmp = nullptr;
    double* xs = nullptr;  // solution copy for the host-fab path
    double* scratch_fc[3] = {nullptr, nullptr, nullptr};
    // reductions
    double* red_partials = nullptr;
    unsigned* red_counter = nullptr;
    double* dscal = nullptr;  // device scalars
    double* hscal = nullptr;  // pinned host mirror
    int m = 5;
    // inertial-step work arrays (allocated on the first step)
    bool step_ready = false;
    double* sb[128] = {nullptr};
    // the filtered stochastic stresses (filtering_width != 0): two sets of
    // dim + 2 * edge-set arrays in the context's precision, on first use
    void* stoch_filt = nullptr;
    // CUDA graphs of the preconditioner applications inside GMRES, keyed by
    // the operand pointers and the prepared coefficients (-1 auto, 0 off,
    // 1 on)
    int graph_mode = -1;
    // the coarse multigrid levels in one CTA (-1 default: on, 0 off)
    int coarse_mode = -1;
    // the row-tile fused smoother on large FP32 levels (-1 default: on, 0 off)
    int fused_mode = -1;
    int tune_mode = -1;           // smoother autotuner (fhd_ctx_set_tune)
    int sms = 148;                // multiprocessors of the device
    int smem_optin = 48 * 1024;   // shared memory a block may opt in to
    int smem_sm = 0;              // shared memory of one multiprocessor
    unsigned* dev_err = nullptr;  // set by a kernel whose bounded wait ran out
    struct PreconGraph {
        unsigned long long key = 0;
        cudaGraphExec_t exec = nullptr;
        cudaGraph_t graph = nullptr;             // kept while ev_nodes is not empty
        std::vector<cudaGraphNode_t> ev_nodes;   // profiling records, capture order
        long long launches = 0;
        int vcycles = 0;
        long long prof_launches = 0;
        double prof_bytes = 0.0;
        long long used = 0;
    };
    std::vector<PreconGraph> graphs;
    long long graph_clock = 0;
    bool capturing = false;
    bool cap_fail = false;
    std::vector<cudaGraphNode_t> cap_nodes;
    // optional timing of the finest-level smoother launches (CUDA events on
    // the context stream) with their algorithmic bytes
    bool prof = false;
    std::vector<cudaEvent_t> prof_ev;  // start/stop pairs
    size_t prof_used = 0;
    double prof_bytes = 0.0;
    long long prof_launches = 0;
};

namespace fhd {
// Reservoirs (bc codes 101 NO_SLIP_RESERVOIR, 201 SLIP_RESERVOIR) are no-slip
// and slip walls for the velocity and the pressure (the NO_SLIP / SLIP
// ranges of adv_bc_level_build and ell_bc_level_build, src_lowMach/
// define_bc_tower.f90:225-250, 301-355) and for the stochastic momentum flux
// (mflux_bc_2d / _3d,
// stochastic_m_fluxdiv.f90:363-451).  Their mass exchange -- Dirichlet
// concentrations on the boundary face (scalar_bc, inhomogeneous_bc_val.f90:
// 39-41) and the sqrt(2) random flux through it (stoch_mass_bc,
// stochastic_mass_fluxdiv.f90:216-368) -- is not built: the mass-flux entries
// and the multispecies steps refuse a context with reservoirs.
inline int refuse_reservoirs(const fhd_ctx* c, const char* where) {
    if (!c->reservoirs) return 0;
    set_last_error(std::string(where) + ": the mass exchange of reservoirs (bc codes 101, 201) is not built");
    return FHD_ERR_UNSUPPORTED;
}

constexpr int NSCAL = 256;
// scalar slots
constexpr int S_H = 0;        // H column, 1..m+1
constexpr int S_NRM = 128;    // norm squares
constexpr int S_MEAN = 140;   // mean sums
constexpr int S_Y = 160;      // least-squares y (m <= 64)
// the multigrids' own convergence checks (stag_mg_max_vcycles,
// mg_max_vcycles > 1): apart from the norms GMRES holds across a
// preconditioner application
constexpr int S_MG = 232;

inline RedSlot slot(fhd_ctx* c, int i) {
    RedSlot r;
    r.partials = c->red_partials + (size_t)i * 0;  // partials shared: reductions are stream-ordered
    r.counter = c->red_counter;
    r.out = c->dscal + i;
    return r;
}

int precon(fhd_ctx* ctx, CSVec<double> b, SVec<double> x);
int stokes_apply(fhd_ctx* ctx, CSVec<double> x, CSVec<double> rhs, SVec<double> out, int mode);
int prepare(fhd_ctx* ctx, const double* const alpha_fc[], const double* beta, const double* const beta_ed[],
            const double* gamma, double theta);
int stag_mg_solve_dev(fhd_ctx* ctx, double* const phi[], const double* const rhs[]);
int gmres_dev(fhd_ctx* ctx, CSVec<double> b, SVec<double> x, double* norm_pre_rhs, fhd_solve_stats* st);
int sync_scalars(fhd_ctx* ctx, int first, int count);
int dev_err_check(fhd_ctx* ctx);
int mass_fluxdiv(fhd_ctx* ctx, const fhd_mixture_params* mp, const fhd_stoch_params* sp, const double* const rho[],
                 double dt, const double* weights, int n_rngs, const double* const W[], double* const fluxdiv[]);
// compute_sqrtLonsager_fc on the high wall face of direction d (stored by
// neither layout): plane[r + ns*c] holds nc / n[d] values, in-plane index
// u + n_u v over the other two directions u < v
int sqrtL_high_wall_plane(fhd_ctx* ctx, const fhd_mixture_params* mp, const fhd_stoch_params* sp,
                          const double* const rho[], int d, double* const plane[]);
}  // namespace fhd
