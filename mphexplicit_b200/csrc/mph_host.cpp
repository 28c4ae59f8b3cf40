// mph_host.cpp — the C ABI (include/mph_b200.h): set-up constants, device
// state, the per-step launch sequence, read-back and output.
//
// Step sequence of the FP64 form (the reference's loop body,
// main.cpp:386-431):
//   k_move        Convection + Wall + PeriodicBoundary + max displacement
//   [rebuild]     cell index -> bitonic sort -> cell ranges -> reorder ->
//                 neighbour list   (when the displacement test fires)
//   k_sweep_a     DensityA, GravityCenter, DensityP, DivergenceP, coefficients,
//                 PressureP/PressureA values
//   k_sweep_b     all forces, gravity, acceleration
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <string>
#include <vector>
#include <algorithm>

#include <nvtx3/nvToolsExt.h>
#include "mph_internal.h"
#include "mph_io.h"
#include "mph_mixed.h"
#include "mph_learned.h"
#include "mph_text.h"

using mph::SimConst;
using mph::StepScalars;

// Per-kernel CUDA-event timing on the context stream (mph_profile_*).
struct Profiler {
    struct Pending {
        int id;
        int count;
        cudaEvent_t a, b;
    };
    bool on = false;
    std::vector<std::string> names;
    std::vector<long long> launches;
    std::vector<double> ms;
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
};

// The learned form's device buffers and counters (MPH_MODE_LEARNED).
struct LearnedState {
    mph_model* model = nullptr;
    int judge_interval = 20;
    double tol = 1e-2;
    int* eoff = nullptr;        // CSR offsets of the fluid particles' edges [nf + 1]
    int* bsum = nullptr;        // scan scratch
    int* ei = nullptr;          // edge -> i
    int* ej = nullptr;          // edge -> j
    float4* eforce = nullptr;   // edge-MLP pair forces
    long long ecap = 0, ne = 0;
    bool edges_valid = false;
    float4* lsum = nullptr;     // per-particle learned force
    double4* force_j = nullptr; // the judge's forces and velocities
    double4* vel_j = nullptr;
    double* sums = nullptr;     // device [3]
    double* h_sums = nullptr;   // pinned [3]
    int fallback_left = 0;
    mph_learned_info info{};
};

// mph_step in the FP64 form for more than one step: one executable graph per
// parity of the velocity ping-pong, replayed once per step, whose conditional
// nodes take the host's per-step decisions (the rebuild test, made by the
// move kernel's last block, and the table check); made for the buffers and
// table capacities they were captured with.
struct StepGraphs {
    cudaGraphExec_t exec[2] = {nullptr, nullptr};  // by the vcur of the step
    int cur = -1, cap = -1, cap_s = -1;
    const int* nlist = nullptr;
    const int* nlist_s = nullptr;
    int launches_step = 0, launches_rebuild = 0;  // kernels per step and per rebuild
    bool enabled = true;  // mph_set_step_graphs
};

// mph_step_read_state: the copy stream (packs and device-to-host copies), its
// events and the velocities' staging buffer; made by the first call.
struct ReadBack {
    cudaStream_t copy = nullptr;
    cudaEvent_t ev[2] = {};
    double* stage_v = nullptr;  // [n][3]
};

struct mph_ctx {
    int mode = MPH_MODE_FP64;
    bool cell_walk = false;  // MPH_MIXED_CELL_WALK
    int n_fluid = 0;
    LearnedState lrn;
    int dim = 3;
    int n = 0;
    mph_params p{};
    mph_grid_header h{};
    mph_constants c{};
    SimConst sc{};
    cudaStream_t stream = nullptr;
    mph::DevFP64 d;
    mph::MixedState* mixed = nullptr;
    StepScalars* h_scal = nullptr;  // pinned
    double time = 0.0;
    long long step = 0, rebuilds = 0;
    bool virial_valid = false;
    bool dens_a_valid = false;  // DensityA / PressureA hold the values of the last step
    bool wall_force_valid = true;  // the walls' Force holds the values of the last step
    int lazy_pos = -1;             // pos buffer holding the last step's positions after mph_set_state
    int max_neighbors = 0;
    long long launches = 0;
    ReadBack rb;
    StepGraphs sg;
    Profiler prof;
    std::string err;
    mph::TextWriter* text = nullptr;  // *.prof / *.vtk writer thread, made by the first write
};

static thread_local std::string g_err;

static cudaEvent_t take_event(mph_ctx* ctx) {
    Profiler& p = ctx->prof;
    if (!p.pool.empty()) {
        cudaEvent_t e = p.pool.back();
        p.pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Brackets one launch (or one group of launches) of a named kernel: counts it,
// marks it as an NVTX range (visible to Nsight Systems on the host timeline)
// and, when profiling is on, records CUDA events around it on the ctx stream.
struct Launch {
    mph_ctx* ctx;
    int id = -1;
    int count = 1;
    cudaEvent_t a = nullptr;
    Launch(mph_ctx* c, const char* name) : ctx(c) {
        nvtxRangePushA(name);
        Profiler& p = ctx->prof;
        if (!p.on) return;
        for (size_t k = 0; k < p.names.size(); ++k)
            if (p.names[k] == name) id = (int)k;
        if (id < 0) {
            id = (int)p.names.size();
            p.names.push_back(name);
            p.launches.push_back(0);
            p.ms.push_back(0.0);
        }
        a = take_event(ctx);
        cudaEventRecord(a, ctx->stream);
    }
    ~Launch() {
        nvtxRangePop();
        ctx->launches += count;
        if (id < 0) return;
        cudaEvent_t b = take_event(ctx);
        cudaEventRecord(b, ctx->stream);
        ctx->prof.pending.push_back({id, count, a, b});
    }
};

static int fail(mph_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    g_err = msg;
    return code;
}

int mph::set_thread_error(int code, const std::string& msg) { return fail(nullptr, code, msg); }

#define CUDA_TRY(ctx, expr)                                                                \
    do {                                                                                   \
        cudaError_t e_ = (expr);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(ctx, MPH_ERR_CUDA, std::string(#expr ": ") + cudaGetErrorString(e_)); \
    } while (0)

// ---------------------------------------------------------------------------
// set-up constants: initializeWeight (main.cpp:836-954), initializeFluid's
// CofK/CofA (971-983), initializeWall (994-1033), initializeDomain (1035-1084).
// Evaluated on the host in the reference's expression order.
static double shape_wa(int dim, double swa, double r, double h) {
    const double hp = dim == 2 ? h * h : h * h * h;
    return 1.0 / swa * 1.0 / hp * (r / h) * (1.0 - (r / h)) * (1.0 - (r / h));
}
static double shape_wp(int dim, double swp, double r, double h) {
    const double hp = dim == 2 ? h * h : h * h * h;
    return 1.0 / swp * 1.0 / hp * ((1.0 - r / h) * (1.0 - r / h));
}

extern "C" int mph_compute_constants(const mph_params* p, const mph_grid_header* h, int dim, mph_constants* c) {
    if (!p || !h || !c || (dim != 2 && dim != 3)) return fail(nullptr, MPH_ERR_ARG, "bad arguments");
    if (!(h->particle_spacing > 0.0)) return fail(nullptr, MPH_ERR_ARG, "particle spacing must be > 0");
    std::memset(c, 0, sizeof(*c));
    const double l0 = h->particle_spacing;
    c->dim = dim;
    c->particle_volume = dim == 2 ? l0 * l0 : l0 * l0 * l0;
    c->radius_a = p->radius_ratio_a * l0;
    c->radius_g = p->radius_ratio_a * l0;  // RadiusRatioG = RadiusRatioA (main.cpp:838)
    c->radius_p = p->radius_ratio_p * l0;
    c->radius_v = p->radius_ratio_v * l0;
    if (dim == 2) {
        c->swa = 1.0 / 2.0 * 2.0 / 15.0 * M_PI / l0 / l0;
        c->swg = 1.0 / 2.0 * 1.0 / 3.0 * M_PI / l0 / l0;
        c->swp = 1.0 / 2.0 * 1.0 / 3.0 * M_PI / l0 / l0;
        c->swv = 1.0 / 2.0 * 1.0 / 3.0 * M_PI / l0 / l0;
        c->r2g = 1.0 / 2.0 * 1.0 / 30.0 * M_PI * c->radius_g * c->radius_g / l0 / l0 / c->swg;
    } else {
        c->swa = 1.0 / 3.0 * 1.0 / 5.0 * M_PI / l0 / l0 / l0;
        c->swg = 1.0 / 3.0 * 2.0 / 5.0 * M_PI / l0 / l0 / l0;
        c->swp = 1.0 / 3.0 * 2.0 / 5.0 * M_PI / l0 / l0 / l0;
        c->swv = 1.0 / 3.0 * 2.0 / 5.0 * M_PI / l0 / l0 / l0;
        c->r2g = 1.0 / 3.0 * 4.0 / 105.0 * M_PI * c->radius_g * c->radius_g / l0 / l0 / l0 / c->swg;
    }
    for (int which = 0; which < 2; ++which) {  // lattice sums N0a, N0p: origin excluded, r^2 <= R^2
        const double R = which == 0 ? c->radius_a : c->radius_p;
        const int range = (int)(R / l0 + 3.0);
        const int zr = dim == 2 ? 0 : range;
        double sum = 0.0;
        int count = 0;
        for (int ix = -range; ix <= range; ++ix)
            for (int iy = -range; iy <= range; ++iy)
                for (int iz = -zr; iz <= zr; ++iz) {
                    if (ix == 0 && iy == 0 && iz == 0) continue;
                    const double x = l0 * ((double)ix), y = l0 * ((double)iy), z = l0 * ((double)iz);
                    const double r2 = dim == 2 ? x * x + y * y : x * x + y * y + z * z;
                    if (r2 <= R * R) {
                        const double r = std::sqrt(r2);
                        sum += which == 0 ? shape_wa(dim, c->swa, r, R) : shape_wp(dim, c->swp, r, R);
                        ++count;
                    }
                }
        if (which == 0) { c->n0a = sum; c->n0a_count = count; }
        else            { c->n0p = sum; c->n0p_count = count; }
    }
    double integN, integX;
    if (dim == 2) { c->cof_k = 0.350778153; integN = 0.024679383; integX = 0.226126699; }
    else          { c->cof_k = 0.326976006; integN = 0.021425779; integX = 0.233977488; }
    for (int t = 0; t < MPH_TYPE_COUNT; ++t)
        c->cof_a[t] = p->surface_tension[t] / ((c->radius_g / l0) * (integN + c->cof_k * c->cof_k * integX));
    for (int t = 2; t < MPH_TYPE_COUNT; ++t) {  // theta = |omega|^2, no sqrt, as in the reference
        const double* w = p->wall_omega[t];
        double nrm[3] = {0.0, 0.0, 0.0}, q[4];
        const double th = std::fabs(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        if (th != 0.0)
            for (int d = 0; d < 3; ++d) nrm[d] = w[d] / th;
        q[0] = nrm[0] * std::sin(th * p->dt / 2.0);
        q[1] = nrm[1] * std::sin(th * p->dt / 2.0);
        q[2] = nrm[2] * std::sin(th * p->dt / 2.0);
        q[3] = std::cos(th * p->dt / 2.0);
        double(*R)[3] = c->wall_rotation[t];
        R[0][0] = q[0] * q[0] - q[1] * q[1] - q[2] * q[2] + q[3] * q[3];
        R[0][1] = 2.0 * (q[0] * q[1] - q[2] * q[3]);
        R[0][2] = 2.0 * (q[0] * q[2] + q[1] * q[3]);
        R[1][0] = 2.0 * (q[0] * q[1] + q[2] * q[3]);
        R[1][1] = -q[0] * q[0] + q[1] * q[1] - q[2] * q[2] + q[3] * q[3];
        R[1][2] = 2.0 * (q[1] * q[2] - q[0] * q[3]);
        R[2][0] = 2.0 * (q[0] * q[2] - q[1] * q[3]);
        R[2][1] = 2.0 * (q[1] * q[2] + q[0] * q[3]);
        R[2][2] = -q[0] * q[0] - q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    }
    double mr = 0.0;
    mr = c->radius_a > mr ? c->radius_a : mr;
    mr = c->radius_g > mr ? c->radius_g : mr;
    mr = c->radius_p > mr ? c->radius_p : mr;
    mr = c->radius_v > mr ? c->radius_v : mr;
    c->max_radius = mr;
    const double margin = 0.1 * l0;
    double cc[3];
    for (int d = 0; d < 3; ++d) c->domain_width[d] = h->domain_max[d] - h->domain_min[d];
    cc[0] = std::floor((h->domain_max[0] - h->domain_min[0]) / (mr + margin));
    cc[1] = std::floor((h->domain_max[1] - h->domain_min[1]) / (mr + margin));
    cc[2] = dim == 2 ? 1 : std::floor((h->domain_max[2] - h->domain_min[2]) / (mr + margin));
    for (int d = 0; d < 3; ++d) c->cell_count[d] = (int)cc[d];
    c->total_cell_count = (int)(cc[0] * cc[1] * cc[2]);
    for (int d = 0; d < 3; ++d) c->cell_width[d] = c->domain_width[d] / c->cell_count[d];
    return MPH_OK;
}

// Kernel constants derived from mph_constants, in the reference's order.
int mph::make_simconst(const mph_params& p, const mph_grid_header& h, const mph_constants& c, int dim, int n,
                       SimConst& s, std::string& msg) {
    std::memset(&s, 0, sizeof(s));
    const double l0 = h.particle_spacing;
    s.n = n;
    s.dim = dim;
    s.tot = c.total_cell_count;
    for (int d = 0; d < 3; ++d) {
        s.cc[d] = c.cell_count[d];
        s.dmin[d] = h.domain_min[d];
        s.width[d] = c.domain_width[d];
        s.half_width[d] = 0.5 * c.domain_width[d];
        {
            const double q = 0.75 * c.domain_width[d];
            std::memcpy(&s.q75_bits[d], &q, sizeof(q));
        }
        s.cell_width[d] = c.cell_width[d];
    }
    if (s.cc[0] < 1 || s.cc[1] < 1 || s.cc[2] < 1 || s.tot < 1)
        { msg = "domain narrower than one cell of MaxRadius+MARGIN"; return MPH_ERR_GEOMETRY; }
    if ((long long)s.cc[0] * s.cc[1] * s.cc[2] > (1LL << 29))
        { msg = "too many cells"; return MPH_ERR_GEOMETRY; }
    const double rm = c.max_radius + 0.1 * l0;  // MaxRadius + MARGIN
    s.rm2 = rm * rm;
    const double rs = (c.radius_p + 0.1 * l0) * (1.0 + 1e-9);  // RadiusP + MARGIN, with room for rounding
    s.rs2 = rs * rs;
    s.range[0] = (int)std::ceil(rm / c.cell_width[0]);
    s.range[1] = (int)std::ceil(rm / c.cell_width[1]);
    s.range[2] = dim == 2 ? 0 : (int)std::ceil(rm / c.cell_width[2]);
    for (int d = 0; d < 3; ++d)  // the reference asserts 2*range+1 <= 3 (main.cpp:1347-1349)
        if (2 * s.range[d] + 1 > 3) { msg = "cell narrower than MaxRadius+MARGIN"; return MPH_ERR_GEOMETRY; }
    int pe = 0;
    while ((n >> pe) != 0) ++pe;  // smallest power of two above n (main.cpp:612-617)
    if (pe > 30) { msg = "too many particles"; return MPH_ERR_ARG; }
    s.pow2 = 1 << pe;
    s.dt = p.dt;
    s.l0 = l0;
    s.vol = c.particle_volume;
    s.vol_over_l0 = c.particle_volume / l0;
    s.n0a = c.n0a;
    s.n0p = c.n0p;
    s.r2g = c.r2g;
    s.cof_k = c.cof_k;
    s.ra = c.radius_a; s.rg = c.radius_g; s.rp = c.radius_p; s.rv = c.radius_v;
    s.ra2 = s.ra * s.ra; s.rg2 = s.rg * s.rg; s.rp2 = s.rp * s.rp; s.rv2 = s.rv * s.rv;
    auto hp = [dim](double h) { return dim == 2 ? h * h : h * h * h; };
    // 1.0/Sw * 1.0/h^D evaluated as ((1.0/Sw)*1.0)/h^D, main.cpp:215-284
    s.ca = 1.0 / c.swa * 1.0 / hp(s.ra);
    s.cg = 1.0 / c.swg * 1.0 / hp(s.rg);
    s.cp = 1.0 / c.swp * 1.0 / hp(s.rp);
    s.cv = 1.0 / c.swv * 1.0 / hp(s.rv);
    s.inv_ra = 1.0 / s.ra; s.inv_rg = 1.0 / s.rg; s.inv_rp = 1.0 / s.rp; s.inv_rv = 1.0 / s.rv;
    s.m2_rg = -2.0 / s.rg; s.m2_rp = -2.0 / s.rp; s.m2_rv = -2.0 / s.rv;
    s.visc_c = dim == 2 ? 8.0 : 10.0;
    s.inv_r2g = 1.0 / s.r2g;
    s.rg_eq_ra = s.rg == s.ra;
    s.rv_eq_ra = s.rv == s.ra;
    for (int t = 0; t < MPH_TYPE_COUNT; ++t)
        for (int u = 0; u < MPH_TYPE_COUNT; ++u) {
            const double mi = p.shear_viscosity[t], mj = p.shear_viscosity[u];
            const double muij = 2.0 * (mi * mj) / (mi + mj);
            s.visc_mu[t][u] = s.visc_c * muij;
        }
    const double margin = 0.1 * l0;
    s.shift_thr = 0.5 * margin * 0.5 * margin;  // main.cpp:1102
    s.has_st = 0;
    s.ratio_all_one = 1;
    for (int t = 0; t < MPH_TYPE_COUNT; ++t) {
        s.density[t] = p.density[t];
        s.bulk_modulus[t] = p.bulk_modulus[t];
        s.bulk_viscosity[t] = p.bulk_viscosity[t];
        s.shear_viscosity[t] = p.shear_viscosity[t];
        s.cof_a[t] = c.cof_a[t];
        s.a_k[t] = c.cof_a[t] * (c.cof_k) * (c.cof_k);
        if (c.cof_a[t] != 0.0) s.has_st = 1;
        for (int u = 0; u < MPH_TYPE_COUNT; ++u) {
            s.ratio[t][u] = p.interaction_ratio[t][u];
            if (p.interaction_ratio[t][u] != 1.0) s.ratio_all_one = 0;
        }
        for (int d = 0; d < 3; ++d) {
            s.wall_velocity[t][d] = p.wall_velocity[t][d];
            s.wall_omega[t][d] = p.wall_omega[t][d];
            for (int e = 0; e < 3; ++e) s.wall_rot[t][d][e] = c.wall_rotation[t][d][e];
        }
    }
    for (int d = 0; d < 3; ++d) s.gravity[d] = p.gravity[d];
    return MPH_OK;
}

static int fill_simconst(mph_ctx* ctx) {
    std::string msg;
    const int st = mph::make_simconst(ctx->p, ctx->h, ctx->c, ctx->dim, ctx->n, ctx->sc, msg);
    if (st != MPH_OK) return fail(ctx, st, msg);
    return MPH_OK;
}

// ---------------------------------------------------------------------------
template <class T>
static int dalloc(mph_ctx* ctx, T** ptr, size_t count) {
    *ptr = nullptr;
    if (count == 0) count = 1;
    const cudaError_t e = cudaMalloc((void**)ptr, count * sizeof(T));
    if (e != cudaSuccess)
        return fail(ctx, MPH_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    return MPH_OK;
}

static void free_fp64(mph::DevFP64& d) {
    void* ptrs[] = {d.pidx[0], d.pidx[1], d.type[0], d.type[1], d.pos[0], d.pos[1], d.vel[0], d.vel[1],
                    d.snap, d.pos32, d.force, d.dens_a, d.strain_p, d.div_p, d.press, d.gc, d.virial_p, d.keys,
                    d.vals, d.cellstart, d.ncount, d.nlist, d.ncount_s, d.nlist_s, d.wall_center, d.staging,
                    d.scal};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    d = mph::DevFP64();
}

#define TRY(expr)                       \
    do {                                \
        const int st_ = (expr);         \
        if (st_ != MPH_OK) return st_;  \
    } while (0)

static int alloc_fp64(mph_ctx* ctx) {
    mph::DevFP64& d = ctx->d;
    const size_t n = (size_t)ctx->n, P = (size_t)ctx->sc.pow2, tot = (size_t)ctx->sc.tot;
    for (int k = 0; k < 2; ++k) {
        TRY(dalloc(ctx, &d.pidx[k], n));
        TRY(dalloc(ctx, &d.type[k], n));
        TRY(dalloc(ctx, &d.pos[k], n));
        TRY(dalloc(ctx, &d.vel[k], n));
    }
    TRY(dalloc(ctx, &d.snap, n));
    TRY(dalloc(ctx, &d.pos32, n));
    TRY(dalloc(ctx, &d.force, n));
    TRY(dalloc(ctx, &d.dens_a, n));
    TRY(dalloc(ctx, &d.strain_p, n));
    TRY(dalloc(ctx, &d.div_p, n));
    TRY(dalloc(ctx, &d.press, n));
    TRY(dalloc(ctx, &d.gc, n));
    TRY(dalloc(ctx, &d.virial_p, n));
    TRY(dalloc(ctx, &d.keys, P));
    TRY(dalloc(ctx, &d.vals, P));
    TRY(dalloc(ctx, &d.cellstart, 2 * tot + 1));
    TRY(dalloc(ctx, &d.ncount, n));
    TRY(dalloc(ctx, &d.wall_center, 12));
    TRY(dalloc(ctx, &d.staging, 3 * n));
    TRY(dalloc(ctx, &d.scal, 1));
    CUDA_TRY(ctx, cudaMemsetAsync(d.gc, 0, n * sizeof(double4), ctx->stream));
    CUDA_TRY(ctx, cudaMemsetAsync(d.force, 0, n * sizeof(double4), ctx->stream));
    CUDA_TRY(ctx, cudaMemsetAsync(d.virial_p, 0, n * sizeof(double), ctx->stream));
    CUDA_TRY(ctx, cudaMemsetAsync(d.scal, 0, sizeof(StepScalars), ctx->stream));
    return MPH_OK;
}

// Initial list length: lattice points within the cut-off, with head room for
// compression; the build grows it when a longer list appears.
static int initial_capacity(const mph_ctx* ctx, double r2) {
    const double ratio = std::sqrt(r2) / ctx->h.particle_spacing;
    const int r = (int)ratio + 1;
    int cnt = 0;
    const int zr = ctx->dim == 2 ? 0 : r;
    for (int x = -r; x <= r; ++x)
        for (int y = -r; y <= r; ++y)
            for (int z = -zr; z <= zr; ++z)
                if (x * x + y * y + z * z <= ratio * ratio) ++cnt;
    int cap = (int)(cnt * 1.25) + 8;
    cap = (cap + 31) / 32 * 32;
    return cap;
}

static int grow_table(mph_ctx* ctx, int need, int** table, int* capacity) {
    int cap = (int)(need * 1.15) + 8;
    cap = (cap + 31) / 32 * 32;
    if (*table) cudaFree(*table);
    *table = nullptr;
    *capacity = 0;
    TRY(dalloc(ctx, table, (size_t)cap * (size_t)ctx->n));
    *capacity = cap;
    return MPH_OK;
}

static int grow_list(mph_ctx* ctx, int need) { return grow_table(ctx, need, &ctx->d.nlist, &ctx->d.cap); }

// The short sublist (the list's entries within RadiusP+MARGIN, in list order)
// serves the pressure loops of both sweeps, with and without surface tension.
static bool uses_short_list(const mph_ctx* ctx) {
    (void)ctx;
    return true;
}

// calculateCellParticle + calculateNeighbor (main.cpp:1111-1596).
static int build_lists(mph_ctx* ctx);

static int rebuild_fp64(mph_ctx* ctx) {
    mph::DevFP64& d = ctx->d;
    const SimConst& s = ctx->sc;
    cudaStream_t st = ctx->stream;
    const int a = d.cur, b = 1 - d.cur, va = d.vcur, vb = 1 - d.vcur;
    { Launch L(ctx, "cell_index"); mph::launch_cell_index(s, d.pos[a], d.type[a], d.keys, d.vals, st); }
    { Launch L(ctx, "bitonic_sort"); L.count = mph::launch_bitonic_sort(s, d.keys, d.vals, st); }
    { Launch L(ctx, "cell_ranges"); mph::launch_cell_ranges(s, d.keys, d.cellstart, st); }
    {
        Launch L(ctx, "reorder");
        mph::launch_reorder(s, d.vals, d.pidx[a], d.type[a], d.pos[a], d.vel[va], d.pidx[b], d.type[b], d.pos[b],
                            d.vel[vb], d.snap, st);
    }
    d.cur = b;
    d.vcur = vb;
    return build_lists(ctx);
}

// calculateNeighbor on the current (just reordered) positions: the list and
// the short sublist, growing their tables and building again while a list is
// longer than its table.
static int build_lists(mph_ctx* ctx) {
    mph::DevFP64& d = ctx->d;
    const SimConst& s = ctx->sc;
    cudaStream_t st = ctx->stream;
    const bool sl = uses_short_list(ctx);
    int max_short = 0;
    for (int attempt = 0; attempt < 3; ++attempt) {
        CUDA_TRY(ctx, cudaMemsetAsync(&d.scal->max_neighbors, 0, sizeof(int), st));
        CUDA_TRY(ctx, cudaMemsetAsync(&d.scal->max_short, 0, sizeof(int), st));
        {
            Launch L(ctx, "neighbor_list");
            mph::launch_pos32(s, d.pos[d.cur], d.pos32, st);
            mph::launch_neighbor_list(s, d.pos[d.cur], d.pos32, d.cellstart, d.ncount, d.nlist, d.cap,
                                      sl ? d.ncount_s : nullptr, sl ? d.nlist_s : nullptr, d.cap_s, d.scal, st);
            L.count = 2;
        }
        CUDA_TRY(ctx, cudaGetLastError());
        CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_scal, d.scal, sizeof(StepScalars), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(ctx, cudaStreamSynchronize(st));
        ctx->max_neighbors = ctx->h_scal->max_neighbors;
        max_short = sl ? ctx->h_scal->max_short : 0;
        if (ctx->max_neighbors <= d.cap && max_short <= d.cap_s) break;
        if (ctx->max_neighbors > d.cap) TRY(grow_list(ctx, ctx->max_neighbors));
        if (max_short > d.cap_s) TRY(grow_table(ctx, max_short, &d.nlist_s, &d.cap_s));
    }
    if (ctx->max_neighbors > d.cap || max_short > d.cap_s)
        return fail(ctx, MPH_ERR_CAPACITY, "neighbour table could not grow");
    // the overflow flag of the attempts that grew the table is not an error
    CUDA_TRY(ctx, cudaMemsetAsync(&d.scal->flags, 0, sizeof(int), st));
    ctx->lrn.edges_valid = false;
    return MPH_OK;
}

static void sweep_a(mph_ctx* ctx, bool advance_wall) {
    mph::DevFP64& d = ctx->d;
    Launch L(ctx, "sweep_a");
    mph::launch_sweep_a(ctx->sc, d.cellstart, d.pos[d.cur], d.vel[d.vcur], d.ncount, d.nlist, d.ncount_s, d.nlist_s,
                        d.dens_a, d.strain_p, d.div_p, d.press, d.gc, advance_wall ? d.wall_center : nullptr,
                        ctx->stream);
    ctx->dens_a_valid = ctx->sc.has_st;  // without surface tension, computed when read
    ctx->lazy_pos = -1;                  // this step's positions are the current ones
}

// DensityA / PressureA of the last step, for a reader (FP64 and learned forms
// without surface tension, where the step itself does not need them).
// The positions the last step used: the current ones, or their copy when
// mph_set_state has replaced them since.
static const double4* step_positions(mph_ctx* ctx) {
    return ctx->d.pos[ctx->lazy_pos >= 0 ? ctx->lazy_pos : ctx->d.cur];
}

static void ensure_density_a(mph_ctx* ctx) {
    if (ctx->mixed || ctx->dens_a_valid) return;
    mph::DevFP64& d = ctx->d;
    Launch L(ctx, "density_a");
    mph::launch_density_a(ctx->sc, step_positions(ctx), d.ncount, d.nlist, d.dens_a, d.gc, ctx->stream);
    ctx->dens_a_valid = true;
}

// The walls' Force of the last step (output only: walls do not move by it),
// from the arrays the step's force sweep read, which stay until the next step.
static void ensure_wall_force(mph_ctx* ctx) {
    if (ctx->mixed || ctx->wall_force_valid) return;
    mph::DevFP64& d = ctx->d;
    Launch L(ctx, "wall_force");
    const bool sl = uses_short_list(ctx);
    mph::launch_sweep_b(ctx->sc, d.cellstart, step_positions(ctx), nullptr, nullptr, d.press, d.gc, d.ncount,
                        d.nlist, sl ? d.ncount_s : nullptr, sl ? d.nlist_s : nullptr, d.force, d.scal, ctx->stream,
                        nullptr, nullptr, nullptr, 2);
    ctx->wall_force_valid = true;
}

static int validate_inputs(int n, const int* type, const double* xyz, const double* vel) {
    for (int i = 0; i < n; ++i) {
        if (type[i] < 0 || type[i] >= MPH_TYPE_COUNT) return fail(nullptr, MPH_ERR_ARG, "particle type outside 0..3");
        for (int d = 0; d < 3; ++d)
            if (!std::isfinite(xyz[3 * (size_t)i + d]) || !std::isfinite(vel[3 * (size_t)i + d]))
                return fail(nullptr, MPH_ERR_NONFINITE, "non-finite position or velocity in the input");
    }
    return MPH_OK;
}

extern "C" void mph_destroy(mph_ctx* ctx) {
    if (!ctx) return;
    delete ctx->text;  // finishes the files still being written
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    free_fp64(ctx->d);
    for (auto& q : ctx->prof.pending) { cudaEventDestroy(q.a); cudaEventDestroy(q.b); }
    for (cudaEvent_t e : ctx->prof.pool) cudaEventDestroy(e);
    if (ctx->mixed) mph::mixed_destroy(ctx->mixed);
    {
        LearnedState& L = ctx->lrn;
        cudaFree(L.eoff);
        cudaFree(L.bsum);
        cudaFree(L.ei);
        cudaFree(L.ej);
        cudaFree(L.eforce);
        cudaFree(L.lsum);
        cudaFree(L.force_j);
        cudaFree(L.vel_j);
        cudaFree(L.sums);
        if (L.h_sums) cudaFreeHost(L.h_sums);
    }
    if (ctx->h_scal) cudaFreeHost(ctx->h_scal);
    {
        ReadBack& R = ctx->rb;
        if (R.copy) cudaStreamSynchronize(R.copy);
        for (cudaEvent_t e : R.ev)
            if (e) cudaEventDestroy(e);
        cudaFree(R.stage_v);
        if (R.copy) cudaStreamDestroy(R.copy);
    }
    for (cudaGraphExec_t& e : ctx->sg.exec)
        if (e) cudaGraphExecDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

static int create_impl(mph_ctx* ctx, const int* type, const double* xyz, const double* vel) {
    CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    CUDA_TRY(ctx, cudaMallocHost((void**)&ctx->h_scal, sizeof(StepScalars)));
    TRY(alloc_fp64(ctx));
    mph::DevFP64& d = ctx->d;
    const size_t n = (size_t)ctx->n;
    cudaStream_t st = ctx->stream;
    std::vector<int> pidx(n);
    for (size_t i = 0; i < n; ++i) pidx[i] = (int)i;  // main.cpp:645-647
    CUDA_TRY(ctx, cudaMemcpyAsync(d.pidx[0], pidx.data(), n * sizeof(int), cudaMemcpyHostToDevice, st));
    CUDA_TRY(ctx, cudaMemcpyAsync(d.type[0], type, n * sizeof(int), cudaMemcpyHostToDevice, st));
    CUDA_TRY(ctx, cudaMemcpyAsync(d.staging, xyz, 3 * n * sizeof(double), cudaMemcpyHostToDevice, st));
    { Launch L(ctx, "unpack3"); mph::launch_unpack3(ctx->n, d.staging, d.pos[0], d.type[0], st); }
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    CUDA_TRY(ctx, cudaMemcpyAsync(d.staging, vel, 3 * n * sizeof(double), cudaMemcpyHostToDevice, st));
    { Launch L(ctx, "unpack3"); mph::launch_unpack3(ctx->n, d.staging, d.vel[0], nullptr, st); }
    double wc[12];
    for (int t = 0; t < 4; ++t)
        for (int k = 0; k < 3; ++k) wc[3 * t + k] = ctx->p.wall_center[t][k];
    CUDA_TRY(ctx, cudaMemcpyAsync(d.wall_center, wc, sizeof(wc), cudaMemcpyHostToDevice, st));
    d.cur = 0;
    d.vcur = 0;
    // start-up: calculateCellParticle, calculateNeighbor, DensityA, GravityCenter,
    // DensityP (main.cpp:358-364)
    if (ctx->mode == MPH_MODE_MIXED || ctx->mode == MPH_MODE_MIXED_P64) {
        TRY(mph::mixed_create(&ctx->mixed, ctx->sc, ctx->c, d, ctx->mode == MPH_MODE_MIXED_P64, st, &ctx->err));
        mph::mixed_set_cell_walk(ctx->mixed, ctx->cell_walk);
    } else {
        TRY(grow_list(ctx, initial_capacity(ctx, ctx->sc.rm2)));
        if (uses_short_list(ctx)) {
            TRY(dalloc(ctx, &d.ncount_s, n));
            TRY(grow_table(ctx, initial_capacity(ctx, ctx->sc.rs2), &d.nlist_s, &d.cap_s));
        }
        TRY(rebuild_fp64(ctx));
        sweep_a(ctx, false);
    }
    CUDA_TRY(ctx, cudaGetLastError());
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return MPH_OK;
}

extern "C" int mph_create(const mph_params* p, const mph_grid_header* h, int dim, int mode, const int* type,
                          const double* xyz, const double* vel, mph_ctx** out) {
    if (!out) return fail(nullptr, MPH_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!p || !h || !type || !xyz || !vel) return fail(nullptr, MPH_ERR_ARG, "NULL argument");
    if (dim != 2 && dim != 3) return fail(nullptr, MPH_ERR_ARG, "dim must be 2 or 3");
    const bool walk = (mode & MPH_MIXED_CELL_WALK) != 0;
    mode &= ~MPH_MIXED_CELL_WALK;
    if (mode != MPH_MODE_FP64 && mode != MPH_MODE_MIXED && mode != MPH_MODE_MIXED_P64 && mode != MPH_MODE_LEARNED)
        return fail(nullptr, MPH_ERR_ARG, "unknown mode");
    if (walk && mode != MPH_MODE_MIXED && mode != MPH_MODE_MIXED_P64)
        return fail(nullptr, MPH_ERR_ARG, "MPH_MIXED_CELL_WALK applies to the mixed forms only");
    if (h->particle_count <= 0) return fail(nullptr, MPH_ERR_ARG, "particle_count must be > 0");
    if (!(p->dt > 0.0) || !std::isfinite(p->dt)) return fail(nullptr, MPH_ERR_ARG, "Dt must be finite and > 0");
    for (int d = 0; d < 3; ++d)
        if (!(h->domain_max[d] > h->domain_min[d])) return fail(nullptr, MPH_ERR_ARG, "empty domain");
    TRY(validate_inputs(h->particle_count, type, xyz, vel));
    mph_ctx* ctx = new mph_ctx();
    ctx->mode = mode;
    ctx->cell_walk = walk;
    for (int i = 0; i < h->particle_count; ++i) ctx->n_fluid += type[i] < 2 ? 1 : 0;
    ctx->dim = dim;
    ctx->n = h->particle_count;
    ctx->p = *p;
    ctx->h = *h;
    ctx->time = h->time;
    int st = mph_compute_constants(p, h, dim, &ctx->c);
    if (st == MPH_OK) st = fill_simconst(ctx);
    if (st == MPH_OK) st = create_impl(ctx, type, xyz, vel);
    if (st != MPH_OK) {
        g_err = ctx->err.empty() ? g_err : ctx->err;
        mph_destroy(ctx);
        return st;
    }
    *out = ctx;
    return MPH_OK;
}

static int read_scalars(mph_ctx* ctx) {
    CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_scal, ctx->d.scal, sizeof(StepScalars), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return MPH_OK;
}

static int check_flags(mph_ctx* ctx) {
    const int f = ctx->h_scal->flags;
    if (f & mph::DEVFLAG_NONFINITE) return fail(ctx, MPH_ERR_NONFINITE, "non-finite velocity produced by a step");
    if (f & mph::DEVFLAG_NEIGHBOR_OVERFLOW) return fail(ctx, MPH_ERR_CAPACITY, "neighbour table overflow");
    if (f) return fail(ctx, MPH_ERR_DEVICE, "device error flag " + std::to_string(f));
    return MPH_OK;
}

// One FP64 step up to the pair sweeps: convection, wall motion, periodic wrap
// and the displacement test, then the list rebuild when it fires
// (main.cpp:387-403).  The positions are the step's final ones after this.
static int step_fp64_head(mph_ctx* ctx) {
    mph::DevFP64& d = ctx->d;
    const SimConst& s = ctx->sc;
    cudaStream_t st = ctx->stream;
    CUDA_TRY(ctx, cudaMemsetAsync(&d.scal->max_shift2_bits, 0, sizeof(unsigned long long), st));
    {
        Launch L(ctx, "move");
        mph::launch_move(s, d.cellstart, d.pos[d.cur], d.vel[d.vcur], d.snap, d.wall_center, d.scal, st);
    }
    TRY(read_scalars(ctx));
    TRY(check_flags(ctx));
    double ms;
    std::memcpy(&ms, &ctx->h_scal->max_shift2_bits, sizeof(double));
    if (ms > s.shift_thr) {  // neighborCalculation() == 1 (main.cpp:1102)
        TRY(rebuild_fp64(ctx));
        ++ctx->rebuilds;
    }
    return MPH_OK;
}

// ---- the FP64 step as CUDA graphs --------------------------------------------

// Adds an IF node after the work captured so far on st and makes it the
// capture's only dependency; *body is the graph the node runs.
static int add_if_node(mph_ctx* ctx, cudaStream_t st, cudaGraphConditionalHandle h, cudaGraph_t* body) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    CUDA_TRY(ctx, cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) return fail(ctx, MPH_ERR_CUDA, "step graph: no active capture");
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeIf;
    p.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    CUDA_TRY(ctx, cudaGraphAddNode(&node, g, deps, nd, &p));
    *body = p.conditional.phGraph_out[0];
    CUDA_TRY(ctx, cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    return MPH_OK;
}

// Captures one FP64 step for vcur == v:
//   move (its last block makes the rebuild test and sets both conditionals)
//   -> IF rebuild { cell index, bitonic sort, cell ranges, reorder (then copied
//   back into the buffers this graph holds), pos32, neighbour list, table
//   check } -> IF sweep { sweep A, force sweep }
// The kernels and arguments of step_fp64, so the same bits.
static int capture_step(mph_ctx* ctx, int v, cudaGraphExec_t* out, int* launches_step, int* launches_rebuild) {
    mph::DevFP64& d = ctx->d;
    const SimConst& s = ctx->sc;
    cudaStream_t st = ctx->stream;
    const int a = d.cur, b = 1 - d.cur, va = v, vb = 1 - v;
    const size_t n = (size_t)ctx->n;
    const bool sl = uses_short_list(ctx);
    const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
    cudaGraph_t g = nullptr, g_reb = nullptr, g_sw = nullptr;
    cudaGraphConditionalHandle h_reb = 0, h_sw = 0;
    int rc = MPH_OK;
    auto ck = [&](cudaError_t e) {
        if (e != cudaSuccess && rc == MPH_OK)
            rc = fail(ctx, MPH_ERR_CUDA, std::string("step graph: ") + cudaGetErrorString(e));
        return rc == MPH_OK;
    };
    auto end_capture = [&]() {
        cudaGraph_t tmp = nullptr;
        ck(cudaStreamEndCapture(st, &tmp));
        ck(cudaGetLastError());
    };
    int ls = 0, lr = 0;
    if (ck(cudaGraphCreate(&g, 0)) && ck(cudaGraphConditionalHandleCreate(&h_reb, g, 0, 0)) &&
        ck(cudaGraphConditionalHandleCreate(&h_sw, g, 0, 0)) &&
        ck(cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, mode))) {
        mph::launch_move_graph(s, d.cellstart, d.pos[a], d.vel[va], d.snap, d.wall_center, d.scal, h_reb, h_sw, st);
        ls += 1;
        if (rc == MPH_OK) rc = add_if_node(ctx, st, h_reb, &g_reb);
        if (rc == MPH_OK) rc = add_if_node(ctx, st, h_sw, &g_sw);
        end_capture();
    }
    if (rc == MPH_OK && ck(cudaStreamBeginCaptureToGraph(st, g_reb, nullptr, nullptr, 0, mode))) {
        mph::launch_cell_index(s, d.pos[a], d.type[a], d.keys, d.vals, st);
        lr += 1 + mph::launch_bitonic_sort(s, d.keys, d.vals, st);
        mph::launch_cell_ranges(s, d.keys, d.cellstart, st);
        mph::launch_reorder(s, d.vals, d.pidx[a], d.type[a], d.pos[a], d.vel[va], d.pidx[b], d.type[b], d.pos[b],
                            d.vel[vb], d.snap, st);
        ck(cudaMemcpyAsync(d.pos[a], d.pos[b], n * sizeof(double4), cudaMemcpyDeviceToDevice, st));
        ck(cudaMemcpyAsync(d.vel[va], d.vel[vb], n * sizeof(double4), cudaMemcpyDeviceToDevice, st));
        ck(cudaMemcpyAsync(d.pidx[a], d.pidx[b], n * sizeof(int), cudaMemcpyDeviceToDevice, st));
        ck(cudaMemcpyAsync(d.type[a], d.type[b], n * sizeof(int), cudaMemcpyDeviceToDevice, st));
        ck(cudaMemsetAsync(&d.scal->max_neighbors, 0, sizeof(int), st));
        ck(cudaMemsetAsync(&d.scal->max_short, 0, sizeof(int), st));
        mph::launch_pos32(s, d.pos[a], d.pos32, st);
        mph::launch_neighbor_list(s, d.pos[a], d.pos32, d.cellstart, d.ncount, d.nlist, d.cap,
                                  sl ? d.ncount_s : nullptr, sl ? d.nlist_s : nullptr, d.cap_s, d.scal, st);
        mph::launch_graph_list_check(d.scal, d.cap, d.cap_s, sl ? 1 : 0, h_sw, st);
        lr += 6;
        end_capture();
    }
    if (rc == MPH_OK && ck(cudaStreamBeginCaptureToGraph(st, g_sw, nullptr, nullptr, 0, mode))) {
        mph::launch_sweep_a(s, d.cellstart, d.pos[a], d.vel[va], d.ncount, d.nlist, d.ncount_s, d.nlist_s,
                            d.dens_a, d.strain_p, d.div_p, d.press, d.gc, d.wall_center, st);
        mph::launch_sweep_b(s, d.cellstart, d.pos[a], d.vel[va], d.vel[vb], d.press, d.gc, d.ncount, d.nlist,
                            sl ? d.ncount_s : nullptr, sl ? d.nlist_s : nullptr, d.force, d.scal, st, nullptr,
                            nullptr, nullptr, 1);
        ls += 2;
        end_capture();
    }
    if (rc == MPH_OK) ck(cudaGraphInstantiate(out, g, 0));
    if (g) cudaGraphDestroy(g);
    *launches_step = ls;
    *launches_rebuild = lr;
    return rc;
}

static void drop_step_graphs(mph_ctx* ctx) {
    StepGraphs& G = ctx->sg;
    for (cudaGraphExec_t& e : G.exec)
        if (e) {
            cudaGraphExecDestroy(e);
            e = nullptr;
        }
    G.cur = -1;
}

static int ensure_step_graphs(mph_ctx* ctx) {
    StepGraphs& G = ctx->sg;
    const mph::DevFP64& d = ctx->d;
    if (G.exec[0] && G.exec[1] && G.cur == d.cur && G.cap == d.cap && G.cap_s == d.cap_s && G.nlist == d.nlist &&
        G.nlist_s == d.nlist_s)
        return MPH_OK;
    drop_step_graphs(ctx);
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    for (int v = 0; v < 2; ++v) {
        const int rc = capture_step(ctx, v, &G.exec[v], &G.launches_step, &G.launches_rebuild);
        if (rc != MPH_OK) {
            drop_step_graphs(ctx);
            return rc;
        }
    }
    G.cur = d.cur;
    G.cap = d.cap;
    G.cap_s = d.cap_s;
    G.nlist = d.nlist;
    G.nlist_s = d.nlist_s;
    return MPH_OK;
}

// nsteps FP64 steps as graph launches with no host round trip in between;
// the host reads the batch's counters at the end.  A list that outgrew its
// table stops the batch after that step's reorder: the host then grows the
// table, builds the list again from the same positions, finishes that step
// and runs the rest.  A non-finite velocity is reported at the end of the
// batch (the host path reports it at the next step's move).
static int step_fp64(mph_ctx* ctx, int nsteps);

static int step_fp64_graphs(mph_ctx* ctx, int nsteps) {
    StepGraphs& G = ctx->sg;
    mph::DevFP64& d = ctx->d;
    cudaStream_t st = ctx->stream;
    TRY(ensure_step_graphs(ctx));
    // the graphs' move accumulates into a cleared maximum and clears it again
    CUDA_TRY(ctx, cudaMemsetAsync(&d.scal->max_shift2_bits, 0, sizeof(unsigned long long), st));
    CUDA_TRY(ctx, cudaMemsetAsync(&d.scal->stop, 0, 4 * sizeof(int), st));  // stop, steps, rebuilds, blocks
    for (int k = 0; k < nsteps; ++k) CUDA_TRY(ctx, cudaGraphLaunch(G.exec[(d.vcur + k) & 1], st));
    TRY(read_scalars(ctx));
    const StepScalars& h = *ctx->h_scal;
    const int stopped = h.stop, reb = h.rebuilds_done;
    const int done = h.steps_done - stopped;  // steps moved, less the one whose list overflowed
    for (int k = 0; k < done; ++k) ctx->time += ctx->p.dt;  // main.cpp:449, one step at a time
    ctx->step += done;
    if (done & 1) d.vcur = 1 - d.vcur;
    ctx->rebuilds += reb;
    ctx->launches += (long long)G.launches_step * (done + stopped) + (long long)G.launches_rebuild * reb;
    static_assert(offsetof(StepScalars, blocks_done) == offsetof(StepScalars, stop) + 3 * sizeof(int),
                  "stop, steps_done, rebuilds_done and blocks_done are cleared together");
    if (reb > 0) {
        ctx->max_neighbors = h.max_neighbors;
        ctx->lrn.edges_valid = false;
    }
    ctx->dens_a_valid = ctx->sc.has_st;
    ctx->lazy_pos = -1;
    ctx->wall_force_valid = false;
    ctx->virial_valid = false;
    if (h.flags & ~mph::DEVFLAG_NEIGHBOR_OVERFLOW) return check_flags(ctx);
    if (!stopped) {
        if (done != nsteps) return fail(ctx, MPH_ERR_DEVICE, "step graph: a step did not complete");
        return MPH_OK;
    }
    // the stopped step: moved, sorted and reordered; build its lists with room
    CUDA_TRY(ctx, cudaMemsetAsync(&d.scal->flags, 0, sizeof(int), st));
    TRY(build_lists(ctx));
    sweep_a(ctx, true);
    {
        Launch L(ctx, "sweep_b");
        const bool sl = uses_short_list(ctx);
        mph::launch_sweep_b(ctx->sc, d.cellstart, d.pos[d.cur], d.vel[d.vcur], d.vel[1 - d.vcur], d.press, d.gc,
                            d.ncount, d.nlist, sl ? d.ncount_s : nullptr, sl ? d.nlist_s : nullptr, d.force, d.scal,
                            st, nullptr, nullptr, nullptr, 1);
        ctx->wall_force_valid = false;
    }
    d.vcur = 1 - d.vcur;
    CUDA_TRY(ctx, cudaGetLastError());
    ctx->time += ctx->p.dt;
    ++ctx->step;
    const int rest = nsteps - done - 1;
    return rest > 0 ? step_fp64(ctx, rest) : MPH_OK;
}

static int step_fp64(mph_ctx* ctx, int nsteps) {
    // several steps: graph replay (per-kernel profiling needs the host path)
    if (nsteps > 1 && ctx->sg.enabled && !ctx->prof.on) return step_fp64_graphs(ctx, nsteps);
    mph::DevFP64& d = ctx->d;
    const SimConst& s = ctx->sc;
    cudaStream_t st = ctx->stream;
    for (int k = 0; k < nsteps; ++k) {
        TRY(step_fp64_head(ctx));
        sweep_a(ctx, true);
        {
            Launch L(ctx, "sweep_b");
            const bool sl = uses_short_list(ctx);
            mph::launch_sweep_b(s, d.cellstart, d.pos[d.cur], d.vel[d.vcur], d.vel[1 - d.vcur], d.press, d.gc,
                                d.ncount, d.nlist, sl ? d.ncount_s : nullptr, sl ? d.nlist_s : nullptr, d.force,
                                d.scal, st, nullptr, nullptr, nullptr, 1);
            ctx->wall_force_valid = false;  // computed when read
        }
        d.vcur = 1 - d.vcur;
        CUDA_TRY(ctx, cudaGetLastError());
        ctx->time += ctx->p.dt;  // main.cpp:449
        ++ctx->step;
    }
    ctx->virial_valid = false;
    return MPH_OK;
}

// The mixed form: same step order, its own kernels (k_mixed.cu).
static int step_mixed(mph_ctx* ctx, int nsteps) {
    mph::DevFP64& d = ctx->d;
    const SimConst& s = ctx->sc;
    cudaStream_t st = ctx->stream;
    for (int k = 0; k < nsteps; ++k) {
        CUDA_TRY(ctx, cudaMemsetAsync(&d.scal->max_shift2_bits, 0, sizeof(unsigned long long), st));
        {
            Launch L(ctx, "mix_move");
            mph::mixed_move(ctx->mixed, s, d, st);
        }
        TRY(read_scalars(ctx));
        TRY(check_flags(ctx));
        double ms;
        std::memcpy(&ms, &ctx->h_scal->max_shift2_bits, sizeof(double));
        if (ms > s.shift_thr) {
            Launch L(ctx, "mix_rebuild");
            const int rc = mph::mixed_rebuild(ctx->mixed, s, d, st, &ctx->err, &L.count);
            if (rc != MPH_OK) return fail(ctx, rc, ctx->err);
            ++ctx->rebuilds;
        }
        {
            Launch L(ctx, "mix_sweep_a");
            mph::mixed_sweep_a(ctx->mixed, s, d, true, st);
        }
        {
            Launch L(ctx, "mix_sweep_b");
            L.count = mph::mixed_sweep_b(ctx->mixed, s, d, st);
        }
        d.vcur = 1 - d.vcur;
        CUDA_TRY(ctx, cudaGetLastError());
        ctx->time += ctx->p.dt;  // main.cpp:449
        ++ctx->step;
    }
    ctx->virial_valid = false;
    return MPH_OK;
}

// ---- the learned form --------------------------------------------------------

// CSR edges of the fluid particles' neighbour lists (after each rebuild).
static int build_edges(mph_ctx* ctx) {
    LearnedState& L = ctx->lrn;
    mph::DevFP64& d = ctx->d;
    cudaStream_t st = ctx->stream;
    const int nf = ctx->n_fluid;
    if (!L.eoff) {
        TRY(dalloc(ctx, &L.eoff, (size_t)nf + 1));
        TRY(dalloc(ctx, &L.bsum, (size_t)mph::edge_scan_blocks(nf) + 1));
    }
    {
        Launch Lc(ctx, "edge_offsets");
        Lc.count = 3;
        mph::launch_edge_offsets(d.ncount, nf, L.eoff, L.bsum, st);
    }
    int ne = 0;
    CUDA_TRY(ctx, cudaMemcpyAsync(&ne, L.eoff + nf, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (ne > L.ecap) {
        cudaFree(L.ei);
        cudaFree(L.ej);
        cudaFree(L.eforce);
        L.ei = L.ej = nullptr;
        L.eforce = nullptr;
        L.ecap = 0;
        const long long cap = (long long)(ne * 1.2) + 1024;
        TRY(dalloc(ctx, &L.ei, (size_t)cap));
        TRY(dalloc(ctx, &L.ej, (size_t)cap));
        if (ctx->mode == MPH_MODE_LEARNED) TRY(dalloc(ctx, &L.eforce, (size_t)cap));
        L.ecap = cap;
    }
    L.ne = ne;
    {
        Launch Lc(ctx, "edge_fill");
        mph::launch_edge_fill(d.ncount, d.nlist, ctx->n, nf, L.eoff, L.ei, L.ej, st);
    }
    CUDA_TRY(ctx, cudaGetLastError());
    L.edges_valid = true;
    return MPH_OK;
}

static int learned_buffers(mph_ctx* ctx) {
    LearnedState& L = ctx->lrn;
    if (L.lsum) return MPH_OK;
    const size_t n = (size_t)ctx->n;
    TRY(dalloc(ctx, &L.lsum, n));
    TRY(dalloc(ctx, &L.force_j, n));
    TRY(dalloc(ctx, &L.vel_j, n));
    TRY(dalloc(ctx, &L.sums, 3));
    CUDA_TRY(ctx, cudaMallocHost((void**)&L.h_sums, 3 * sizeof(double)));
    return MPH_OK;
}

static void plain_sweep_b(mph_ctx* ctx, double4* vel_out, double4* force) {
    mph::DevFP64& d = ctx->d;
    Launch L(ctx, "sweep_b");
    const bool sl = uses_short_list(ctx);
    mph::launch_sweep_b(ctx->sc, d.cellstart, d.pos[d.cur], d.vel[d.vcur], vel_out, d.press, d.gc, d.ncount, d.nlist,
                        sl ? d.ncount_s : nullptr, sl ? d.nlist_s : nullptr, force, d.scal, ctx->stream);
}

// The FP64 step with the learned pair terms, the judge and the fallback.
static int step_learned(mph_ctx* ctx, int nsteps) {
    LearnedState& L = ctx->lrn;
    if (!L.model) return fail(ctx, MPH_ERR_STATE, "no model attached (mph_set_learned)");
    mph::DevFP64& d = ctx->d;
    const SimConst& s = ctx->sc;
    cudaStream_t st = ctx->stream;
    TRY(learned_buffers(ctx));
    mph::mlp::Model* md = mph::model_of(L.model);
    for (int k = 0; k < nsteps; ++k) {
        CUDA_TRY(ctx, cudaMemsetAsync(&d.scal->max_shift2_bits, 0, sizeof(unsigned long long), st));
        {
            Launch Lm(ctx, "move");
            mph::launch_move(s, d.cellstart, d.pos[d.cur], d.vel[d.vcur], d.snap, d.wall_center, d.scal, st);
        }
        TRY(read_scalars(ctx));
        TRY(check_flags(ctx));
        double ms;
        std::memcpy(&ms, &ctx->h_scal->max_shift2_bits, sizeof(double));
        if (ms > s.shift_thr) {
            TRY(rebuild_fp64(ctx));
            ++ctx->rebuilds;
        }
        sweep_a(ctx, true);
        double4* vout = d.vel[1 - d.vcur];
        if (L.fallback_left > 0) {
            plain_sweep_b(ctx, vout, d.force);
            --L.fallback_left;
            ++L.info.plain_steps;
        } else {
            if (!L.edges_valid) TRY(build_edges(ctx));
            mph::mlp::EdgeSource es{};
            es.pos = d.pos[d.cur];
            es.vel = d.press;
            es.ei = L.ei;
            es.ej = L.ej;
            es.ne = L.ne;
            for (int q = 0; q < 3; ++q) {
                es.width[q] = s.width[q];
                es.half_width[q] = s.half_width[q];
            }
            es.inv_l0 = 1.0 / s.l0;
            es.rv2 = s.rv2;
            {
                Launch Lm(ctx, "mlp_edges");
                if (mph::mlp::model_apply_edges(md, es, L.eforce, st, &Lm.count, &ctx->err) != 0)
                    return fail(ctx, MPH_ERR_CUDA, ctx->err);
            }
            {
                Launch Lb(ctx, "sweep_b_learned");
                // the learned sweep evaluates only the pairs within RadiusP
                const bool sl = uses_short_list(ctx);
                mph::launch_sweep_b(s, d.cellstart, d.pos[d.cur], d.vel[d.vcur], vout, d.press, d.gc,
                                    sl ? d.ncount_s : d.ncount, sl ? d.nlist_s : d.nlist, nullptr, nullptr,
                                    d.force, d.scal, st, L.eoff, L.eforce, L.lsum);
            }
            bool use = true;
            if (L.info.steps % L.judge_interval == 0) {
                plain_sweep_b(ctx, L.vel_j, L.force_j);
                CUDA_TRY(ctx, cudaMemsetAsync(L.sums, 0, 3 * sizeof(double), st));
                {
                    Launch Lc(ctx, "force_compare");
                    mph::launch_force_compare(ctx->n_fluid, d.force, L.force_j, L.lsum, L.sums, st);
                }
                CUDA_TRY(ctx, cudaMemcpyAsync(L.h_sums, L.sums, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
                CUDA_TRY(ctx, cudaStreamSynchronize(st));
                std::string merr;
                if (mph::mlp::model_error_flag(md, &merr) != 0) return fail(ctx, MPH_ERR_DEVICE, merr);
                const double e = L.h_sums[1] > 0.0 ? std::sqrt(L.h_sums[0] / L.h_sums[1]) : 0.0;
                ++L.info.judged;
                L.info.last_force_error = e;
                L.info.max_force_error = std::max(L.info.max_force_error, e);
                // The judged error is the replaced terms' own relative error
                // (the network's output against the FP64 PressureA +
                // DiffuseInterface + ViscosityV it stands for); where those
                // terms are negligible against the total force (a fluid at
                // rest has none) it is the error of the total force.
                double judged_error = e;
                if (L.h_sums[2] > 1e-12 * L.h_sums[1]) {
                    const double te = std::sqrt(L.h_sums[0] / L.h_sums[2]);
                    L.info.last_term_error = te;
                    L.info.max_term_error = std::max(L.info.max_term_error, te);
                    judged_error = te;
                } else {
                    L.info.last_term_error = 0.0;
                }
                if (judged_error <= L.tol)
                    L.info.max_accepted_error = std::max(L.info.max_accepted_error, judged_error);
                if (!(judged_error <= L.tol)) {  // fall back: take the judge's step
                    use = false;
                    ++L.info.fallbacks;
                    ++L.info.plain_steps;
                    L.fallback_left = L.judge_interval - 1;
                    const size_t bytes = (size_t)ctx->n * sizeof(double4);
                    CUDA_TRY(ctx, cudaMemcpyAsync(vout, L.vel_j, bytes, cudaMemcpyDeviceToDevice, st));
                    CUDA_TRY(ctx, cudaMemcpyAsync(d.force, L.force_j, bytes, cudaMemcpyDeviceToDevice, st));
                }
            }
            if (use) ++L.info.learned_steps;
        }
        ++L.info.steps;
        d.vcur = 1 - d.vcur;
        CUDA_TRY(ctx, cudaGetLastError());
        ctx->time += ctx->p.dt;
        ++ctx->step;
    }
    ctx->virial_valid = false;
    return MPH_OK;
}

extern "C" int mph_set_learned(mph_ctx* ctx, mph_model* m, int judge_interval, double tolerance) {
    if (!ctx) return fail(nullptr, MPH_ERR_ARG, "ctx is NULL");
    if (ctx->mode != MPH_MODE_LEARNED) return fail(ctx, MPH_ERR_STATE, "the context is not in MPH_MODE_LEARNED");
    if (!m || judge_interval < 1 || !(tolerance > 0.0)) return fail(ctx, MPH_ERR_ARG, "bad arguments");
    ctx->lrn.model = m;
    ctx->lrn.judge_interval = judge_interval;
    ctx->lrn.tol = tolerance;
    ctx->lrn.fallback_left = 0;
    return MPH_OK;
}

extern "C" int mph_learned_stats(mph_ctx* ctx, mph_learned_info* info) {
    if (!ctx || !info) return fail(ctx, MPH_ERR_ARG, "bad arguments");
    *info = ctx->lrn.info;
    info->edges = ctx->lrn.ne;
    return MPH_OK;
}

extern "C" int mph_collect_samples(mph_ctx* ctx, mph_dataset* ds, long long max_samples, unsigned long long seed) {
    if (!ctx || !ds || max_samples < 0) return fail(ctx, MPH_ERR_ARG, "bad arguments");
    if (ctx->mixed) return fail(ctx, MPH_ERR_STATE, "samples come from the FP64 neighbour list (FP64 or learned form)");
    if (!ctx->lrn.edges_valid) TRY(build_edges(ctx));
    long long got = 0;
    float4* dst = mph::dataset_reserve(ds, max_samples, &got);
    if (got < max_samples) return fail(ctx, MPH_ERR_CAPACITY, "dataset is full");
    mph::DevFP64& d = ctx->d;
    {
        Launch L(ctx, "collect");
        mph::launch_collect(ctx->sc, d.pos[d.cur], d.press, d.gc, ctx->lrn.ei, ctx->lrn.ej, ctx->lrn.ne, got, seed, dst,
                            ctx->stream);
    }
    CUDA_TRY(ctx, cudaGetLastError());
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    mph::dataset_commit(ds, got);
    return MPH_OK;
}

extern "C" int mph_step(mph_ctx* ctx, int nsteps) {
    if (!ctx || nsteps < 0) return fail(ctx, MPH_ERR_ARG, "bad arguments");
    if (ctx->mixed) return step_mixed(ctx, nsteps);
    if (ctx->mode == MPH_MODE_LEARNED) return step_learned(ctx, nsteps);
    return step_fp64(ctx, nsteps);
}

extern "C" int mph_set_sweep_layout(mph_ctx* ctx, int layout) {
    if (!ctx) return fail(nullptr, MPH_ERR_ARG, "ctx is NULL");
    if (layout < 0 || layout > 2) return fail(ctx, MPH_ERR_ARG, "layout must be 0, 1 or 2");
    ctx->sc.sweep_layout = layout;
    drop_step_graphs(ctx);  // they hold the constants by value
    return MPH_OK;
}

extern "C" int mph_set_step_graphs(mph_ctx* ctx, int enable) {
    if (!ctx) return fail(nullptr, MPH_ERR_ARG, "ctx is NULL");
    ctx->sg.enabled = enable != 0;
    if (!enable) drop_step_graphs(ctx);
    return MPH_OK;
}

extern "C" int mph_synchronize(mph_ctx* ctx) {
    if (!ctx) return fail(nullptr, MPH_ERR_ARG, "ctx is NULL");
    TRY(read_scalars(ctx));
    return check_flags(ctx);
}

// The mixed form keeps its own particle order between rebuilds; bring the
// FP64 buffers up to date before any read-back.
static int sync_state(mph_ctx* ctx) {
    ensure_density_a(ctx);
    ensure_wall_force(ctx);
    if (ctx->mixed) {
        Launch L(ctx, "mix_export");
        const int rc = mph::mixed_export(ctx->mixed, ctx->sc, ctx->d, ctx->stream, &ctx->err, &L.count);
        if (rc != MPH_OK) return fail(ctx, rc, ctx->err);
    }
    return MPH_OK;
}

extern "C" int mph_get_info(mph_ctx* ctx, mph_info* info) {
    if (!ctx || !info) return fail(ctx, MPH_ERR_ARG, "bad arguments");
    TRY(sync_state(ctx));
    std::memset(info, 0, sizeof(*info));
    info->particle_count = ctx->n;
    int cs[3] = {0, 0, 0};
    const int tot = ctx->sc.tot;
    CUDA_TRY(ctx, cudaMemcpyAsync(&cs[0], ctx->d.cellstart, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(&cs[1], ctx->d.cellstart + tot, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(&cs[2], ctx->d.cellstart + 2 * tot, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    std::vector<int> nc(ctx->n);
    CUDA_TRY(ctx, cudaMemcpyAsync(nc.data(), ctx->d.ncount, nc.size() * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    long long total = 0;
    for (int v : nc) total += v;
    info->fluid_particle_begin = cs[0];
    info->fluid_particle_end = cs[1];
    info->wall_particle_begin = cs[1];
    info->wall_particle_end = cs[2];
    info->neighbor_ind_count = total;
    info->max_neighbor_count = ctx->mixed ? mph::mixed_max_neighbors(ctx->mixed) : ctx->max_neighbors;
    info->neighbor_capacity = ctx->mixed ? mph::mixed_capacity(ctx->mixed) : ctx->d.cap;
    info->step = ctx->step;
    info->rebuild_count = ctx->rebuilds;
    info->time = ctx->time;
    info->mode = ctx->mode | (ctx->cell_walk ? MPH_MIXED_CELL_WALK : 0);
    return MPH_OK;
}

extern "C" int mph_get_constants(mph_ctx* ctx, mph_constants* c) {
    if (!ctx || !c) return fail(ctx, MPH_ERR_ARG, "bad arguments");
    *c = ctx->c;
    return MPH_OK;
}

static int d2h_vec3(mph_ctx* ctx, const double4* src, double* dst) {
    { Launch L(ctx, "pack3"); mph::launch_pack3(ctx->n, src, ctx->d.staging, ctx->stream); }
    CUDA_TRY(ctx, cudaMemcpyAsync(dst, ctx->d.staging, 3 * (size_t)ctx->n * sizeof(double), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return MPH_OK;
}

template <class T>
static int d2h(mph_ctx* ctx, T* dst, const T* src, size_t count) {
    if (!dst) return MPH_OK;
    CUDA_TRY(ctx, cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
    return MPH_OK;
}

extern "C" int mph_get_state(mph_ctx* ctx, int* particle_index, int* type, double* xyz, double* vel, double* force,
                             int* neighbor_count, double* density_a, double* vol_strain_p, double* virial_pressure) {
    if (!ctx) return fail(nullptr, MPH_ERR_ARG, "ctx is NULL");
    // the mixed forms compute these output-only arrays on demand
    if (force || neighbor_count || density_a) TRY(sync_state(ctx));
    mph::DevFP64& d = ctx->d;
    const size_t n = (size_t)ctx->n;
    TRY(d2h(ctx, particle_index, d.pidx[d.cur], n));
    TRY(d2h(ctx, type, d.type[d.cur], n));
    TRY(d2h(ctx, neighbor_count, d.ncount, n));
    TRY(d2h(ctx, density_a, d.dens_a, n));
    TRY(d2h(ctx, vol_strain_p, d.strain_p, n));
    TRY(d2h(ctx, virial_pressure, d.virial_p, n));
    if (xyz) TRY(d2h_vec3(ctx, d.pos[d.cur], xyz));
    if (vel) TRY(d2h_vec3(ctx, d.vel[d.vcur], vel));
    if (force) TRY(d2h_vec3(ctx, d.force, force));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return MPH_OK;
}

static int readback_init(mph_ctx* ctx) {
    ReadBack& R = ctx->rb;
    if (R.copy) return MPH_OK;
    CUDA_TRY(ctx, cudaStreamCreateWithFlags(&R.copy, cudaStreamNonBlocking));
    for (cudaEvent_t& e : R.ev) CUDA_TRY(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    TRY(dalloc(ctx, &R.stage_v, 3 * (size_t)ctx->n));
    return MPH_OK;
}

// The device address of a host buffer of `count` doubles when all of it is
// pinned and mapped (cudaHostAlloc memory always is under unified addressing;
// cudaHostRegister memory when registered mapped), else nullptr.
static double* mapped_host(double* p, size_t count) {
    if (!p || count == 0) return nullptr;
    cudaPointerAttributes a{}, b{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess || cudaPointerGetAttributes(&b, p + count - 1) != cudaSuccess) {
        cudaGetLastError();  // pageable memory on older runtimes reports an error: not an error here
        return nullptr;
    }
    if (a.type != cudaMemoryTypeHost || b.type != cudaMemoryTypeHost || !a.devicePointer || !b.devicePointer)
        return nullptr;
    if ((char*)b.devicePointer - (char*)a.devicePointer != (ptrdiff_t)((count - 1) * sizeof(double))) return nullptr;
    return (double*)a.devicePointer;
}

// The FP64 form's last step with its read-back overlapped.  The positions are
// final once the move and any rebuild are done: they are packed and copied on
// a copy stream while the sweeps run.  The velocities: with a pinned, mapped
// host buffer the force sweep stores each particle's new velocity into it as
// well as into device memory (24 B per particle over PCIe while the sweep
// runs); otherwise they are packed and copied after the sweep.  Same kernels
// and inputs: the bits of mph_step + mph_get_state.
static int step_fp64_read(mph_ctx* ctx, double* xyz, double* vel) {
    TRY(readback_init(ctx));
    ReadBack& R = ctx->rb;
    mph::DevFP64& d = ctx->d;
    const SimConst& s = ctx->sc;
    cudaStream_t st = ctx->stream;
    const size_t n = (size_t)ctx->n;
    double* vh = mapped_host(vel, 3 * n);
    TRY(step_fp64_head(ctx));
    CUDA_TRY(ctx, cudaEventRecord(R.ev[0], st));  // positions final
    sweep_a(ctx, true);
    double4* vout = d.vel[1 - d.vcur];
    {
        Launch L(ctx, "sweep_b");
        const bool sl = uses_short_list(ctx);
        mph::launch_sweep_b(s, d.cellstart, d.pos[d.cur], d.vel[d.vcur], vout, d.press, d.gc, d.ncount, d.nlist,
                            sl ? d.ncount_s : nullptr, sl ? d.nlist_s : nullptr, d.force, d.scal, st, nullptr,
                            nullptr, nullptr, 1, 0, -1, vh);
        ctx->wall_force_valid = false;  // computed when read
    }
    CUDA_TRY(ctx, cudaEventRecord(R.ev[1], st));  // velocities final
    // copies, enqueued after the compute so pageable buffers do not hold it back
    if (xyz) {
        CUDA_TRY(ctx, cudaStreamWaitEvent(R.copy, R.ev[0], 0));
        mph::launch_pack3(ctx->n, d.pos[d.cur], d.staging, R.copy);
        ++ctx->launches;
        CUDA_TRY(ctx, cudaMemcpyAsync(xyz, d.staging, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, R.copy));
    }
    if (vel && !vh) {
        CUDA_TRY(ctx, cudaStreamWaitEvent(R.copy, R.ev[1], 0));
        mph::launch_pack3(ctx->n, vout, R.stage_v, R.copy);
        ++ctx->launches;
        CUDA_TRY(ctx, cudaMemcpyAsync(vel, R.stage_v, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, R.copy));
    }
    d.vcur = 1 - d.vcur;
    CUDA_TRY(ctx, cudaGetLastError());
    ctx->time += ctx->p.dt;  // main.cpp:449
    ++ctx->step;
    ctx->virial_valid = false;
    CUDA_TRY(ctx, cudaStreamSynchronize(R.copy));
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return MPH_OK;
}

extern "C" int mph_step_read_state(mph_ctx* ctx, int nsteps, double* xyz, double* vel) {
    if (!ctx || nsteps < 1) return fail(ctx, MPH_ERR_ARG, "bad arguments");
    if (ctx->mixed || ctx->mode == MPH_MODE_LEARNED) {  // no overlap: the step, then the read
        TRY(mph_step(ctx, nsteps));
        return mph_get_state(ctx, nullptr, nullptr, xyz, vel, nullptr, nullptr, nullptr, nullptr, nullptr);
    }
    if (nsteps > 1) TRY(step_fp64(ctx, nsteps - 1));
    return step_fp64_read(ctx, xyz, vel);
}

extern "C" int mph_set_state(mph_ctx* ctx, const double* xyz, const double* vel) {
    if (!ctx) return fail(nullptr, MPH_ERR_ARG, "ctx is NULL");
    mph::DevFP64& d = ctx->d;
    const size_t n = (size_t)ctx->n;
    cudaStream_t st = ctx->stream;
    // The last step's output-only fields (DensityA without surface tension, the
    // walls' Force) are computed when read, from the positions that step used:
    // keep a copy of those in the idle ping-pong buffer before they are replaced.
    if (xyz && !ctx->mixed && ctx->lazy_pos < 0 && (!ctx->dens_a_valid || !ctx->wall_force_valid)) {
        CUDA_TRY(ctx, cudaMemcpyAsync(d.pos[1 - d.cur], d.pos[d.cur], n * sizeof(double4), cudaMemcpyDeviceToDevice,
                                      st));
        ctx->lazy_pos = 1 - d.cur;
    }
    // with the read-back's velocity buffer (made by mph_step_read_state) both
    // copies are queued before the unpacks, back to back on the copy engine
    double* sv = (xyz && vel && ctx->rb.stage_v) ? ctx->rb.stage_v : nullptr;
    if (xyz) CUDA_TRY(ctx, cudaMemcpyAsync(d.staging, xyz, 3 * n * sizeof(double), cudaMemcpyHostToDevice, st));
    if (sv) CUDA_TRY(ctx, cudaMemcpyAsync(sv, vel, 3 * n * sizeof(double), cudaMemcpyHostToDevice, st));
    if (xyz) {
        Launch L(ctx, "unpack3");
        mph::launch_unpack3(ctx->n, d.staging, d.pos[d.cur], d.type[d.cur], st);
    }
    if (vel) {
        if (!sv) {
            sv = d.staging;
            CUDA_TRY(ctx, cudaMemcpyAsync(sv, vel, 3 * n * sizeof(double), cudaMemcpyHostToDevice, st));
        }
        Launch L(ctx, "unpack3");
        mph::launch_unpack3(ctx->n, sv, d.vel[d.vcur], nullptr, st);
    }
    if (ctx->mixed) TRY(mph::mixed_import(ctx->mixed, ctx->sc, ctx->d, st, &ctx->err));
    CUDA_TRY(ctx, cudaGetLastError());
    return MPH_OK;
}

extern "C" int mph_get_fields(mph_ctx* ctx, double* divergence_p, double* pressure_p, double* pressure_a,
                              double* gravity_center) {
    if (!ctx) return fail(nullptr, MPH_ERR_ARG, "ctx is NULL");
    TRY(sync_state(ctx));
    mph::DevFP64& d = ctx->d;
    const size_t n = (size_t)ctx->n;
    TRY(d2h(ctx, divergence_p, d.div_p, n));
    if (pressure_p || pressure_a) {  // PressureP rides in velp.w, PressureA in gc.w
        std::vector<double4> vp(n), ga(n);
        CUDA_TRY(ctx, cudaMemcpyAsync(vp.data(), d.press, n * sizeof(double4), cudaMemcpyDeviceToHost, ctx->stream));
        CUDA_TRY(ctx, cudaMemcpyAsync(ga.data(), d.gc, n * sizeof(double4), cudaMemcpyDeviceToHost, ctx->stream));
        CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        for (size_t i = 0; i < n; ++i) {
            if (pressure_p) pressure_p[i] = vp[i].w;
            if (pressure_a) pressure_a[i] = ga[i].w;
        }
    }
    if (gravity_center) TRY(d2h_vec3(ctx, d.gc, gravity_center));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return MPH_OK;
}

extern "C" int mph_get_cells(mph_ctx* ctx, int* cell_index, int* fb, int* fe, int* wb, int* we) {
    if (!ctx) return fail(nullptr, MPH_ERR_ARG, "ctx is NULL");
    if (ctx->mixed) return fail(ctx, MPH_ERR_STATE, "cell data is kept by the FP64 form only");
    const int tot = ctx->sc.tot;
    std::vector<int> cs(2 * (size_t)tot + 1);
    TRY(d2h(ctx, cell_index, ctx->d.keys, (size_t)ctx->n));
    CUDA_TRY(ctx, cudaMemcpyAsync(cs.data(), ctx->d.cellstart, cs.size() * sizeof(int), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    for (int c = 0; c < tot; ++c) {
        if (fb) fb[c] = cs[c];
        if (fe) fe[c] = cs[c + 1];
        if (wb) wb[c] = cs[c + tot];
        if (we) we[c] = cs[c + tot + 1];
    }
    return MPH_OK;
}

extern "C" int mph_get_neighbors(mph_ctx* ctx, long long* ptr, int* ind, long long ind_capacity) {
    if (!ctx || !ptr) return fail(ctx, MPH_ERR_ARG, "bad arguments");
    if (ctx->mixed) return fail(ctx, MPH_ERR_STATE, "the neighbour list is kept by the FP64 form only");
    const size_t n = (size_t)ctx->n;
    std::vector<int> nc(n);
    CUDA_TRY(ctx, cudaMemcpyAsync(nc.data(), ctx->d.ncount, n * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    ptr[0] = 0;
    for (size_t i = 0; i < n; ++i) ptr[i + 1] = ptr[i] + nc[i];
    if (!ind) return MPH_OK;
    if (ptr[n] > ind_capacity) return fail(ctx, MPH_ERR_ARG, "ind_capacity too small");
    const int cap = ctx->d.cap;
    std::vector<int> tab((size_t)cap * n);
    CUDA_TRY(ctx, cudaMemcpyAsync(tab.data(), ctx->d.nlist, tab.size() * sizeof(int), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < nc[i]; ++k) ind[ptr[i] + k] = tab[(size_t)k * n + i];
    return MPH_OK;
}

extern "C" int mph_compute_virial(mph_ctx* ctx) {
    if (!ctx) return fail(nullptr, MPH_ERR_ARG, "ctx is NULL");
    mph::DevFP64& d = ctx->d;
    if (ctx->mixed) {  // FP32 pair terms over the mixed form's own table (output only)
        TRY(sync_state(ctx));
        {
            Launch L(ctx, "mix_virial");
            const int rc = mph::mixed_virial(ctx->mixed, ctx->sc, d, ctx->stream, &ctx->err);
            if (rc != MPH_OK) return fail(ctx, rc, ctx->err);
        }
        CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        ctx->virial_valid = true;
        return MPH_OK;
    }
    ensure_density_a(ctx);  // the virial reads PressureA
    {
        Launch L(ctx, "virial");
        mph::launch_virial(ctx->sc, d.pos[d.cur], d.vel[d.vcur], d.press, d.gc, d.ncount, d.nlist, d.virial_p,
                           ctx->stream);
    }
    CUDA_TRY(ctx, cudaGetLastError());
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->virial_valid = true;
    return MPH_OK;
}

// ---- output files, formatted on the device ----------------------------------
static int text_submit(mph_ctx* ctx, mph::TextDoc& doc, const char* path, const char* what) {
    if (!ctx->text) {
        int dev = 0;
        CUDA_TRY(ctx, cudaGetDevice(&dev));
        try {
            ctx->text = new mph::TextWriter(dev);
        } catch (const std::exception& e) {  // no exception crosses the C ABI
            return fail(ctx, MPH_ERR_NOMEM, std::string("text writer thread: ") + e.what());
        }
    }
    std::string err;
    Launch L(ctx, what);
    const int st = ctx->text->submit(doc, ctx->stream, path, &err, &L.count);
    if (st != MPH_OK) return fail(ctx, st, err);
    return MPH_OK;
}

// writeVtkFile (main.cpp:698-834): the same sections, each particle's lines
// formatted by the device in the context's (cell-sorted) order.
extern "C" int mph_write_vtk_async(mph_ctx* ctx, const char* path) {
    if (!ctx || !path) return fail(ctx, MPH_ERR_ARG, "bad arguments");
    TRY(sync_state(ctx));
    mph::DevFP64& d = ctx->d;
    const int n = ctx->n;
    char h[256];
    mph::TextDoc doc;
    doc.nsec = doc.nblocks = doc.head_used = 0;
    bool ok = true;
    std::snprintf(h, sizeof(h),
                  "# vtk DataFile Version 2.0\nUnstructured Grid Example\nASCII\nDATASET UNSTRUCTURED_GRID\n"
                  "POINTS %d float\n", n);
    ok &= mph::text_add(doc, h, mph::kRecVec3f, n, d.pos[d.cur]);
    std::snprintf(h, sizeof(h), "CELLS %d %d\n", n, 2 * n);
    ok &= mph::text_add(doc, h, mph::kRecCell, n);
    std::snprintf(h, sizeof(h), "\nCELL_TYPES %d\n", n);
    ok &= mph::text_add(doc, h, mph::kRecOne, n);
    std::snprintf(h, sizeof(h), "\n\nPOINT_DATA %d\nSCALARS label float 1\nLOOKUP_TABLE default\n", n);
    ok &= mph::text_add(doc, h, mph::kRecInt, n, d.type[d.cur]);
    ok &= mph::text_add(doc, "\nSCALARS DensityA float 1\nLOOKUP_TABLE default\n", mph::kRecScalarf, n, d.dens_a);
    ok &= mph::text_add(doc, "\nSCALARS VolStrainP float 1\nLOOKUP_TABLE default\n", mph::kRecScalarf, n,
                        d.strain_p);
    ok &= mph::text_add(doc, "\nSCALARS VirialPressureAtParticle float 1\nLOOKUP_TABLE default\n",
                        mph::kRecScalarf, n, d.virial_p);
    ok &= mph::text_add(doc, "\nSCALARS neighbor float 1\nLOOKUP_TABLE default\n", mph::kRecInt, n, d.ncount);
    ok &= mph::text_add(doc, "\nVECTORS velocity float\n", mph::kRecVec3f, n, d.vel[d.vcur]);
    ok &= mph::text_add(doc, "\nVECTORS force float\n", mph::kRecVec3f, n, d.force);
    ok &= mph::text_add(doc, "\n", mph::kRecNone, 0);
    if (!ok) return fail(ctx, MPH_ERR_STATE, "vtk document does not fit its tables");
    return text_submit(ctx, doc, path, "text_vtk");
}

// writeProfFile (main.cpp:672-696), formatted by the device.
extern "C" int mph_write_prof_async(mph_ctx* ctx, const char* path) {
    if (!ctx || !path) return fail(ctx, MPH_ERR_ARG, "bad arguments");
    mph::DevFP64& d = ctx->d;
    const mph_grid_header& g = ctx->h;
    char h[256];
    std::snprintf(h, sizeof(h), "%e\n%d %e %e %e %e %e %e %e\n", ctx->time, g.particle_count, g.particle_spacing,
                  g.domain_min[0], g.domain_max[0], g.domain_min[1], g.domain_max[1], g.domain_min[2],
                  g.domain_max[2]);
    mph::TextDoc doc;
    doc.nsec = doc.nblocks = doc.head_used = 0;
    if (!mph::text_add(doc, h, mph::kRecProf, ctx->n, d.pos[d.cur], d.vel[d.vcur], d.type[d.cur]))
        return fail(ctx, MPH_ERR_STATE, "prof document does not fit its tables");
    return text_submit(ctx, doc, path, "text_prof");
}

extern "C" int mph_output_wait(mph_ctx* ctx) {
    if (!ctx) return fail(nullptr, MPH_ERR_ARG, "ctx is NULL");
    if (!ctx->text) return MPH_OK;
    std::string err;
    const int st = ctx->text->wait(&err);
    if (st != MPH_OK) return fail(ctx, st, err);
    return MPH_OK;
}

extern "C" int mph_write_vtk(mph_ctx* ctx, const char* path) {
    TRY(mph_write_vtk_async(ctx, path));
    return mph_output_wait(ctx);
}

extern "C" int mph_write_vtk_arrays(const char* path, int n, const int* type, const double* xyz, const double* vel,
                                    const double* force, const int* neighbor_count, const double* density_a,
                                    const double* vol_strain_p, const double* virial_pressure) {
    if (!path || n < 0 || (n > 0 && (!type || !xyz || !vel || !force || !neighbor_count || !density_a ||
                                     !vol_strain_p || !virial_pressure)))
        return fail(nullptr, MPH_ERR_ARG, "bad arguments");
    const int st = mph::write_vtk_host(path, n, type, xyz, vel, force, neighbor_count, density_a, vol_strain_p,
                                       virial_pressure);
    if (st != MPH_OK) return fail(nullptr, st, std::string("cannot write ") + path);
    return MPH_OK;
}

extern "C" int mph_write_prof(mph_ctx* ctx, const char* path) {
    TRY(mph_write_prof_async(ctx, path));
    return mph_output_wait(ctx);
}

extern "C" int mph_write_checkpoint(mph_ctx* ctx, const char* path) {
    if (!ctx || !path) return fail(ctx, MPH_ERR_ARG, "bad arguments");
    const size_t n = (size_t)ctx->n;
    std::vector<int> type(n), pidx(n);
    std::vector<double> x(3 * n), v(3 * n);
    TRY(mph_get_state(ctx, pidx.data(), type.data(), x.data(), v.data(), nullptr, nullptr, nullptr, nullptr, nullptr));
    double wc[12];
    CUDA_TRY(ctx, cudaMemcpyAsync(wc, ctx->d.wall_center, sizeof(wc), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    mph_params p = ctx->p;
    for (int t = 2; t < MPH_TYPE_COUNT; ++t)  // the wall centres reached (calculateWall, main.cpp:2013-2053)
        for (int k = 0; k < 3; ++k) p.wall_center[t][k] = wc[3 * t + k];
    mph_grid_header h = ctx->h;
    h.time = ctx->time;
    const int st = mph_write_checkpoint_arrays(path, &p, &h, ctx->dim, ctx->step, type.data(), pidx.data(), x.data(),
                                               v.data());
    if (st != MPH_OK) return fail(ctx, st, std::string("cannot write ") + path);
    return MPH_OK;
}

extern "C" int mph_conserved_sums(mph_ctx* ctx, double out[5]) {
    if (!ctx || !out) return fail(ctx, MPH_ERR_ARG, "bad arguments");
    TRY(sync_state(ctx));
    mph::DevFP64& d = ctx->d;
    const int nb = (ctx->n + 255) / 256;
    double* part = nullptr;
    TRY(dalloc(ctx, &part, 5 * (size_t)nb));
    { Launch L(ctx, "conserved"); mph::launch_conserved(ctx->sc, d.cellstart, d.pos[d.cur], d.vel[d.vcur], part, ctx->stream); }
    std::vector<double> h(5 * (size_t)nb);
    cudaError_t e = cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(part);
    if (e != cudaSuccess) return fail(ctx, MPH_ERR_CUDA, cudaGetErrorString(e));
    for (int k = 0; k < 5; ++k) out[k] = 0.0;
    for (int b = 0; b < nb; ++b)
        for (int k = 0; k < 5; ++k) out[k] += h[5 * (size_t)b + k];
    return MPH_OK;
}

extern "C" int mph_check_exact_division(long long n, unsigned long long seed, long long* mismatches,
                                        double* first) {
    if (!mismatches || n < 0) return fail(nullptr, MPH_ERR_ARG, "bad arguments");
    unsigned long long* d_count = nullptr;
    double* d_first = nullptr;
    cudaError_t e = cudaMalloc((void**)&d_count, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc((void**)&d_first, 2 * sizeof(double));
    if (e == cudaSuccess) e = cudaMemset(d_count, 0, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(d_first, 0, 2 * sizeof(double));
    if (e == cudaSuccess) {
        mph::check_division(seed, n, d_count, d_first, 0);
        e = cudaGetLastError();
    }
    unsigned long long cnt = 0;
    double f[2] = {0.0, 0.0};
    if (e == cudaSuccess) e = cudaMemcpy(&cnt, d_count, sizeof(cnt), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(f, d_first, sizeof(f), cudaMemcpyDeviceToHost);
    if (d_count) cudaFree(d_count);
    if (d_first) cudaFree(d_first);
    if (e != cudaSuccess) return fail(nullptr, MPH_ERR_CUDA, cudaGetErrorString(e));
    *mismatches = (long long)cnt;
    if (first) { first[0] = f[0]; first[1] = f[1]; }
    return MPH_OK;
}

extern "C" void* mph_stream(mph_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

extern "C" long long mph_launch_count(mph_ctx* ctx) { return ctx ? ctx->launches : -1; }

static int profile_collect(mph_ctx* ctx) {
    Profiler& p = ctx->prof;
    if (p.pending.empty()) return MPH_OK;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    for (const auto& q : p.pending) {
        float ms = 0.0f;
        CUDA_TRY(ctx, cudaEventElapsedTime(&ms, q.a, q.b));
        p.ms[q.id] += ms;
        p.launches[q.id] += q.count;
        p.pool.push_back(q.a);
        p.pool.push_back(q.b);
    }
    p.pending.clear();
    return MPH_OK;
}

extern "C" int mph_profile_enable(mph_ctx* ctx, int enable) {
    if (!ctx) return fail(nullptr, MPH_ERR_ARG, "ctx is NULL");
    TRY(profile_collect(ctx));
    Profiler& p = ctx->prof;
    p.on = enable != 0;
    if (p.on) {
        p.names.clear();
        p.launches.clear();
        p.ms.clear();
    }
    return MPH_OK;
}

extern "C" int mph_profile_read(mph_ctx* ctx, mph_kernel_stat* out, int capacity, int* count) {
    if (!ctx || !count || (capacity > 0 && !out)) return fail(ctx, MPH_ERR_ARG, "bad arguments");
    TRY(profile_collect(ctx));
    const Profiler& p = ctx->prof;
    *count = (int)p.names.size();
    for (int k = 0; k < (int)p.names.size() && k < capacity; ++k) {
        std::snprintf(out[k].name, sizeof(out[k].name), "%s", p.names[k].c_str());
        out[k].launches = p.launches[k];
        out[k].total_ms = p.ms[k];
    }
    return MPH_OK;
}

extern "C" int mph_last_error(mph_ctx* ctx, char* buf, int len) {
    if (!buf || len <= 0) return MPH_ERR_ARG;
    const std::string& m = ctx ? ctx->err : g_err;
    std::snprintf(buf, (size_t)len, "%s", m.c_str());
    return MPH_OK;
}

extern "C" const char* mph_version(void) { return "mph_b200 0.1 (sm_100a)"; }
