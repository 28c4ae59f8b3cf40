// mph_internal.h — device constants, context layout and kernel launchers of the
// B200 MPH-WC explicit step.  Shared by the host orchestration (mph_host.cpp)
// and the CUDA translation units (k_cells.cu, k_fp64.cu, k_mixed.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include "mph_b200.h"

namespace mph {

// Everything a step kernel needs that is fixed between rebuilds, passed by
// value (kernel parameter space) so no constant-memory upload is needed.
// The kernel-shape prefactors are evaluated on the host in the reference's
// operation order (main.cpp:214-284): e.g. wa = ((ca*q)*(1-q))*(1-q) with
// ca = (1/Swa)/h^D and q = r/h.
struct SimConst {
    int n;                 // particle count
    int dim;
    int tot;               // TotalCellCount
    int cc[3];             // CellCount
    int range[3];          // stencil half-width per axis (1, or 0 for z in 2-D)
    int pow2;              // PowerParticleCount
    int has_st;            // any surface tension -> diffuse-interface terms
    int ratio_all_one;     // InteractionRatio == 1 everywhere
    double dmin[3], width[3], half_width[3], cell_width[3];
    // bits of 0.75*width: Mod(x, w) needs no division when 0 <= x < 0.75 w,
    // tested as one unsigned compare of x's bit pattern (negative x, -0.0
    // and NaN have the sign bit set and compare above every positive bound)
    unsigned long long q75_bits[3];
    double dt, l0, vol, vol_over_l0;
    double n0a, n0p, r2g, cof_k;
    double ra, rg, rp, rv;             // radii
    double ra2, rg2, rp2, rv2;         // radius*radius
    double rm2;                        // (MaxRadius+MARGIN)^2, neighbour cut-off
    double rs2;                        // ((RadiusP+MARGIN)(1+1e-9))^2, cut-off of the short sublist
    double ca, cg, cp, cv;             // (1/Sw)/h^D for wa, wg/dwg, wp/dwp, dwv
    double inv_ra, inv_rg, inv_rp, inv_rv;  // 1.0/h
    double m2_rg, m2_rp, m2_rv;        // -2.0/h
    double visc_c;                     // 8 (2-D) or 10 (3-D)
    double inv_r2g;                    // RN(1/R2g)
    int rg_eq_ra, rv_eq_ra;            // radii equal: r/h shared
    int sweep_layout;                  // FP64 sweeps: 0 by size, 1 thread per particle, 2 warp per particle
    // visc_c * muij per type pair, muij = 2*(mu_i*mu_j)/(mu_i+mu_j) (main.cpp:1968)
    double visc_mu[MPH_TYPE_COUNT][MPH_TYPE_COUNT];
    double shift_thr;                  // 0.5*MARGIN*0.5*MARGIN
    double density[MPH_TYPE_COUNT], bulk_modulus[MPH_TYPE_COUNT];
    double bulk_viscosity[MPH_TYPE_COUNT], shear_viscosity[MPH_TYPE_COUNT];
    double cof_a[MPH_TYPE_COUNT], a_k[MPH_TYPE_COUNT];  // a_k = CofA*CofK*CofK
    double ratio[MPH_TYPE_COUNT][MPH_TYPE_COUNT];
    double gravity[3];
    double wall_velocity[MPH_TYPE_COUNT][3], wall_omega[MPH_TYPE_COUNT][3];
    double wall_rot[MPH_TYPE_COUNT][3][3];
};

// Small per-step device scalars (one cache line, read back with one copy).
struct StepScalars {
    unsigned long long max_shift2_bits;  // max |shift|^2 as ordered bits (>= 0)
    int flags;                           // MPH_DEVFLAG_*
    int max_neighbors;                   // longest list of the last build
    int rebuild;                         // decision of the last move kernel
    int max_short, max_long;             // longest short / long part (mixed table)
    int stop;                            // step graphs: a list overflowed, the later steps skip
    int steps_done;                      // step graphs: steps started (moved) in this batch
    int rebuilds_done;                   // step graphs: rebuilds started in this batch
    unsigned blocks_done;                // step graphs: move blocks finished in this launch
    int pad[5];
};

enum : int {
    DEVFLAG_NEIGHBOR_OVERFLOW = 1,
    DEVFLAG_NONFINITE = 2,
    DEVFLAG_CELL_RANGE = 4,
};

// Device buffers of the FP64 form.  Arrays are in cell-sorted order.
struct DevFP64 {
    int* pidx[2] = {nullptr, nullptr};
    int* type[2] = {nullptr, nullptr};
    double4* pos[2] = {nullptr, nullptr};   // x,y,z,(double)type
    double4* vel[2] = {nullptr, nullptr};   // vx,vy,vz,0
    int cur = 0;                            // index of the current pos/type/pidx
    int vcur = 0;                           // index of the current velocity
    double4* snap = nullptr;                // NeighborCalculatedPosition
    float4* pos32 = nullptr;                // FP32 x - dmin for the list build's prefilter
    double4* force = nullptr;
    double* dens_a = nullptr;
    double* strain_p = nullptr;
    double* div_p = nullptr;
    double4* press = nullptr;               // {vx, vy, vz, PressureP} before the acceleration
    double4* gc = nullptr;                  // {GravityCenter, PressureA}
    double* virial_p = nullptr;
    int* keys = nullptr;                    // CellIndex (sorted), pow2 entries
    int* vals = nullptr;                    // CellParticle, pow2 entries
    int* cellstart = nullptr;               // 2*tot+1: #keys below each key value
    int* ncount = nullptr;                  // NeighborCount
    int* nlist = nullptr;                   // [cap][n] column-major list
    int cap = 0;
    int* ncount_s = nullptr;                // short sublist: the entries
    int* nlist_s = nullptr;                 // within rs2, in list order, [cap_s][n]
    int cap_s = 0;
    double* wall_center = nullptr;          // [4][3], advanced on the device
    double* staging = nullptr;              // [n][3] pack/unpack buffer
    StepScalars* scal = nullptr;
};

// ---- kernel launchers (k_cells.cu) ----------------------------------------
void launch_cell_index(const SimConst& c, const double4* pos, const int* type, int* keys,
                       int* vals, cudaStream_t s);
int launch_bitonic_sort(const SimConst& c, int* keys, int* vals, cudaStream_t s);  // returns #launches
void launch_cell_ranges(const SimConst& c, const int* keys, int* cellstart, cudaStream_t s);
void launch_reorder(const SimConst& c, const int* vals, const int* pidx_in, const int* type_in,
                    const double4* pos_in, const double4* vel_in, int* pidx_out, int* type_out,
                    double4* pos_out, double4* vel_out, double4* snap, cudaStream_t s);
// FP32 prefilter of the neighbour-list build: per axis whether it takes part,
// the domain width, and the FP32 distance squared above which no candidate
// can pass the exact FP64 test.
struct Prefilter {
    int use[3];
    float width[3];
    float r2_hi;   // per pair: FP32 distance squared at or below it for every pair within rm
    float r2_box;  // per candidate: FP32 distance squared to the box around a warp's particles
    float r2_lo;   // FP32 distance squared at or below it: within rm in FP64 for certain (-1: never)
    float rs2_lo, rs2_hi;  // the same two bounds for the short radius rs
};
Prefilter make_prefilter(const SimConst& c);
// FP32 positions relative to the domain origin (the prefilter's input).
void launch_pos32(const SimConst& c, const double4* pos, float4* pos32, cudaStream_t s);
// nlist_s != nullptr: also the short sublist (entries within rs2, in list
// order; its longest length in scal->max_short).  pos32 (launch_pos32) feeds
// the FP32 prefilter that skips candidates surely beyond the cut-off (the
// list is the same).  One warp per cell key.
void launch_neighbor_list(const SimConst& c, const double4* pos, const float4* pos32, const int* cellstart,
                          int* ncount, int* nlist, int cap, int* ncount_s, int* nlist_s, int cap_s,
                          StepScalars* scal, cudaStream_t s);
void launch_pack3(int n, const double4* src, double* dst, cudaStream_t s);

// ---- step graphs (FP64 form) ------------------------------------------------
// after a list build: a list longer than its table stops the batch (sweep = 0)
void launch_graph_list_check(StepScalars* scal, int cap, int cap_s, int short_list,
                             cudaGraphConditionalHandle sweep, cudaStream_t s);
// the move of a step graph (k_fp64.cu): as launch_move, and its last block
// makes the rebuild test of main.cpp:1102 (rebuild = 1 when it fires; sweep =
// 1 unless the batch stopped, when the move does nothing), counts the step
// and clears the maximum shift for the next step
void launch_move_graph(const SimConst& c, const int* cellstart, double4* pos, double4* vel, const double4* snap,
                       const double* wall_center, StepScalars* scal, cudaGraphConditionalHandle rebuild,
                       cudaGraphConditionalHandle sweep, cudaStream_t s);
void launch_unpack3(int n, const double* src, double4* dst, const int* type, cudaStream_t s);

// ---- kernel launchers (k_fp64.cu) -----------------------------------------
void launch_move(const SimConst& c, const int* cellstart, double4* pos, double4* vel,
                 const double4* snap, const double* wall_center, StepScalars* scal,
                 cudaStream_t s);
// Sweep A's DensityP and DivergenceP visit the short sublist (ncount_s,
// nlist_s); with surface tension DensityA and GravityCenter the whole list.
void launch_sweep_a(const SimConst& c, const int* cellstart, const double4* pos,
                    const double4* vel, const int* ncount, const int* nlist, const int* ncount_s,
                    const int* nlist_s, double* dens_a, double* strain_p, double* div_p, double4* press,
                    double4* gc, double* wall_center, cudaStream_t s);
// DensityA and PressureA alone (into dens_a and gc[].w), in k_sweep_a's
// order: what sweep A leaves out when there is no surface tension.
void launch_density_a(const SimConst& c, const double4* pos, const int* ncount, const int* nlist, double* dens_a,
                      double4* gc, cudaStream_t s);
// eforce != nullptr: the learned form (edge-MLP pair forces replace the
// PressureA, DiffuseInterface and ViscosityV terms; see k_sweep_b; it then
// needs only the pairs within RadiusP, so the short sublist may be passed).
// part: 0 every particle; 1 the fluid (walls copy their velocity, their
// force is not written); 2 the walls' forces alone (vel_out unused).
// ncount_s / nlist_s (not learned): the short sublist, over which the
// PressureP force runs as its own loop (same result).
// [i0, i1): the particles (sorted order) this launch computes; i1 < 0 means
// all n.  Every particle's result depends on the inputs alone, so a sweep
// split into ranges gives the same bits as one launch.  vel_host (part 1): a
// device-accessible [n][3] view of pinned host memory that also receives
// each particle's new velocity.
void launch_sweep_b(const SimConst& c, const int* cellstart, const double4* pos,
                    const double4* vel_in, double4* vel_out, const double4* press,
                    const double4* gc, const int* ncount, const int* nlist, const int* ncount_s,
                    const int* nlist_s, double4* force, StepScalars* scal, cudaStream_t s,
                    const int* eoff = nullptr, const float4* eforce = nullptr, float4* lsum = nullptr,
                    int part = 0, int i0 = 0, int i1 = -1, double* vel_host = nullptr);

// ---- learned form (k_fp64.cu) ---------------------------------------------
// CSR edges of the fluid particles' lists (i < nf): eoff[0..nf] = exclusive
// prefix of ncount (bsum: scratch of edge_scan_blocks(nf) ints), then
// ei/ej = (i, list entry) for every edge, self entries included.
int edge_scan_blocks(int nf);
void launch_edge_offsets(const int* ncount, int nf, int* eoff, int* bsum, cudaStream_t s);
void launch_edge_fill(const int* ncount, const int* nlist, int n, int nf, const int* eoff, int* ei, int* ej,
                      cudaStream_t s);
// `count` training samples (3 float4 each) of edges drawn at random from the
// ne CSR edges: features of the pair and its FP64 PressureA + DiffuseInterface
// + ViscosityV force on i as target (valid = 0 outside every radius or j == i)
void launch_collect(const SimConst& c, const double4* pos, const double4* press, const double4* gc,
                    const int* ei, const int* ej, long long ne, long long count, unsigned long long seed,
                    float4* out, cudaStream_t s);
// sums over fluid particles of |F_a - F_b|^2, |F_b|^2, |F_b - F_a + L|^2
void launch_force_compare(int nf, const double4* fa, const double4* fb, const float4* lsum, double* sums3,
                          cudaStream_t s);
void launch_virial(const SimConst& c, const double4* pos, const double4* vel, const double4* press,
                   const double4* gc, const int* ncount, const int* nlist, double* virial_p,
                   cudaStream_t s);
int check_division(unsigned long long seed, long long n, unsigned long long* d_count, double* d_first,
                   cudaStream_t s);
void launch_conserved(const SimConst& c, const int* cellstart, const double4* pos,
                      const double4* vel, double* out5, cudaStream_t s);

// Kernel constants of one scene from its parameters, header and set-up
// constants (mph_compute_constants), evaluated in the reference's order
// (mph_host.cpp); on failure returns the status and sets msg.
int make_simconst(const mph_params& p, const mph_grid_header& h, const mph_constants& c, int dim, int n,
                  SimConst& s, std::string& msg);

// Sets the calling thread's message for mph_last_error(NULL, ...) and returns code.
int set_thread_error(int code, const std::string& msg);

}  // namespace mph
