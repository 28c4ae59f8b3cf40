// k_batch.cu — the batched form: many independent MPH-WC scenes of one
// dimension stepped together on sm_100a (mph_batch_* in mph_b200.h).
//
// All scenes share one set of particle arrays; scene s owns the slots
// [pbase[s], pbase[s+1]), kept sorted by the scene's own cell id (the CellId of
// main.cpp:96-100; wall and fluid particles share one cell range here).  One
// step of every scene is
//   move     convection (main.cpp:1605-1615), periodic wrap (2306-2317) and the
//            rebuild test of neighborCalculation (1086-1108), per scene;
//   rebuild  a stable counting sort by cell of the scenes whose test fired
//            (histogram, per-scene scan, place, rank + gather, commit); each
//            of these kernels returns at once when no scene asked for it, so
//            the host never waits on the decision;
//   sweep A  DensityP, DivergenceP (+ DensityA, GravityCenter with surface
//            tension) and the PressureP / PressureA values (1631-1662,
//            1665-1740, 1831-1906);
//   sweep B  PressureP, PressureA, DiffuseInterface and ViscosityV forces,
//            gravity, acceleration (1742-2010).
// Both sweeps are persistent kernels: every CTA takes (scene, cell tile) items
// from a queue, stages the tile and its one-cell halo in shared memory and
// evaluates the tile's pairs from there; no neighbour list is stored.  Staged
// positions are tile-relative, split into a part on a power-of-two grid and
// an FP32 remainder, so x_j - x_i is the true displacement rounded once to
// FP32.  The density sweep's DensityP / DivergenceP pairs are evaluated in
// FP64 on that displacement (the pressure is a bulk modulus times a small
// difference of two numbers near N0p), every other pair term in FP32 with
// the mixed form's formulas (Kahan-compensated short-range force sums);
// positions and velocities are integrated in FP64.  A tile whose halo does not fit in
// shared memory is split in two until it does.  mph_batch_step replays K steps
// as one CUDA graph; mph_batch_autotune times the candidate tile shapes on the
// batch itself and keeps the fastest.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include <nvtx3/nvToolsExt.h>
#include "mph_internal.h"
#include "mph_pair32.cuh"

namespace mph {
namespace {

constexpr int kStack = 64;         // pending sub-tiles per CTA
constexpr int kMaxThreads = 256;   // CTA size bound of the sweeps
constexpr int kGraphSteps = MPH_BATCH_GRAPH_STEPS;  // steps per captured graph

enum : int {
    BERR_CAPACITY = 1,   // a one-cell tile did not fit in shared memory
    BERR_NONFINITE = 2,  // NaN/Inf velocity
};

// Per-scene constants: FP64 values for the integration, FP32 values for the
// pair terms (field names follow MixConst so the shared pair helpers apply).
struct alignas(16) BScene {
    int n, pbase, cbase, tot;
    int cc[3], tile[3];
    int has_st, ratio_all_one, uniform_mu, pad0;
    double dmin[3], width[3], inv_width[3], cell_width[3], half_width[3];
    double dt, shift_thr, grid, inv_grid, vol_d, n0p_d;
    double rp2_d, inv_rp_d, cp_d, cp_m2_d;  // FP64 density pairs
    double gravity[3];
    double density[MPH_TYPE_COUNT], bulk_modulus_d[MPH_TYPE_COUNT], bulk_viscosity_d[MPH_TYPE_COUNT];
    float cut2_a, cut2_b, short_r2;
    float rp2_pre;                      // RP^2 a little widened: FP32 pre-filter of the FP64 density pairs
    float ra2, rp2, rv2, rg2;
    float inv_ra, inv_rp, inv_rv, inv_rg;
    float ca, cp, cg, cv;
    float cp_m2, cg_m2, ca_inv;
    float p_a, p_b, v_a, v_b;
    float vol, vol_over_l0, n0a, n0p, inv_r2g_rg, l0;
    float visc_mu[MPH_TYPE_COUNT][MPH_TYPE_COUNT];
    float ratio[MPH_TYPE_COUNT][MPH_TYPE_COUNT];
    float a_k[MPH_TYPE_COUNT], cof_a[MPH_TYPE_COUNT];
};
static_assert(sizeof(BScene) % 16 == 0, "BScene is copied as 16-byte words");

// Kernel arguments (by value): sizes and device pointers, fixed between
// set-ups so that captured graphs stay valid.
struct BatchDev {
    int n, S, n_items, cap;
    int hmax, ncol;               // halo cells / interior columns of the largest tile
    const BScene* scenes;
    const int* sid;               // scene of every slot
    const int4* items;            // (scene, x0, y0, z0) of every tile, largest first
    double4* pos;                 // x, y, z, (double)type
    double4* vel;
    double4* snap;                // positions at the scene's last sort
    int* pidx;                    // index in the scene's input order
    double4* pos_t;
    double4* vel_t;
    int* pidx_t;
    int* key;                     // global cell of a re-sorted particle
    int* slot;
    int* tmp;
    int* counts;                  // [cells], zero between sorts
    int* start;                   // [cells + 1]: first slot of every cell
    float4* vp;                   // sweep A -> B: 2-D (vx, vy, P, type), 3-D (vx, vy, vz, P)
    float4* gc;                   // sweep A -> B: (GravityCenter, PressureA)
    int* flags;                   // [S]: the scene's rebuild test fired
    int* ctl;                     // [8] see below
};
// ctl: 0 any scene to sort, 1 error bits, 2/3 sweep A queue head/done,
// 4/5 sweep B queue head/done, 6 scene sorts so far, 7 tile splits so far.

__device__ __forceinline__ double bmod(double x, double w) { return x - w * floor(x / w); }
__device__ __forceinline__ double bmod_fast(double x, double w) {
    return (x >= 0.0 && x < 0.75 * w) ? x : bmod(x, w);
}
__device__ __forceinline__ int wrapi(int v, int m) { return ((v % m) + m) % m; }

// ---- per step: move -----------------------------------------------------------

__global__ void __launch_bounds__(256) k_bt_move(BatchDev b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.n) return;
    const int s = b.sid[i];
    const BScene& c = b.scenes[s];
    double4 p = b.pos[i];
    if ((int)p.w < 2) {
        const double4 v = b.vel[i];
        p.x += v.x * c.dt;
        p.y += v.y * c.dt;
        p.z += v.z * c.dt;
    }
    p.x = bmod_fast(p.x - c.dmin[0], c.width[0]) + c.dmin[0];
    p.y = bmod_fast(p.y - c.dmin[1], c.width[1]) + c.dmin[1];
    p.z = bmod_fast(p.z - c.dmin[2], c.width[2]) + c.dmin[2];
    b.pos[i] = p;
    const double4 q = b.snap[i];
    const double d0 = bmod_fast(p.x - q.x + c.half_width[0], c.width[0]) - c.half_width[0];
    const double d1 = bmod_fast(p.y - q.y + c.half_width[1], c.width[1]) - c.half_width[1];
    const double d2 = bmod_fast(p.z - q.z + c.half_width[2], c.width[2]) - c.half_width[2];
    if (d0 * d0 + d1 * d1 + d2 * d2 > c.shift_thr) {
        b.flags[s] = 1;
        b.ctl[0] = 1;
    }
}

// ---- rebuild: stable counting sort of the flagged scenes ----------------------

__global__ void __launch_bounds__(256) k_bt_hist(BatchDev b) {
    if (b.ctl[0] == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.n) return;
    const int s = b.sid[i];
    if (!b.flags[s]) return;
    const BScene& c = b.scenes[s];
    const double4 p = b.pos[i];
    const int cx = wrapi((int)floor((p.x - c.dmin[0]) / c.cell_width[0]), c.cc[0]);
    const int cy = wrapi((int)floor((p.y - c.dmin[1]) / c.cell_width[1]), c.cc[1]);
    const int cz = wrapi((int)floor((p.z - c.dmin[2]) / c.cell_width[2]), c.cc[2]);
    const int key = c.cbase + (cx * c.cc[1] + cy) * c.cc[2] + cz;
    b.key[i] = key;
    b.slot[i] = atomicAdd(&b.counts[key], 1);
}

// One block per scene: exclusive scan of the scene's cell counts into start
// (offset by the scene's first slot), counts reset to zero.
__global__ void __launch_bounds__(1024) k_bt_scan(BatchDev b) {
    if (b.ctl[0] == 0) return;
    const int s = blockIdx.x;
    if (!b.flags[s]) return;
    __shared__ int part[1024];
    const BScene& c = b.scenes[s];
    int* counts = b.counts + c.cbase;
    int* out = b.start + c.cbase;
    const int m = c.tot, t = threadIdx.x;
    const int chunk = (m + blockDim.x - 1) / blockDim.x;
    const int lo = min(m, t * chunk), hi = min(m, lo + chunk);
    int sum = 0;
    for (int k = lo; k < hi; ++k) sum += counts[k];
    part[t] = sum;
    __syncthreads();
    for (int off = 1; off < (int)blockDim.x; off <<= 1) {  // Hillis-Steele inclusive scan
        const int v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = c.pbase + part[t] - sum;
    for (int k = lo; k < hi; ++k) {
        out[k] = run;
        run += counts[k];
        counts[k] = 0;
    }
}

__global__ void __launch_bounds__(256) k_bt_place(BatchDev b) {
    if (b.ctl[0] == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.n || !b.flags[b.sid[i]]) return;
    b.tmp[b.start[b.key[i]] + b.slot[i]] = i;
}

// Order each cell's particles by their previous slot (a stable sort) and
// gather the state into the temporaries.
__global__ void __launch_bounds__(256) k_bt_gather(BatchDev b) {
    if (b.ctl[0] == 0) return;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= b.n || !b.flags[b.sid[p]]) return;
    const int i = b.tmp[p];
    const int key = b.key[i];
    const int lo = b.start[key], hi = b.start[key + 1];
    int rank = 0;
    for (int q = lo; q < hi; ++q) rank += b.tmp[q] < i;
    const int dst = lo + rank;
    b.pos_t[dst] = b.pos[i];
    b.vel_t[dst] = b.vel[i];
    b.pidx_t[dst] = b.pidx[i];
}

__global__ void __launch_bounds__(256) k_bt_commit(BatchDev b) {
    if (b.ctl[0] == 0) return;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= b.n || !b.flags[b.sid[p]]) return;
    const double4 x = b.pos_t[p];
    b.pos[p] = x;
    b.snap[p] = x;
    b.vel[p] = b.vel_t[p];
    b.pidx[p] = b.pidx_t[p];
}

// ---- the sweeps ----------------------------------------------------------------

template <int DIM, int SWEEP, bool ST>
struct Smem {
    // staged per particle: P (2-D hi.xy lo.xy; 3-D hi.xyz type), L (3-D lo.xyz),
    // V (sweep A: velocity; sweep B: vp), G (sweep B with surface tension: gc)
    static constexpr int kL = DIM == 3 ? 1 : 0;
    static constexpr int kG = (SWEEP == 1 && ST) ? 1 : 0;
    static constexpr int kVec = 2 + kL + kG;
    static size_t bytes(int cap, int hmax, int ncol) {
        return (size_t)cap * 16 * kVec + (size_t)(2 * hmax + 1 + ncol + 1) * 4 + (size_t)cap * 2 + 16;
    }
};

template <int DIM, int SWEEP, bool ST>
__global__ void __launch_bounds__(kMaxThreads) k_bt_sweep(BatchDev b) {
    using SM = Smem<DIM, SWEEP, ST>;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ BScene sc;
    __shared__ int4 stack[kStack];
    __shared__ int s_item, s_sp;
    const int cap = b.cap, tid = threadIdx.x, bd = blockDim.x, lane = tid & 31, warp = tid >> 5;
    float4* sP = reinterpret_cast<float4*>(smem);
    float4* sL = sP + cap;
    float4* sV = sL + (size_t)cap * SM::kL;
    float4* sG = sV + cap;
    int* hb = reinterpret_cast<int*>(sG + (size_t)cap * SM::kG);  // [hmax + 1] staged begin of each halo cell
    int* hsrc = hb + b.hmax + 1;                                   // [hmax] first slot of each halo cell
    int* col = hsrc + b.hmax;                                      // [ncol + 1] interior prefix per column
    unsigned short* sH = reinterpret_cast<unsigned short*>(col + b.ncol + 1);
    int* qhead = b.ctl + (SWEEP == 0 ? 2 : 4);

    if (SWEEP == 0 && blockIdx.x == 0) {  // the sorts of this step are done: clear the requests
        for (int s = tid; s < b.S; s += bd)
            if (b.flags[s]) {
                atomicAdd(&b.ctl[6], 1);
                b.flags[s] = 0;
            }
        if (tid == 0) b.ctl[0] = 0;
    }
    int cur = -1;
    for (;;) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(qhead, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= b.n_items) break;
        const int4 it = b.items[item];
        if (it.x != cur) {
            const int4* src = reinterpret_cast<const int4*>(b.scenes + it.x);
            int4* dst = reinterpret_cast<int4*>(&sc);
            for (int k = tid; k < (int)(sizeof(BScene) / 16); k += bd) dst[k] = src[k];
            cur = it.x;
            __syncthreads();
        }
        if (tid == 0) {
            const int t0 = min(sc.tile[0], sc.cc[0] - it.y), t1 = min(sc.tile[1], sc.cc[1] - it.z);
            const int t2 = DIM == 3 ? min(sc.tile[2], sc.cc[2] - it.w) : 1;
            stack[0] = make_int4(it.y, it.z, it.w, t0 | (t1 << 8) | (t2 << 16));
            s_sp = 1;
        }
        for (;;) {
            __syncthreads();
            if (s_sp == 0) break;
            const int4 e = stack[s_sp - 1];
            __syncthreads();
            if (tid == 0) --s_sp;
            const int x0 = e.x, y0 = e.y, z0 = e.z;
            const int t0 = e.w & 255, t1 = (e.w >> 8) & 255, t2 = (e.w >> 16) & 255;
            const int H1 = t1 + 2, H2 = DIM == 3 ? t2 + 2 : 1, H = (t0 + 2) * H1 * H2;
            // halo cells: first slot and count
            for (int h = tid; h < H; h += bd) {
                const int a = h / (H1 * H2), bb = (h / H2) % H1, cz = h % H2;
                const int cx = wrapi(x0 - 1 + a, sc.cc[0]), cy = wrapi(y0 - 1 + bb, sc.cc[1]);
                const int czz = DIM == 3 ? wrapi(z0 - 1 + cz, sc.cc[2]) : 0;
                const int key = sc.cbase + (cx * sc.cc[1] + cy) * sc.cc[2] + czz;
                const int s0 = b.start[key];
                hsrc[h] = s0;
                hb[h] = b.start[key + 1] - s0;
            }
            __syncthreads();
            if (warp == 0) {  // exclusive scan of the counts, hb[H] = total
                int run = 0;
                for (int base = 0; base < H; base += 32) {
                    const int v = base + lane < H ? hb[base + lane] : 0;
                    int x = v;
                    for (int o = 1; o < 32; o <<= 1) {
                        const int y = __shfl_up_sync(0xffffffffu, x, o);
                        if (lane >= o) x += y;
                    }
                    if (base + lane < H) hb[base + lane] = run + x - v;
                    run += __shfl_sync(0xffffffffu, x, 31);
                }
                if (lane == 0) hb[H] = run;
            }
            __syncthreads();
            const int total = hb[H];
            if (total > cap) {  // split the tile along its longest axis
                if (tid == 0) {
                    const int ax = (DIM == 3 && t2 >= t0 && t2 >= t1) ? 2 : (t1 > t0 ? 1 : 0);
                    const int len = ax == 0 ? t0 : ax == 1 ? t1 : t2;
                    if (len <= 1 || s_sp + 2 > kStack) {
                        atomicOr(&b.ctl[1], BERR_CAPACITY);
                    } else {
                        const int h0 = len / 2, h1 = len - h0;
                        int4 lo = e, hi = e;
                        const int sh = 8 * ax;
                        lo.w = (e.w & ~(255 << sh)) | (h0 << sh);
                        hi.w = (e.w & ~(255 << sh)) | (h1 << sh);
                        if (ax == 0) hi.x += h0;
                        else if (ax == 1) hi.y += h0;
                        else hi.z += h0;
                        stack[s_sp] = lo;
                        stack[s_sp + 1] = hi;
                        s_sp += 2;
                        atomicAdd(&b.ctl[7], 1);
                    }
                }
                continue;
            }
            if (total == 0) continue;
            // interior columns: (a in 1..t0) in 2-D, (a, b) in 1..t0 x 1..t1 in 3-D
            const int ncol = DIM == 3 ? t0 * t1 : t0;
            auto col_begin = [&](int k, int& lo, int& hi) {
                const int a = DIM == 3 ? 1 + k / t1 : 1 + k, bb = DIM == 3 ? 1 + k % t1 : 1;
                if (DIM == 3) {
                    const int base = (a * H1 + bb) * H2;
                    lo = hb[base + 1];
                    hi = hb[base + t2 + 1];
                } else {
                    lo = hb[a * H1 + 1];
                    hi = hb[a * H1 + t1 + 1];
                }
            };
            if (warp == 0) {
                int run = 0;
                for (int base = 0; base < ncol; base += 32) {
                    int v = 0;
                    if (base + lane < ncol) {
                        int lo, hi;
                        col_begin(base + lane, lo, hi);
                        v = hi - lo;
                    }
                    int x = v;
                    for (int o = 1; o < 32; o <<= 1) {
                        const int y = __shfl_up_sync(0xffffffffu, x, o);
                        if (lane >= o) x += y;
                    }
                    if (base + lane < ncol) col[base + lane] = run + x - v;
                    run += __shfl_sync(0xffffffffu, x, 31);
                }
                if (lane == 0) col[ncol] = run;
            }
            // stage every halo particle: tile-relative hi/lo coordinates
            const double ox = sc.dmin[0] + (double)(x0 - 1) * sc.cell_width[0];
            const double oy = sc.dmin[1] + (double)(y0 - 1) * sc.cell_width[1];
            const double oz = sc.dmin[2] + (double)(z0 - 1) * sc.cell_width[2];
            for (int q = tid; q < total; q += bd) {
                int lo = 0, hi = H;  // largest h with hb[h] <= q (skips empty cells)
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (hb[mid] <= q) lo = mid;
                    else hi = mid - 1;
                }
                const int h = lo;
                const int g = hsrc[h] + (q - hb[h]);
                const int a = h / (H1 * H2), bb = (h / H2) % H1, cz = h % H2;
                const double4 p = b.pos[g];
                double d[3] = {p.x - ox, p.y - oy, p.z - oz};
                const int hc[3] = {a, bb, cz};
                float fh[3], fl[3];
#pragma unroll
                for (int k = 0; k < DIM; ++k) {
                    const double ec = ((double)hc[k] + 0.5) * sc.cell_width[k];
                    d[k] -= sc.width[k] * rint((d[k] - ec) * sc.inv_width[k]);
                    const double qh = rint(d[k] * sc.inv_grid) * sc.grid;
                    fh[k] = (float)qh;
                    fl[k] = (float)(d[k] - qh);
                }
                const int type = (int)p.w;
                if (DIM == 2) {
                    sP[q] = make_float4(fh[0], fh[1], fl[0], fl[1]);
                } else {
                    sP[q] = make_float4(fh[0], fh[1], fh[2], __int_as_float(type));
                    sL[q] = make_float4(fl[0], fl[1], fl[2], 0.0f);
                }
                if (SWEEP == 0) {
                    const double4 v = b.vel[g];
                    sV[q] = DIM == 2 ? make_float4((float)v.x, (float)v.y, 0.0f, __int_as_float(type))
                                     : make_float4((float)v.x, (float)v.y, (float)v.z, 0.0f);
                } else {
                    sV[q] = b.vp[g];
                    if (ST) sG[q] = b.gc[g];
                }
                sH[q] = (unsigned short)h;
            }
            __syncthreads();
            const int nin = col[ncol];
            for (int k = tid; k < nin; k += bd) {
                int lo = 0, hi = ncol;  // column of interior particle k
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (col[mid] <= k) lo = mid;
                    else hi = mid - 1;
                }
                int cb, ce;
                col_begin(lo, cb, ce);
                const int si = cb + (k - col[lo]);
                const int h = sH[si];
                const int a = h / (H1 * H2), bb = (h / H2) % H1, cz = h % H2;
                const int g = hsrc[h] + (si - hb[h]);
                const float4 pi = sP[si];
                float4 li = make_float4(0.f, 0.f, 0.f, 0.f);
                if (DIM == 3) li = sL[si];
                const float4 vi = sV[si];
                const int ti = DIM == 2 ? __float_as_int(vi.w) : __float_as_int(pi.w);
                if (SWEEP == 1 && ti >= 2) continue;  // walls never accelerate
                // runs of three cells along the last axis: 3 in 2-D, 9 in 3-D
                auto run_of = [&](int r, int& rb, int& re) {
                    if (DIM == 2) {
                        const int base = (a + r - 1) * H1 + bb;
                        rb = hb[base - 1];
                        re = hb[base + 2];
                    } else {
                        const int base = ((a + r / 3 - 1) * H1 + (bb + r % 3 - 1)) * H2 + cz;
                        rb = hb[base - 1];
                        re = hb[base + 2];
                    }
                };
                auto disp = [&](int j, float& dx, float& dy, float& dz) {
                    const float4 pj = sP[j];
                    if (DIM == 2) {
                        dx = (pj.x - pi.x) + (pj.z - pi.z);
                        dy = (pj.y - pi.y) + (pj.w - pi.w);
                        dz = 0.0f;
                    } else {
                        const float4 lj = sL[j];
                        dx = (pj.x - pi.x) + (lj.x - li.x);
                        dy = (pj.y - pi.y) + (lj.y - li.y);
                        dz = (pj.z - pi.z) + (lj.z - li.z);
                    }
                };
                auto type_of = [&](int j) {
                    return DIM == 2 ? __float_as_int(sV[j].w) : __float_as_int(sP[j].w);
                };
                const bool st = ST && sc.has_st;
                const bool ratio1 = sc.ratio_all_one;
                // Pairs within sqrt(cut2) in the runs' order: each chunk of up to 64
                // candidates is filtered into a bit mask first, then only the set
                // bits are visited, so the lanes of a warp run the pair terms
                // together instead of under divergent distance tests.
                auto for_near = [&](float cut2, auto&& visit) {
                    for (int r = 0; r < (DIM == 2 ? 3 : 9); ++r) {
                        int rb, re;
                        run_of(r, rb, re);
                        for (int base = rb; base < re; base += 64) {
                            const int cnt = min(64, re - base);
                            unsigned long long m = 0ull;
                            for (int q = 0; q < cnt; ++q) {
                                float dx, dy, dz;
                                disp(base + q, dx, dy, dz);
                                if (dx * dx + dy * dy + dz * dz < cut2) m |= 1ull << q;
                            }
                            if (si >= base && si < base + cnt) m &= ~(1ull << (si - base));
                            while (m != 0ull) {
                                const int j = base + __ffsll((long long)m) - 1;
                                m &= m - 1ull;
                                float dx, dy, dz;
                                disp(j, dx, dy, dz);
                                visit(j, dx, dy, dz, dx * dx + dy * dy + dz * dz);
                            }
                        }
                    }
                };
                if (SWEEP == 0) {
                    double spd = 0.0, sdd = 0.0;  // DensityP, DivergenceP: FP64 pairs
                    float sa = 0.f, cak = 0.f, g0 = 0.f, g1 = 0.f, g2 = 0.f;
                    for_near(sc.cut2_a, [&](int j, float dx, float dy, float dz, float r2) {
                            const float rinv = rsqrt_nr(r2);
                            const float rr = r2 * rinv;
                            if (r2 <= sc.rp2_pre) {
                                // FP64 displacement: the hi parts' difference is exact in FP32,
                                // the lo parts carry the rest
                                const float4 pj = sP[j];
                                double dd[3];
                                if (DIM == 2) {
                                    dd[0] = (double)(pj.x - pi.x) + ((double)pj.z - (double)pi.z);
                                    dd[1] = (double)(pj.y - pi.y) + ((double)pj.w - (double)pi.w);
                                    dd[2] = 0.0;
                                } else {
                                    const float4 lj = sL[j];
                                    dd[0] = (double)(pj.x - pi.x) + ((double)lj.x - (double)li.x);
                                    dd[1] = (double)(pj.y - pi.y) + ((double)lj.y - (double)li.y);
                                    dd[2] = (double)(pj.z - pi.z) + ((double)lj.z - (double)li.z);
                                }
                                const double r2d = dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2];
                                if (r2d <= sc.rp2_d) {
                                    const double y = rsqrt_dnr(r2d);
                                    const double q = 1.0 - r2d * y * sc.inv_rp_d;
                                    spd += sc.cp_d * q * q;  // wp
                                    const double dw = sc.cp_m2_d * q;
                                    const float4 vj = sV[j];
                                    double ue = ((double)vj.x - (double)vi.x) * dd[0] +
                                                ((double)vj.y - (double)vi.y) * dd[1];
                                    if (DIM == 3) ue += ((double)vj.z - (double)vi.z) * dd[2];
                                    sdd -= ue * y * dw;
                                }
                            }
                            if (ST && st) {
                                const int tj = type_of(j);
                                if (ratio1) st_density<false>(sc, ti, tj, r2, rr, dx, dy, dz, sa, cak, g0, g1, g2);
                                else st_density<true>(sc, ti, tj, r2, rr, dx, dy, dz, sa, cak, g0, g1, g2);
                            }
                    });
                    const double strain = spd - sc.n0p_d;
                    const double div = sdd;
                    double kappa = sc.bulk_modulus_d[ti];
                    if (strain < 0.0) kappa = 0.0;
                    const double pp = -sc.bulk_viscosity_d[ti] * div + kappa * strain;
                    if (ST) {
                        float pa = 0.0f;
                        if (st) {
                            const float dens = sa - cak;
                            pa = sc.cof_a[ti] * (dens - sc.n0a) / sc.l0;
                            if (sc.n0a <= dens) pa = 0.0f;
                        }
                        b.gc[g] = make_float4(g0, g1, g2, pa);
                    }
                    b.vp[g] = DIM == 2 ? make_float4(vi.x, vi.y, (float)pp, vi.w)
                                       : make_float4(vi.x, vi.y, vi.z, (float)pp);
                } else {
                    const float Pi = DIM == 2 ? vi.z : vi.w;
                    float4 gi = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (ST) gi = sG[si];
                    const float ai = sc.a_k[ti];
                    const float mu_u = sc.visc_mu[ti][ti];
                    float fx = 0.f, fy = 0.f, fz = 0.f, cx = 0.f, cy = 0.f, cz2 = 0.f;  // short range, Kahan
                    float gx = 0.f, gy = 0.f, gz = 0.f;                                  // long range
                    for_near(sc.cut2_b, [&](int j, float dx, float dy, float dz, float r2) {
                            const float rinv = rsqrt_nr(r2);
                            const float rr = r2 * rinv;
                            const float4 vj = sV[j];
                            const float Pj = DIM == 2 ? vj.z : vj.w;
                            const int tj = (sc.uniform_mu && ratio1 && !st) ? ti : type_of(j);
                            float s = 0.0f;
                            if (r2 < sc.rp2) s += (Pi + Pj) * fmaf(sc.p_b, rr, sc.p_a) * rinv;
                            if (r2 < sc.rv2) {
                                const float mu = sc.uniform_mu ? mu_u : sc.visc_mu[ti][tj];
                                float ud = (vj.x - vi.x) * dx + (vj.y - vi.y) * dy;
                                if (DIM == 3) ud += (vj.z - vi.z) * dz;
                                s += mu * ud * fmaf(sc.v_b, rr, sc.v_a) * (rinv * rinv * rinv);
                            }
                            float3 t = make_float3(0.f, 0.f, 0.f);
                            if (ST && st) {
                                if (ratio1) s += st_terms<false>(sc, ti, tj, r2, rr, rinv, dx, dy, dz, gi, sG[j], ai, t);
                                else s += st_terms<true>(sc, ti, tj, r2, rr, rinv, dx, dy, dz, gi, sG[j], ai, t);
                            }
                            if (r2 < sc.short_r2) {
                                kahan_add(fx, cx, fmaf(s, dx, t.x));
                                kahan_add(fy, cy, fmaf(s, dy, t.y));
                                if (DIM == 3) kahan_add(fz, cz2, fmaf(s, dz, t.z));
                            } else {
                                gx += fmaf(s, dx, t.x);
                                gy += fmaf(s, dy, t.y);
                                if (DIM == 3) gz += fmaf(s, dz, t.z);
                            }
                    });
                    double F0 = ((double)fx - (double)cx) + (double)gx;
                    double F1 = ((double)fy - (double)cy) + (double)gy;
                    double F2 = ((double)fz - (double)cz2) + (double)gz;
                    const double mass = sc.density[ti] * sc.vol_d;
                    F0 += mass * sc.gravity[0];
                    F1 += mass * sc.gravity[1];
                    F2 += mass * sc.gravity[2];
                    double4 v = b.vel[g];
                    v.x += F0 / mass * sc.dt;
                    v.y += F1 / mass * sc.dt;
                    v.z += F2 / mass * sc.dt;
                    if (!(isfinite(v.x) && isfinite(v.y) && isfinite(v.z))) atomicOr(&b.ctl[1], BERR_NONFINITE);
                    b.vel[g] = v;
                }
            }
        }
    }
    // every CTA has drawn past the end of the queue: the last one resets it
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        if (atomicAdd(qhead + 1, 1) == (int)gridDim.x - 1) {
            qhead[0] = 0;
            qhead[1] = 0;
            __threadfence();
        }
    }
}

inline int nblocks(long long n, int t) { return (int)((n + t - 1) / t); }

using SweepFn = void (*)(BatchDev);

template <int DIM>
SweepFn sweep_fn(int sweep, bool st) {
    if (sweep == 0) return st ? k_bt_sweep<DIM, 0, true> : k_bt_sweep<DIM, 0, false>;
    return st ? k_bt_sweep<DIM, 1, true> : k_bt_sweep<DIM, 1, false>;
}

size_t sweep_smem(int dim, int sweep, bool st, int cap, int hmax, int ncol) {
    if (dim == 2) {
        if (sweep == 0) return st ? Smem<2, 0, true>::bytes(cap, hmax, ncol) : Smem<2, 0, false>::bytes(cap, hmax, ncol);
        return st ? Smem<2, 1, true>::bytes(cap, hmax, ncol) : Smem<2, 1, false>::bytes(cap, hmax, ncol);
    }
    if (sweep == 0) return st ? Smem<3, 0, true>::bytes(cap, hmax, ncol) : Smem<3, 0, false>::bytes(cap, hmax, ncol);
    return st ? Smem<3, 1, true>::bytes(cap, hmax, ncol) : Smem<3, 1, false>::bytes(cap, hmax, ncol);
}

}  // namespace
}  // namespace mph

using mph::BatchDev;
using mph::BScene;

// ---------------------------------------------------------------------------
// host side

struct BatchProfile {
    bool on = false;
    std::vector<std::string> names;
    std::vector<long long> launches;
    std::vector<double> ms;
    struct Pending {
        int id, count;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
};

struct mph_batch {
    int dim = 2, S = 0, n = 0, n_fluid = 0, cells = 0;
    int tile[3] = {8, 8, 1}, threads = 256, occ = 2;
    int cap = 0, hmax = 0, ncol = 0, n_items = 0, grid_a = 0, grid_b = 0, sms = 0;
    size_t smem_a = 0, smem_b = 0;
    bool has_st = false;
    std::vector<BScene> hs;
    std::vector<int> pbase;
    std::vector<std::vector<int>> cell_count;  // per scene: particles per cell at creation
    cudaStream_t stream = nullptr;
    BatchDev d{};
    BScene* d_scenes = nullptr;
    int4* d_items = nullptr;
    int* d_sid = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long steps = 0, launches = 0;
    int* h_ctl = nullptr;  // pinned [8]
    BatchProfile prof;
    std::string err;
};

static thread_local std::string g_batch_err;

static int bfail(mph_batch* b, int code, const std::string& msg) {
    if (b) b->err = msg;
    g_batch_err = msg;
    return code;
}

#define BTRY(b, expr)                                                                        \
    do {                                                                                     \
        cudaError_t e_ = (expr);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return bfail(b, MPH_ERR_CUDA, std::string(#expr ": ") + cudaGetErrorString(e_)); \
    } while (0)

template <class T>
static cudaError_t balloc(T** p, size_t n) {
    *p = nullptr;
    return cudaMalloc((void**)p, (n ? n : 1) * sizeof(T));
}

static void free_graph(mph_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

extern "C" void mph_batch_destroy(mph_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    free_graph(b);
    BatchDev& d = b->d;
    void* ptrs[] = {b->d_scenes, b->d_items, b->d_sid, d.pos, d.vel, d.snap, d.pidx, d.pos_t, d.vel_t, d.pidx_t,
                    d.key, d.slot, d.tmp, d.counts, d.start, d.vp, d.gc, d.flags, d.ctl};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (auto& pe : b->prof.pending) {
        cudaEventDestroy(pe.a);
        cudaEventDestroy(pe.b);
    }
    if (b->h_ctl) cudaFreeHost(b->h_ctl);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

// Pair constants of one scene (the mixed form's, from the FP64 values).
static void fill_bscene(BScene& s, const mph::SimConst& c, const mph_constants& k) {
    std::memset(&s, 0, sizeof(s));
    s.n = c.n;
    s.tot = c.tot;
    for (int d = 0; d < 3; ++d) {
        s.cc[d] = c.cc[d];
        s.dmin[d] = c.dmin[d];
        s.width[d] = c.width[d];
        s.inv_width[d] = 1.0 / c.width[d];
        s.cell_width[d] = c.cell_width[d];
        s.half_width[d] = c.half_width[d];
        s.gravity[d] = c.gravity[d];
    }
    s.has_st = c.has_st;
    s.ratio_all_one = c.ratio_all_one;
    s.uniform_mu = 1;
    for (int t = 0; t < MPH_TYPE_COUNT; ++t)
        for (int u = 0; u < MPH_TYPE_COUNT; ++u)
            if (c.visc_mu[t][u] != c.visc_mu[0][0]) s.uniform_mu = 0;
    s.dt = c.dt;
    s.shift_thr = c.shift_thr;
    s.vol_d = c.vol;
    for (int t = 0; t < MPH_TYPE_COUNT; ++t) {
        s.density[t] = c.density[t];
        s.bulk_modulus_d[t] = c.bulk_modulus[t];
        s.bulk_viscosity_d[t] = c.bulk_viscosity[t];
        s.a_k[t] = (float)c.a_k[t];
        s.cof_a[t] = (float)c.cof_a[t];
        for (int u = 0; u < MPH_TYPE_COUNT; ++u) {
            s.visc_mu[t][u] = (float)c.visc_mu[t][u];
            s.ratio[t][u] = (float)c.ratio[t][u];
        }
    }
    const double margin = 0.1 * c.l0, rs = k.radius_p + margin;
    s.short_r2 = (float)(rs * rs);
    s.ra2 = (float)c.ra2;
    s.rp2 = (float)c.rp2;
    s.rv2 = (float)c.rv2;
    s.rg2 = (float)c.rg2;
    // the density sums take r^2 <= R^2 (main.cpp:1684), the forces r^2 < R^2:
    // pairs are selected by r^2 < cut2 in FP32, so cut2_a lies a little above
    // (the FP64 test r^2 <= RP^2 decides the pressure pairs)
    s.rp2_pre = (float)(c.rp2 * (1.0 + 1e-5));
    s.cut2_a = std::nextafter(c.has_st ? std::max(s.rp2_pre, std::max(s.ra2, s.rg2)) : s.rp2_pre, INFINITY);
    s.cut2_b = std::max(s.rp2, s.rv2);
    if (c.has_st) s.cut2_b = std::max(s.cut2_b, std::max(s.ra2, s.rg2));
    s.inv_ra = (float)(1.0 / c.ra);
    s.inv_rp = (float)(1.0 / c.rp);
    s.inv_rv = (float)(1.0 / c.rv);
    s.inv_rg = (float)(1.0 / c.rg);
    s.ca = (float)c.ca;
    s.cp = (float)c.cp;
    s.cg = (float)c.cg;
    s.cv = (float)c.cv;
    s.cp_m2 = (float)(c.cp * c.m2_rp);
    s.cg_m2 = (float)(c.cg * c.m2_rg);
    s.ca_inv = (float)(c.ca * c.inv_ra);
    s.p_a = (float)(c.cp * c.m2_rp * c.vol);
    s.p_b = (float)(-c.cp * c.m2_rp * c.vol / c.rp);
    s.v_a = (float)(-c.cv * c.m2_rv * c.vol);
    s.v_b = (float)(c.cv * c.m2_rv * c.vol / c.rv);
    s.vol = (float)c.vol;
    s.vol_over_l0 = (float)c.vol_over_l0;
    s.n0a = (float)c.n0a;
    s.n0p = (float)c.n0p;
    s.n0p_d = c.n0p;
    s.rp2_d = c.rp2;
    s.inv_rp_d = 1.0 / c.rp;
    s.cp_d = c.cp;
    s.cp_m2_d = c.cp * c.m2_rp;
    s.inv_r2g_rg = (float)(c.rg / c.r2g);
    s.l0 = (float)c.l0;
}

// Tiles, items (largest first by the particle count at creation), staging
// capacity, shared memory and persistent grid sizes for tile t and CTA size.
static int configure(mph_batch* b, const int t[3], int threads, int ctas_per_sm = 2) {
    const int dim = b->dim;
    if (threads < 64 || threads > mph::kMaxThreads || threads % 32 != 0)
        return bfail(b, MPH_ERR_ARG, "threads must be a multiple of 32 in [64, 256]");
    for (int d = 0; d < dim; ++d)
        if (t[d] < 1 || t[d] > 64) return bfail(b, MPH_ERR_ARG, "tile sides must be in [1, 64]");
    int tmax[3] = {1, 1, 1};
    struct Item {
        int4 v;
        long long cost;
    };
    std::vector<Item> items;
    long long max_halo = 0;
    for (int s = 0; s < b->S; ++s) {
        BScene& sc = b->hs[s];
        for (int d = 0; d < 3; ++d) sc.tile[d] = 1;
        for (int d = 0; d < dim; ++d) sc.tile[d] = std::max(1, std::min(t[d], sc.cc[d] - 2));  // distinct halo cells
        for (int d = 0; d < 3; ++d) tmax[d] = std::max(tmax[d], sc.tile[d]);
        const std::vector<int>& cnt = b->cell_count[s];
        auto cell_n = [&](int x, int y, int z) {
            x = (x % sc.cc[0] + sc.cc[0]) % sc.cc[0];
            y = (y % sc.cc[1] + sc.cc[1]) % sc.cc[1];
            z = (z % sc.cc[2] + sc.cc[2]) % sc.cc[2];
            return (long long)cnt[((size_t)x * sc.cc[1] + y) * sc.cc[2] + z];
        };
        const int zc = dim == 3 ? sc.cc[2] : 1;
        for (int x0 = 0; x0 < sc.cc[0]; x0 += sc.tile[0])
            for (int y0 = 0; y0 < sc.cc[1]; y0 += sc.tile[1])
                for (int z0 = 0; z0 < zc; z0 += sc.tile[2]) {
                    const int t0 = std::min(sc.tile[0], sc.cc[0] - x0), t1 = std::min(sc.tile[1], sc.cc[1] - y0);
                    const int t2 = dim == 3 ? std::min(sc.tile[2], sc.cc[2] - z0) : 1;
                    long long in = 0, halo = 0;
                    const int hz0 = dim == 3 ? -1 : 0, hz1 = dim == 3 ? t2 + 1 : 1;
                    for (int a = -1; a <= t0; ++a)
                        for (int c = -1; c <= t1; ++c)
                            for (int z = hz0; z < hz1; ++z) {
                                const long long v = cell_n(x0 + a, y0 + c, z0 + z);
                                halo += v;
                                if (a >= 0 && a < t0 && c >= 0 && c < t1 && (dim == 2 || (z >= 0 && z < t2))) in += v;
                            }
                    max_halo = std::max(max_halo, halo);
                    items.push_back({make_int4(s, x0, y0, z0), in});
                }
        // the grid of the hi parts: |tile-relative coordinate| < 2^24 grid
        double ext = 0.0;
        for (int d = 0; d < dim; ++d) ext = std::max(ext, (sc.tile[d] + 2.5) * sc.cell_width[d]);
        sc.grid = std::ldexp(1.0, (int)std::ceil(std::log2(ext)) - 23);
        sc.inv_grid = 1.0 / sc.grid;
    }
    std::stable_sort(items.begin(), items.end(), [](const Item& x, const Item& y) { return x.cost > y.cost; });
    const int hmax = (tmax[0] + 2) * (tmax[1] + 2) * (dim == 3 ? tmax[2] + 2 : 1);
    const int ncol = dim == 3 ? tmax[0] * tmax[1] : tmax[0];
    if (hmax > 65535) return bfail(b, MPH_ERR_ARG, "tile too large");
    // staging capacity: the largest halo at creation with head room, bounded by
    // the shared memory of two resident CTAs per SM
    int dev = 0;
    cudaGetDevice(&dev);
    int smem_optin = 0;
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    // shared memory for ctas_per_sm resident CTAs (228 KB per SM, 1 KB reserved per CTA)
    const int occ = std::max(1, std::min(ctas_per_sm, 8));
    const size_t budget = std::min<size_t>((size_t)smem_optin, (size_t)228 * 1024 / occ - 1024) - sizeof(BScene) - 2048;
    int cap = (int)std::min<long long>(max_halo + max_halo / 8 + 32, 1 << 20);
    while (cap > 64 && std::max(mph::sweep_smem(dim, 0, b->has_st, cap, hmax, ncol),
                                mph::sweep_smem(dim, 1, b->has_st, cap, hmax, ncol)) > budget)
        cap -= 32;
    // free old items, upload new
    if (b->d_items) cudaFree(b->d_items);
    b->d_items = nullptr;
    std::vector<int4> hv(items.size());
    for (size_t k = 0; k < items.size(); ++k) hv[k] = items[k].v;
    BTRY(b, balloc(&b->d_items, hv.size()));
    BTRY(b, cudaMemcpyAsync(b->d_items, hv.data(), hv.size() * sizeof(int4), cudaMemcpyHostToDevice, b->stream));
    BTRY(b, cudaMemcpyAsync(b->d_scenes, b->hs.data(), b->hs.size() * sizeof(BScene), cudaMemcpyHostToDevice,
                            b->stream));
    for (int d = 0; d < 3; ++d) b->tile[d] = t[d];
    if (dim == 2) b->tile[2] = 1;
    b->threads = threads;
    b->occ = occ;
    b->cap = cap;
    b->hmax = hmax;
    b->ncol = ncol;
    b->n_items = (int)items.size();
    b->smem_a = mph::sweep_smem(dim, 0, b->has_st, cap, hmax, ncol);
    b->smem_b = mph::sweep_smem(dim, 1, b->has_st, cap, hmax, ncol);
    int g[2];
    for (int sw = 0; sw < 2; ++sw) {
        mph::SweepFn f = dim == 2 ? mph::sweep_fn<2>(sw, b->has_st) : mph::sweep_fn<3>(sw, b->has_st);
        const size_t sm = sw == 0 ? b->smem_a : b->smem_b;
        BTRY(b, cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        int per = 0;
        BTRY(b, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, f, threads, sm));
        if (per < 1) return bfail(b, MPH_ERR_ARG, "sweep kernel does not fit on an SM with this tile");
        g[sw] = std::max(1, std::min(per * b->sms, b->n_items));
    }
    b->grid_a = g[0];
    b->grid_b = g[1];
    BatchDev& d = b->d;
    d.n_items = b->n_items;
    d.cap = cap;
    d.hmax = hmax;
    d.ncol = ncol;
    d.items = b->d_items;
    free_graph(b);
    return MPH_OK;
}

// Launch groups: an NVTX range each, and CUDA events around them when
// profiling is enabled (direct launches).
struct BLaunch {
    mph_batch* b;
    int id = -1, count;
    cudaEvent_t a = nullptr;
    BLaunch(mph_batch* bb, const char* name, int c) : b(bb), count(c) {
        nvtxRangePushA(name);
        BatchProfile& p = b->prof;
        if (!p.on) return;
        for (size_t k = 0; k < p.names.size(); ++k)
            if (p.names[k] == name) id = (int)k;
        if (id < 0) {
            id = (int)p.names.size();
            p.names.push_back(name);
            p.launches.push_back(0);
            p.ms.push_back(0.0);
        }
        cudaEventCreate(&a);
        cudaEventRecord(a, b->stream);
    }
    ~BLaunch() {
        nvtxRangePop();
        b->launches += count;
        if (id < 0) return;
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        cudaEventRecord(e, b->stream);
        b->prof.pending.push_back({id, count, a, e});
    }
};

static void launch_rebuild(mph_batch* b) {
    const BatchDev& d = b->d;
    const int nb = mph::nblocks(b->n, 256);
    mph::k_bt_hist<<<nb, 256, 0, b->stream>>>(d);
    mph::k_bt_scan<<<b->S, 1024, 0, b->stream>>>(d);
    mph::k_bt_place<<<nb, 256, 0, b->stream>>>(d);
    mph::k_bt_gather<<<nb, 256, 0, b->stream>>>(d);
    mph::k_bt_commit<<<nb, 256, 0, b->stream>>>(d);
}

static void launch_sweep(mph_batch* b, int sw) {
    mph::SweepFn f = b->dim == 2 ? mph::sweep_fn<2>(sw, b->has_st) : mph::sweep_fn<3>(sw, b->has_st);
    f<<<sw == 0 ? b->grid_a : b->grid_b, b->threads, sw == 0 ? b->smem_a : b->smem_b, b->stream>>>(b->d);
}

// One step as direct launches: move, the five (usually empty) sort kernels,
// sweep A, sweep B.
static void launch_step(mph_batch* b) {
    {
        BLaunch l(b, "batch_move", 1);
        mph::k_bt_move<<<mph::nblocks(b->n, 256), 256, 0, b->stream>>>(b->d);
    }
    {
        BLaunch l(b, "batch_rebuild", 5);
        launch_rebuild(b);
    }
    {
        BLaunch l(b, "batch_sweep_a", 1);
        launch_sweep(b, 0);
    }
    {
        BLaunch l(b, "batch_sweep_b", 1);
        launch_sweep(b, 1);
    }
}

static int ensure_graph(mph_batch* b) {
    if (b->exec) return MPH_OK;
    BTRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const long long before = b->launches;
    for (int k = 0; k < mph::kGraphSteps; ++k) launch_step(b);
    b->launches = before;
    cudaGraph_t g = nullptr;
    BTRY(b, cudaStreamEndCapture(b->stream, &g));
    b->graph = g;
    BTRY(b, cudaGraphInstantiate(&b->exec, g, 0));
    return MPH_OK;
}

static int check_ctl(mph_batch* b) {
    BTRY(b, cudaMemcpyAsync(b->h_ctl, b->d.ctl, 8 * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    BTRY(b, cudaStreamSynchronize(b->stream));
    const int e = b->h_ctl[1];
    if (e & mph::BERR_CAPACITY)
        return bfail(b, MPH_ERR_CAPACITY, "a one-cell tile and its halo exceed the staging capacity");
    if (e & mph::BERR_NONFINITE) return bfail(b, MPH_ERR_NONFINITE, "non-finite velocity");
    return MPH_OK;
}

extern "C" int mph_batch_create(int n_scenes, const mph_params* params, const mph_grid_header* headers, int dim,
                                const int* type, const double* xyz, const double* vel, mph_batch** out) {
    if (!out) return bfail(nullptr, MPH_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (n_scenes < 1 || !params || !headers || !type || !xyz || !vel || (dim != 2 && dim != 3))
        return bfail(nullptr, MPH_ERR_ARG, "bad arguments");
    mph_batch* b = new mph_batch();
    b->dim = dim;
    b->S = n_scenes;
    b->hs.resize(n_scenes);
    b->pbase.assign(n_scenes + 1, 0);
    b->cell_count.resize(n_scenes);
    long long ntot = 0, ctot = 0;
    for (int s = 0; s < n_scenes; ++s) {
        const mph_params& p = params[s];
        const mph_grid_header& h = headers[s];
        if (h.particle_count < 1) {
            mph_batch_destroy(b);
            return bfail(nullptr, MPH_ERR_ARG, "every scene needs particles");
        }
        for (int t = 2; t < MPH_TYPE_COUNT; ++t)
            for (int k = 0; k < 3; ++k)
                if (p.wall_velocity[t][k] != 0.0 || p.wall_omega[t][k] != 0.0) {
                    mph_batch_destroy(b);
                    return bfail(nullptr, MPH_ERR_ARG, "the batched form takes static walls only");
                }
        mph_constants k{};
        int st = mph_compute_constants(&p, &h, dim, &k);
        mph::SimConst sc{};
        std::string msg;
        if (st == MPH_OK) st = mph::make_simconst(p, h, k, dim, h.particle_count, sc, msg);
        else msg = "scene constants";
        if (st == MPH_OK && (sc.cc[0] < 3 || sc.cc[1] < 3 || (dim == 3 && sc.cc[2] < 3))) {
            st = MPH_ERR_GEOMETRY;
            msg = "the batched form needs at least 3 cells per axis";
        }
        if (st != MPH_OK) {
            mph_batch_destroy(b);
            return bfail(nullptr, st, "scene " + std::to_string(s) + ": " + msg);
        }
        BScene& bs = b->hs[s];
        fill_bscene(bs, sc, k);
        bs.pbase = (int)ntot;
        bs.cbase = (int)ctot;
        b->pbase[s] = (int)ntot;
        if (sc.has_st) b->has_st = true;
        ntot += h.particle_count;
        ctot += sc.tot;
        if (ntot > (1LL << 30) || ctot > (1LL << 30)) {
            mph_batch_destroy(b);
            return bfail(nullptr, MPH_ERR_ARG, "batch too large");
        }
    }
    b->pbase[n_scenes] = (int)ntot;
    b->n = (int)ntot;
    b->cells = (int)ctot;
    std::vector<double4> hp(ntot), hvv(ntot);
    std::vector<int> hpi(ntot), hsid(ntot), hflags(n_scenes, 1);
    for (int s = 0; s < n_scenes; ++s) {
        const BScene& sc = b->hs[s];
        std::vector<int>& cnt = b->cell_count[s];
        cnt.assign((size_t)sc.tot, 0);
        for (int q = 0; q < headers[s].particle_count; ++q) {
            const long long i = (long long)sc.pbase + q;
            const int t = type[i];
            if (t < 0 || t >= MPH_TYPE_COUNT) {
                mph_batch_destroy(b);
                return bfail(nullptr, MPH_ERR_ARG, "particle type out of range");
            }
            for (int k = 0; k < 3; ++k)
                if (!std::isfinite(xyz[3 * i + k]) || !std::isfinite(vel[3 * i + k])) {
                    mph_batch_destroy(b);
                    return bfail(nullptr, MPH_ERR_ARG, "non-finite input");
                }
            hp[i] = make_double4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], (double)t);
            const bool wall = t >= 2;  // static walls: calculateWall gives them zero velocity (main.cpp:2013-2053)
            hvv[i] = wall ? make_double4(0, 0, 0, 0) : make_double4(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2], 0);
            hpi[i] = q;
            hsid[i] = s;
            if (t < 2) ++b->n_fluid;
            int c3[3];
            const double x3[3] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
            for (int k = 0; k < 3; ++k) {
                const double w = sc.width[k];
                double xr = x3[k] - sc.dmin[k];
                xr -= w * std::floor(xr / w);
                c3[k] = std::min(sc.cc[k] - 1, std::max(0, (int)std::floor(xr / sc.cell_width[k])));
            }
            ++cnt[((size_t)c3[0] * sc.cc[1] + c3[1]) * sc.cc[2] + c3[2]];
        }
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    BatchDev& d = b->d;
    const size_t n = (size_t)ntot;
    if (e == cudaSuccess) e = balloc(&b->d_scenes, (size_t)n_scenes);
    if (e == cudaSuccess) e = balloc(&b->d_sid, n);
    if (e == cudaSuccess) e = balloc(&d.pos, n);
    if (e == cudaSuccess) e = balloc(&d.vel, n);
    if (e == cudaSuccess) e = balloc(&d.snap, n);
    if (e == cudaSuccess) e = balloc(&d.pidx, n);
    if (e == cudaSuccess) e = balloc(&d.pos_t, n);
    if (e == cudaSuccess) e = balloc(&d.vel_t, n);
    if (e == cudaSuccess) e = balloc(&d.pidx_t, n);
    if (e == cudaSuccess) e = balloc(&d.key, n);
    if (e == cudaSuccess) e = balloc(&d.slot, n);
    if (e == cudaSuccess) e = balloc(&d.tmp, n);
    if (e == cudaSuccess) e = balloc(&d.counts, (size_t)ctot);
    if (e == cudaSuccess) e = balloc(&d.start, (size_t)ctot + 1);
    if (e == cudaSuccess) e = balloc(&d.vp, n);
    if (e == cudaSuccess) e = balloc(&d.gc, n);
    if (e == cudaSuccess) e = balloc(&d.flags, (size_t)n_scenes);
    if (e == cudaSuccess) e = balloc(&d.ctl, 8);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&b->h_ctl, 8 * sizeof(int));
    if (e != cudaSuccess) {
        const std::string m = std::string("batch allocation: ") + cudaGetErrorString(e);
        mph_batch_destroy(b);
        return bfail(nullptr, MPH_ERR_NOMEM, m);
    }
    d.n = b->n;
    d.S = n_scenes;
    d.scenes = b->d_scenes;
    d.sid = b->d_sid;
    const int end = (int)ntot;
    const int ctl0[8] = {1, 0, 0, 0, 0, 0, 0, 0};  // sort every scene once
    cudaStream_t st = b->stream;
    e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMemcpyAsync(d.pos, hp.data(), n * sizeof(double4), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d.vel, hvv.data(), n * sizeof(double4), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d.pidx, hpi.data(), n * sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_sid, hsid.data(), n * sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d.counts, 0, (size_t)ctot * sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d.vp, 0, n * sizeof(float4), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d.gc, 0, n * sizeof(float4), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d.start + ctot, &end, sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d.flags, hflags.data(), hflags.size() * sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d.ctl, ctl0, sizeof(ctl0), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // host vectors go out of scope below
    if (e != cudaSuccess) {
        const std::string m = std::string("batch upload: ") + cudaGetErrorString(e);
        mph_batch_destroy(b);
        return bfail(nullptr, MPH_ERR_CUDA, m);
    }
    const int t2d[3] = {8, 8, 1}, t3d[3] = {2, 2, 4};  // defaults until mph_batch_autotune / set_tiles
    int rc = configure(b, dim == 2 ? t2d : t3d, 256);
    if (rc == MPH_OK) {
        // the initial sort of every scene (the reference's start-up neighbour
        // build, main.cpp:357-359)
        launch_rebuild(b);
        b->launches += 5;
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemsetAsync(d.flags, 0, (size_t)n_scenes * sizeof(int), st);
        if (e == cudaSuccess) e = cudaMemsetAsync(d.ctl, 0, 8 * sizeof(int), st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = bfail(b, MPH_ERR_CUDA, std::string("initial sort: ") + cudaGetErrorString(e));
    }
    if (rc != MPH_OK) {
        const std::string m = b->err;
        mph_batch_destroy(b);
        return bfail(nullptr, rc, m);
    }
    *out = b;
    return MPH_OK;
}

extern "C" int mph_batch_step(mph_batch* b, int nsteps) {
    if (!b || nsteps < 0) return bfail(b, MPH_ERR_ARG, "bad arguments");
    if (b->prof.on) {
        for (int k = 0; k < nsteps; ++k) launch_step(b);
    } else {
        int left = nsteps;
        if (left >= mph::kGraphSteps) {
            const int rc = ensure_graph(b);
            if (rc != MPH_OK) return rc;
            for (; left >= mph::kGraphSteps; left -= mph::kGraphSteps) {
                BTRY(b, cudaGraphLaunch(b->exec, b->stream));
                b->launches += 8LL * mph::kGraphSteps;
            }
        }
        for (; left > 0; --left) launch_step(b);
    }
    BTRY(b, cudaGetLastError());
    b->steps += nsteps;
    return MPH_OK;
}

extern "C" int mph_batch_synchronize(mph_batch* b) {
    if (!b) return bfail(nullptr, MPH_ERR_ARG, "batch is NULL");
    return check_ctl(b);
}

extern "C" int mph_batch_get_state(mph_batch* b, double* xyz, double* vel) {
    if (!b || !xyz || !vel) return bfail(b, MPH_ERR_ARG, "bad arguments");
    const int rc = check_ctl(b);
    if (rc != MPH_OK) return rc;
    const size_t n = (size_t)b->n;
    std::vector<double4> hp(n), hv(n);
    std::vector<int> hpi(n);
    BTRY(b, cudaMemcpyAsync(hp.data(), b->d.pos, n * sizeof(double4), cudaMemcpyDeviceToHost, b->stream));
    BTRY(b, cudaMemcpyAsync(hv.data(), b->d.vel, n * sizeof(double4), cudaMemcpyDeviceToHost, b->stream));
    BTRY(b, cudaMemcpyAsync(hpi.data(), b->d.pidx, n * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    BTRY(b, cudaStreamSynchronize(b->stream));
    for (int s = 0; s < b->S; ++s)
        for (int p = b->pbase[s]; p < b->pbase[s + 1]; ++p) {
            const size_t o = 3 * ((size_t)b->pbase[s] + hpi[p]);
            xyz[o] = hp[p].x;
            xyz[o + 1] = hp[p].y;
            xyz[o + 2] = hp[p].z;
            vel[o] = hv[p].x;
            vel[o + 1] = hv[p].y;
            vel[o + 2] = hv[p].z;
        }
    return MPH_OK;
}

extern "C" int mph_batch_set_tiles(mph_batch* b, int tx, int ty, int tz, int threads, int ctas_per_sm) {
    if (!b) return bfail(nullptr, MPH_ERR_ARG, "batch is NULL");
    if (ctas_per_sm < 0 || ctas_per_sm > 8) return bfail(b, MPH_ERR_ARG, "ctas_per_sm must be in [0, 8]");
    BTRY(b, cudaStreamSynchronize(b->stream));
    const int t[3] = {tx, ty, b->dim == 3 ? tz : 1};
    return configure(b, t, threads, ctas_per_sm > 0 ? ctas_per_sm : b->occ);
}

extern "C" int mph_batch_get_info(mph_batch* b, mph_batch_info* info) {
    if (!b || !info) return bfail(b, MPH_ERR_ARG, "bad arguments");
    const int rc = check_ctl(b);
    if (rc != MPH_OK) return rc;
    std::memset(info, 0, sizeof(*info));
    info->dim = b->dim;
    info->scenes = b->S;
    info->particles = b->n;
    info->fluid_particles = b->n_fluid;
    for (int d = 0; d < 3; ++d) info->tile[d] = b->tile[d];
    info->threads = b->threads;
    info->ctas_per_sm = b->occ;
    info->items = b->n_items;
    info->capacity = b->cap;
    info->grid_a = b->grid_a;
    info->grid_b = b->grid_b;
    info->graph_steps = mph::kGraphSteps;
    info->steps = b->steps;
    info->scene_rebuilds = b->h_ctl[6];
    info->tile_splits = b->h_ctl[7];
    info->launches = b->launches;
    return MPH_OK;
}

// Device state a trial may change: saved before the autotuner's trials and
// put back after each.
struct BatchBackup {
    double4 *pos = nullptr, *vel = nullptr, *snap = nullptr;
    int *pidx = nullptr, *start = nullptr, *flags = nullptr, *ctl = nullptr;
};

static int backup_copy(mph_batch* b, BatchBackup& k, bool save) {
    const size_t n = (size_t)b->n;
    auto cp = [&](void* bk, void* live, size_t bytes) {
        return save ? cudaMemcpyAsync(bk, live, bytes, cudaMemcpyDeviceToDevice, b->stream)
                    : cudaMemcpyAsync(live, bk, bytes, cudaMemcpyDeviceToDevice, b->stream);
    };
    BTRY(b, cp(k.pos, b->d.pos, n * sizeof(double4)));
    BTRY(b, cp(k.vel, b->d.vel, n * sizeof(double4)));
    BTRY(b, cp(k.snap, b->d.snap, n * sizeof(double4)));
    BTRY(b, cp(k.pidx, b->d.pidx, n * sizeof(int)));
    BTRY(b, cp(k.start, b->d.start, ((size_t)b->cells + 1) * sizeof(int)));
    BTRY(b, cp(k.flags, b->d.flags, (size_t)b->S * sizeof(int)));
    BTRY(b, cp(k.ctl, b->d.ctl, 8 * sizeof(int)));
    return MPH_OK;
}

extern "C" int mph_batch_autotune(mph_batch* b, int steps, mph_batch_trial* trials, int capacity, int* count) {
    if (!b || steps < 1) return bfail(b, MPH_ERR_ARG, "bad arguments");
    int rc = check_ctl(b);
    if (rc != MPH_OK) return rc;
    std::vector<std::array<int, 5>> cand;  // tile x, y, z, CTA size, CTAs per SM the staging is sized for
    if (b->dim == 2) {
        const int ts[][2] = {{4, 4}, {4, 8}, {8, 4}, {8, 8}, {8, 16}, {16, 8}, {12, 12}, {16, 16}};
        for (auto& t : ts)
            for (int th : {128, 256})
                for (int oc : {2, 3, 4}) cand.push_back({t[0], t[1], 1, th, oc});
    } else {
        const int ts[][3] = {{1, 2, 2}, {2, 2, 2}, {2, 2, 4}, {2, 4, 4}, {4, 4, 4}, {1, 1, 4}, {1, 2, 4}};
        for (auto& t : ts)
            for (int th : {128, 256})
                for (int oc : {1, 2}) cand.push_back({t[0], t[1], t[2], th, oc});
    }
    const bool prof = b->prof.on;
    b->prof.on = false;
    const long long steps0 = b->steps, launches0 = b->launches;
    const int keep[3] = {b->tile[0], b->tile[1], b->tile[2]}, keep_threads = b->threads, keep_occ = b->occ;
    BatchBackup k;
    const size_t n = (size_t)b->n;
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = balloc(&k.pos, n);
    if (e == cudaSuccess) e = balloc(&k.vel, n);
    if (e == cudaSuccess) e = balloc(&k.snap, n);
    if (e == cudaSuccess) e = balloc(&k.pidx, n);
    if (e == cudaSuccess) e = balloc(&k.start, (size_t)b->cells + 1);
    if (e == cudaSuccess) e = balloc(&k.flags, (size_t)b->S);
    if (e == cudaSuccess) e = balloc(&k.ctl, 8);
    auto release = [&]() {
        void* ptrs[] = {k.pos, k.vel, k.snap, k.pidx, k.start, k.flags, k.ctl};
        for (void* p : ptrs)
            if (p) cudaFree(p);
    };
    if (e != cudaSuccess) {
        release();
        return bfail(b, MPH_ERR_NOMEM, std::string("autotune backup: ") + cudaGetErrorString(e));
    }
    rc = backup_copy(b, k, true);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e300;
    int best_i = -1, nt = 0;
    const int rounds = std::max(1, (steps + mph::kGraphSteps - 1) / mph::kGraphSteps);
    for (size_t ci = 0; ci < cand.size() && rc == MPH_OK; ++ci) {
        const int t[3] = {cand[ci][0], cand[ci][1], cand[ci][2]};
        rc = configure(b, t, cand[ci][3], cand[ci][4]);
        if (rc != MPH_OK) {  // a shape this GPU cannot hold: skip it
            cudaGetLastError();
            rc = MPH_OK;
            continue;
        }
        rc = backup_copy(b, k, false);
        if (rc == MPH_OK) rc = mph_batch_step(b, mph::kGraphSteps);  // warm-up, builds the graph
        if (rc != MPH_OK) break;
        cudaEventRecord(e0, b->stream);
        for (int r = 0; r < rounds && rc == MPH_OK; ++r) rc = mph_batch_step(b, mph::kGraphSteps);
        cudaEventRecord(e1, b->stream);
        if (rc == MPH_OK) rc = check_ctl(b);
        if (rc != MPH_OK) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double per = ms / (rounds * mph::kGraphSteps);
        if (trials && nt < capacity) {
            trials[nt].tile[0] = b->tile[0];
            trials[nt].tile[1] = b->tile[1];
            trials[nt].tile[2] = b->tile[2];
            trials[nt].threads = b->threads;
            trials[nt].ctas_per_sm = b->occ;
            trials[nt].capacity = b->cap;
            trials[nt].ms_per_step = per;
        }
        ++nt;
        if (per < best) {
            best = per;
            best_i = (int)ci;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc == MPH_OK) rc = backup_copy(b, k, false);
    if (rc == MPH_OK) {
        if (best_i >= 0) {
            const int t[3] = {cand[best_i][0], cand[best_i][1], cand[best_i][2]};
            rc = configure(b, t, cand[best_i][3], cand[best_i][4]);
        } else {
            rc = configure(b, keep, keep_threads, keep_occ);
        }
    }
    if (rc == MPH_OK) {
        e = cudaStreamSynchronize(b->stream);
        if (e != cudaSuccess) rc = bfail(b, MPH_ERR_CUDA, cudaGetErrorString(e));
    }
    release();
    b->steps = steps0;
    b->launches = launches0;
    b->prof.on = prof;
    if (count) *count = nt;
    return rc;
}

extern "C" void* mph_batch_stream(mph_batch* b) { return b ? (void*)b->stream : nullptr; }

extern "C" int mph_batch_profile_enable(mph_batch* b, int enable) {
    if (!b) return bfail(nullptr, MPH_ERR_ARG, "batch is NULL");
    BTRY(b, cudaStreamSynchronize(b->stream));
    for (auto& pe : b->prof.pending) {
        cudaEventDestroy(pe.a);
        cudaEventDestroy(pe.b);
    }
    b->prof = BatchProfile();
    b->prof.on = enable != 0;
    return MPH_OK;
}

extern "C" int mph_batch_profile_read(mph_batch* b, mph_kernel_stat* out, int capacity, int* count) {
    if (!b) return bfail(nullptr, MPH_ERR_ARG, "batch is NULL");
    BTRY(b, cudaStreamSynchronize(b->stream));
    BatchProfile& p = b->prof;
    for (auto& pe : p.pending) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, pe.a, pe.b);
        p.ms[pe.id] += ms;
        p.launches[pe.id] += pe.count;
        cudaEventDestroy(pe.a);
        cudaEventDestroy(pe.b);
    }
    p.pending.clear();
    const int nn = (int)p.names.size();
    for (int k = 0; k < nn && k < capacity && out; ++k) {
        std::memset(out[k].name, 0, sizeof(out[k].name));
        std::strncpy(out[k].name, p.names[k].c_str(), sizeof(out[k].name) - 1);
        out[k].launches = p.launches[k];
        out[k].total_ms = p.ms[k];
    }
    if (count) *count = nn;
    return MPH_OK;
}

extern "C" int mph_batch_last_error(mph_batch* b, char* buf, int len) {
    const std::string& m = b ? b->err : g_batch_err;
    if (buf && len > 0) {
        std::strncpy(buf, m.c_str(), (size_t)len - 1);
        buf[len - 1] = 0;
    }
    return (int)m.size();
}
