// k_mixed.cu — the mixed-precision MPH-WC step on sm_100a.
//
// Same physics and step order as the reference loop (main.cpp:386-431), with
//   * a stable counting sort by cell (histogram -> scan -> scatter -> in-cell
//     ordering by previous index) instead of the bitonic network;
//   * FP32 pair arithmetic on cell-relative coordinates: each particle keeps
//     its FP32 offset from the origin of its home cell (the cell of the last
//     list build), and every list entry packs the neighbour index with a 5-bit
//     code of the neighbouring cell's offset, so x_j - x_i = (o_j - o_i) +
//     D[code] never subtracts two large FP32 coordinates;
//   * one neighbour table, entries within RP+margin first, so the density
//     sweep walks the short part only; the force sweep runs for fluid
//     particles only (walls never accelerate);
//   * Kahan-compensated FP32 per-particle sums; FP64 position/velocity
//     integration, FP64 global sums.
// Quantities the reference computes for output only (DensityA without surface
// tension, wall forces) are computed when the state is read back.
#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <vector>
#include "mph_mixed.h"
#include "mph_pair32.cuh"

namespace mph {

namespace {

constexpr int kCodeBits = 5;  // 27 neighbour-cell offsets

// Resident 128-thread blocks per SM the force sweep is compiled for (register
// cap 65536 / (128 * blocks)); set by measurement on the full dam break.
#ifndef MPH_MIXB_MINB_FUSED
#define MPH_MIXB_MINB_FUSED 8
#endif
// ... and of its surface-tension variants (more live values per pair): on the
// 8.5 M-particle two-fluid column 10.06 ms at 8 blocks (some spilling), 10.28
// at 6 and 11.06 at 5, results identical.
#ifndef MPH_MIXB_MINB_ST
#define MPH_MIXB_MINB_ST 8
#endif
// Resident 128-thread blocks per SM of the table-free force sweep.
#ifndef MPH_WALK_MINB
#define MPH_WALK_MINB 6
#endif

struct MixConst {
    int n, tot, dim, has_st, ratio_all_one, uniform_mu;
    int cap_s;                         // table rows of the short part; the long part follows
    int cc[3], range[3];
    double grid, inv_grid;             // hi-part grid (a power of two, metres)
    float dhi[27][4];                  // cell-origin offset per code: hi part (on the grid)
    float dlo[27][4];                  //                              lo part
    float list_r2, short_r2;           // (MaxRadius+m)^2, (RP+m)^2
    float walk_r2, walk_short2;        // cell walk: (largest force radius + s)^2, (RP + s)^2, s = 8 grid steps
    float ra2, rp2, rv2, rg2;
    float inv_ra, inv_rp, inv_rv, inv_rg;
    float ca, cp, cg, cv;              // (1/Sw)/h^D
    float cp_m2, cg_m2, cv_m2, ca_inv; // c*(-2/h); ca/h
    float p_a, p_b;                    // pressure:  cp*(-2/rp)*vol * (1 - r/rp) = p_a + p_b*r
    float v_a, v_b;                    // viscosity: -cv*(-2/rv)*vol * (1 - r/rv) = v_a + v_b*r
    float vol, vol_over_l0, n0a, n0p, inv_r2g_rg, l0;
    double p_a_d, p_b_d, v_a_d, v_b_d, cp_d, cp_m2_d, inv_rp_d, n0p_d;  // FP64 pressure core
    float inv_rp_lo, cp_lo;            // 1/RP and Cp as FP32 pairs: (inv_rp, inv_rp_lo), (cp, cp_lo)
    float visc_mu[MPH_TYPE_COUNT][MPH_TYPE_COUNT];
    float ratio[MPH_TYPE_COUNT][MPH_TYPE_COUNT];
    float a_k[MPH_TYPE_COUNT], cof_a[MPH_TYPE_COUNT];
    float bulk_modulus[MPH_TYPE_COUNT], bulk_viscosity[MPH_TYPE_COUNT];
};

__device__ __forceinline__ double omod(double x, double w) { return x - w * floor(x / w); }
__device__ __forceinline__ double omod_fast(double x, double w) {
    return (x >= 0.0 && x < 0.75 * w) ? x : omod(x, w);
}

__device__ __forceinline__ int pack_cell(int x, int y, int z) { return x | (y << 10) | (z << 20); }

// A particle's 32-byte record {hi position + type, velocity + PressureP} in
// one 256-bit read-only load: one L1 sector per neighbour instead of two.
__device__ __forceinline__ void ldg_pv(const float4* __restrict__ pv, int j, float4& p, float4& v) {
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(p.x), "=f"(p.y), "=f"(p.z), "=f"(p.w), "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(pv + 2 * (size_t)j));
}

// Cell-relative position in two FP32 words.  hi lies on a power-of-two grid g
// with |hi| < 2^24 g, so hi_j - hi_i + Dhi (also on the grid) is computed
// exactly; lo = x - hi (|lo| <= g/2) carries the rest.  The pair
// displacement ((hi_j - hi_i) + Dhi) + ((lo_j - lo_i) + Dlo) is then the true
// displacement rounded once to FP32, independent of where the cell sits.
__device__ __forceinline__ void rel32(const SimConst& c, const MixConst& m, const double4& p, int h, float4& hi,
                                      float4& lo) {
    const int hx = h & 1023, hy = (h >> 10) & 1023, hz = (h >> 20) & 1023;
    double d[3] = {p.x - (c.dmin[0] + (double)hx * c.cell_width[0]), p.y - (c.dmin[1] + (double)hy * c.cell_width[1]),
                   p.z - (c.dmin[2] + (double)hz * c.cell_width[2])};
    float h3[3], l3[3];
    for (int k = 0; k < 3; ++k) {
        if (d[k] > c.half_width[k]) d[k] -= c.width[k];  // minimum image from the home cell
        if (d[k] < -c.half_width[k]) d[k] += c.width[k];
        const double q = rint(d[k] * m.inv_grid) * m.grid;
        h3[k] = (float)q;
        l3[k] = (float)(d[k] - q);
    }
    hi = make_float4(h3[0], h3[1], h3[2], __int_as_float((int)p.w));
    lo = make_float4(l3[0], l3[1], l3[2], 0.0f);
}

// The neighbour table holds entries in rows of four: entries 4r..4r+3 of
// particle i are one uint4 at row r, column i (tab[r * n + i]), so a lane
// writes 16 bytes at a time when the table is built and the lanes of a warp
// read consecutive uint4 when it is swept.  Visits entries [0, cnt) in order.
template <class F>
__device__ __forceinline__ void for_entries(const uint4* __restrict__ tab, size_t n, int cnt, F&& f) {
    for (int k = 0; k < cnt; k += 4) {
        const uint4 q = __ldg(tab + (size_t)(k >> 2) * n);
        f(q.x);
        if (k + 1 < cnt) f(q.y);
        if (k + 2 < cnt) f(q.z);
        if (k + 3 < cnt) f(q.w);
    }
}

// ---- counting sort by cell ------------------------------------------------

// Cell key of main.cpp:1115-1133 (walls offset by TotalCellCount), its slot in
// the cell (atomic, order fixed later), the cell histogram.
__global__ void k_mix_cellkey(SimConst c, const double4* __restrict__ pos, int* __restrict__ keys,
                              int* __restrict__ slot, int* __restrict__ counts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const double4 p = pos[i];
    const int cx = ((int)floor((p.x - c.dmin[0]) / c.cell_width[0])) % c.cc[0];
    const int cy = ((int)floor((p.y - c.dmin[1]) / c.cell_width[1])) % c.cc[1];
    const int cz = ((int)floor((p.z - c.dmin[2]) / c.cell_width[2])) % c.cc[2];
    int id = ((cx % c.cc[0] + c.cc[0]) % c.cc[0]) * c.cc[1] * c.cc[2] +
             ((cy % c.cc[1] + c.cc[1]) % c.cc[1]) * c.cc[2] + ((cz % c.cc[2] + c.cc[2]) % c.cc[2]);
    const int t = (int)p.w;
    if (t >= 2 && t < 4) id += c.tot;
    keys[i] = id;
    slot[i] = atomicAdd(&counts[id], 1);
}

// Exclusive scan of counts[0..m) into out[0..m] (out[m] = total), one block:
// each thread scans a contiguous chunk; chunk totals are scanned in shared memory.
__global__ void __launch_bounds__(1024) k_mix_scan(const int* __restrict__ counts, int m, int* __restrict__ out) {
    __shared__ int part[1024];
    const int t = threadIdx.x;
    const int chunk = (m + blockDim.x - 1) / blockDim.x;
    const int b = min(m, t * chunk), e = min(m, b + chunk);
    int s = 0;
    for (int k = b; k < e; ++k) s += counts[k];
    part[t] = s;
    __syncthreads();
    for (int off = 1; off < (int)blockDim.x; off <<= 1) {  // Hillis-Steele inclusive scan
        const int v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = part[t] - s;
    for (int k = b; k < e; ++k) {
        out[k] = run;
        run += counts[k];
    }
    if (t == blockDim.x - 1) out[m] = part[t];
}

__global__ void k_mix_place(int n, const int* __restrict__ keys, const int* __restrict__ slot,
                            const int* __restrict__ start, int* __restrict__ tmp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    tmp[start[keys[i]] + slot[i]] = i;
}

// Order each cell's particles by their previous index (a stable sort overall).
__global__ void k_mix_rank(int n, const int* __restrict__ keys, const int* __restrict__ start,
                           const int* __restrict__ tmp, int* __restrict__ perm, int* __restrict__ sorted_keys) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int i = tmp[p];
    const int key = keys[i];
    const int b = start[key], e = start[key + 1];
    int rank = 0;
    for (int q = b; q < e; ++q) rank += tmp[q] < i;
    perm[b + rank] = i;
    sorted_keys[b + rank] = key;
}

// ---- list build -------------------------------------------------------------

// Home cell and FP32 positions after a sort (sorted order).
__global__ void k_mix_home(SimConst c, MixConst m, const double4* __restrict__ pos, const int* __restrict__ keys,
                           const double4* __restrict__ vel, int* __restrict__ home, float4* __restrict__ phl,
                           float4* __restrict__ p32, float4* __restrict__ v32) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    int k = keys[i];
    if (k >= c.tot) k -= c.tot;
    const int h = pack_cell(k / (c.cc[1] * c.cc[2]), (k / c.cc[2]) % c.cc[1], k % c.cc[2]);
    home[i] = h;
    float4 hi, lo;
    rel32(c, m, pos[i], h, hi, lo);
    phl[2 * (size_t)i] = hi;
    phl[2 * (size_t)i + 1] = lo;
    p32[i] = hi;
    const double4 v = vel[i];
    v32[i] = make_float4((float)v.x, (float)v.y, (float)v.z, 0.0f);
}

// Neighbour table, one warp per home key (the particles of one cell, fluid
// keys then the wall keys of the same cells): the lanes share the 3^D stencil
// (same visiting order as main.cpp:1356-1392) and walk it in step, 32 home
// particles at a time.  Each candidate range is read 32 records at a time
// (coalesced, into shared memory) and every lane tests all of them in FP32 on
// the cell-relative hi parts.  Entries are (j << 5 | code): pairs within
// RP+margin go to rows [0, cap_s), the rest within MaxRadius+margin to rows
// [cap_s, cap_s + cap_l), each part in stencil order.  Self is excluded.
// Walls without a fluid neighbour get no list (their pressure is never used).
constexpr int kMixListWarps = 4;

__global__ void __launch_bounds__(32 * kMixListWarps, 6)
k_mix_list(SimConst c, MixConst m, const float4* __restrict__ p32, const int* __restrict__ cellstart,
           unsigned* __restrict__ list, int cap_l, int* __restrict__ cnt_short, int* __restrict__ cnt_all,
           StepScalars* __restrict__ scal) {
    __shared__ float4 cand[kMixListWarps][32];
    __shared__ int2 sten[kMixListWarps][27];  // the stencil in visiting order: cell, offset code
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int key = blockIdx.x * kMixListWarps + wib;
    if (key >= 2 * c.tot) return;  // whole warp
    const int hb = cellstart[key], he = cellstart[key + 1];
    if (hb == he) return;
    const int ci = key >= c.tot ? key - c.tot : key;
    const int ic[3] = {ci / (c.cc[1] * c.cc[2]), (ci / c.cc[2]) % c.cc[1], ci % c.cc[2]};
    int jmin[3], w[3];
    for (int d = 0; d < 3; ++d) {
        const int r = c.range[d];
        w[d] = 2 * r + 1;
        const int b = (2 * r) - (ic[d] + r) % c.cc[d];
        jmin[d] = b > 0 ? b : 0;
    }
    // lane s < w0*w1*w2 computes stencil slot s of the visiting order (x
    // outer, z inner), once for all the key's chunks
    const int nsl = w[0] * w[1] * w[2];  // at most 27: range <= 1 on every axis
    if (lane < nsl) {
        const int ax = (jmin[0] + lane / (w[1] * w[2])) % w[0], ay = (jmin[1] + (lane / w[2]) % w[1]) % w[1],
                  az = (jmin[2] + lane % w[2]) % w[2];
        const int cx = ((ic[0] - c.range[0] + ax) % c.cc[0] + c.cc[0]) % c.cc[0];
        const int cy = ((ic[1] - c.range[1] + ay) % c.cc[1] + c.cc[1]) % c.cc[1];
        const int cz = ((ic[2] - c.range[2] + az) % c.cc[2] + c.cc[2]) % c.cc[2];
        sten[wib][lane] = make_int2(cx * c.cc[1] * c.cc[2] + cy * c.cc[2] + cz,
                                    (ax - c.range[0] + 1) * 9 + (ay - c.range[1] + 1) * 3 + (az - c.range[2] + 1));
    }
    __syncwarp();
    const int nf = cellstart[c.tot];
    const size_t n = (size_t)c.n;
    const int cap_s = m.cap_s;
    float4* cw = cand[wib];
    const float kInf = __int_as_float(0x7f800000);
    for (int h0 = hb; h0 < he; h0 += 32) {
        const int i = h0 + lane;
        const bool active = i < he;
        const float4 pi = p32[active ? i : hb];
        const bool is_wall = i >= nf;
        // box of the chunk's hi positions: the hi values, the cell offsets and
        // their sums and differences are exact on the hi grid, so a candidate
        // whose distance to the box is beyond the cut-off is no lane's neighbour
        float b0x = active ? pi.x : kInf, b0y = active ? pi.y : kInf, b0z = active ? pi.z : kInf;
        float b1x = active ? pi.x : -kInf, b1y = active ? pi.y : -kInf, b1z = active ? pi.z : -kInf;
        for (int o = 16; o > 0; o >>= 1) {
            b0x = fminf(b0x, __shfl_xor_sync(0xffffffffu, b0x, o));
            b0y = fminf(b0y, __shfl_xor_sync(0xffffffffu, b0y, o));
            b0z = fminf(b0z, __shfl_xor_sync(0xffffffffu, b0z, o));
            b1x = fmaxf(b1x, __shfl_xor_sync(0xffffffffu, b1x, o));
            b1y = fmaxf(b1y, __shfl_xor_sync(0xffffffffu, b1y, o));
            b1z = fmaxf(b1z, __shfl_xor_sync(0xffffffffu, b1z, o));
        }
        uint4* const ls = reinterpret_cast<uint4*>(list) + i;
        uint4* const ll = reinterpret_cast<uint4*>(list) + (size_t)(cap_s >> 2) * n + i;
        int cs = 0, cl = 0;
        unsigned s0 = 0, s1 = 0, s2 = 0, s3 = 0, l0 = 0, l1 = 0, l2 = 0, l3 = 0;  // rows being filled
        auto push = [n](unsigned e, int& cnt, int cap, uint4* row0, unsigned& b0, unsigned& b1, unsigned& b2,
                        unsigned& b3) {
            switch (cnt & 3) {
                case 0: b0 = e; break;
                case 1: b1 = e; break;
                case 2: b2 = e; break;
                default:
                    b3 = e;
                    if (cnt < cap) row0[(size_t)(cnt >> 2) * n] = make_uint4(b0, b1, b2, b3);
            }
            ++cnt;
        };
        bool any_fluid = !is_wall;  // a wall needs a list only if a fluid particle is within reach
        for (int sl = 0; sl < nsl; ++sl) {
            const int2 st = sten[wib][sl];
            const int cell = st.x, code = st.y;
            const float ox = m.dhi[code][0] - pi.x, oy = m.dhi[code][1] - pi.y, oz = m.dhi[code][2] - pi.z;
            for (int kind = 0; kind < 2; ++kind) {
                const int off = kind ? c.tot : 0;
                const int b = cellstart[cell + off], e = cellstart[cell + off + 1];
                for (int cb = b; cb < e; cb += 32) {
                    bool near = false;
                    float4 qc;
                    if (cb + lane < e) {
                        qc = p32[cb + lane];
                        const float ax = qc.x + m.dhi[code][0], ay = qc.y + m.dhi[code][1],
                                    az = qc.z + m.dhi[code][2];
                        const float ex = fmaxf(0.f, fmaxf(b0x - ax, ax - b1x));
                        const float ey = fmaxf(0.f, fmaxf(b0y - ay, ay - b1y));
                        const float ez = fmaxf(0.f, fmaxf(b0z - az, az - b1z));
                        near = ex * ex + ey * ey + ez * ez < m.list_r2;
                    }
                    const unsigned kept = __ballot_sync(0xffffffffu, near);
                    __syncwarp();
                    if (near) {
                        qc.w = __int_as_float(cb + lane);
                        cw[__popc(kept & ((1u << lane) - 1u))] = qc;
                    }
                    __syncwarp();
                    if (!active) continue;
                    const int mm = __popc(kept);
                    for (int t = 0; t < mm; ++t) {
                        const float4 q = cw[t];
                        const int j = __float_as_int(q.w);
                        const float dx = q.x + ox, dy = q.y + oy, dz = q.z + oz;
                        const float r2 = dx * dx + dy * dy + dz * dz;
                        if (r2 < m.list_r2 && j != i) {
                            if (kind == 0) any_fluid = true;
                            const unsigned entry = ((unsigned)j << kCodeBits) | (unsigned)code;
                            if (r2 < m.short_r2) push(entry, cs, cap_s, ls, s0, s1, s2, s3);
                            else push(entry, cl, cap_l, ll, l0, l1, l2, l3);
                        }
                    }
                }
            }
        }
        if (!active) continue;
        if ((cs & 3) != 0 && cs < cap_s) ls[(size_t)(cs >> 2) * n] = make_uint4(s0, s1, s2, s3);
        if ((cl & 3) != 0 && cl < cap_l) ll[(size_t)(cl >> 2) * n] = make_uint4(l0, l1, l2, l3);
        if (is_wall && !any_fluid) cs = cl = 0;
        cnt_short[i] = cs;
        cnt_all[i] = cs + cl;
        atomicMax(&scal->max_neighbors, cs + cl);
        atomicMax(&scal->max_short, cs);
        atomicMax(&scal->max_long, cl);
        if (cs > cap_s || cl > cap_l) atomicOr(&scal->flags, DEVFLAG_NEIGHBOR_OVERFLOW);
    }
}

// ---- per step -----------------------------------------------------------------

// Convection, wall motion, periodic wrap and the displacement maximum (the
// same FP64 expressions as the FP64 form's move), plus the FP32 copies of
// position (home-relative, hi/lo) and velocity for the pair sweeps.
__global__ void __launch_bounds__(256)
k_mix_move(SimConst c, MixConst m, const int* __restrict__ cellstart, double4* __restrict__ pos,
           double4* __restrict__ vel, const double4* __restrict__ snap, const double* __restrict__ wall_center,
           const int* __restrict__ home, float4* __restrict__ phl, float4* __restrict__ p32,
           float4* __restrict__ v32, StepScalars* __restrict__ scal) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double s2 = 0.0;
    if (i < c.n) {
        const int nf = cellstart[c.tot], we = cellstart[2 * c.tot];
        double4 p = pos[i];
        double4 v = vel[i];
        if (i < nf) {
            p.x += v.x * c.dt;
            p.y += v.y * c.dt;
            p.z += v.z * c.dt;
        } else if (i < we) {
            const int t = (int)p.w;
            const double* C = wall_center + 3 * t;
            const double(*R)[3] = c.wall_rot[t];
            const double* W = c.wall_omega[t];
            const double* U = c.wall_velocity[t];
            double r0 = p.x - C[0], r1 = p.y - C[1], r2 = p.z - C[2];
            r0 = R[0][0] * r0 + R[0][1] * r1 + R[0][2] * r2;
            r1 = R[1][0] * r0 + R[1][1] * r1 + R[1][2] * r2;
            r2 = R[2][0] * r0 + R[2][1] * r1 + R[2][2] * r2;
            v.x = W[1] * r2 - W[2] * r1 + U[0];
            v.y = W[2] * r0 - W[0] * r2 + U[1];
            v.z = W[0] * r1 - W[1] * r0 + U[2];
            vel[i] = v;
            p.x = r0 + C[0] + U[0] * c.dt;
            p.y = r1 + C[1] + U[1] * c.dt;
            p.z = r2 + C[2] + U[2] * c.dt;
        }
        p.x = omod_fast(p.x - c.dmin[0], c.width[0]) + c.dmin[0];
        p.y = omod_fast(p.y - c.dmin[1], c.width[1]) + c.dmin[1];
        p.z = omod_fast(p.z - c.dmin[2], c.width[2]) + c.dmin[2];
        pos[i] = p;
        float4 hi, lo;
        rel32(c, m, p, home[i], hi, lo);
        phl[2 * (size_t)i] = hi;
        phl[2 * (size_t)i + 1] = lo;
        p32[i] = hi;
        v32[i] = make_float4((float)v.x, (float)v.y, (float)v.z, 0.0f);
        const double4 q = snap[i];
        const double d0 = omod_fast(p.x - q.x + c.half_width[0], c.width[0]) - c.half_width[0];
        const double d1 = omod_fast(p.y - q.y + c.half_width[1], c.width[1]) - c.half_width[1];
        const double d2 = omod_fast(p.z - q.z + c.half_width[2], c.width[2]) - c.half_width[2];
        s2 = d0 * d0 + d1 * d1 + d2 * d2;
        if (!(s2 > 0.0)) s2 = 0.0;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double t = __shfl_xor_sync(0xffffffffu, s2, o);
        s2 = t > s2 ? t : s2;
    }
    __shared__ double red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double mx = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) mx = red[w] > mx ? red[w] : mx;
        if (mx > 0.0) atomicMax(&scal->max_shift2_bits, (unsigned long long)__double_as_longlong(mx));
    }
}

// Offset tables in shared memory: per-lane codes differ, and shared memory
// serves divergent addresses in one access where the constant bank serialises.
struct SharedTables {
    float4 dhi[27];
    float4 dlo[27];
    float mu[MPH_TYPE_COUNT * MPH_TYPE_COUNT];
};

__device__ __forceinline__ void load_tables(const MixConst& m, SharedTables& t) {
    for (int k = threadIdx.x; k < 27; k += blockDim.x) {
        t.dhi[k] = make_float4(m.dhi[k][0], m.dhi[k][1], m.dhi[k][2], 0.f);
        t.dlo[k] = make_float4(m.dlo[k][0], m.dlo[k][1], m.dlo[k][2], 0.f);
    }
    for (int k = threadIdx.x; k < 16; k += blockDim.x) t.mu[k] = m.visc_mu[k / 4][k % 4];
    __syncthreads();
}

// One DensityP term wp = Cp (1 - r/RP)^2 as an unevaluated sum of two FP32
// numbers, added to the pair sum (sh, sl), with FP32 operations only.  The
// displacement arrives as its exact hi part (grid multiples) and its small lo
// part; error-free transformations (Knuth's TwoSum, Dekker's Fast2Sum, the
// FMA product error a*b - RN(a*b); Muller et al., Handbook of Floating-Point
// Arithmetic, chs. 4-5) carry r^2, r, 1 - r/RP and the square to about 2^-44
// relative.  The strain is a small difference of a sum near N0p, so the
// per-term rounding of plain FP32 (~1e-7 relative) would dominate the error.
__device__ __forceinline__ void wp_df(const MixConst& m, float hx, float hy, float hz, float lx, float ly,
                                      float lz, float& sh, float& sl) {
    // renormalise each axis so that hi is the FP32 rounding of hi + lo
    { const float t = hx + lx; lx -= t - hx; hx = t; }
    { const float t = hy + ly; ly -= t - hy; hy = t; }
    { const float t = hz + lz; lz -= t - hz; hz = t; }
    const float px = hx * hx, py = hy * hy, pz = hz * hz;
    const float ex = fmaf(hx, hx, -px), ey = fmaf(hy, hy, -py), ez = fmaf(hz, hz, -pz);
    const float s1 = px + py;
    float bb = s1 - px;
    const float e1 = (px - (s1 - bb)) + (py - bb);
    const float s2 = s1 + pz;
    bb = s2 - s1;
    const float e2 = (s1 - (s2 - bb)) + (pz - bb);
    float lo = e1 + e2 + ex + ey + ez + 2.0f * (hx * lx + hy * ly + hz * lz);
    const float hi = s2 + lo;
    lo -= hi - s2;
    // r = sqrt(hi + lo): r0 + rl
    const float y = rsqrt_nr(hi);
    const float r0 = hi * y;
    const float rl = (fmaf(-r0, r0, hi) + lo) * (0.5f * y);
    // q = 1 - r / RP: qh + ql
    const float t = r0 * m.inv_rp;
    const float te = fmaf(r0, m.inv_rp, -t) + r0 * m.inv_rp_lo + rl * m.inv_rp;
    const float qh = 1.0f - t;
    const float ql = ((1.0f - qh) - t) - te;
    // w = Cp q^2: wh + wl
    const float p2 = qh * qh;
    const float p2e = fmaf(qh, qh, -p2) + 2.0f * qh * ql;
    const float wh = m.cp * p2;
    const float wl = fmaf(m.cp, p2, -wh) + m.cp * p2e + m.cp_lo * p2;
    // (sh, sl) += (wh, wl)
    const float sn = sh + wh;
    bb = sn - sh;
    const float se = (sh - (sn - bb)) + (wh - bb);
    sh = sn;
    sl += se + wl;
}

// Sweep A: DensityP and DivergenceP over the short part of the list with the
// exact FP32 displacement (S64: pair arithmetic in FP64, the displacement
// assembled in FP64 from the hi/lo parts, FP32 velocities), plus, with
// surface tension, DensityA and GravityCenter over all of it; epilogue:
// coefficients, PressureP, PressureA (main.cpp:1631-1662, 1735-1740, 1831-1906).
template <bool ST, bool RATIO, bool S64>
__global__ void __launch_bounds__(128)
k_mix_a(MixConst m, const float4* __restrict__ phl, const float4* __restrict__ v32,
        const unsigned* __restrict__ list, const int* __restrict__ cnt_short, const int* __restrict__ cnt_all,
        float4* __restrict__ pv, float4* __restrict__ gca, double* __restrict__ strain_out,
        double* __restrict__ div_out, double* __restrict__ dens_a_out, double* __restrict__ wall_center,
        const SimConst c, const double4* __restrict__ vel64,
        double4* __restrict__ press64) {
    __shared__ SharedTables tb;
    load_tables(m, tb);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (wall_center != nullptr && blockIdx.x == 0 && threadIdx.x < 12) {
        const int t = threadIdx.x / 3, d = threadIdx.x % 3;
        if (t >= 2) wall_center[3 * t + d] += c.wall_velocity[t][d] * c.dt;
    }
    if (i >= m.n) return;
    const float4 pi = phl[2 * (size_t)i];
    const float4 li = phl[2 * (size_t)i + 1];
    const float4 vi = v32[i];
    const int ti = __float_as_int(pi.w);
    const int ns = cnt_short[i];
    const int na = ST ? cnt_all[i] : ns;
    const size_t n = (size_t)m.n;
    float sph = 0.f, spl = 0.f, sd = 0.f, cdk = 0.f;
    double spd = 0.0, sdd = 0.0;
    float sa = 0.f, cak = 0.f, g0 = 0.f, g1 = 0.f, g2 = 0.f;
    const uint4* tab = reinterpret_cast<const uint4*>(list) + i;
    for_entries(tab, n, ns, [&](unsigned e) {
        const int j = (int)(e >> kCodeBits), code = (int)(e & 31u);
        float4 pj, lj;
        ldg_pv(phl, j, pj, lj);  // {hi, lo} in one 256-bit load
        const float4 dh = tb.dhi[code], dl = tb.dlo[code];
        float dx, dy, dz;
        if (S64) {
            // FP64 displacement: the hi difference plus the cell offset is exact in
            // FP32 (grid multiples), the lo parts carry the rest to ~1e-14 l0
            const double dxd = (double)((pj.x - pi.x) + dh.x) + (((double)lj.x - (double)li.x) + (double)dl.x);
            const double dyd = (double)((pj.y - pi.y) + dh.y) + (((double)lj.y - (double)li.y) + (double)dl.y);
            const double dzd = (double)((pj.z - pi.z) + dh.z) + (((double)lj.z - (double)li.z) + (double)dl.z);
            const double r2d = dxd * dxd + dyd * dyd + dzd * dzd;
            if (r2d <= c.rp2) {
                const double y = rsqrt_dnr(r2d);
                const double q = 1.0 - r2d * y * m.inv_rp_d;
                spd += m.cp_d * q * q;
                const double dw = m.cp_m2_d * q;
                const float4 vj = v32[j];
                sdd -= (((double)vj.x - (double)vi.x) * dxd + ((double)vj.y - (double)vi.y) * dyd +
                        ((double)vj.z - (double)vi.z) * dzd) * y * dw;
            }
            dx = (float)dxd;
            dy = (float)dyd;
            dz = (float)dzd;
        } else {
            dx = ((pj.x - pi.x) + dh.x) + ((lj.x - li.x) + dl.x);
            dy = ((pj.y - pi.y) + dh.y) + ((lj.y - li.y) + dl.y);
            dz = ((pj.z - pi.z) + dh.z) + ((lj.z - li.z) + dl.z);
        }
        const float r2 = dx * dx + dy * dy + dz * dz;
        const float rinv = rsqrt_nr(r2);
        const float r = r2 * rinv;
        if (!S64 && r2 <= m.rp2) {
            wp_df(m, (pj.x - pi.x) + dh.x, (pj.y - pi.y) + dh.y, (pj.z - pi.z) + dh.z, (lj.x - li.x) + dl.x,
                  (lj.y - li.y) + dl.y, (lj.z - li.z) + dl.z, sph, spl);  // wp
            const float q = 1.0f - r * m.inv_rp;
            const float dw = m.cp_m2 * q;                        // dwpdr
            const float4 vj = v32[j];
            const float ue = ((vj.x - vi.x) * dx + (vj.y - vi.y) * dy + (vj.z - vi.z) * dz) * rinv;
            kahan_add(sd, cdk, -ue * dw);
        }
        if (ST) st_density<RATIO>(m, ti, __float_as_int(pj.w), r2, r, dx, dy, dz, sa, cak, g0, g1, g2);
    });
    if (ST) {  // surface tension only: the long part
        for_entries(tab + (size_t)(m.cap_s >> 2) * n, n, na - ns, [&](unsigned e) {
            const int j = (int)(e >> kCodeBits), code = (int)(e & 31u);
            const float4 pj = phl[2 * (size_t)j];
            const float4 dh = tb.dhi[code];
            const float dx = (pj.x - pi.x) + dh.x, dy = (pj.y - pi.y) + dh.y, dz = (pj.z - pi.z) + dh.z;
            const float r2 = dx * dx + dy * dy + dz * dz;
            st_density<RATIO>(m, ti, __float_as_int(pj.w), r2, r2 * rsqrtf(r2), dx, dy, dz, sa, cak, g0, g1, g2);
        });
    }
    double strain, div;
    if (S64) {
        strain = spd - m.n0p_d;
        div = sdd;
    } else {
        // the pair sum is exact to ~2^-44: N0p is subtracted in FP64 (the
        // strain is a small difference of two numbers near N0p)
        strain = ((double)sph + (double)spl) - m.n0p_d;
        div = (double)sd - (double)cdk;
    }
    double kappa = c.bulk_modulus[ti];
    if (strain < 0.0) kappa = 0.0;
    const double pp = -c.bulk_viscosity[ti] * div + kappa * strain;
    float pa = 0.0f;
    if (ST) {
        const float dens = sa - cak;
        pa = m.cof_a[ti] * (dens - m.n0a) / m.l0;
        if (m.n0a <= dens) pa = 0.0f;
        dens_a_out[i] = dens;
        gca[i] = make_float4(g0, g1, g2, pa);
    }
    pv[2 * (size_t)i] = pi;
    pv[2 * (size_t)i + 1] = make_float4(vi.x, vi.y, vi.z, (float)pp);
    if (S64) {
        const double4 vid = vel64[i];
        press64[i] = make_double4(vid.x, vid.y, vid.z, pp);
    }
    strain_out[i] = strain;
    div_out[i] = div;
}

// Sweep B for fluid particles (WALLS: for the wall particles, output only),
// FP32 in both mixed forms (the FP64 density sweep of MPH_MODE_MIXED_P64 sets
// the pressures this sweep reads).  The short part of the list: exact
// displacement, PressureP + ViscosityV (+ the surface-tension terms), Kahan
// sums.  The long part: the hi displacement, ViscosityV (+ surface tension),
// plain FP32 sum.  Then gravity and the FP64 velocity update
// (main.cpp:1908-2010).
template <bool ST, bool RATIO, bool WALLS>
__global__ void __launch_bounds__(128, ST ? MPH_MIXB_MINB_ST : MPH_MIXB_MINB_FUSED)
k_mix_b(MixConst m, SimConst c, const int* __restrict__ cellstart, const float4* __restrict__ phl,
        const float4* __restrict__ pv, const float4* __restrict__ gca,
        const unsigned* __restrict__ list, const int* __restrict__ cnt_short, const int* __restrict__ cnt_all,
        const double4* __restrict__ vel, double4* __restrict__ vel_out, double4* __restrict__ force,
        StepScalars* __restrict__ scal) {
    __shared__ SharedTables tb;
    load_tables(m, tb);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    const int nf = cellstart[c.tot];
    if (WALLS ? i < nf : i >= nf) {
        if (!WALLS) vel_out[i] = vel[i];
        return;
    }
    const float4 pi = phl[2 * (size_t)i];
    const float4 li = phl[2 * (size_t)i + 1];
    const float4 vi = pv[2 * (size_t)i + 1];
    const int ti = __float_as_int(pi.w);
    float4 gi = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ST) gi = gca[i];
    const float ai = m.a_k[ti];
    const int ns = cnt_short[i], na = cnt_all[i];
    const size_t n = (size_t)m.n;
    const float mu_u = tb.mu[ti * 4 + ti];
    float fx = 0.f, fy = 0.f, fz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;  // short part, Kahan
    float gx = 0.f, gy = 0.f, gz = 0.f;                                 // long part
    const uint4* tab = reinterpret_cast<const uint4*>(list) + i;
    for_entries(tab, n, ns, [&](unsigned e) {
        const int j = (int)(e >> kCodeBits), code = (int)(e & 31u);
        float4 pj, vj;
        ldg_pv(pv, j, pj, vj);
        const float4 lj = phl[2 * (size_t)j + 1];
        const float4 dh = tb.dhi[code], dl = tb.dlo[code];
        const float dx = ((pj.x - pi.x) + dh.x) + ((lj.x - li.x) + dl.x);
        const float dy = ((pj.y - pi.y) + dh.y) + ((lj.y - li.y) + dl.y);
        const float dz = ((pj.z - pi.z) + dh.z) + ((lj.z - li.z) + dl.z);
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (!(r2 < m.rv2 || r2 < m.rp2 || (ST && (r2 < m.ra2 || r2 < m.rg2)))) return;
        const float rinv = rsqrt_nr(r2);
        const float r = r2 * rinv;
        const int tj = __float_as_int(pj.w);
        float s = 0.0f;
        if (r2 < m.rp2) s += (vi.w + vj.w) * fmaf(m.p_b, r, m.p_a) * rinv;
        if (r2 < m.rv2) {
            const float mu = m.uniform_mu ? mu_u : tb.mu[ti * 4 + tj];
            const float ud = (vj.x - vi.x) * dx + (vj.y - vi.y) * dy + (vj.z - vi.z) * dz;
            s += mu * ud * fmaf(m.v_b, r, m.v_a) * (rinv * rinv * rinv);
        }
        float3 t = make_float3(0.f, 0.f, 0.f);
        if (ST) s += st_terms<RATIO>(m, ti, tj, r2, r, rinv, dx, dy, dz, gi, gca[j], ai, t);
        kahan_add(fx, cx, fmaf(s, dx, t.x));
        kahan_add(fy, cy, fmaf(s, dy, t.y));
        kahan_add(fz, cz, fmaf(s, dz, t.z));
    });
    // long part: a row of four pairs per iteration, their gathers issued
    // together so a thread keeps four independent loads in flight
    auto long_pair = [&](unsigned e, const float4& pj, const float4& vj) {
        const int code = (int)(e & 31u);
        const float4 dh = tb.dhi[code];
        const float dx = (pj.x - pi.x) + dh.x, dy = (pj.y - pi.y) + dh.y, dz = (pj.z - pi.z) + dh.z;
        const float r2 = dx * dx + dy * dy + dz * dz;
        const float rinv = rsqrtf(r2);
        float s = 0.0f;
        if (r2 < m.rv2) {
            const float r = r2 * rinv;
            const float mu = m.uniform_mu ? mu_u : tb.mu[ti * 4 + __float_as_int(pj.w)];
            const float ud = (vj.x - vi.x) * dx + (vj.y - vi.y) * dy + (vj.z - vi.z) * dz;
            s = mu * ud * fmaf(m.v_b, r, m.v_a) * (rinv * rinv * rinv);
        }
        if (ST) {
            if (r2 < m.ra2 || r2 < m.rg2) {
                const int j = (int)(e >> kCodeBits);
                float3 t = make_float3(0.f, 0.f, 0.f);
                s += st_terms<RATIO>(m, ti, __float_as_int(pj.w), r2, r2 * rinv, rinv, dx, dy, dz, gi, gca[j], ai, t);
                gx += t.x;
                gy += t.y;
                gz += t.z;
            }
        }
        gx = fmaf(s, dx, gx);
        gy = fmaf(s, dy, gy);
        gz = fmaf(s, dz, gz);
    };
    const uint4* tl = tab + (size_t)(m.cap_s >> 2) * n;
    const int nl = na - ns;
    for (int k = 0; k < nl; k += 4) {
        const uint4 q = __ldg(tl + (size_t)(k >> 2) * n);
        const unsigned e[4] = {q.x, q.y, q.z, q.w};
        float4 pj[4], vj[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k + u < nl) ldg_pv(pv, (int)(e[u] >> kCodeBits), pj[u], vj[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k + u < nl) long_pair(e[u], pj[u], vj[u]);
    }
    double F0 = ((double)fx - (double)cx) + (double)gx;
    double F1 = ((double)fy - (double)cy) + (double)gy;
    double F2 = ((double)fz - (double)cz) + (double)gz;
    if (WALLS) {
        force[i] = make_double4(F0, F1, F2, 0.0);
        return;
    }
    double4 v = vel[i];
    const double mass = c.density[ti] * c.vol;
    F0 += mass * c.gravity[0];
    F1 += mass * c.gravity[1];
    F2 += mass * c.gravity[2];
    v.x += F0 / mass * c.dt;
    v.y += F1 / mass * c.dt;
    v.z += F2 / mass * c.dt;
    if (!(isfinite(v.x) && isfinite(v.y) && isfinite(v.z))) atomicOr(&scal->flags, DEVFLAG_NONFINITE);
    force[i] = make_double4(F0, F1, F2, 0.0);
    vel_out[i] = v;
}

// The force sweep without the long table (MPH_MIXED_CELL_WALK).  One warp per
// home key walks the 3^D stencil in the table build's order (main.cpp:
// 1356-1392), reading each candidate range 32 records at a time (coalesced).
// A lane keeps its candidate when the candidate's hi position lies within
// the largest force radius of the bounding box of the warp's own particles;
// the kept records go to the warp's stage in shared memory (compacted by a
// ballot), and every lane evaluates every kept candidate against its own
// particle, reading the stage with broadcast loads.  Pair terms as in k_mix_b:
// where the hi-only distance is within RP (plus the hi/lo slack) the exact
// hi/lo displacement and Kahan sums, beyond it the hi displacement and plain
// sums.  Then gravity and the FP64 velocity update (main.cpp:1908-2010).  Wall
// keys carry their velocities over (walls never accelerate).
constexpr int kWalkWarps = 4;

struct WalkRec {
    float4 p;  // hi position + the cell offset's hi part (home-relative), type bits
    float4 v;  // velocity, PressureP
    float4 l;  // lo position + the cell offset's lo part, index bits
};

template <bool ST, bool RATIO>
__global__ void __launch_bounds__(32 * kWalkWarps, MPH_WALK_MINB)
k_mix_b_walk(MixConst m, SimConst c, const int* __restrict__ cellstart, const float4* __restrict__ phl,
             const float4* __restrict__ pv, const float4* __restrict__ gca, const double4* __restrict__ vel,
             double4* __restrict__ vel_out, double4* __restrict__ force, StepScalars* __restrict__ scal) {
    __shared__ WalkRec stage_all[kWalkWarps][32];
    __shared__ float4 gstage_all[kWalkWarps][ST ? 32 : 1];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int key = blockIdx.x * kWalkWarps + wib;
    if (key >= 2 * c.tot) return;  // whole warp
    const int hb = cellstart[key], he = cellstart[key + 1];
    if (hb == he) return;
    if (key >= c.tot) {  // wall key
        for (int i = hb + lane; i < he; i += 32) vel_out[i] = vel[i];
        return;
    }
    WalkRec* const stage = stage_all[wib];
    float4* const gstage = gstage_all[wib];
    const int ic[3] = {key / (c.cc[1] * c.cc[2]), (key / c.cc[2]) % c.cc[1], key % c.cc[2]};
    int jmin[3], w[3];
    for (int d = 0; d < 3; ++d) {
        const int r = c.range[d];
        w[d] = 2 * r + 1;
        const int b = (2 * r) - (ic[d] + r) % c.cc[d];
        jmin[d] = b > 0 ? b : 0;
    }
    const float kInf = __int_as_float(0x7f800000);
    for (int h0 = hb; h0 < he; h0 += 32) {
        const int i = h0 + lane;
        const bool act = i < he;
        const int ii = act ? i : hb;
        const float4 pi = phl[2 * (size_t)ii];
        const float4 li = phl[2 * (size_t)ii + 1];
        const float4 vi = pv[2 * (size_t)ii + 1];
        const int ti = __float_as_int(pi.w);
        float4 gi = make_float4(0.f, 0.f, 0.f, 0.f);
        if (ST) gi = gca[ii];
        const float ai = m.a_k[ti];
        const float mu_u = m.visc_mu[ti][ti];
        // bounding box of the chunk's hi positions
        float b0x = act ? pi.x : kInf, b0y = act ? pi.y : kInf, b0z = act ? pi.z : kInf;
        float b1x = act ? pi.x : -kInf, b1y = act ? pi.y : -kInf, b1z = act ? pi.z : -kInf;
        for (int o = 16; o > 0; o >>= 1) {
            b0x = fminf(b0x, __shfl_xor_sync(0xffffffffu, b0x, o));
            b0y = fminf(b0y, __shfl_xor_sync(0xffffffffu, b0y, o));
            b0z = fminf(b0z, __shfl_xor_sync(0xffffffffu, b0z, o));
            b1x = fmaxf(b1x, __shfl_xor_sync(0xffffffffu, b1x, o));
            b1y = fmaxf(b1y, __shfl_xor_sync(0xffffffffu, b1y, o));
            b1z = fmaxf(b1z, __shfl_xor_sync(0xffffffffu, b1z, o));
        }
        float fx = 0.f, fy = 0.f, fz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;  // within RP: Kahan
        float gx = 0.f, gy = 0.f, gz = 0.f;                                 // beyond
        for (int jx = jmin[0]; jx < jmin[0] + w[0]; ++jx)
            for (int jy = jmin[1]; jy < jmin[1] + w[1]; ++jy)
                for (int jz = jmin[2]; jz < jmin[2] + w[2]; ++jz) {
                    const int ax = jx % w[0], ay = jy % w[1], az = jz % w[2];
                    const int ncx = ((ic[0] - c.range[0] + ax) % c.cc[0] + c.cc[0]) % c.cc[0];
                    const int ncy = ((ic[1] - c.range[1] + ay) % c.cc[1] + c.cc[1]) % c.cc[1];
                    const int ncz = ((ic[2] - c.range[2] + az) % c.cc[2] + c.cc[2]) % c.cc[2];
                    const int cell = ncx * c.cc[1] * c.cc[2] + ncy * c.cc[2] + ncz;
                    const int code = (ax - c.range[0] + 1) * 9 + (ay - c.range[1] + 1) * 3 + (az - c.range[2] + 1);
                    const float dhx = m.dhi[code][0], dhy = m.dhi[code][1], dhz = m.dhi[code][2];
                    const float dlx = m.dlo[code][0], dly = m.dlo[code][1], dlz = m.dlo[code][2];
                    for (int kind = 0; kind < 2; ++kind) {
                        const int off = kind ? c.tot : 0;
                        const int b = cellstart[cell + off], e = cellstart[cell + off + 1];
                        for (int cb = b; cb < e; cb += 32) {
                            const int t = cb + lane;
                            bool keep = false;
                            float4 pj, vj, lj;
                            if (t < e) {
                                ldg_pv(pv, t, pj, vj);
                                lj = phl[2 * (size_t)t + 1];
                                pj.x += dhx;  // exact: both on the hi grid
                                pj.y += dhy;
                                pj.z += dhz;
                                const float ex = fmaxf(0.0f, fmaxf(b0x - pj.x, pj.x - b1x));
                                const float ey = fmaxf(0.0f, fmaxf(b0y - pj.y, pj.y - b1y));
                                const float ez = fmaxf(0.0f, fmaxf(b0z - pj.z, pj.z - b1z));
                                keep = ex * ex + ey * ey + ez * ez < m.walk_r2;
                            }
                            const unsigned kept = __ballot_sync(0xffffffffu, keep);
                            if (keep) {
                                const int slot = __popc(kept & ((1u << lane) - 1u));
                                stage[slot].p = pj;
                                stage[slot].v = vj;
                                stage[slot].l = make_float4(lj.x + dlx, lj.y + dly, lj.z + dlz, __int_as_float(t));
                                if (ST) gstage[slot] = gca[t];
                            }
                            __syncwarp();
                            const int cnt = __popc(kept);
                            if (act) {
                                for (int q = 0; q < cnt; ++q) {
                                    const float4 A = stage[q].p;
                                    const float hx = A.x - pi.x, hy = A.y - pi.y, hz = A.z - pi.z;  // exact
                                    const float r2h = hx * hx + hy * hy + hz * hz;
                                    if (!(r2h < m.walk_r2)) continue;
                                    const float4 L = stage[q].l;
                                    const int j = __float_as_int(L.w);
                                    if (j == i) continue;
                                    const float4 V = stage[q].v;
                                    const int tj = __float_as_int(A.w);
                                    if (r2h < m.walk_short2) {
                                        const float dx = hx + (L.x - li.x);
                                        const float dy = hy + (L.y - li.y);
                                        const float dz = hz + (L.z - li.z);
                                        const float r2 = dx * dx + dy * dy + dz * dz;
                                        if (!(r2 < m.rv2 || r2 < m.rp2 || (ST && (r2 < m.ra2 || r2 < m.rg2)))) continue;
                                        const float rinv = rsqrt_nr(r2);
                                        const float r = r2 * rinv;
                                        float sc = 0.0f;
                                        if (r2 < m.rp2) sc += (vi.w + V.w) * fmaf(m.p_b, r, m.p_a) * rinv;
                                        if (r2 < m.rv2) {
                                            const float mu = m.uniform_mu ? mu_u : m.visc_mu[ti][tj];
                                            const float ud = (V.x - vi.x) * dx + (V.y - vi.y) * dy + (V.z - vi.z) * dz;
                                            sc += mu * ud * fmaf(m.v_b, r, m.v_a) * (rinv * rinv * rinv);
                                        }
                                        float3 tt = make_float3(0.f, 0.f, 0.f);
                                        if (ST) sc += st_terms<RATIO>(m, ti, tj, r2, r, rinv, dx, dy, dz, gi, gstage[q], ai, tt);
                                        kahan_add(fx, cx, fmaf(sc, dx, tt.x));
                                        kahan_add(fy, cy, fmaf(sc, dy, tt.y));
                                        kahan_add(fz, cz, fmaf(sc, dz, tt.z));
                                    } else {
                                        const float rinv = rsqrtf(r2h);
                                        float sc = 0.0f;
                                        if (r2h < m.rv2) {
                                            const float r = r2h * rinv;
                                            const float mu = m.uniform_mu ? mu_u : m.visc_mu[ti][tj];
                                            const float ud = (V.x - vi.x) * hx + (V.y - vi.y) * hy + (V.z - vi.z) * hz;
                                            sc = mu * ud * fmaf(m.v_b, r, m.v_a) * (rinv * rinv * rinv);
                                        }
                                        if (ST) {
                                            if (r2h < m.ra2 || r2h < m.rg2) {
                                                float3 tt = make_float3(0.f, 0.f, 0.f);
                                                sc += st_terms<RATIO>(m, ti, tj, r2h, r2h * rinv, rinv, hx, hy, hz, gi,
                                                                      gstage[q], ai, tt);
                                                gx += tt.x;
                                                gy += tt.y;
                                                gz += tt.z;
                                            }
                                        }
                                        gx = fmaf(sc, hx, gx);
                                        gy = fmaf(sc, hy, gy);
                                        gz = fmaf(sc, hz, gz);
                                    }
                                }
                            }
                            __syncwarp();
                        }
                    }
                }
        if (!act) continue;
        double F0 = ((double)fx - (double)cx) + (double)gx;
        double F1 = ((double)fy - (double)cy) + (double)gy;
        double F2 = ((double)fz - (double)cz) + (double)gz;
        double4 v = vel[i];
        const double mass = c.density[ti] * c.vol;
        F0 += mass * c.gravity[0];
        F1 += mass * c.gravity[1];
        F2 += mass * c.gravity[2];
        v.x += F0 / mass * c.dt;
        v.y += F1 / mass * c.dt;
        v.z += F2 / mass * c.dt;
        if (!(isfinite(v.x) && isfinite(v.y) && isfinite(v.z))) atomicOr(&scal->flags, DEVFLAG_NONFINITE);
        force[i] = make_double4(F0, F1, F2, 0.0);
        vel_out[i] = v;
    }
}

// DensityA over the whole list (output only, without surface tension).
__global__ void k_mix_density_a(MixConst m, const float4* __restrict__ p32, const unsigned* __restrict__ list,
                                const int* __restrict__ cnt_short, const int* __restrict__ cnt_all,
                                double* __restrict__ dens_a_out) {
    __shared__ SharedTables tb;
    load_tables(m, tb);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    const float4 pi = p32[i];
    const int ti = __float_as_int(pi.w);
    const size_t n = (size_t)m.n;
    float sa = 0.f, ck = 0.f;
    const int ns = cnt_short[i], na = cnt_all[i];
    const uint4* tab = reinterpret_cast<const uint4*>(list) + i;
    auto visit = [&](unsigned e) {
        const int j = (int)(e >> kCodeBits), code = (int)(e & 31u);
        const float4 pj = p32[j];
        const float4 dh = tb.dhi[code];
        const float dx = (pj.x - pi.x) + dh.x, dy = (pj.y - pi.y) + dh.y, dz = (pj.z - pi.z) + dh.z;
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 <= m.ra2) {
            const float r = sqrtf(r2);
            const float q = r * m.inv_ra;
            const float ratio = m.ratio_all_one ? 1.0f : m.ratio[ti][__float_as_int(pj.w)];
            kahan_add(sa, ck, ratio * m.ca * q * (1.0f - q) * (1.0f - q));
        }
    };
    for_entries(tab, n, ns, visit);
    for_entries(tab + (size_t)(m.cap_s >> 2) * n, n, na - ns, visit);
    dens_a_out[i] = sa - ck;
}

// Virial pressure at particles for the mixed forms (output only; the FP64
// form's k_virial restates main.cpp:2057-2302).  Only the trace of the pair
// stress enters VirialPressureAtParticle = -trace / D, so each term reduces to
// a scalar per pair (x = x_j - x_i, r = |x|, e = x / r):
//   PressureP  (r < RP): P_i dwpdr(r) r
//   PressureA  (r < RA): PA_i ratio_ij dwadr(r) r
//   ViscosityV (r < RV): 0.5 C mu_ij (u_ij . e) (-dwvdr(r))
//   DiffuseInterface (r < RG): a_i (GC_i . x) ratio_ij (wg + dwgdr r) Rg / R2g / l0
// in FP32 on the exact cell-relative displacement, Kahan-compensated, with
// the velocities after the step (the reference calls it after
// calculateAcceleration, main.cpp:432-435).
template <bool ST, bool RATIO>
__global__ void __launch_bounds__(128)
k_mix_virial(MixConst m, const float4* __restrict__ phl, const float4* __restrict__ pv,
             const float4* __restrict__ gca, const double4* __restrict__ vel, const unsigned* __restrict__ list,
             const int* __restrict__ cnt_short, const int* __restrict__ cnt_all, double* __restrict__ virial) {
    __shared__ SharedTables tb;
    load_tables(m, tb);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    const float4 pi = phl[2 * (size_t)i];
    const float4 li = phl[2 * (size_t)i + 1];
    const int ti = __float_as_int(pi.w);
    const float ppi = pv[2 * (size_t)i + 1].w;
    const float4 gi = ST ? gca[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const double4 vd = vel[i];
    const float vix = (float)vd.x, viy = (float)vd.y, viz = (float)vd.z;
    const float ai = m.a_k[ti];
    const float inv_l0 = 1.0f / m.l0;
    const size_t n = (size_t)m.n;
    float tr = 0.f, ck = 0.f;
    auto visit = [&](unsigned e) {
        const int j = (int)(e >> kCodeBits), code = (int)(e & 31u);
        const float4 pj = phl[2 * (size_t)j];
        const float4 lj = phl[2 * (size_t)j + 1];
        const float4 dh = tb.dhi[code], dl = tb.dlo[code];
        const float dx = ((pj.x - pi.x) + dh.x) + ((lj.x - li.x) + dl.x);
        const float dy = ((pj.y - pi.y) + dh.y) + ((lj.y - li.y) + dl.y);
        const float dz = ((pj.z - pi.z) + dh.z) + ((lj.z - li.z) + dl.z);
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (!(r2 < m.rv2 || r2 < m.rp2 || (ST && (r2 < m.ra2 || r2 < m.rg2)))) return;
        const float r = sqrtf(r2);
        const int tj = __float_as_int(pj.w);
        const float ratio = RATIO ? m.ratio[ti][tj] : 1.0f;
        float t = 0.f;
        if (r2 < m.rp2) t += ppi * (m.cp_m2 * (1.0f - r * m.inv_rp)) * r;
        if (ST && r2 < m.ra2) {
            const float q = r * m.inv_ra;
            t += gi.w * ratio * (m.ca_inv * (1.0f - q) * (1.0f - 3.0f * q)) * r;
        }
        if (r2 < m.rv2) {
            const double4 vj = vel[j];
            const float ue = (((float)vj.x - vix) * dx + ((float)vj.y - viy) * dy + ((float)vj.z - viz) * dz) / r;
            t += 0.5f * tb.mu[ti * 4 + tj] * ue * (-(m.cv_m2 * (1.0f - r * m.inv_rv)));
        }
        if (ST && r2 < m.rg2) {
            const float q = 1.0f - r * m.inv_rg;
            const float gx = gi.x * dx + gi.y * dy + gi.z * dz;
            t += ai * gx * ratio * (m.cg * q * q + m.cg_m2 * q * r) * m.inv_r2g_rg * inv_l0;
        }
        kahan_add(tr, ck, t);
    };
    const uint4* tab = reinterpret_cast<const uint4*>(list) + i;
    const int ns = cnt_short[i], na = cnt_all[i];
    for_entries(tab, n, ns, visit);
    for_entries(tab + (size_t)(m.cap_s >> 2) * n, n, na - ns, visit);
    virial[i] = -((double)tr - (double)ck) / (double)m.dim;
}

// NeighborCount for output: the list counts plus self (the reference lists
// self), except walls without a fluid neighbour, whose list is empty there
// (main.cpp:1416).
__global__ void k_mix_counts(int n, const int* __restrict__ cnt_all, const int* __restrict__ cellstart, int tot,
                             int* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = cnt_all[i];
    out[i] = c > 0 ? c + 1 : (i < cellstart[tot] ? 1 : 0);
}

inline int blocks(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

struct MixedState {
    MixConst mc;
    int* keys_unsorted = nullptr;
    int* slot = nullptr;
    int* counts = nullptr;
    int* tmp = nullptr;
    int* home = nullptr;
    float4* phl = nullptr;  // [2n]: {hi position + type, lo position} per particle (home-cell relative)
    float4* p32 = nullptr;  // [n]: the hi parts alone, for the table build
    float4* v32 = nullptr;
    float4* pv = nullptr;  // [2n]: {hi position + type, (v, PressureP)} per particle, written by sweep A
    float4* gca = nullptr;
    unsigned* list = nullptr;
    int cap = 0;          // cap_s + cap_l rows
    int cap_l = 0;        // rows of the long part (mc.cap_s: the short part)
    int max_short = 0, max_long = 0;
    int* cnt_short = nullptr;
    int* cnt_all = nullptr;
    StepScalars* h_scal = nullptr;
    int max_neighbors = 0;
    bool exported = false;
    bool s64 = false;  // FP64 pressure core (MPH_MODE_MIXED_P64)
    bool walk = false; // force sweep by cell walk (MPH_MIXED_CELL_WALK)
};

static void mfree(MixedState* m) {
    void* ptrs[] = {m->keys_unsorted, m->slot, m->counts, m->tmp, m->home, m->phl, m->p32, m->v32, m->pv,
                    m->gca, m->list, m->cnt_short, m->cnt_all};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (m->h_scal) cudaFreeHost(m->h_scal);
}

#define MTRY(expr)                                                                     \
    do {                                                                               \
        cudaError_t e_ = (expr);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            if (err) *err = std::string(#expr ": ") + cudaGetErrorString(e_);          \
            return MPH_ERR_CUDA;                                                       \
        }                                                                              \
    } while (0)

template <class T>
static cudaError_t malloc_n(T** p, size_t n) {
    return cudaMalloc((void**)p, (n ? n : 1) * sizeof(T));
}

static int grow_list(MixedState* m, int need_s, int need_l, int n, std::string* err) {
    const int cs = ((int)(need_s * 1.15) + 8 + 7) / 8 * 8, cl = ((int)(need_l * 1.15) + 8 + 7) / 8 * 8;
    if (m->list) cudaFree(m->list);
    m->list = nullptr;
    m->cap = m->cap_l = m->mc.cap_s = 0;
    MTRY(malloc_n(&m->list, (size_t)(cs + cl) * (size_t)n));
    m->mc.cap_s = cs;
    m->cap_l = cl;
    m->cap = cs + cl;
    return MPH_OK;
}

// Counting sort by cell, reorder the FP64 state, home cells, list build.
int mixed_rebuild(MixedState* m, const SimConst& c, DevFP64& d, cudaStream_t s, std::string* err, int* launches) {
    const int n = c.n, nb = 2 * c.tot;
    const int a = d.cur, b = 1 - d.cur, va = d.vcur, vb = 1 - d.vcur;
    int nl = 0;
    MTRY(cudaMemsetAsync(m->counts, 0, sizeof(int) * (size_t)(nb + 1), s));
    k_mix_cellkey<<<blocks(n, 256), 256, 0, s>>>(c, d.pos[a], m->keys_unsorted, m->slot, m->counts);
    k_mix_scan<<<1, 1024, 0, s>>>(m->counts, nb, d.cellstart);
    k_mix_place<<<blocks(n, 256), 256, 0, s>>>(n, m->keys_unsorted, m->slot, d.cellstart, m->tmp);
    k_mix_rank<<<blocks(n, 256), 256, 0, s>>>(n, m->keys_unsorted, d.cellstart, m->tmp, d.vals, d.keys);
    launch_reorder(c, d.vals, d.pidx[a], d.type[a], d.pos[a], d.vel[va], d.pidx[b], d.type[b], d.pos[b], d.vel[vb],
                   d.snap, s);
    d.cur = b;
    d.vcur = vb;
    k_mix_home<<<blocks(n, 256), 256, 0, s>>>(c, m->mc, d.pos[d.cur], d.keys, d.vel[d.vcur], m->home, m->phl,
                                              m->p32, m->v32);
    nl += 6;
    for (int attempt = 0; attempt < 3; ++attempt) {
        MTRY(cudaMemsetAsync(&d.scal->max_neighbors, 0, sizeof(int), s));
        MTRY(cudaMemsetAsync(&d.scal->max_short, 0, 2 * sizeof(int), s));
        k_mix_list<<<blocks(2LL * c.tot, kMixListWarps), 32 * kMixListWarps, 0, s>>>(c, m->mc, m->p32, d.cellstart,
                                                                                   m->list, m->cap_l,
                                                  m->cnt_short, m->cnt_all, d.scal);
        ++nl;
        MTRY(cudaGetLastError());
        MTRY(cudaMemcpyAsync(m->h_scal, d.scal, sizeof(StepScalars), cudaMemcpyDeviceToHost, s));
        MTRY(cudaStreamSynchronize(s));
        m->max_neighbors = m->h_scal->max_neighbors;
        m->max_short = m->h_scal->max_short;
        m->max_long = m->h_scal->max_long;
        if (m->max_short <= m->mc.cap_s && m->max_long <= m->cap_l) break;
        const int st = grow_list(m, std::max(m->max_short, m->mc.cap_s), std::max(m->max_long, m->cap_l), n, err);
        if (st != MPH_OK) return st;
    }
    if (launches) *launches = nl;
    if (m->max_short > m->mc.cap_s || m->max_long > m->cap_l) {
        if (err) *err = "mixed neighbour table could not grow";
        return MPH_ERR_CAPACITY;
    }
    MTRY(cudaMemsetAsync(&d.scal->flags, 0, sizeof(int), s));
    m->exported = false;
    return MPH_OK;
}

void mixed_sweep_a(MixedState* m, const SimConst& c, DevFP64& d, bool advance_wall, cudaStream_t s) {
    const int nb = blocks(c.n, 128);
    double* wc = advance_wall ? d.wall_center : nullptr;
#define MIX_A(ST, RATIO, S64)                                                                                   \
    k_mix_a<ST, RATIO, S64><<<nb, 128, 0, s>>>(m->mc, m->phl, m->v32, m->list, m->cnt_short,          \
                                               m->cnt_all, m->pv, m->gca, d.strain_p, d.div_p, d.dens_a, wc, c, \
                                               d.vel[d.vcur], d.press)
#define MIX_A2(ST, RATIO) \
    if (m->s64) MIX_A(ST, RATIO, true); else MIX_A(ST, RATIO, false)
    if (m->mc.has_st) {
        if (m->mc.ratio_all_one) { MIX_A2(true, false); } else { MIX_A2(true, true); }
    } else {
        if (m->mc.ratio_all_one) { MIX_A2(false, false); } else { MIX_A2(false, true); }
    }
#undef MIX_A2
#undef MIX_A
    m->exported = false;
}

template <bool WALLS>
static void launch_b(MixedState* m, const SimConst& c, DevFP64& d, cudaStream_t s) {
    const int nb = blocks(c.n, 128);
    double4* vout = WALLS ? nullptr : d.vel[1 - d.vcur];
#define MIX_B1(ST, RATIO)                                                                                   \
    k_mix_b<ST, RATIO, WALLS><<<nb, 128, 0, s>>>(m->mc, c, d.cellstart, m->phl, m->pv, m->gca,   \
                                                 m->list, m->cnt_short, m->cnt_all, d.vel[d.vcur], vout,   \
                                                 d.force, d.scal)
    if (m->mc.has_st) {
        if (m->mc.ratio_all_one) { MIX_B1(true, false); } else { MIX_B1(true, true); }
    } else {
        if (m->mc.ratio_all_one) { MIX_B1(false, false); } else { MIX_B1(false, true); }
    }
#undef MIX_B1
}

static void launch_b_walk(MixedState* m, const SimConst& c, DevFP64& d, cudaStream_t s) {
    const int nb = (2 * c.tot + kWalkWarps - 1) / kWalkWarps;
#define MIX_W(ST, RATIO)                                                                                      \
    k_mix_b_walk<ST, RATIO><<<nb, 32 * kWalkWarps, 0, s>>>(m->mc, c, d.cellstart, m->phl, m->pv, m->gca,    \
                                                          d.vel[d.vcur], d.vel[1 - d.vcur], d.force, d.scal)
    if (m->mc.has_st) {
        if (m->mc.ratio_all_one) { MIX_W(true, false); } else { MIX_W(true, true); }
    } else {
        if (m->mc.ratio_all_one) { MIX_W(false, false); } else { MIX_W(false, true); }
    }
#undef MIX_W
}

int mixed_sweep_b(MixedState* m, const SimConst& c, DevFP64& d, cudaStream_t s) {
    if (m->walk) launch_b_walk(m, c, d, s);
    else launch_b<false>(m, c, d, s);
    m->exported = false;
    return 1;
}

void mixed_set_cell_walk(MixedState* m, bool on) { m->walk = on; }

void mixed_move(MixedState* m, const SimConst& c, DevFP64& d, cudaStream_t s) {
    k_mix_move<<<blocks(c.n, 256), 256, 0, s>>>(c, m->mc, d.cellstart, d.pos[d.cur], d.vel[d.vcur], d.snap,
                                                d.wall_center, m->home, m->phl, m->p32, m->v32, d.scal);
    m->exported = false;
}

int mixed_create(MixedState** out, const SimConst& c, const mph_constants& k, DevFP64& d, bool fp64_pressure,
                 cudaStream_t s, std::string* err) {
    *out = nullptr;
    if (c.cc[0] > 1024 || c.cc[1] > 1024 || c.cc[2] > 1024) {
        if (err) *err = "mixed form: at most 1024 cells per axis";
        return MPH_ERR_GEOMETRY;
    }
    if ((long long)c.n >= (1LL << (32 - kCodeBits))) {
        if (err) *err = "mixed form: too many particles for the packed list";
        return MPH_ERR_ARG;
    }
    MixedState* m = new MixedState();
    m->s64 = fp64_pressure;
    MixConst& mc = m->mc;
    std::memset(&mc, 0, sizeof(mc));
    mc.n = c.n;
    mc.tot = c.tot;
    mc.dim = c.dim;
    mc.has_st = c.has_st;
    mc.ratio_all_one = c.ratio_all_one;
    for (int dd = 0; dd < 3; ++dd) {
        mc.cc[dd] = c.cc[dd];
        mc.range[dd] = c.range[dd];
    }
    // hi-part grid: a power of two g with 2.2 cell widths below 2^24 g
    const double cwmax = std::max(c.cell_width[0], std::max(c.cell_width[1], c.cell_width[2]));
    mc.grid = std::ldexp(1.0, (int)std::ceil(std::log2(2.2 * cwmax)) - 24);
    mc.inv_grid = 1.0 / mc.grid;
    for (int code = 0; code < 27; ++code) {
        const int dc[3] = {code / 9 - 1, (code / 3) % 3 - 1, code % 3 - 1};
        for (int dd = 0; dd < 3; ++dd) {
            const double off = dc[dd] * c.cell_width[dd];
            const double q = std::rint(off * mc.inv_grid) * mc.grid;
            mc.dhi[code][dd] = (float)q;
            mc.dlo[code][dd] = (float)(off - q);
        }
        mc.dhi[code][3] = mc.dlo[code][3] = 0.0f;
    }
    mc.uniform_mu = 1;
    for (int t = 0; t < MPH_TYPE_COUNT; ++t)
        for (int u = 0; u < MPH_TYPE_COUNT; ++u)
            if (c.visc_mu[t][u] != c.visc_mu[0][0]) mc.uniform_mu = 0;
    const double margin = 0.1 * c.l0;
    const double rl = k.max_radius + margin, rs = k.radius_p + margin;
    mc.list_r2 = (float)(rl * rl);
    mc.short_r2 = (float)(rs * rs);
    {
        // the hi-only distance is within 3 * 1.5 grid steps of the exact one
        // (the lo parts of both particles and of the cell offset): 8 steps of slack
        double rf = std::max(c.rv, c.rp);
        if (c.has_st) rf = std::max(rf, std::max(c.ra, c.rg));
        const double sl = 8.0 * mc.grid;
        mc.walk_r2 = (float)((rf + sl) * (rf + sl));
        mc.walk_short2 = (float)((c.rp + sl) * (c.rp + sl));
    }
    mc.ra2 = (float)c.ra2;
    mc.rp2 = (float)c.rp2;
    mc.rv2 = (float)c.rv2;
    mc.rg2 = (float)c.rg2;
    mc.inv_ra = (float)(1.0 / c.ra);
    mc.inv_rp = (float)(1.0 / c.rp);
    mc.inv_rv = (float)(1.0 / c.rv);
    mc.inv_rg = (float)(1.0 / c.rg);
    mc.ca = (float)c.ca;
    mc.cp = (float)c.cp;
    mc.cg = (float)c.cg;
    mc.cv = (float)c.cv;
    mc.cp_m2 = (float)(c.cp * c.m2_rp);
    mc.cg_m2 = (float)(c.cg * c.m2_rg);
    mc.cv_m2 = (float)(c.cv * c.m2_rv);
    mc.ca_inv = (float)(c.ca * c.inv_ra);
    mc.p_a = (float)(c.cp * c.m2_rp * c.vol);
    mc.p_b = (float)(-c.cp * c.m2_rp * c.vol / c.rp);
    mc.v_a = (float)(-c.cv * c.m2_rv * c.vol);
    mc.v_b = (float)(c.cv * c.m2_rv * c.vol / c.rv);
    mc.p_a_d = c.cp * c.m2_rp * c.vol;
    mc.p_b_d = -c.cp * c.m2_rp * c.vol / c.rp;
    mc.v_a_d = -c.cv * c.m2_rv * c.vol;
    mc.v_b_d = c.cv * c.m2_rv * c.vol / c.rv;
    mc.cp_d = c.cp;
    mc.cp_m2_d = c.cp * c.m2_rp;
    mc.inv_rp_d = 1.0 / c.rp;
    mc.n0p_d = c.n0p;
    mc.inv_rp_lo = (float)(1.0 / c.rp - (double)mc.inv_rp);
    mc.cp_lo = (float)(c.cp - (double)mc.cp);
    mc.vol = (float)c.vol;
    mc.vol_over_l0 = (float)c.vol_over_l0;
    mc.n0a = (float)c.n0a;
    mc.n0p = (float)c.n0p;
    mc.inv_r2g_rg = (float)(c.rg / c.r2g);
    mc.l0 = (float)c.l0;
    for (int t = 0; t < MPH_TYPE_COUNT; ++t) {
        mc.a_k[t] = (float)c.a_k[t];
        mc.cof_a[t] = (float)c.cof_a[t];
        mc.bulk_modulus[t] = (float)c.bulk_modulus[t];
        mc.bulk_viscosity[t] = (float)c.bulk_viscosity[t];
        for (int u = 0; u < MPH_TYPE_COUNT; ++u) {
            mc.visc_mu[t][u] = (float)c.visc_mu[t][u];
            mc.ratio[t][u] = (float)c.ratio[t][u];
        }
    }
    const size_t n = (size_t)c.n;
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = malloc_n(&m->keys_unsorted, n);
    if (e == cudaSuccess) e = malloc_n(&m->slot, n);
    if (e == cudaSuccess) e = malloc_n(&m->counts, 2 * (size_t)c.tot + 1);
    if (e == cudaSuccess) e = malloc_n(&m->tmp, n);
    if (e == cudaSuccess) e = malloc_n(&m->home, n);
    if (e == cudaSuccess) e = malloc_n(&m->phl, 2 * n);
    if (e == cudaSuccess) e = malloc_n(&m->p32, n);
    if (e == cudaSuccess) e = malloc_n(&m->v32, n);
    if (e == cudaSuccess) e = malloc_n(&m->pv, 2 * n);
    if (e == cudaSuccess) e = malloc_n(&m->gca, n);
    if (e == cudaSuccess) e = malloc_n(&m->cnt_short, n);
    if (e == cudaSuccess) e = malloc_n(&m->cnt_all, n);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&m->h_scal, sizeof(StepScalars));
    if (e == cudaSuccess) e = cudaMemsetAsync(m->gca, 0, n * sizeof(float4), s);
    if (e != cudaSuccess) {
        if (err) *err = std::string("mixed form allocation: ") + cudaGetErrorString(e);
        mfree(m);
        delete m;
        return MPH_ERR_NOMEM;
    }
    // initial table: lattice points within the short and the long cut-off, with head room
    const double ratio = rl / c.l0, rs_l0 = rs / c.l0;
    const int r = (int)ratio + 1, zr = c.dim == 2 ? 0 : r;
    int lat_s = 0, lat_l = 0;
    for (int x = -r; x <= r; ++x)
        for (int y = -r; y <= r; ++y)
            for (int z = -zr; z <= zr; ++z) {
                const double q2 = x * x + y * y + z * z;
                if (q2 <= rs_l0 * rs_l0) ++lat_s;
                else if (q2 <= ratio * ratio) ++lat_l;
            }
    int st = grow_list(m, (int)(lat_s * 1.1) + 4, (int)(lat_l * 1.1) + 8, c.n, err);
    if (st == MPH_OK) st = mixed_rebuild(m, c, d, s, err, nullptr);
    if (st == MPH_OK) {
        mixed_sweep_a(m, c, d, false, s);
        e = cudaGetLastError();
        if (e != cudaSuccess) {
            if (err) *err = cudaGetErrorString(e);
            st = MPH_ERR_CUDA;
        }
    }
    if (st != MPH_OK) {
        mfree(m);
        delete m;
        return st;
    }
    *out = m;
    return MPH_OK;
}

int mixed_export(MixedState* m, const SimConst& c, DevFP64& d, cudaStream_t s, std::string* err, int* launches) {
    int nl = 0;
    if (!m->exported) {
        if (!m->mc.has_st) {
            k_mix_density_a<<<blocks(c.n, 128), 128, 0, s>>>(m->mc, m->p32, m->list, m->cnt_short, m->cnt_all,
                                                               d.dens_a);
            ++nl;
        }
        launch_b<true>(m, c, d, s);  // wall forces
        k_mix_counts<<<blocks(c.n, 256), 256, 0, s>>>(c.n, m->cnt_all, d.cellstart, c.tot, d.ncount);
        nl += 2;
        MTRY(cudaGetLastError());
        m->exported = true;
    }
    if (launches) *launches = nl;
    return MPH_OK;
}

int mixed_virial(MixedState* m, const SimConst& c, DevFP64& d, cudaStream_t s, std::string* err) {
    const int nb = blocks(c.n, 128);
#define MIX_V(ST, RATIO)                                                                                    \
    k_mix_virial<ST, RATIO><<<nb, 128, 0, s>>>(m->mc, m->phl, m->pv, m->gca, d.vel[d.vcur], m->list,        \
                                               m->cnt_short, m->cnt_all, d.virial_p)
    if (m->mc.has_st) {
        if (m->mc.ratio_all_one) { MIX_V(true, false); } else { MIX_V(true, true); }
    } else {
        if (m->mc.ratio_all_one) { MIX_V(false, false); } else { MIX_V(false, true); }
    }
#undef MIX_V
    MTRY(cudaGetLastError());
    return MPH_OK;
}

int mixed_import(MixedState* m, const SimConst& c, DevFP64& d, cudaStream_t s, std::string* err) {
    // positions/velocities changed from the host: refresh the FP32 copies
    k_mix_home<<<blocks(c.n, 256), 256, 0, s>>>(c, m->mc, d.pos[d.cur], d.keys, d.vel[d.vcur], m->home, m->phl,
                                                m->p32, m->v32);
    MTRY(cudaGetLastError());
    m->exported = false;
    return MPH_OK;
}

void mixed_mark_stale(MixedState* m) { m->exported = false; }
int mixed_max_neighbors(const MixedState* m) { return m ? m->max_neighbors : 0; }
int mixed_capacity(const MixedState* m) { return m ? m->cap : 0; }

void mixed_destroy(MixedState* m) {
    if (!m) return;
    mfree(m);
    delete m;
}

}  // namespace mph
