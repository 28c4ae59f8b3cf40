// k_cells.cu — cell assignment, bitonic cell sort, per-cell ranges, reorder and
// the Verlet neighbour list of the FP64 form (sm_100a).
//
// This is integer/index work plus the FP64 distance test of the list build.
// The results are bit-exact against the reference:
//   * cell index:      main.cpp:1115-1133 (same floor/modulo expressions);
//   * sort:            the reference's bitonic compare-exchange network
//                      (main.cpp:1137-1158), pass for pass, so ties inside a
//                      cell end in the same order and the permutation matches;
//   * per-cell ranges: main.cpp:1160-1247 (begin/end equal the number of sorted
//                      keys below each key value, found here by binary search);
//   * neighbour list:  main.cpp:1329-1596, same stencil order, self included,
//                      wall particles without a fluid neighbour get no list.
// Compiled with -fmad=false so the distance test is not FMA-contracted.
#include <cmath>
#include "mph_internal.h"

namespace mph {

namespace {

constexpr int kLogLocal = 12;               // 4096 keys per shared-memory block
constexpr int kLocal = 1 << kLogLocal;
constexpr int kSortThreads = 1024;

__device__ __forceinline__ double omod(double x, double w) { return x - w * floor(x / w); }

// Mod(x,w) of main.cpp:70.  When 0 <= x < 0.75 w the quotient rounds below 1,
// floor gives +0 and the expression returns x exactly; skip the division then.
__device__ __forceinline__ double omod_fast(double x, double w) {
    return (x >= 0.0 && x < 0.75 * w) ? x : omod(x, w);
}

__device__ __forceinline__ int cell_id(const SimConst& c, int ix, int iy, int iz) {  // main.cpp:96-100
    return ((ix % c.cc[0] + c.cc[0]) % c.cc[0]) * c.cc[1] * c.cc[2] +
           ((iy % c.cc[1] + c.cc[1]) % c.cc[1]) * c.cc[2] + ((iz % c.cc[2] + c.cc[2]) % c.cc[2]);
}

__global__ void k_cell_index(SimConst c, const double4* __restrict__ pos, const int* __restrict__ type,
                             int* __restrict__ keys, int* __restrict__ vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.pow2) return;
    if (i < c.n) {
        const double4 p = pos[i];
        const int cx = ((int)floor((p.x - c.dmin[0]) / c.cell_width[0])) % c.cc[0];
        const int cy = ((int)floor((p.y - c.dmin[1]) / c.cell_width[1])) % c.cc[1];
        const int cz = ((int)floor((p.z - c.dmin[2]) / c.cell_width[2])) % c.cc[2];
        int id = cell_id(c, cx, cy, cz);
        const int t = type[i];
        if (t >= 2 && t < 4) id += c.tot;
        keys[i] = id;
        vals[i] = i;
    } else {
        keys[i] = 2 * c.tot;
        vals[i] = c.n;
    }
}

// One compare-exchange of pass (m, dist): element i (bit log2(dist) clear) and
// i|dist; ascending when bit m+1 of i is clear (main.cpp:1146-1148).
__device__ __forceinline__ void cmpx(int* k, int* v, int a, int b, bool up) {
    const int ka = k[a], kb = k[b];
    if ((ka > kb) == up) {
        const int va = v[a], vb = v[b];
        k[a] = kb; k[b] = ka;
        v[a] = vb; v[b] = va;
    }
}

// All passes whose distance is below the block size, for main-stage m in
// [m_begin, m_end); for each m the sub-stages with dist < block run here.
// Block b owns keys [b*L, (b+1)*L).
__global__ void __launch_bounds__(kSortThreads)
k_bitonic_local(int* __restrict__ keys, int* __restrict__ vals, int L, int logL, int m_begin, int m_end) {
    __shared__ int sk[kLocal];
    __shared__ int sv[kLocal];
    const int base = blockIdx.x * L;
    for (int t = threadIdx.x; t < L; t += blockDim.x) {
        sk[t] = keys[base + t];
        sv[t] = vals[base + t];
    }
    __syncthreads();
    const int half = L >> 1;
    for (int m = m_begin; m < m_end; ++m) {
        // sub-stages with dist = 2^(m-k) < L, i.e. log2(dist) <= min(m, logL-1)
        const int top = m < logL - 1 ? m : logL - 1;
        for (int ld = top; ld >= 0; --ld) {
            const int dist = 1 << ld;
            for (int t = threadIdx.x; t < half; t += blockDim.x) {
                const int i = ((t >> ld) << (ld + 1)) | (t & (dist - 1));
                const bool up = (((base + i) >> m) & 2) == 0;
                cmpx(sk, sv, i, i | dist, up);
            }
            __syncthreads();
        }
    }
    for (int t = threadIdx.x; t < L; t += blockDim.x) {
        keys[base + t] = sk[t];
        vals[base + t] = sv[t];
    }
}

// One pass with dist >= block size, one pair per thread.
__global__ void k_bitonic_global(int* __restrict__ keys, int* __restrict__ vals, int npairs, int m, int ld) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npairs) return;
    const int dist = 1 << ld;
    const int i = ((t >> ld) << (ld + 1)) | (t & (dist - 1));
    const bool up = ((i >> m) & 2) == 0;
    cmpx(keys, vals, i, i | dist, up);
}

// cellstart[b] = number of sorted keys below b, b in [0, 2*tot].  These are
// the reference's CellFluidParticleBegin/End (b < tot) and
// CellWallParticleBegin/End (b >= tot) after its prefix sum (main.cpp:1191-1247).
__global__ void k_cell_ranges(const int* __restrict__ keys, int n, int nb, int* __restrict__ cellstart) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (keys[mid] < b) lo = mid + 1; else hi = mid;
    }
    cellstart[b] = lo;
}

// Gather by the sorted CellParticle (main.cpp:1262-1325); the snapshot of the
// positions for the rebuild test is taken here (main.cpp:1587-1595: the
// positions do not change between the reorder and the end of the build).
__global__ void k_reorder(int n, const int* __restrict__ vals, const int* __restrict__ pidx_in,
                          const int* __restrict__ type_in, const double4* __restrict__ pos_in,
                          const double4* __restrict__ vel_in, int* __restrict__ pidx_out,
                          int* __restrict__ type_out, double4* __restrict__ pos_out,
                          double4* __restrict__ vel_out, double4* __restrict__ snap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = vals[i];
    pidx_out[i] = pidx_in[s];
    type_out[i] = type_in[s];
    const double4 p = pos_in[s];
    pos_out[i] = p;
    snap[i] = p;
    vel_out[i] = vel_in[s];
}

// Neighbour list (main.cpp:1329-1585), one warp per home key: the particles
// of one cell (fluid keys, then the wall keys of the same cells) share their
// 3^D stencil and its visiting order, so the warp walks it in step, 32 home
// particles at a time (one per lane).  Each candidate range is read 32
// candidates at a time (one coalesced FP32 record per lane into shared
// memory); every lane then tests all of them against its own particle with
// the FP32 prefilter, giving a bit mask, and runs the exact FP64 test of the
// reference only over the set bits, in ascending order.  A lane's entries
// are therefore the reference's, in the reference's order: fluid candidates
// of the 27 cells, then wall candidates (a wall with no fluid neighbour
// skips the walls, main.cpp:1416), self included, each range ascending.
//
// The count and the fill of the reference are one pass: entries go to a
// column-major [cap][n] table; a list longer than cap is still counted,
// raises DEVFLAG_NEIGHBOR_OVERFLOW and the host rebuilds with a larger table.
// With nlist_s, the entries within rs2 also go, in the same order, to the
// short sublist: a particle moves at most MARGIN/2 between builds (the
// rebuild test of main.cpp:1086-1108), so every pair within RadiusP until the
// next build is in it, and a sum over the pairs within RadiusP visits them in
// list order.
//
// Prefilter: FP32 positions relative to the domain origin (k_pos32) give a
// displacement within the bound of make_prefilter of the one the exact FP64
// test computes, so a candidate whose FP32 distance squared exceeds pf.r2_hi
// cannot pass that test and is skipped.  An axis with fewer than 4 cells
// contributes nothing to the FP32 distance (its minimum image need not be the
// neighbouring cell's), which only keeps more candidates.
constexpr int kListWarps = 4;  // warps (home keys) per 128-thread block

#ifndef MPH_LIST_MINB
#define MPH_LIST_MINB 6
#endif
template <bool ALL3>  // every axis in the FP32 prefilter (pf.use all set)
__global__ void __launch_bounds__(32 * kListWarps, MPH_LIST_MINB)
k_neighbor_list(SimConst c, const double4* __restrict__ pos, const float4* __restrict__ pos32, Prefilter pf,
                const int* __restrict__ cellstart, int* __restrict__ ncount, int* __restrict__ nlist, int cap,
                int* __restrict__ ncount_s, int* __restrict__ nlist_s, int cap_s, StepScalars* __restrict__ scal) {
    __shared__ float4 cand[kListWarps][32];
    __shared__ int4 sten[kListWarps][27];  // the stencil in visiting order: cell, FP32 image offsets
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int key = blockIdx.x * kListWarps + wib;  // home key in [0, 2*tot)
    if (key >= 2 * c.tot) return;                   // whole warp
    const int hb = cellstart[key], he = cellstart[key + 1];
    if (hb == he) return;
    // the stencil of the home cell as main.cpp:1356-1392 computes it from the
    // key (a wall's key carries +TotalCellCount: its icx is cx + cc[0])
    const int icx = (key / (c.cc[1] * c.cc[2])) % c.tot;
    const int ic[3] = {icx, (key / c.cc[2]) % c.cc[1], key % c.cc[2]};
    int jmin[3], w[3], home[3];
    for (int d = 0; d < 3; ++d) {
        const int r = c.range[d];
        w[d] = 2 * r + 1;
        home[d] = ic[d] % c.cc[d];
        const int b = (2 * r) - (ic[d] + r) % c.cc[d];  // main.cpp:1376-1381
        jmin[d] = b > 0 ? b : 0;
    }
    // stencil slot s of axis d: the cell coordinate (main.cpp:1360-1372) and
    // the FP32 image offset (0, or -+ the domain width where the slot wraps)
    auto slot = [&](int d, int s_, float& off) {
        const int raw = home[d] - c.range[d] + s_;
        off = raw < 0 ? -pf.width[d] : (raw >= c.cc[d] ? pf.width[d] : 0.0f);
        return ((ic[d] - c.range[d] + s_) % c.cc[d] + c.cc[d]) % c.cc[d];
    };
    // lane s < w0*w1*w2 computes stencil slot s of the loop order of
    // main.cpp:1356-1392 (x outer, z inner), once for all the key's chunks
    const int nsl = w[0] * w[1] * w[2];  // at most 27: range <= 1 on every axis
    if (lane < nsl) {
        const int a0 = lane / (w[1] * w[2]), a1 = (lane / w[2]) % w[1], a2 = lane % w[2];
        float gx, gy, gz;
        const int cx = slot(0, (jmin[0] + a0) % w[0], gx), cy = slot(1, (jmin[1] + a1) % w[1], gy),
                  cz = slot(2, (jmin[2] + a2) % w[2], gz);
        sten[wib][lane] = make_int4(cell_id(c, cx, cy, cz), __float_as_int(gx), __float_as_int(gy),
                                    __float_as_int(gz));
    }
    __syncwarp();
    const int wall_begin = cellstart[c.tot], wall_end = cellstart[2 * c.tot];
    const size_t n = (size_t)c.n;
    const bool short_list = nlist_s != nullptr;
    float4* cw = cand[wib];
    const float kInf = __int_as_float(0x7f800000);
    for (int h0 = hb; h0 < he; h0 += 32) {
        const int i = h0 + lane;
        const bool active = i < he;
        const double4 pi = pos[active ? i : hb];
        const float4 fi = pos32[active ? i : hb];
        const bool is_wall = wall_begin <= i && i < wall_end;
        int cnt = 0, cnt_s = 0;
        // box of the chunk's FP32 positions: a candidate farther than the
        // cut-off from it is no lane's neighbour (Prefilter::r2_box)
        float b0x = active ? fi.x : kInf, b0y = active ? fi.y : kInf, b0z = active ? fi.z : kInf;
        float b1x = active ? fi.x : -kInf, b1y = active ? fi.y : -kInf, b1z = active ? fi.z : -kInf;
        for (int o = 16; o > 0; o >>= 1) {
            b0x = fminf(b0x, __shfl_xor_sync(0xffffffffu, b0x, o));
            b0y = fminf(b0y, __shfl_xor_sync(0xffffffffu, b0y, o));
            b0z = fminf(b0z, __shfl_xor_sync(0xffffffffu, b0z, o));
            b1x = fmaxf(b1x, __shfl_xor_sync(0xffffffffu, b1x, o));
            b1y = fmaxf(b1y, __shfl_xor_sync(0xffffffffu, b1y, o));
            b1z = fmaxf(b1z, __shfl_xor_sync(0xffffffffu, b1z, o));
        }
        for (int kind = 0; kind < 2; ++kind) {
            // main.cpp:1416: a wall with no fluid neighbour gets no wall entries
            const bool take = active && !(kind == 1 && is_wall && cnt == 0);
            const int off = kind ? c.tot : 0;
            for (int sl = 0; sl < nsl; ++sl) {
                const int4 st = sten[wib][sl];
                const int cell = st.x;
                const float gx = __int_as_float(st.y), gy = __int_as_float(st.z), gz = __int_as_float(st.w);
                const float ox = (ALL3 || pf.use[0]) ? gx - fi.x : 0.f;
                const float oy = (ALL3 || pf.use[1]) ? gy - fi.y : 0.f;
                const float oz = (ALL3 || pf.use[2]) ? gz - fi.z : 0.f;
                const int b = cellstart[cell + off], e = cellstart[cell + off + 1];
                for (int cb = b; cb < e; cb += 32) {
                    // the candidates near the box, compacted in order into the stage
                    bool near = false;
                    float4 q;
                    if (cb + lane < e) {
                        q = pos32[cb + lane];
                        const float ax = q.x + gx, ay = q.y + gy, az = q.z + gz;
                        const float ex = (ALL3 || pf.use[0]) ? fmaxf(0.f, fmaxf(b0x - ax, ax - b1x)) : 0.f;
                        const float ey = (ALL3 || pf.use[1]) ? fmaxf(0.f, fmaxf(b0y - ay, ay - b1y)) : 0.f;
                        const float ez = (ALL3 || pf.use[2]) ? fmaxf(0.f, fmaxf(b0z - az, az - b1z)) : 0.f;
                        near = __fmaf_rn(ex, ex, __fmaf_rn(ey, ey, __fmul_rn(ez, ez))) <= pf.r2_box;
                    }
                    const unsigned kept = __ballot_sync(0xffffffffu, near);
                    __syncwarp();
                    if (near) {
                        q.w = __int_as_float(lane);
                        cw[__popc(kept & ((1u << lane) - 1u))] = q;
                    }
                    __syncwarp();
                    const int m = __popc(kept);
                    // per candidate of the stage: may be within rm (mask), needs the
                    // FP64 test (exact: in a shell of the rm or the rs bound), within
                    // rs for certain (in_s)
                    unsigned mask = 0u, exact = 0u, in_s = 0u;
                    if (take) {
                        for (int t = 0; t < m; ++t) {
                            const float4 q = cw[t];
                            const float fx = (ALL3 || pf.use[0]) ? q.x + ox : 0.f;
                            const float fy = (ALL3 || pf.use[1]) ? q.y + oy : 0.f;
                            const float fz = (ALL3 || pf.use[2]) ? q.z + oz : 0.f;
                            // FMA: fewer roundings than the bound allows for
                            const float r2f = __fmaf_rn(fx, fx, __fmaf_rn(fy, fy, __fmul_rn(fz, fz)));
                            if (r2f <= pf.r2_hi) {
                                const unsigned bit = 1u << t;
                                mask |= bit;
                                if (r2f > pf.r2_lo || (short_list && r2f > pf.rs2_lo && r2f <= pf.rs2_hi))
                                    exact |= bit;
                                else if (r2f <= pf.rs2_lo)
                                    in_s |= bit;
                            }
                        }
                    }
                    while (mask) {
                        const int t = __ffs(mask) - 1;
                        const unsigned bit = mask & (0u - mask);
                        mask &= mask - 1u;
                        const int j = cb + __float_as_int(cw[t].w);
                        bool in = true, in_short = (in_s & bit) != 0u;
                        if (exact & bit) {
                            const double4 pj = pos[j];
                            const double q0 = omod_fast(pj.x - pi.x + c.half_width[0], c.width[0]) - c.half_width[0];
                            const double q1 = omod_fast(pj.y - pi.y + c.half_width[1], c.width[1]) - c.half_width[1];
                            const double q2 = omod_fast(pj.z - pi.z + c.half_width[2], c.width[2]) - c.half_width[2];
                            const double r2 = q0 * q0 + q1 * q1 + q2 * q2;
                            in = r2 <= c.rm2;
                            in_short = r2 <= c.rs2;
                        }
                        if (in) {
                            if (cnt < cap) nlist[(size_t)cnt * n + i] = j;
                            cnt++;
                            if (short_list && in_short) {
                                if (cnt_s < cap_s) nlist_s[(size_t)cnt_s * n + i] = j;
                                cnt_s++;
                            }
                        }
                    }
                }
            }
        }
        if (active) {
            ncount[i] = cnt;
            atomicMax(&scal->max_neighbors, cnt);
            if (cnt > cap) atomicOr(&scal->flags, DEVFLAG_NEIGHBOR_OVERFLOW);
            if (short_list) {
                ncount_s[i] = cnt_s;
                atomicMax(&scal->max_short, cnt_s);
                if (cnt_s > cap_s) atomicOr(&scal->flags, DEVFLAG_NEIGHBOR_OVERFLOW);
            }
        }
    }
}

// FP32 copies of the positions relative to the domain origin, for the list
// build's prefilter: Mod(x - dmin, W) in [0, W), the coordinate of the
// particle's image in the cell its CellId names (main.cpp:96-100).
__global__ void k_pos32(SimConst c, const double4* __restrict__ pos, float4* __restrict__ pos32) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const double4 p = pos[i];
    pos32[i] = make_float4((float)omod(p.x - c.dmin[0], c.width[0]), (float)omod(p.y - c.dmin[1], c.width[1]),
                           (float)omod(p.z - c.dmin[2], c.width[2]), 0.f);
}

__global__ void k_pack3(int n, const double4* __restrict__ src, double* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 p = src[i];
    dst[3 * (size_t)i + 0] = p.x;
    dst[3 * (size_t)i + 1] = p.y;
    dst[3 * (size_t)i + 2] = p.z;
}

__global__ void k_unpack3(int n, const double* __restrict__ src, double4* __restrict__ dst,
                          const int* __restrict__ type) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double w = type ? (double)type[i] : 0.0;
    dst[i] = make_double4(src[3 * (size_t)i], src[3 * (size_t)i + 1], src[3 * (size_t)i + 2], w);
}

inline int blocks(long long n, int t) { return (int)((n + t - 1) / t); }

// Table check of a step graph's rebuild (one thread): a list longer than its
// table stops the batch and skips this step's sweeps.
__global__ void k_graph_list_check(StepScalars* scal, int cap, int cap_s, int short_list,
                                   cudaGraphConditionalHandle sweep) {
    if (scal->max_neighbors > cap || (short_list && scal->max_short > cap_s)) {
        scal->stop = 1;
        cudaGraphSetConditional(sweep, 0u);
    }
}

}  // namespace

void launch_graph_list_check(StepScalars* scal, int cap, int cap_s, int short_list,
                             cudaGraphConditionalHandle sweep, cudaStream_t s) {
    k_graph_list_check<<<1, 1, 0, s>>>(scal, cap, cap_s, short_list, sweep);
}

void launch_cell_index(const SimConst& c, const double4* pos, const int* type, int* keys, int* vals,
                       cudaStream_t s) {
    k_cell_index<<<blocks(c.pow2, 256), 256, 0, s>>>(c, pos, type, keys, vals);
}

// The reference's network (main.cpp:1137-1158): for m in [0, log2 P), k in [0, m],
// dist = 2^(m-k).  Passes with dist below the shared-memory block run inside
// k_bitonic_local; the others one launch each.  Same passes, same order.
int launch_bitonic_sort(const SimConst& c, int* keys, int* vals, cudaStream_t s) {
    const int P = c.pow2;
    int logP = 0;
    while ((1 << logP) < P) ++logP;
    if (logP == 0) return 0;
    const int logL = logP < kLogLocal ? logP : kLogLocal;
    const int L = 1 << logL;
    const int nblk = P / L;
    const int thr = (L / 2) < kSortThreads ? (L / 2) : kSortThreads;
    int launches = 0;
    // every main stage m < logL is entirely local
    k_bitonic_local<<<nblk, thr, 0, s>>>(keys, vals, L, logL, 0, logL);
    ++launches;
    for (int m = logL; m < logP; ++m) {
        for (int ld = m; ld >= logL; --ld) {
            k_bitonic_global<<<blocks(P / 2, 256), 256, 0, s>>>(keys, vals, P / 2, m, ld);
            ++launches;
        }
        k_bitonic_local<<<nblk, thr, 0, s>>>(keys, vals, L, logL, m, m + 1);
        ++launches;
    }
    return launches;
}

void launch_cell_ranges(const SimConst& c, const int* keys, int* cellstart, cudaStream_t s) {
    const int nb = 2 * c.tot + 1;
    k_cell_ranges<<<blocks(nb, 256), 256, 0, s>>>(keys, c.n, nb, cellstart);
}

void launch_reorder(const SimConst& c, const int* vals, const int* pidx_in, const int* type_in,
                    const double4* pos_in, const double4* vel_in, int* pidx_out, int* type_out,
                    double4* pos_out, double4* vel_out, double4* snap, cudaStream_t s) {
    k_reorder<<<blocks(c.n, 256), 256, 0, s>>>(c.n, vals, pidx_in, type_in, pos_in, vel_in, pidx_out,
                                               type_out, pos_out, vel_out, snap);
}

// Bound of the prefilter (see k_neighbor_list).  An FP32 coordinate in
// [0, W) is within 2^-24 W of its FP64 value (two coordinates: 2 * 2^-24 W);
// a component is formed as q + (offset - p_i) with |offset - p_i| < 2W
// (2 * 2^-24 W more) and a small result (less than 2^-24 W more), so each
// component is within e = 5 * 2^-24 * W of the FP64 minimum-image
// displacement (W rounded to FP32 for the offset adds 2^-24 W), which is
// itself within 2^-50 W of the true one.  The FP32 distance is then within
// sqrt(3) e < 2e of the FP64 one, and the FP32 sum of squares (three
// roundings: a product and two FMAs) within a factor 1 + 2^-21 of its exact
// value: a candidate the FP64 test accepts (r <= rm)
// has an FP32 distance squared below (rm + 2e)^2 (1 + 2^-20), rounded up to
// the next float.  e is taken as 8 * 2^-24 * W for room.
// The box test of a candidate (its image q + offset against the box of the
// FP32 positions of the warp's particles) bounds each axis' gap by the
// component for every particle in the box, within the same e (the image sum
// q + offset rounds once, within 2^-24 2W): a candidate within rm of any of
// them has a box distance squared below (rm + 2e)^2 (1 + 2^-20); r2_box takes
// 4e for room.
Prefilter make_prefilter(const SimConst& c) {
    Prefilter pf{};
    double wmax = 0.0;
    for (int d = 0; d < 3; ++d) {
        pf.use[d] = c.cc[d] >= 4 && c.range[d] == 1;
        pf.width[d] = (float)c.width[d];
        if (pf.use[d]) wmax = std::fmax(wmax, c.width[d]);
    }
    const double e = 8.0 * std::ldexp(wmax, -24);
    const double rm = std::sqrt(c.rm2);
    const double t = (rm + 2.0 * e) * (rm + 2.0 * e) * (1.0 + std::ldexp(1.0, -20));
    pf.r2_hi = std::nextafter((float)t, 3.0e38f);
    const double tb = (rm + 4.0 * e) * (rm + 4.0 * e) * (1.0 + std::ldexp(1.0, -20));
    pf.r2_box = std::nextafter((float)tb, 3.0e38f);
    // The other side of the same bounds: an FP32 distance squared at or below
    // (R - 2e)^2 (1 - 2^-20), rounded down to the previous float, puts the FP64
    // distance below R - 2e + 2e = R, so the FP64 test r2 <= R^2 holds for
    // certain and is skipped; only the candidates in the shell between the two
    // bounds take it.  Valid when every axis is compared in FP32 (an axis left
    // out of the prefilter contributes 0 in FP32 but not in FP64), or the axis
    // left out is the flat one of a 2-D run.
    bool all_axes = true;
    for (int d = 0; d < 3; ++d)
        if (!pf.use[d] && !(c.dim == 2 && d == 2)) all_axes = false;
    auto lo_bound = [&](double r) {
        if (!all_axes || r <= 2.0 * e) return -1.0f;
        const double t2 = (r - 2.0 * e) * (r - 2.0 * e) * (1.0 - std::ldexp(1.0, -20));
        return std::nextafter((float)t2, -1.0f);
    };
    const double rs = std::sqrt(c.rs2);
    pf.r2_lo = lo_bound(rm);
    pf.rs2_lo = lo_bound(rs);
    pf.rs2_hi = all_axes ? std::nextafter((float)((rs + 2.0 * e) * (rs + 2.0 * e) * (1.0 + std::ldexp(1.0, -20))),
                                          3.0e38f)
                         : 3.0e38f;
    return pf;
}

void launch_pos32(const SimConst& c, const double4* pos, float4* pos32, cudaStream_t s) {
    k_pos32<<<blocks(c.n, 256), 256, 0, s>>>(c, pos, pos32);
}

void launch_neighbor_list(const SimConst& c, const double4* pos, const float4* pos32, const int* cellstart,
                          int* ncount, int* nlist, int cap, int* ncount_s, int* nlist_s, int cap_s,
                          StepScalars* scal, cudaStream_t s) {
    const long long keys = 2LL * c.tot;
    const Prefilter pf = make_prefilter(c);
    const int nb = (int)((keys + kListWarps - 1) / kListWarps);
    if (pf.use[0] && pf.use[1] && pf.use[2])
        k_neighbor_list<true><<<nb, 32 * kListWarps, 0, s>>>(c, pos, pos32, pf, cellstart, ncount, nlist, cap,
                                                              ncount_s, nlist_s, cap_s, scal);
    else
        k_neighbor_list<false><<<nb, 32 * kListWarps, 0, s>>>(c, pos, pos32, pf, cellstart, ncount, nlist, cap,
                                                               ncount_s, nlist_s, cap_s, scal);
}

void launch_pack3(int n, const double4* src, double* dst, cudaStream_t s) {
    k_pack3<<<blocks(n, 256), 256, 0, s>>>(n, src, dst);
}

void launch_unpack3(int n, const double* src, double4* dst, const int* type, cudaStream_t s) {
    k_unpack3<<<blocks(n, 256), 256, 0, s>>>(n, src, dst, type);
}

}  // namespace mph
