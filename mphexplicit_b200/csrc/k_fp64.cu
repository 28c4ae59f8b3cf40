// k_fp64.cu — the plain FP64 MPH-WC step on sm_100a, bit-exact against the
// reference's x86-64 build.
//
// The reference runs eight neighbour sweeps per step (main.cpp:1665-1985).
// Here they are two, one thread per particle, list order kept:
//   sweep A = DensityA + GravityCenter + DensityP + DivergenceP
//             (four independent sums over the same list) and, in the epilogue,
//             PhysicalCoefficients + PressureP value + PressureA value;
//   sweep B = PressureP + PressureA + DiffuseInterface + ViscosityV forces,
//             each in its own accumulator, added to Force in the reference's
//             order, then Gravity + Acceleration (velocity double-buffered).
// plus one per-particle kernel for Convection + Wall + PeriodicBoundary +
// the rebuild test.  Every FP expression keeps the reference's association
// order; the file is compiled with -fmad=false and uses IEEE division and
// square root, so each operation rounds exactly as on the CPU.
#include "mph_internal.h"
#include "mph_exact.cuh"

// Resident 128-thread blocks per SM the sweeps are compiled for (register cap
// 65536 / (128 * blocks)); latency hiding vs. spills, set by measurement on
// the full dam break.  Both sweeps keep the next neighbour's records in
// flight: sweep A at 7 (72 registers; at 8 it spills), the force sweep at 6
// (80 registers, a few spills outside the neighbour loops: 3.08 ms against
// 3.13 ms at 5 blocks and 3.16 ms at 4, with the pressure loop split off).
#ifndef MPH_SWEEP_MINB
#define MPH_SWEEP_MINB 7
#endif
#ifndef MPH_SWEEPB_MINB
#define MPH_SWEEPB_MINB 6
#endif
// The surface-tension variants hold more live values per pair; at the
// bounds above they spilled (140 B in the force sweep) and ran the 8.5 M
// particle two-fluid column's step at 40.6 + 13.9 ms.  Measured on that
// column: the force sweep 26.7 ms at 4 blocks (no spills) and 29.6 ms at 3,
// sweep A 12.5 ms at 5 (13.3 at 6); results bit-identical.  With the pressure
// loops over the short sublist (SPLIT): 26.0 and 10.2 ms.
#ifndef MPH_SWEEP_MINB_ST
#define MPH_SWEEP_MINB_ST 5
#endif
#ifndef MPH_SWEEPB_MINB_ST
#define MPH_SWEEPB_MINB_ST 4
#endif

namespace mph {

namespace {

__device__ __forceinline__ double omod(double x, double w) { return x - w * floor(x / w); }

// Mod(x,w), main.cpp:70.  When 0 <= x < 0.75 w the rounded quotient is below 1,
// floor gives +0 and x - w*0 == x exactly: the division is skipped then.
__device__ __forceinline__ double omod_fast(double x, double w) {
    return (x >= 0.0 && x < 0.75 * w) ? x : omod(x, w);
}

// The same Mod with the range test as one unsigned compare of x's bits
// against those of 0.75 w (SimConst::q75_bits): equal to omod_fast for every x
// except -0.0, which takes omod and gives +0.0 instead of -0.0; the callers
// then subtract half_width (non-zero), so their results are the same.
__device__ __forceinline__ double omod_q(double x, double w, unsigned long long q75) {
    return ((unsigned long long)__double_as_longlong(x) < q75) ? x : omod(x, w);
}

// Minimum-image displacement x_j - x_i (main.cpp:1680 and every sweep).
__device__ __forceinline__ void disp(const SimConst& c, const double4& pi, const double4& pj, double* x) {
    x[0] = omod_q(pj.x - pi.x + c.half_width[0], c.width[0], c.q75_bits[0]) - c.half_width[0];
    x[1] = omod_q(pj.y - pi.y + c.half_width[1], c.width[1], c.q75_bits[1]) - c.half_width[1];
    x[2] = omod_q(pj.z - pi.z + c.half_width[2], c.width[2], c.q75_bits[2]) - c.half_width[2];
}

// Kernel shapes, main.cpp:214-284, with q = r/h computed by division.
__device__ __forceinline__ double f_dwadr(const SimConst& c, double r) {
    const double q = r / c.ra;
    return ((c.ca * (1.0 - q)) * (1.0 - 3.0 * q)) * c.inv_ra;
}
__device__ __forceinline__ double f_wg(const SimConst& c, double r) {
    const double q = r / c.rg;
    return c.cg * ((1.0 - q) * (1.0 - q));
}
__device__ __forceinline__ double f_dwgdr(const SimConst& c, double r) {
    const double q = r / c.rg;
    return c.cg * (c.m2_rg * (1.0 - q));
}
__device__ __forceinline__ double f_dwpdr(const SimConst& c, double r) {
    const double q = r / c.rp;
    return c.cp * (c.m2_rp * (1.0 - q));
}
__device__ __forceinline__ double f_dwvdr(const SimConst& c, double r) {
    const double q = r / c.rv;
    return c.cv * (c.m2_rv * (1.0 - q));
}

__device__ __forceinline__ int type_of(const double4& p) { return (int)p.w; }

// Convection (main.cpp:1605-1615), Wall (2013-2043), PeriodicBoundary
// (2306-2317) and the displacement maximum of neighborCalculation (1086-1100).
// GRAPH (a step graph's move): nothing to do once the batch stopped; the last
// block to finish makes the rebuild test on the maximum (main.cpp:1102) and
// sets the graph's conditionals, counts the step and clears the maximum for
// the next step's move.
template <bool GRAPH>
__global__ void __launch_bounds__(256)
k_move(SimConst c, const int* __restrict__ cellstart, double4* __restrict__ pos, double4* __restrict__ vel,
       const double4* __restrict__ snap, const double* __restrict__ wall_center, StepScalars* __restrict__ scal,
       cudaGraphConditionalHandle h_rebuild, cudaGraphConditionalHandle h_sweep) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool stopped = GRAPH && *reinterpret_cast<volatile int*>(&scal->stop) != 0;
    double s2 = 0.0;
    if (i < c.n && !stopped) {
        const int nf = cellstart[c.tot], we = cellstart[2 * c.tot];
        double4 p = pos[i];
        if (i < nf) {
            const double4 v = vel[i];
            p.x += v.x * c.dt;
            p.y += v.y * c.dt;
            p.z += v.z * c.dt;
        } else if (i < we) {
            const int t = type_of(p);
            const double* C = wall_center + 3 * t;
            const double (*R)[3] = c.wall_rot[t];
            const double* W = c.wall_omega[t];
            const double* U = c.wall_velocity[t];
            double r0 = p.x - C[0], r1 = p.y - C[1], r2 = p.z - C[2];
            r0 = R[0][0] * r0 + R[0][1] * r1 + R[0][2] * r2;   // in place, as main.cpp:2033-2035
            r1 = R[1][0] * r0 + R[1][1] * r1 + R[1][2] * r2;
            r2 = R[2][0] * r0 + R[2][1] * r1 + R[2][2] * r2;
            double4 v = vel[i];
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
        const double4 q = snap[i];
        double d[3];
        d[0] = omod_fast(p.x - q.x + c.half_width[0], c.width[0]) - c.half_width[0];
        d[1] = omod_fast(p.y - q.y + c.half_width[1], c.width[1]) - c.half_width[1];
        d[2] = omod_fast(p.z - q.z + c.half_width[2], c.width[2]) - c.half_width[2];
        s2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        if (!(s2 > 0.0)) s2 = 0.0;  // a NaN never wins the reference's `>` test
    }
    // block maximum, then one atomic on the ordered bit pattern (s2 >= 0)
    for (int o = 16; o > 0; o >>= 1) {
        const double t = __shfl_xor_sync(0xffffffffu, s2, o);
        s2 = t > s2 ? t : s2;
    }
    __shared__ double red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = red[w] > m ? red[w] : m;
        if (m > 0.0) atomicMax(&scal->max_shift2_bits, (unsigned long long)__double_as_longlong(m));
        if (GRAPH) {
            __threadfence();
            if (atomicAdd(&scal->blocks_done, 1u) == gridDim.x - 1) {  // the last block
                __threadfence();
                const unsigned long long bits = atomicAdd(&scal->max_shift2_bits, 0ull);
                const bool rebuild = !stopped && __longlong_as_double((long long)bits) > c.shift_thr;
                cudaGraphSetConditional(h_rebuild, rebuild ? 1u : 0u);
                cudaGraphSetConditional(h_sweep, stopped ? 0u : 1u);
                if (rebuild) scal->rebuilds_done += 1;
                if (!stopped) scal->steps_done += 1;
                scal->max_shift2_bits = 0ull;
                scal->blocks_done = 0u;
            }
        }
    }
}

// Kernel shapes as functions of q = r/h (main.cpp:214-284; the reference's
// (1.0/h) factor is the rounded reciprocal inv_h, as there).
__device__ __forceinline__ double s_wa(const SimConst& c, double q) { return ((c.ca * q) * (1.0 - q)) * (1.0 - q); }
__device__ __forceinline__ double s_dwa(const SimConst& c, double q) {
    return ((c.ca * (1.0 - q)) * (1.0 - 3.0 * q)) * c.inv_ra;
}
__device__ __forceinline__ double s_wg(const SimConst& c, double q) { return c.cg * ((1.0 - q) * (1.0 - q)); }
__device__ __forceinline__ double s_dwg(const SimConst& c, double q) { return c.cg * (c.m2_rg * (1.0 - q)); }
__device__ __forceinline__ double s_wp(const SimConst& c, double q) { return c.cp * ((1.0 - q) * (1.0 - q)); }
__device__ __forceinline__ double s_dwp(const SimConst& c, double q) { return c.cp * (c.m2_rp * (1.0 - q)); }
__device__ __forceinline__ double s_dwv(const SimConst& c, double q) { return c.cv * (c.m2_rv * (1.0 - q)); }

// Sweep A: DensityA (main.cpp:1665-1692), GravityCenter (1695-1727),
// DensityP (1831-1858), DivergenceP (1860-1896), then
// calculatePhysicalCoefficients (1631-1662) and the PressureP / PressureA
// values (1904-1906, 1735-1740).  Every division of the reference is an
// exactly rounded div_rn (mph_exact.cuh) against one reciprocal per pair.
// DA: DensityA and PressureA are computed here, over the whole list.  Without
// surface tension the step does not use them (PressureA is zero and its force
// terms are not evaluated), so the step leaves them to k_density_a, run only
// when they are read, and visits only the short sublist (the pairs that can
// lie within RadiusP, in list order).
// SPLIT (with surface tension): DensityP and DivergenceP over the short
// sublist (ncount_p, nlist_p: the list's entries within RadiusP+MARGIN, in list
// order, so the same sums), DensityA and GravityCenter over the list; the
// pressure block then no longer runs with most lanes masked off.
template <bool ST, bool RATIO, bool DA, bool SPLIT>
__global__ void __launch_bounds__(128, ST ? MPH_SWEEP_MINB_ST : MPH_SWEEP_MINB)
k_sweep_a(SimConst c, const double4* __restrict__ pos, const double4* __restrict__ vel,
          const int* __restrict__ ncount, const int* __restrict__ nlist, const int* __restrict__ ncount_p,
          const int* __restrict__ nlist_p, double* __restrict__ dens_a,
          double* __restrict__ strain_p, double* __restrict__ div_p, double4* __restrict__ velp,
          double4* __restrict__ gcpa, double* __restrict__ wall_center) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (wall_center != nullptr && blockIdx.x == 0 && threadIdx.x < 12) {
        // WallCenter += WallVelocity*Dt (main.cpp:2048-2052); the move kernel of
        // this step has already used the old value.
        const int t = threadIdx.x / 3, d = threadIdx.x % 3;
        if (t >= 2) wall_center[3 * t + d] += c.wall_velocity[t][d] * c.dt;
    }
    if (i >= c.n) return;
    const double4 pi = pos[i];
    const double4 vi = vel[i];
    const int ti = type_of(pi);
    const int cnt = ncount[i];
    const size_t n = (size_t)c.n;
    double sum_a = 0.0, sum_p = 0.0, sum_d = 0.0;
    double g0 = 0.0, g1 = 0.0, g2 = 0.0;
    if (SPLIT) {  // DensityP, DivergenceP over the short sublist (main.cpp:1831-1896)
        const int cs = ncount_p[i];
        const int* lq = nlist_p + i;
        int q1 = cs > 0 ? __ldg(lq) : i;
        int q2 = cs > 1 ? __ldg(lq + n) : i;
        lq += 2 * n;
        double4 qn = pos[q1], qv = vel[q1];
        for (int k = 0; k < cs; ++k) {
            const int j = q1;
            const double4 pj = qn;
            const double4 vjn = qv;
            q1 = q2;
            if (k + 2 < cs) q2 = __ldg(lq);
            lq += n;
            if (k + 1 < cs) {
                qn = pos[q1];
                qv = vel[q1];
            }
            if (j == i) continue;
            double x[3];
            disp(c, pi, pj, x);
            const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            if (!(r2 <= c.rp2)) continue;
            const double r = sqrt(r2);
            const double qp = div_rs(r, c.rp, c.inv_rp);
            sum_p += s_wp(c, qp);
            const double dw = s_dwp(c, qp);
            const double ri = __drcp_rn(r);
            const double e0 = div_rs(x[0], r, ri), e1 = div_rs(x[1], r, ri), e2 = div_rs(x[2], r, ri);
            const double u0 = vjn.x - vi.x, u1 = vjn.y - vi.y, u2 = vjn.z - vi.z;
            sum_d -= u0 * e0 * dw;
            sum_d -= u1 * e1 * dw;
            sum_d -= u2 * e2 * dw;
        }
    }
    // indices two entries ahead, the neighbour's position and velocity one ahead
    const int* lp = nlist + i;
    int j1 = cnt > 0 ? __ldg(lp) : i;
    int j2 = cnt > 1 ? __ldg(lp + n) : i;
    lp += 2 * n;
    double4 pn = pos[j1], vq = vel[j1];
    for (int k = 0; k < cnt; ++k) {
        const int j = j1;
        const double4 pj = pn;
        const double4 vjn = vq;
        j1 = j2;
        if (k + 2 < cnt) j2 = __ldg(lp);
        lp += n;
        if (k + 1 < cnt) {
            pn = pos[j1];
            vq = vel[j1];
        }
        if (j == i) continue;
        double x[3];
        disp(c, pi, pj, x);
        const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        // R*R - r2 >= 0 (main.cpp:1683 and the other density sums) is r2 <= R*R:
        // with gradual underflow a - b is zero only when a == b, and its sign exact
        const bool in_a = DA && (r2 <= c.ra2);
        const bool in_p = !SPLIT && r2 <= c.rp2;
        const bool in_g = ST && (r2 <= c.rg2);
        if (!(in_a || in_p || in_g)) continue;
        const double r = sqrt(r2);
        double ratio = 1.0;
        if (RATIO) ratio = c.ratio[ti][type_of(pj)];
        const double qa = div_rs(r, c.ra, c.inv_ra);
        if (in_a) {
            const double w = RATIO ? ratio * s_wa(c, qa) : s_wa(c, qa);
            sum_a += w;
        }
        if (ST && in_g) {
            const double qg = c.rg_eq_ra ? qa : div_rs(r, c.rg, c.inv_rg);
            const double w = RATIO ? ratio * s_wg(c, qg) : s_wg(c, qg);
            g0 += div_rs(x[0] * w, c.r2g, c.inv_r2g) * c.rg;
            g1 += div_rs(x[1] * w, c.r2g, c.inv_r2g) * c.rg;
            g2 += div_rs(x[2] * w, c.r2g, c.inv_r2g) * c.rg;
        }
        if (in_p) {
            const double qp = div_rs(r, c.rp, c.inv_rp);
            sum_p += s_wp(c, qp);
            const double dw = s_dwp(c, qp);
            const double ri = __drcp_rn(r);
            const double e0 = div_rs(x[0], r, ri), e1 = div_rs(x[1], r, ri), e2 = div_rs(x[2], r, ri);
            const double u0 = vjn.x - vi.x, u1 = vjn.y - vi.y, u2 = vjn.z - vi.z;
            sum_d -= u0 * e0 * dw;
            sum_d -= u1 * e1 * dw;
            sum_d -= u2 * e2 * dw;
        }
    }
    if (DA) dens_a[i] = sum_a;
    const double strain = sum_p - c.n0p;
    strain_p[i] = strain;
    div_p[i] = sum_d;
    double kappa = c.bulk_modulus[ti];
    if (strain < 0.0) kappa = 0.0;
    const double lambda = c.bulk_viscosity[ti];
    const double pp = -lambda * sum_d + kappa * strain;
    double pa = 0.0;
    if (DA) {
        pa = c.cof_a[ti] * (sum_a - c.n0a) / c.l0;
        if (c.n0a <= sum_a) pa = 0.0;
    }
    // sweep B gathers {v, PressureP} and {GravityCenter, PressureA} per neighbour
    velp[i] = make_double4(vi.x, vi.y, vi.z, pp);
    gcpa[i] = make_double4(g0, g1, g2, pa);
}

// DensityA (main.cpp:1665-1692) and PressureA (1735-1740) alone, for the
// readers of a form without surface tension: the pairs of k_sweep_a's DensityA
// sum in the same list order with the same arithmetic, from the positions
// that sweep used (the step changes only velocities after it), so the values
// are those the reference holds after the step.
template <bool RATIO>
__global__ void __launch_bounds__(128) k_density_a(SimConst c, const double4* __restrict__ pos,
                                                   const int* __restrict__ ncount, const int* __restrict__ nlist,
                                                   double* __restrict__ dens_a, double4* __restrict__ gcpa) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const double4 pi = pos[i];
    const int ti = type_of(pi);
    const int cnt = ncount[i];
    const size_t n = (size_t)c.n;
    double sum_a = 0.0;
    for (int k = 0; k < cnt; ++k) {
        const int j = __ldg(nlist + (size_t)k * n + i);
        if (j == i) continue;
        const double4 pj = pos[j];
        double x[3];
        disp(c, pi, pj, x);
        const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        if (!(r2 <= c.ra2)) continue;
        const double r = sqrt(r2);
        const double qa = div_rs(r, c.ra, c.inv_ra);
        sum_a += RATIO ? c.ratio[ti][type_of(pj)] * s_wa(c, qa) : s_wa(c, qa);
    }
    dens_a[i] = sum_a;
    double pa = c.cof_a[ti] * (sum_a - c.n0a) / c.l0;
    if (c.n0a <= sum_a) pa = 0.0;
    reinterpret_cast<double*>(gcpa + i)[3] = pa;
}

// Sweep B: PressureP force (main.cpp:1908-1938), PressureA force
// (1742-1775), DiffuseInterface (1782-1828, aj uses the type of i as in the
// reference), ViscosityV (1943-1984); Force = 0 + fP + fA + fDI + fV, then
// Gravity (1988-1998) and Acceleration (2000-2010) for fluid particles.
// LRN: the learned form.  The PressureA, DiffuseInterface and ViscosityV pair
// terms are not evaluated; fluid particle i adds instead the sum of its
// edge-MLP pair forces eforce[eoff[i] .. eoff[i+1]) (FP32, in edge order),
// which is also stored in lsum[i].
// SPLIT (not learned): the PressureP force visits only
// pairs within RadiusP, all of which are in the short sublist, in list order
// (the argument of k_neighbor_list), so that sum runs as its own loop over the
// short sublist and the main loop carries ViscosityV alone.  The terms and
// their order in each sum are the reference's; the main loop no longer runs
// the pressure block under a branch that some lane takes on nearly every
// entry while most lanes wait.
template <bool ST, bool RATIO, bool LRN, bool SPLIT>
__global__ void __launch_bounds__(128, ST ? MPH_SWEEPB_MINB_ST : MPH_SWEEPB_MINB)
k_sweep_b(SimConst c, const int* __restrict__ cellstart, const double4* __restrict__ pos,
          const double4* __restrict__ velp, double4* __restrict__ vel_out, const double4* __restrict__ gcpa,
          const int* __restrict__ ncount, const int* __restrict__ nlist, const int* __restrict__ ncount_s,
          const int* __restrict__ nlist_s, double4* __restrict__ force,
          StepScalars* __restrict__ scal, const int* __restrict__ eoff, const float4* __restrict__ eforce,
          float4* __restrict__ lsum, int part, int i0, int i1, double* __restrict__ vel_host) {
    const int i = i0 + (int)(blockIdx.x * blockDim.x + threadIdx.x);  // particles [i0, i1)
    if (i >= i1) return;
    const int nf = cellstart[c.tot];
    const double4 vi = velp[i];   // .w = PressureP
    // part 1: fluid only; a wall keeps its velocity (what the full sweep
    // writes for it) and its force is left for part 2 (output only)
    if (part == 1 && i >= nf) {
        vel_out[i] = make_double4(vi.x, vi.y, vi.z, 0.0);
        if (vel_host) {
            vel_host[3 * (size_t)i] = vi.x;
            vel_host[3 * (size_t)i + 1] = vi.y;
            vel_host[3 * (size_t)i + 2] = vi.z;
        }
        return;
    }
    if (part == 2 && i < nf) return;
    const double4 pi = pos[i];
    const int ti = type_of(pi);
    const double ai = c.a_k[ti];
    double4 gci = make_double4(0, 0, 0, 0);
    if (ST) gci = gcpa[i];        // .w = PressureA
    const int cnt = ncount[i];
    const size_t n = (size_t)c.n;
    double fp0 = 0.0, fp1 = 0.0, fp2 = 0.0;
    double fa0 = 0.0, fa1 = 0.0, fa2 = 0.0;
    double fd0 = 0.0, fd1 = 0.0, fd2 = 0.0;
    double fv0 = 0.0, fv1 = 0.0, fv2 = 0.0;
    if (SPLIT) {  // PressureP force (main.cpp:1908-1938) over the short sublist
        // indices two entries ahead, the neighbour's records one entry ahead
        const int cs = ncount_s[i];
        const int* lq = nlist_s + i;
        int q1 = cs > 0 ? __ldg(lq) : i;
        int q2 = cs > 1 ? __ldg(lq + n) : i;
        lq += 2 * n;
        double4 qn = pos[q1];
        double qp1 = velp[q1].w;
        for (int k = 0; k < cs; ++k) {
            const int j = q1;
            const double4 pj = qn;
            const double pjp = qp1;  // PressureP of j
            q1 = q2;
            if (k + 2 < cs) q2 = __ldg(lq);
            lq += n;
            if (k + 1 < cs) {
                qn = pos[q1];
                qp1 = velp[q1].w;
            }
            if (j == i) continue;
            double x[3];
            disp(c, pi, pj, x);
            const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            if (!(r2 < c.rp2)) continue;
            const double r = sqrt(r2);
            const double ri = __drcp_rn(r);
            const double qp = div_rs(r, c.rp, c.inv_rp);
            const double dw = s_dwp(c, qp);
            const double gw0 = div_rs(dw * x[0], r, ri), gw1 = div_rs(dw * x[1], r, ri),
                         gw2 = div_rs(dw * x[2], r, ri);
            const double ps = vi.w + pjp;
            fp0 += ps * gw0 * c.vol;
            fp1 += ps * gw1 * c.vol;
            fp2 += ps * gw2 * c.vol;
        }
    }
    // software pipeline: list indices two entries ahead, the neighbour's two
    // records (position, velocity + PressureP) one entry ahead, so their
    // gathers overlap the previous pair's FP64 arithmetic
    const int* lp = nlist + i;
    int j1 = cnt > 0 ? __ldg(lp) : i;
    int j2 = cnt > 1 ? __ldg(lp + n) : i;
    lp += 2 * n;
    double4 pn = pos[j1], vn1 = velp[j1];
    for (int k = 0; k < cnt; ++k) {
        const int j = j1;
        const double4 pj = pn;
        const double4 vj = vn1;   // .w = PressureP of j
        j1 = j2;
        if (k + 2 < cnt) j2 = __ldg(lp);
        lp += n;
        if (k + 1 < cnt) {
            pn = pos[j1];
            vn1 = velp[j1];
        }
        if (j == i) continue;
        double x[3];
        disp(c, pi, pj, x);
        const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        // Without surface tension every CofA is 0, PressureA is +-0 and each
        // PressureA term adds a signed zero to a sum that starts at +0: the sum
        // stays +0 exactly, so the term is skipped (ST == false).
        // R*R - r2 > 0 (main.cpp:1926 and the other force sums) is r2 < R*R
        const bool in_p = !SPLIT && r2 < c.rp2;
        const bool in_a = !LRN && ST && (r2 < c.ra2);
        const bool in_g = !LRN && ST && (r2 < c.rg2);
        const bool in_v = !LRN && r2 < c.rv2;
        if (!(in_p || in_a || in_g || in_v)) continue;
        const int tj = type_of(pj);
        const double r = sqrt(r2);
        const double ri = __drcp_rn(r);
        const double e0 = div_rs(x[0], r, ri), e1 = div_rs(x[1], r, ri), e2 = div_rs(x[2], r, ri);
        const double qa = div_rs(r, c.ra, c.inv_ra);
        double rij = 1.0, rji = 1.0;
        if (RATIO) { rij = c.ratio[ti][tj]; rji = c.ratio[tj][ti]; }
        if (in_p) {
            const double qp = div_rs(r, c.rp, c.inv_rp);
            const double dw = s_dwp(c, qp);
            const double gw0 = div_rs(dw * x[0], r, ri), gw1 = div_rs(dw * x[1], r, ri),
                         gw2 = div_rs(dw * x[2], r, ri);
            const double ps = vi.w + vj.w;
            fp0 += ps * gw0 * c.vol;
            fp1 += ps * gw1 * c.vol;
            fp2 += ps * gw2 * c.vol;
        }
        if (in_a) {
            const double dwa = s_dwa(c, qa);
            const double dwij = RATIO ? rij * dwa : dwa;
            const double dwji = RATIO ? rji * dwa : dwa;
            const double s = gci.w * dwij + gcpa[j].w * dwji;
            fa0 += s * e0 * c.vol;
            fa1 += s * e1 * c.vol;
            fa2 += s * e2 * c.vol;
        }
        if (ST && in_g) {
            const double4 gcj = gcpa[j];
            const double aj = ai;
            const double qg = c.rg_eq_ra ? qa : div_rs(r, c.rg, c.inv_rg);
            const double wg = s_wg(c, qg);
            const double wij = RATIO ? rij * wg : wg;
            const double wji = RATIO ? rji * wg : wg;
            fd0 -= div_rs(aj * gcj.x * wji - ai * gci.x * wij, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
            fd1 -= div_rs(aj * gcj.y * wji - ai * gci.y * wij, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
            fd2 -= div_rs(aj * gcj.z * wji - ai * gci.z * wij, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
            const double dg = s_dwg(c, qg);
            const double dwij = RATIO ? rij * dg : dg;
            const double dwji = RATIO ? rji * dg : dg;
            double gr = 0.0;
            gr += (aj * gcj.x * dwji - ai * gci.x * dwij) * x[0];
            gr += (aj * gcj.y * dwji - ai * gci.y * dwij) * x[1];
            gr += (aj * gcj.z * dwji - ai * gci.z * dwij) * x[2];
            fd0 -= div_rs((gr) * e0, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
            fd1 -= div_rs((gr) * e1, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
            fd2 -= div_rs((gr) * e2, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
        }
        if (in_v) {
            const double qv = c.rv_eq_ra ? qa : div_rs(r, c.rv, c.inv_rv);
            const double dw = -s_dwv(c, qv);
            const double u0 = vj.x - vi.x, u1 = vj.y - vi.y, u2 = vj.z - vi.z;
            const double cm = c.visc_mu[ti][tj];
            const double dot = u0 * e0 + u1 * e1 + u2 * e2;
            fv0 += div_rs(cm * dot * e0 * dw, r, ri) * c.vol;
            fv1 += div_rs(cm * dot * e1 * dw, r, ri) * c.vol;
            fv2 += div_rs(cm * dot * e2 * dw, r, ri) * c.vol;
        }
    }
    if (LRN) {
        float l0 = 0.f, l1 = 0.f, l2 = 0.f;
        if (i < nf) {
            for (int g = eoff[i], ge = eoff[i + 1]; g < ge; ++g) {
                const float4 q = eforce[g];
                l0 += q.x;
                l1 += q.y;
                l2 += q.z;
            }
        }
        lsum[i] = make_float4(l0, l1, l2, 0.f);
        fv0 = l0;
        fv1 = l1;
        fv2 = l2;
    }
    double F0 = 0.0, F1 = 0.0, F2 = 0.0;   // resetForce (main.cpp:1617-1628)
    F0 += fp0; F1 += fp1; F2 += fp2;
    F0 += fa0; F1 += fa1; F2 += fa2;
    F0 += fd0; F1 += fd1; F2 += fd2;
    F0 += fv0; F1 += fv1; F2 += fv2;
    double4 vn = make_double4(vi.x, vi.y, vi.z, 0.0);
    if (i < nf) {
        const double m = c.density[ti] * c.vol;
        F0 += m * c.gravity[0];
        F1 += m * c.gravity[1];
        F2 += m * c.gravity[2];
        vn.x += F0 / m * c.dt;
        vn.y += F1 / m * c.dt;
        vn.z += F2 / m * c.dt;
        if (!(isfinite(vn.x) && isfinite(vn.y) && isfinite(vn.z))) atomicOr(&scal->flags, DEVFLAG_NONFINITE);
    }
    force[i] = make_double4(F0, F1, F2, 0.0);
    if (part != 2) {
        vel_out[i] = vn;
        if (vel_host) {  // mapped pinned host memory: the read-back travels while the sweep runs
            vel_host[3 * (size_t)i] = vn.x;
            vel_host[3 * (size_t)i + 1] = vn.y;
            vel_host[3 * (size_t)i + 2] = vn.z;
        }
    }
}

// ---- warp per particle (small scenes) ----------------------------------------
// With few particles the thread-per-particle sweeps leave most of the GPU idle
// and each thread's chain of dependent FP64 work over its ~200 list entries
// sets the time.  Here a warp takes one particle: its 32 lanes compute the
// pair terms of 32 consecutive list entries at once (the expressions of
// k_sweep_a / k_sweep_b), then one lane per sum adds the chunk's terms to it
// in list order, each with the operation the thread kernels apply (+= or -=,
// two in a row where they apply two): the same additions in the same order,
// so the same bits.
constexpr int kWarpSweepWarps = 4;

// lane s's sum of k_sweep_b_w: flag bit, first term, second term (-1: none), subtract
struct SumOp {
    unsigned bit;
    int q1, q2;
    bool sub;
};
__device__ __forceinline__ SumOp sweep_b_sum(int s) {
    // fp0..2 (+, bit 1), fv0..2 (+, bit 8), fa0..2 (+, bit 2), fd0..2 (-, -, bit 4)
    if (s < 3) return {1u, s, -1, false};
    if (s < 6) return {8u, s, -1, false};
    if (s < 9) return {2u, s, -1, false};
    return {4u, s, s + 3, true};
}

template <bool ST, bool RATIO>
__global__ void __launch_bounds__(32 * kWarpSweepWarps)
k_sweep_b_w(SimConst c, const int* __restrict__ cellstart, const double4* __restrict__ pos,
            const double4* __restrict__ velp, double4* __restrict__ vel_out, const double4* __restrict__ gcpa,
            const int* __restrict__ ncount, const int* __restrict__ nlist, double4* __restrict__ force,
            StepScalars* __restrict__ scal, int part, double* __restrict__ vel_host) {
    constexpr int NV = ST ? 15 : 6;  // terms per entry: fp 3, fv 3 [, fa 3, fd 3 + 3]
    constexpr int NS = ST ? 12 : 6;  // sums
    __shared__ double tv[kWarpSweepWarps][NV][33];
    __shared__ unsigned tf[kWarpSweepWarps][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int i = blockIdx.x * kWarpSweepWarps + w;
    if (i >= c.n) return;  // whole warp
    const int nf = cellstart[c.tot];
    const double4 vi = velp[i];   // .w = PressureP
    if (part == 1 && i >= nf) {   // a wall keeps its velocity (see k_sweep_b)
        if (lane == 0) {
            vel_out[i] = make_double4(vi.x, vi.y, vi.z, 0.0);
            if (vel_host) {
                vel_host[3 * (size_t)i] = vi.x;
                vel_host[3 * (size_t)i + 1] = vi.y;
                vel_host[3 * (size_t)i + 2] = vi.z;
            }
        }
        return;
    }
    if (part == 2 && i < nf) return;
    const double4 pi = pos[i];
    const int ti = type_of(pi);
    const double ai = c.a_k[ti];
    double4 gci = make_double4(0, 0, 0, 0);
    if (ST) gci = gcpa[i];        // .w = PressureA
    const int cnt = ncount[i];
    const size_t n = (size_t)c.n;
    const SumOp op = sweep_b_sum(lane < NS ? lane : 0);
    double acc = 0.0;
    for (int k0 = 0; k0 < cnt; k0 += 32) {
        const int k = k0 + lane;
        unsigned fl = 0u;
        double v[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) v[q] = 0.0;
        const int j = k < cnt ? __ldg(nlist + (size_t)k * n + i) : i;
        if (j != i) {
            const double4 pj = pos[j];
            double x[3];
            disp(c, pi, pj, x);
            const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            const bool in_p = r2 < c.rp2;
            const bool in_a = ST && (r2 < c.ra2);
            const bool in_g = ST && (r2 < c.rg2);
            const bool in_v = r2 < c.rv2;
            if (in_p || in_a || in_g || in_v) {
                const double4 vj = velp[j];   // .w = PressureP of j
                const int tj = type_of(pj);
                const double r = sqrt(r2);
                const double ri = __drcp_rn(r);
                const double e0 = div_rs(x[0], r, ri), e1 = div_rs(x[1], r, ri), e2 = div_rs(x[2], r, ri);
                const double qa = div_rs(r, c.ra, c.inv_ra);
                double rij = 1.0, rji = 1.0;
                if (RATIO) { rij = c.ratio[ti][tj]; rji = c.ratio[tj][ti]; }
                if (in_p) {
                    const double qp = div_rs(r, c.rp, c.inv_rp);
                    const double dw = s_dwp(c, qp);
                    const double gw0 = div_rs(dw * x[0], r, ri), gw1 = div_rs(dw * x[1], r, ri),
                                 gw2 = div_rs(dw * x[2], r, ri);
                    const double ps = vi.w + vj.w;
                    v[0] = ps * gw0 * c.vol;
                    v[1] = ps * gw1 * c.vol;
                    v[2] = ps * gw2 * c.vol;
                    fl |= 1u;
                }
                if (in_v) {
                    const double qv = c.rv_eq_ra ? qa : div_rs(r, c.rv, c.inv_rv);
                    const double dw = -s_dwv(c, qv);
                    const double u0 = vj.x - vi.x, u1 = vj.y - vi.y, u2 = vj.z - vi.z;
                    const double cm = c.visc_mu[ti][tj];
                    const double dot = u0 * e0 + u1 * e1 + u2 * e2;
                    v[3] = div_rs(cm * dot * e0 * dw, r, ri) * c.vol;
                    v[4] = div_rs(cm * dot * e1 * dw, r, ri) * c.vol;
                    v[5] = div_rs(cm * dot * e2 * dw, r, ri) * c.vol;
                    fl |= 8u;
                }
                if (ST && in_a) {
                    const double dwa = s_dwa(c, qa);
                    const double dwij = RATIO ? rij * dwa : dwa;
                    const double dwji = RATIO ? rji * dwa : dwa;
                    const double sa = gci.w * dwij + gcpa[j].w * dwji;
                    v[6 % NV] = sa * e0 * c.vol;
                    v[7 % NV] = sa * e1 * c.vol;
                    v[8 % NV] = sa * e2 * c.vol;
                    fl |= 2u;
                }
                if (ST && in_g) {
                    const double4 gcj = gcpa[j];
                    const double aj = ai;
                    const double qg = c.rg_eq_ra ? qa : div_rs(r, c.rg, c.inv_rg);
                    const double wg = s_wg(c, qg);
                    const double wij = RATIO ? rij * wg : wg;
                    const double wji = RATIO ? rji * wg : wg;
                    v[9 % NV] = div_rs(aj * gcj.x * wji - ai * gci.x * wij, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
                    v[10 % NV] = div_rs(aj * gcj.y * wji - ai * gci.y * wij, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
                    v[11 % NV] = div_rs(aj * gcj.z * wji - ai * gci.z * wij, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
                    const double dg = s_dwg(c, qg);
                    const double dwij = RATIO ? rij * dg : dg;
                    const double dwji = RATIO ? rji * dg : dg;
                    double gr = 0.0;
                    gr += (aj * gcj.x * dwji - ai * gci.x * dwij) * x[0];
                    gr += (aj * gcj.y * dwji - ai * gci.y * dwij) * x[1];
                    gr += (aj * gcj.z * dwji - ai * gci.z * dwij) * x[2];
                    v[12 % NV] = div_rs((gr) * e0, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
                    v[13 % NV] = div_rs((gr) * e1, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
                    v[14 % NV] = div_rs((gr) * e2, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
                    fl |= 4u;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NV; ++q) tv[w][q][lane] = v[q];
        tf[w][lane] = fl;
        __syncwarp();
        const int m = min(32, cnt - k0);
        if (lane < NS) {
            // branch-free and the same for every lane: acc = (acc - a) - b, with
            // a = -t, b = +0 for a += (acc + t, then - +0 changes nothing, -0
            // included), a = t1, b = t2 for the two -=; an entry without the
            // term keeps acc
            const int q2 = op.q2 < 0 ? 0 : op.q2;
#pragma unroll 4
            for (int e = 0; e < m; ++e) {
                const double t1 = tv[w][op.q1][e];
                const double a = op.sub ? t1 : -t1;
                const double b = op.sub ? tv[w][q2][e] : 0.0;
                const double nx = (acc - a) - b;
                acc = (tf[w][e] & op.bit) ? nx : acc;
            }
        }
        __syncwarp();
    }
    double sums[12];
#pragma unroll
    for (int q = 0; q < 12; ++q) sums[q] = q < NS ? __shfl_sync(0xffffffffu, acc, q) : 0.0;
    if (lane != 0) return;
    const double fp0 = sums[0], fp1 = sums[1], fp2 = sums[2];
    const double fv0 = sums[3], fv1 = sums[4], fv2 = sums[5];
    const double fa0 = sums[6], fa1 = sums[7], fa2 = sums[8];
    const double fd0 = sums[9], fd1 = sums[10], fd2 = sums[11];
    double F0 = 0.0, F1 = 0.0, F2 = 0.0;   // resetForce (main.cpp:1617-1628), as k_sweep_b
    F0 += fp0; F1 += fp1; F2 += fp2;
    F0 += fa0; F1 += fa1; F2 += fa2;
    F0 += fd0; F1 += fd1; F2 += fd2;
    F0 += fv0; F1 += fv1; F2 += fv2;
    double4 vn = make_double4(vi.x, vi.y, vi.z, 0.0);
    if (i < nf) {
        const double m = c.density[ti] * c.vol;
        F0 += m * c.gravity[0];
        F1 += m * c.gravity[1];
        F2 += m * c.gravity[2];
        vn.x += F0 / m * c.dt;
        vn.y += F1 / m * c.dt;
        vn.z += F2 / m * c.dt;
        if (!(isfinite(vn.x) && isfinite(vn.y) && isfinite(vn.z))) atomicOr(&scal->flags, DEVFLAG_NONFINITE);
    }
    force[i] = make_double4(F0, F1, F2, 0.0);
    if (part != 2) {
        vel_out[i] = vn;
        if (vel_host) {
            vel_host[3 * (size_t)i] = vn.x;
            vel_host[3 * (size_t)i + 1] = vn.y;
            vel_host[3 * (size_t)i + 2] = vn.z;
        }
    }
}

// Sweep A, warp per particle: sums DensityA (lane 0, bit 1), DensityP (lane 1,
// bit 2), DivergenceP (lane 2, bit 2, three subtractions per entry) and
// GravityCenter (lanes 3-5, bit 4), as k_sweep_a adds them.
template <bool ST, bool RATIO, bool DA>
__global__ void __launch_bounds__(32 * kWarpSweepWarps)
k_sweep_a_w(SimConst c, const double4* __restrict__ pos, const double4* __restrict__ vel,
            const int* __restrict__ ncount, const int* __restrict__ nlist, double* __restrict__ dens_a,
            double* __restrict__ strain_p, double* __restrict__ div_p, double4* __restrict__ velp,
            double4* __restrict__ gcpa, double* __restrict__ wall_center) {
    __shared__ double tv[kWarpSweepWarps][8][33];
    __shared__ unsigned tf[kWarpSweepWarps][32];
    if (wall_center != nullptr && blockIdx.x == 0 && threadIdx.x < 12) {
        // WallCenter += WallVelocity*Dt (main.cpp:2048-2052), as k_sweep_a
        const int t = threadIdx.x / 3, d = threadIdx.x % 3;
        if (t >= 2) wall_center[3 * t + d] += c.wall_velocity[t][d] * c.dt;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int i = blockIdx.x * kWarpSweepWarps + w;
    if (i >= c.n) return;  // whole warp
    const double4 pi = pos[i];
    const double4 vi = vel[i];
    const int ti = type_of(pi);
    const int cnt = ncount[i];
    const size_t n = (size_t)c.n;
    // lane s's sum: 0 DensityA, 1 DensityP, 2 DivergenceP, 3-5 GravityCenter
    const unsigned bit = lane == 0 ? 1u : (lane < 3 ? 2u : 4u);
    double acc = 0.0;
    for (int k0 = 0; k0 < cnt; k0 += 32) {
        const int k = k0 + lane;
        unsigned fl = 0u;
        double v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = 0.0;
        const int j = k < cnt ? __ldg(nlist + (size_t)k * n + i) : i;
        if (j != i) {
            const double4 pj = pos[j];
            double x[3];
            disp(c, pi, pj, x);
            const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            const bool in_a = DA && (r2 <= c.ra2);
            const bool in_p = r2 <= c.rp2;
            const bool in_g = ST && (r2 <= c.rg2);
            if (in_a || in_p || in_g) {
                const double r = sqrt(r2);
                double ratio = 1.0;
                if (RATIO) ratio = c.ratio[ti][type_of(pj)];
                const double qa = div_rs(r, c.ra, c.inv_ra);
                if (in_a) {
                    v[0] = RATIO ? ratio * s_wa(c, qa) : s_wa(c, qa);
                    fl |= 1u;
                }
                if (ST && in_g) {
                    const double qg = c.rg_eq_ra ? qa : div_rs(r, c.rg, c.inv_rg);
                    const double wgt = RATIO ? ratio * s_wg(c, qg) : s_wg(c, qg);
                    v[5] = div_rs(x[0] * wgt, c.r2g, c.inv_r2g) * c.rg;
                    v[6] = div_rs(x[1] * wgt, c.r2g, c.inv_r2g) * c.rg;
                    v[7] = div_rs(x[2] * wgt, c.r2g, c.inv_r2g) * c.rg;
                    fl |= 4u;
                }
                if (in_p) {
                    const double4 vjn = vel[j];
                    const double qp = div_rs(r, c.rp, c.inv_rp);
                    v[1] = s_wp(c, qp);
                    const double dw = s_dwp(c, qp);
                    const double ri = __drcp_rn(r);
                    const double e0 = div_rs(x[0], r, ri), e1 = div_rs(x[1], r, ri), e2 = div_rs(x[2], r, ri);
                    const double u0 = vjn.x - vi.x, u1 = vjn.y - vi.y, u2 = vjn.z - vi.z;
                    v[2] = u0 * e0 * dw;
                    v[3] = u1 * e1 * dw;
                    v[4] = u2 * e2 * dw;
                    fl |= 2u;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) tv[w][q][lane] = v[q];
        tf[w][lane] = fl;
        __syncwarp();
        const int m = min(32, cnt - k0);
        if (lane < 6) {
            // as in k_sweep_b_w: acc = ((acc - a) - b) - c, a = -t, b = c = +0
            // for a +=, the three DivergenceP terms for lane 2's three -=
            const int q = lane < 2 ? lane : (lane == 2 ? 2 : lane + 2);
            const bool sub = lane == 2;
#pragma unroll 4
            for (int e = 0; e < m; ++e) {
                const double t = tv[w][q][e];
                const double a = sub ? t : -t;
                const double b = sub ? tv[w][3][e] : 0.0;
                const double c3 = sub ? tv[w][4][e] : 0.0;
                const double nx = ((acc - a) - b) - c3;
                acc = (tf[w][e] & bit) ? nx : acc;
            }
        }
        __syncwarp();
    }
    const double sum_a = __shfl_sync(0xffffffffu, acc, 0);
    const double sum_p = __shfl_sync(0xffffffffu, acc, 1);
    const double sum_d = __shfl_sync(0xffffffffu, acc, 2);
    const double g0 = __shfl_sync(0xffffffffu, acc, 3);
    const double g1 = __shfl_sync(0xffffffffu, acc, 4);
    const double g2 = __shfl_sync(0xffffffffu, acc, 5);
    if (lane != 0) return;
    if (DA) dens_a[i] = sum_a;
    const double strain = sum_p - c.n0p;
    strain_p[i] = strain;
    div_p[i] = sum_d;
    double kappa = c.bulk_modulus[ti];
    if (strain < 0.0) kappa = 0.0;
    const double lambda = c.bulk_viscosity[ti];
    const double pp = -lambda * sum_d + kappa * strain;
    double pa = 0.0;
    if (DA) {
        pa = c.cof_a[ti] * (sum_a - c.n0a) / c.l0;
        if (c.n0a <= sum_a) pa = 0.0;
    }
    velp[i] = make_double4(vi.x, vi.y, vi.z, pp);
    gcpa[i] = make_double4(ST ? g0 : 0.0, ST ? g1 : 0.0, ST ? g2 : 0.0, pa);
}

// Self-check of div_rn against the hardware IEEE division: operands with
// random significands and exponents in [-40, 40], plus all-ones significands.
__global__ void k_check_division(unsigned long long seed, long long n, unsigned long long* mismatches,
                                 double* first) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += stride) {
        unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(t + 1);
        auto mix = [](unsigned long long v) {
            v ^= v >> 30; v *= 0xBF58476D1CE4E5B9ull;
            v ^= v >> 27; v *= 0x94D049BB133111EBull;
            return v ^ (v >> 31);
        };
        const unsigned long long a = mix(z), b = mix(z ^ 0xD1B54A32D192ED03ull), e = mix(z + 17);
        unsigned long long ma = a & 0xFFFFFFFFFFFFFull, mb = b & 0xFFFFFFFFFFFFFull;
        if ((e & 15) == 0) mb = 0xFFFFFFFFFFFFFull;
        if ((e & 15) == 1) ma = 0xFFFFFFFFFFFFFull;
        const int ea = (int)((e >> 8) % 81) - 40, eb = (int)((e >> 20) % 81) - 40;
        const unsigned long long sa = (e >> 40) & 1ull;
        const double x = __longlong_as_double((long long)((sa << 63) | ((unsigned long long)(1023 + ea) << 52) | ma));
        const double y = __longlong_as_double((long long)(((unsigned long long)(1023 + eb) << 52) | mb));
        const double q = div_rn(x, y, __drcp_rn(y));
        const double ref = x / y;
        if (__double_as_longlong(q) != __double_as_longlong(ref)) {
            if (atomicAdd(mismatches, 1ull) == 0) { first[0] = x; first[1] = y; }
        }
    }
}

// Virial stress at particles, main.cpp:2057-2302: four sums (PressureP,
// PressureA, ViscosityV, DiffuseInterface) added in that order.
__global__ void __launch_bounds__(128)
k_virial(SimConst c, const double4* __restrict__ pos, const double4* __restrict__ vel,
         const double4* __restrict__ velp, const double4* __restrict__ gc, const int* __restrict__ ncount,
         const int* __restrict__ nlist, double* __restrict__ virial_p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const double4 pi = pos[i];
    const double4 vi = vel[i];
    const int ti = type_of(pi);
    const double2 pri = make_double2(velp[i].w, gc[i].w);   // {PressureP, PressureA}
    const double4 gci = gc[i];
    const double mui = c.shear_viscosity[ti];
    const int cnt = ncount[i];
    const size_t n = (size_t)c.n;
    double S[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    for (int term = 0; term < 4; ++term) {
        double st[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
        for (int k = 0; k < cnt; ++k) {
            const int j = nlist[(size_t)k * n + i];
            if (j == i) continue;
            const double4 pj = pos[j];
            double x[3];
            disp(c, pi, pj, x);
            const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            double f[3];
            if (term == 0) {
                if (!(c.rp2 - r2 > 0)) continue;
                const double r = sqrt(r2);
                const double dw = f_dwpdr(c, r);
                const double g[3] = {dw * x[0] / r, dw * x[1] / r, dw * x[2] / r};
                for (int d = 0; d < 3; ++d) f[d] = (pri.x) * g[d] * c.vol;
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) st[a][b] += 1.0 * f[a] * x[b] / c.vol;
            } else if (term == 1) {
                if (!(c.ra2 - r2 > 0)) continue;
                const double ratio = c.ratio[ti][type_of(pj)];
                const double r = sqrt(r2);
                const double dw = ratio * f_dwadr(c, r);
                const double g[3] = {dw * x[0] / r, dw * x[1] / r, dw * x[2] / r};
                for (int d = 0; d < 3; ++d) f[d] = (pri.y) * g[d] * c.vol;
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) st[a][b] += 1.0 * f[a] * x[b] / c.vol;
            } else if (term == 2) {
                if (!(c.rv2 - r2 > 0)) continue;
                const double r = sqrt(r2);
                const double dw = -f_dwvdr(c, r);
                const double e[3] = {x[0] / r, x[1] / r, x[2] / r};
                const double4 vj = vel[j];
                const double u[3] = {vj.x - vi.x, vj.y - vi.y, vj.z - vi.z};
                const double muj = c.shear_viscosity[type_of(pj)];
                const double muij = 2.0 * (mui * muj) / (mui + muj);
                for (int d = 0; d < 3; ++d)
                    f[d] = c.visc_c * muij * (u[0] * e[0] + u[1] * e[1] + u[2] * e[2]) * e[d] * dw / r * c.vol;
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) st[a][b] += 0.5 * f[a] * x[b] / c.vol;
            } else {
                if (!(c.rg2 - r2 > 0)) continue;
                const double a_ = c.a_k[ti];
                const double ratio = c.ratio[ti][type_of(pj)];
                const double r = sqrt(r2);
                const double w = ratio * f_wg(c, r);
                const double gv[3] = {gci.x, gci.y, gci.z};
                for (int d = 0; d < 3; ++d) f[d] = -a_ * (-gv[d]) * w / c.r2g * c.rg * c.vol_over_l0;
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) st[a][b] += 1.0 * f[a] * x[b] / c.vol;
                const double dw = ratio * f_dwgdr(c, r);
                const double g[3] = {dw * x[0] / r, dw * x[1] / r, dw * x[2] / r};
                double gr = 0.0;
                for (int d = 0; d < 3; ++d) gr += (-gv[d]) * x[d];
                for (int d = 0; d < 3; ++d) f[d] = -a_ * (gr) * g[d] / c.r2g * c.rg * c.vol_over_l0;
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) st[a][b] += 1.0 * f[a] * x[b] / c.vol;
            }
        }
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) S[a][b] += st[a][b];
    }
    if (c.dim == 2) virial_p[i] = -1.0 / 2.0 * (S[0][0] + S[1][1]);
    else virial_p[i] = -1.0 / 3.0 * (S[0][0] + S[1][1] + S[2][2]);
}

// Fluid mass, momentum, kinetic energy: per-block partial sums in a fixed
// order (deterministic), summed on the host.
__global__ void __launch_bounds__(256)
k_conserved(SimConst c, const int* __restrict__ cellstart, const double4* __restrict__ pos,
            const double4* __restrict__ vel, double* __restrict__ partial) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double s[5] = {0, 0, 0, 0, 0};
    if (i < c.n && i < cellstart[c.tot]) {
        const double m = c.density[type_of(pos[i])] * c.vol;
        const double4 v = vel[i];
        s[0] = m;
        s[1] = m * v.x;
        s[2] = m * v.y;
        s[3] = m * v.z;
        s[4] = 0.5 * m * (v.x * v.x + v.y * v.y + v.z * v.z);
    }
    __shared__ double sh[5][256];
    for (int k = 0; k < 5; ++k) sh[k][threadIdx.x] = s[k];
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o)
            for (int k = 0; k < 5; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 5; ++k) partial[5 * (size_t)blockIdx.x + k] = sh[k][0];
}

inline int blocks(long long n, int t) { return (int)((n + t - 1) / t); }

// Small scenes take the warp-per-particle sweeps: below these sizes the
// thread-per-particle sweeps leave most of the GPU idle.  Set by measurement
// (sweep A + force sweep, one B200): 3-D dam breaks 0.065 ms (warp) against
// 0.125 ms (thread) at 21,924 particles, 0.27 against 0.14 ms at 111,096;
// 2-D droplets with surface tension 0.073 against 0.096 ms at 10,000, 0.52
// against 0.36 ms at 40,000.  The ordered sums run on a few lanes of each
// warp, so at scale the thread kernels win.
#ifndef MPH_WARP_SWEEP_MAX_N
#define MPH_WARP_SWEEP_MAX_N 40000
#endif
#ifndef MPH_WARP_SWEEP_MAX_N_2D
#define MPH_WARP_SWEEP_MAX_N_2D 20000
#endif
inline bool use_warp_sweeps(const SimConst& c) {
    if (c.sweep_layout != 0) return c.sweep_layout == 2;
    return c.n <= (c.dim == 2 ? MPH_WARP_SWEEP_MAX_N_2D : MPH_WARP_SWEEP_MAX_N);
}

// ---- learned form ----------------------------------------------------------

// exclusive prefix of ncount[i], i < nf, within blocks of 1024; block totals to bsum
__global__ void __launch_bounds__(1024) k_edge_scan1(const int* __restrict__ ncount, int nf, int* __restrict__ eoff,
                                                     int* __restrict__ bsum) {
    __shared__ int wsum[32];
    const int i = blockIdx.x * 1024 + threadIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int v = i < nf ? ncount[i] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = wsum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        wsum[lane] = t;
    }
    __syncthreads();
    const int before = (w > 0 ? wsum[w - 1] : 0) + x - v;
    if (i < nf) eoff[i] = before;
    if (threadIdx.x == 1023) bsum[blockIdx.x] = before + v;
}

// exclusive prefix of the block totals (one block, chunks of 1024 with a carry)
__global__ void __launch_bounds__(1024) k_edge_scan2(int* __restrict__ bsum, int nb) {
    __shared__ int wsum[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < nb; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < nb ? bsum[i] : 0;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            int t = wsum[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            wsum[lane] = t;
        }
        __syncthreads();
        const int before = carry + (w > 0 ? wsum[w - 1] : 0) + x - v;
        if (i < nb) bsum[i] = before;
        __syncthreads();
        if (threadIdx.x == 1023) carry = before + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) bsum[nb] = carry;
}

__global__ void __launch_bounds__(1024) k_edge_scan3(int* __restrict__ eoff, const int* __restrict__ bsum, int nf,
                                                     int nb) {
    const int i = blockIdx.x * 1024 + threadIdx.x;
    if (i < nf) eoff[i] += bsum[blockIdx.x];
    if (i == 0) eoff[nf] = bsum[nb];
}

__global__ void __launch_bounds__(128) k_edge_fill(const int* __restrict__ ncount, const int* __restrict__ nlist,
                                                   int n, int nf, const int* __restrict__ eoff, int* __restrict__ ei,
                                                   int* __restrict__ ej) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
    const int b = eoff[i], cnt = ncount[i];
    for (int k = 0; k < cnt; ++k) {
        ei[b + k] = i;
        ej[b + k] = nlist[(size_t)k * n + i];
    }
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// One training sample per thread: a random CSR edge (i, j), its inputs and
// the FP64 PressureA + DiffuseInterface + ViscosityV force of j on i, with the
// expressions of k_sweep_b (main.cpp:1742-1828, 1941-1985).
template <bool ST, bool RATIO>
__global__ void __launch_bounds__(128)
k_collect(SimConst c, const double4* __restrict__ pos, const double4* __restrict__ velp,
          const double4* __restrict__ gcpa, const int* __restrict__ ei, const int* __restrict__ ej, long long ne,
          long long count, unsigned long long seed, float4* __restrict__ out) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    const long long g = (long long)(mix64(seed ^ mix64((unsigned long long)q)) % (unsigned long long)ne);
    const int i = ei[g], j = ej[g];
    const double4 pi = pos[i], pj = pos[j];
    double x[3];
    disp(c, pi, pj, x);
    const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
    const bool in_a = ST && (c.ra2 - r2 > 0);
    const bool in_g = ST && (c.rg2 - r2 > 0);
    const bool in_v = c.rv2 - r2 > 0;
    const int ti = type_of(pi), tj = type_of(pj);
    const double4 vi = velp[i], vj = velp[j];
    double f0 = 0.0, f1 = 0.0, f2 = 0.0;
    const bool valid = i != j && (in_a || in_g || in_v);
    const double r = sqrt(r2);
    if (valid) {
        const double ri = __drcp_rn(r);
        const double e0 = div_rn(x[0], r, ri), e1 = div_rn(x[1], r, ri), e2 = div_rn(x[2], r, ri);
        const double qa = div_rn(r, c.ra, c.inv_ra);
        double rij = 1.0, rji = 1.0;
        if (RATIO) { rij = c.ratio[ti][tj]; rji = c.ratio[tj][ti]; }
        if (in_a) {
            const double dwa = s_dwa(c, qa);
            const double s = gcpa[i].w * (RATIO ? rij * dwa : dwa) + gcpa[j].w * (RATIO ? rji * dwa : dwa);
            f0 += s * e0 * c.vol;
            f1 += s * e1 * c.vol;
            f2 += s * e2 * c.vol;
        }
        if (ST && in_g) {
            const double4 gci = gcpa[i], gcj = gcpa[j];
            const double ai = c.a_k[ti], aj = ai;
            const double qg = c.rg_eq_ra ? qa : div_rn(r, c.rg, c.inv_rg);
            const double wg = s_wg(c, qg);
            const double wij = RATIO ? rij * wg : wg, wji = RATIO ? rji * wg : wg;
            f0 -= div_rn(aj * gcj.x * wji - ai * gci.x * wij, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
            f1 -= div_rn(aj * gcj.y * wji - ai * gci.y * wij, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
            f2 -= div_rn(aj * gcj.z * wji - ai * gci.z * wij, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
            const double dg = s_dwg(c, qg);
            const double dwij = RATIO ? rij * dg : dg, dwji = RATIO ? rji * dg : dg;
            double gr = 0.0;
            gr += (aj * gcj.x * dwji - ai * gci.x * dwij) * x[0];
            gr += (aj * gcj.y * dwji - ai * gci.y * dwij) * x[1];
            gr += (aj * gcj.z * dwji - ai * gci.z * dwij) * x[2];
            f0 -= div_rn(gr * e0, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
            f1 -= div_rn(gr * e1, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
            f2 -= div_rn(gr * e2, c.r2g, c.inv_r2g) * c.rg * c.vol_over_l0;
        }
        if (in_v) {
            const double qv = c.rv_eq_ra ? qa : div_rn(r, c.rv, c.inv_rv);
            const double dw = -s_dwv(c, qv);
            const double u0 = vj.x - vi.x, u1 = vj.y - vi.y, u2 = vj.z - vi.z;
            const double dot = u0 * e0 + u1 * e1 + u2 * e2;
            const double cm = c.visc_mu[ti][tj];
            f0 += div_rn(cm * dot * e0 * dw, r, ri) * c.vol;
            f1 += div_rn(cm * dot * e1 * dw, r, ri) * c.vol;
            f2 += div_rn(cm * dot * e2 * dw, r, ri) * c.vol;
        }
    }
    const double il0 = 1.0 / c.l0;
    out[3 * q + 0] = make_float4((float)(x[0] * il0), (float)(x[1] * il0), (float)(x[2] * il0), (float)(r * il0));
    out[3 * q + 1] = make_float4((float)(vj.x - vi.x), (float)(vj.y - vi.y), (float)(vj.z - vi.z),
                                 (float)(ti + 4 * tj));
    out[3 * q + 2] = make_float4((float)f0, (float)f1, (float)f2, valid ? 1.f : 0.f);
}

__global__ void __launch_bounds__(256)
k_force_compare(int nf, const double4* __restrict__ fa, const double4* __restrict__ fb,
                const float4* __restrict__ lsum, double* __restrict__ sums) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    if (i < nf) {
        const double4 a = fa[i], b = fb[i];
        const float4 l = lsum[i];
        const double d0 = a.x - b.x, d1 = a.y - b.y, d2 = a.z - b.z;
        s0 = d0 * d0 + d1 * d1 + d2 * d2;
        s1 = b.x * b.x + b.y * b.y + b.z * b.z;
        const double v0 = (double)l.x - d0, v1 = (double)l.y - d1, v2 = (double)l.z - d2;
        s2 = v0 * v0 + v1 * v1 + v2 * v2;
    }
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&sums[0], s0);
        atomicAdd(&sums[1], s1);
        atomicAdd(&sums[2], s2);
    }
}

}  // namespace

void launch_move(const SimConst& c, const int* cellstart, double4* pos, double4* vel, const double4* snap,
                 const double* wall_center, StepScalars* scal, cudaStream_t s) {
    k_move<false><<<blocks(c.n, 256), 256, 0, s>>>(c, cellstart, pos, vel, snap, wall_center, scal, 0, 0);
}

void launch_move_graph(const SimConst& c, const int* cellstart, double4* pos, double4* vel, const double4* snap,
                       const double* wall_center, StepScalars* scal, cudaGraphConditionalHandle rebuild,
                       cudaGraphConditionalHandle sweep, cudaStream_t s) {
    k_move<true><<<blocks(c.n, 256), 256, 0, s>>>(c, cellstart, pos, vel, snap, wall_center, scal, rebuild,
                                                  sweep);
}

void launch_sweep_a(const SimConst& c, const int* cellstart, const double4* pos, const double4* vel,
                    const int* ncount, const int* nlist, const int* ncount_s, const int* nlist_s, double* dens_a,
                    double* strain_p, double* div_p, double4* press, double4* gc, double* wall_center,
                    cudaStream_t s) {
    (void)cellstart;
    const bool warp = use_warp_sweeps(c);
    const int nb = warp ? blocks(c.n, kWarpSweepWarps) : (blocks(c.n, 128) > 0 ? blocks(c.n, 128) : 1);
    // with surface tension the list (DensityA, GravityCenter) and, when there
    // is one, the short sublist (DensityP, DivergenceP); without, the short
    // sublist alone
    const bool split = c.has_st && nlist_s != nullptr;
#define SWEEP_A(ST, RATIO, SPLIT, CNT, LIST)                                                                      \
    if (warp)                                                                                                     \
        k_sweep_a_w<ST, RATIO, ST><<<nb, 32 * kWarpSweepWarps, 0, s>>>(c, pos, vel, CNT, LIST, dens_a, strain_p,  \
                                                                       div_p, press, gc, wall_center);            \
    else                                                                                                          \
        k_sweep_a<ST, RATIO, ST, SPLIT><<<nb, 128, 0, s>>>(c, pos, vel, CNT, LIST, ncount_s, nlist_s, dens_a,     \
                                                           strain_p, div_p, press, gc, wall_center)
    if (c.has_st) {
        if (split) {
            if (c.ratio_all_one) SWEEP_A(true, false, true, ncount, nlist); else SWEEP_A(true, true, true, ncount, nlist);
        } else {
            if (c.ratio_all_one) SWEEP_A(true, false, false, ncount, nlist); else SWEEP_A(true, true, false, ncount, nlist);
        }
    } else {
        if (c.ratio_all_one) SWEEP_A(false, false, false, ncount_s, nlist_s);
        else SWEEP_A(false, true, false, ncount_s, nlist_s);
    }
#undef SWEEP_A
}

void launch_density_a(const SimConst& c, const double4* pos, const int* ncount, const int* nlist, double* dens_a,
                      double4* gc, cudaStream_t s) {
    const int nb = blocks(c.n, 128) > 0 ? blocks(c.n, 128) : 1;
    if (c.ratio_all_one)
        k_density_a<false><<<nb, 128, 0, s>>>(c, pos, ncount, nlist, dens_a, gc);
    else
        k_density_a<true><<<nb, 128, 0, s>>>(c, pos, ncount, nlist, dens_a, gc);
}

void launch_sweep_b(const SimConst& c, const int* cellstart, const double4* pos, const double4* vel_in,
                    double4* vel_out, const double4* press, const double4* gc, const int* ncount,
                    const int* nlist, const int* ncount_s, const int* nlist_s, double4* force, StepScalars* scal,
                    cudaStream_t s, const int* eoff, const float4* eforce, float4* lsum, int part, int i0,
                    int i1, double* vel_host) {
    (void)vel_in;
    if (i1 < 0) i1 = c.n;
    if (i1 <= i0) return;
    if (!eforce && i0 == 0 && i1 == c.n && use_warp_sweeps(c)) {
        const int nw = blocks(c.n, kWarpSweepWarps);
#define SWEEP_BW(ST, RATIO)                                                                                       \
    k_sweep_b_w<ST, RATIO><<<nw, 32 * kWarpSweepWarps, 0, s>>>(c, cellstart, pos, press, vel_out, gc, ncount,    \
                                                              nlist, force, scal, part, vel_host)
        if (c.has_st) {
            if (c.ratio_all_one) SWEEP_BW(true, false); else SWEEP_BW(true, true);
        } else {
            if (c.ratio_all_one) SWEEP_BW(false, false); else SWEEP_BW(false, true);
        }
#undef SWEEP_BW
        return;
    }
    const int nb = blocks(i1 - i0, 128);
#define SWEEP_B(ST, RATIO, LRN, SPLIT) \
    k_sweep_b<ST, RATIO, LRN, SPLIT><<<nb, 128, 0, s>>>(c, cellstart, pos, press, vel_out, gc, ncount, nlist,        \
                                                        ncount_s, nlist_s, force, scal, eoff, eforce, lsum, part, \
                                                        i0, i1, vel_host)
#define SWEEP_B2(ST, RATIO)                                             \
    if (eforce) SWEEP_B(ST, RATIO, true, false);                        \
    else if (nlist_s) SWEEP_B(ST, RATIO, false, true);                  \
    else SWEEP_B(ST, RATIO, false, false)
    if (c.has_st) {
        if (c.ratio_all_one) { SWEEP_B2(true, false); } else { SWEEP_B2(true, true); }
    } else {
        if (c.ratio_all_one) { SWEEP_B2(false, false); } else { SWEEP_B2(false, true); }
    }
#undef SWEEP_B2
#undef SWEEP_B
}

void launch_virial(const SimConst& c, const double4* pos, const double4* vel, const double4* press,
                   const double4* gc, const int* ncount, const int* nlist, double* virial_p, cudaStream_t s) {
    k_virial<<<blocks(c.n, 128), 128, 0, s>>>(c, pos, vel, press, gc, ncount, nlist, virial_p);
}

int check_division(unsigned long long seed, long long n, unsigned long long* d_count, double* d_first,
                   cudaStream_t s) {
    k_check_division<<<148 * 8, 256, 0, s>>>(seed, n, d_count, d_first);
    return 1;
}

void launch_conserved(const SimConst& c, const int* cellstart, const double4* pos, const double4* vel,
                      double* partial, cudaStream_t s) {
    k_conserved<<<blocks(c.n, 256), 256, 0, s>>>(c, cellstart, pos, vel, partial);
}

int edge_scan_blocks(int nf) { return (nf + 1023) / 1024 + 1; }

void launch_edge_offsets(const int* ncount, int nf, int* eoff, int* bsum, cudaStream_t s) {
    const int nb = (nf + 1023) / 1024;
    if (nb == 0) {
        cudaMemsetAsync(eoff, 0, sizeof(int), s);
        return;
    }
    k_edge_scan1<<<nb, 1024, 0, s>>>(ncount, nf, eoff, bsum);
    k_edge_scan2<<<1, 1024, 0, s>>>(bsum, nb);
    k_edge_scan3<<<nb, 1024, 0, s>>>(eoff, bsum, nf, nb);
}

void launch_edge_fill(const int* ncount, const int* nlist, int n, int nf, const int* eoff, int* ei, int* ej,
                      cudaStream_t s) {
    if (nf > 0) k_edge_fill<<<blocks(nf, 128), 128, 0, s>>>(ncount, nlist, n, nf, eoff, ei, ej);
}

void launch_collect(const SimConst& c, const double4* pos, const double4* press, const double4* gc, const int* ei,
                    const int* ej, long long ne, long long count, unsigned long long seed, float4* out,
                    cudaStream_t s) {
    if (count <= 0 || ne <= 0) return;
    const unsigned nb = (unsigned)((count + 127) / 128);
#define COLLECT(ST, RATIO) k_collect<ST, RATIO><<<nb, 128, 0, s>>>(c, pos, press, gc, ei, ej, ne, count, seed, out)
    if (c.has_st) {
        if (c.ratio_all_one) COLLECT(true, false); else COLLECT(true, true);
    } else {
        if (c.ratio_all_one) COLLECT(false, false); else COLLECT(false, true);
    }
#undef COLLECT
}

void launch_force_compare(int nf, const double4* fa, const double4* fb, const float4* lsum, double* sums3,
                          cudaStream_t s) {
    if (nf > 0) k_force_compare<<<blocks(nf, 256), 256, 0, s>>>(nf, fa, fb, lsum, sums3);
}

}  // namespace mph
