// mph_pair32.cuh — FP32 pair terms shared by the mixed-precision sweeps
// (k_mixed.cu) and the batched sweeps (k_batch.cu).
//
// K is any constants struct with the FP32 fields used below (ratio, ra2,
// inv_ra, ca, ca_inv, rg2, inv_rg, cg, cg_m2, inv_r2g_rg, vol, vol_over_l0),
// all evaluated on the host from the FP64 set-up constants.
#pragma once
#include <cuda_runtime.h>

namespace mph {

// Kahan-compensated accumulation (Kahan 1965): s + t with the lost low-order
// part carried in c; the compensated value is s - c.
__device__ __forceinline__ void kahan_add(float& s, float& c, float t) {
    const float y = t - c;
    const float u = s + y;
    c = (u - s) - y;
    s = u;
}

// 1/sqrt(r2) with one Newton step (rsqrtf is within 2 ulp; the step brings it
// to about 1 ulp), for the pressure terms.
__device__ __forceinline__ float rsqrt_nr(float r2) {
    const float y = rsqrtf(r2);
    return y * fmaf(-0.5f * r2 * y, y, 1.5f);
}

// 1/sqrt(r2) in FP64 from an FP32 seed plus one Newton step (relative error
// ~1e-14), for the FP64 density pairs.
__device__ __forceinline__ double rsqrt_dnr(double r2) {
    const double y = (double)rsqrtf((float)r2);
    return y * (1.5 - 0.5 * r2 * y * y);
}

// Surface-tension sums of the density sweep for one pair: DensityA
// (main.cpp:1665-1692) and GravityCenter (main.cpp:1695-1727).
template <bool RATIO, class K>
__device__ __forceinline__ void st_density(const K& m, int ti, int tj, float r2, float r, float dx, float dy,
                                           float dz, float& sa, float& cak, float& g0, float& g1, float& g2) {
    const float ratio = RATIO ? m.ratio[ti][tj] : 1.0f;
    if (r2 <= m.ra2) {
        const float q = r * m.inv_ra;
        kahan_add(sa, cak, ratio * m.ca * q * (1.0f - q) * (1.0f - q));
    }
    if (r2 <= m.rg2) {
        const float q = 1.0f - r * m.inv_rg;
        const float wgt = ratio * m.cg * q * q * m.inv_r2g_rg;
        g0 += dx * wgt;
        g1 += dy * wgt;
        g2 += dz * wgt;
    }
}

// Surface-tension terms of one pair (PressureA, DiffuseInterface with aj the
// a of i as the reference has it, main.cpp:1742-1828); returns the radial
// part and adds the tangential part to t.
template <bool RATIO, class K>
__device__ __forceinline__ float st_terms(const K& m, int ti, int tj, float r2, float r, float rinv, float dx,
                                          float dy, float dz, const float4& gi, const float4& gj, float ai,
                                          float3& t) {
    const float rij = RATIO ? m.ratio[ti][tj] : 1.0f, rji = RATIO ? m.ratio[tj][ti] : 1.0f;
    float s = 0.0f;
    if (r2 < m.ra2) {
        const float q = r * m.inv_ra;
        const float dwa = m.ca_inv * (1.0f - q) * (1.0f - 3.0f * q);
        s += (gi.w * rij * dwa + gj.w * rji * dwa) * rinv * m.vol;
    }
    if (r2 < m.rg2) {
        const float q = 1.0f - r * m.inv_rg;
        const float wg = m.cg * q * q, dwg = m.cg_m2 * q;
        const float k1 = m.inv_r2g_rg * m.vol_over_l0;
        t.x -= (ai * gj.x * rji * wg - ai * gi.x * rij * wg) * k1;
        t.y -= (ai * gj.y * rji * wg - ai * gi.y * rij * wg) * k1;
        t.z -= (ai * gj.z * rji * wg - ai * gi.z * rij * wg) * k1;
        const float gr = (ai * gj.x * rji * dwg - ai * gi.x * rij * dwg) * dx +
                         (ai * gj.y * rji * dwg - ai * gi.y * rij * dwg) * dy +
                         (ai * gj.z * rji * dwg - ai * gi.z * rij * dwg) * dz;
        s -= gr * rinv * k1;
    }
    return s;
}

}  // namespace mph
