// Edge-MLP surrogate kernels on the 5th-generation tensor cores (tcgen05):
// training (forward + backward with the weight gradients accumulated in
// tensor memory), deterministic gradient reduction, Adam, and inference.
//
// One CTA of 128 threads processes tiles of 128 edges; thread e owns edge
// (row) e of the tile and TMEM lane e.  Thread 0 issues every MMA
// (M = 128, BF16 x BF16 -> FP32) and commits them to an mbarrier; the
// epilogues (bias, SiLU, its derivative, BF16 packing) run on all threads
// between the MMA groups.  Operands live in shared memory in the no-swizzle
// core-matrix layout (mph_tc.cuh), activations stay on chip for the whole
// forward/backward pass of a tile.
//
// Matrix shapes per tile (E = 128 edges, X = inputs, Z/H = pre/post SiLU):
//   forward   Z1 = X W1^T + b1, Z2 = H1 W2^T + b2, Z3 = H2 W3^T + b3,
//             Y = H3 W4^T + b4;   dY = Y - T (valid rows)
//   backward  dW4^T += H3^T dY,   dH3 = dY W4,  dZ3 = dH3 * silu'(Z3)
//             dW3 += dZ3^T H2,  db3 += dZ3^T 1,  dH2 = dZ3 W3, ...
//             dW1 += dZ1^T X,   db1 += dZ1^T 1
// The gradient accumulators (dW1..dW4, db1..db3) stay in TMEM across all the
// tiles of a CTA and are written once per CTA; a second kernel sums the CTA
// partials in a fixed order, so a training step is deterministic.
#include <cuda_bf16.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>
#include "mph_mlp.h"
#include "mph_tc.cuh"

namespace mph {
namespace mlp {
namespace {

using tc::core_off;

constexpr long long kWaitLimit = 1ll << 22;  // mbarrier polls before a wait is abandoned (~1 s)

// Wait control of the MLP kernels: the poll limit of every mbarrier wait, and
// whether the MMA groups are issued (always, except in the wait self-test of
// model_check_wait, where withholding them makes the first wait run out with
// nothing in flight).
struct WaitCtl {
    long long limit;
    int issue;
};

// shared memory of the training kernel (bytes)
constexpr int S_W = 0;  // packed image: W1, W2, W3, W4 (core layout), b1..b4 (FP32)
constexpr int S_X = 75776;
constexpr int S_DY = S_X + TILE * KIN * 2;
constexpr int S_ONE = S_DY + TILE * KOUT * 2;
constexpr int S_H = S_ONE + KOUT * TILE * 2;
constexpr int S_Z1 = S_H + TILE * H * 2;
constexpr int S_Z2 = S_Z1 + TILE * H * 2;
constexpr int S_Z3 = S_Z2 + TILE * H * 2;
constexpr int S_MISC = S_Z3 + TILE * H * 2;
constexpr int S_TRAIN = S_MISC + 256;
static_assert(PK_BYTES <= S_X, "image overlaps the input tile");
static_assert(S_TRAIN <= 227 * 1024, "training kernel exceeds the shared memory of a CTA");

// shared memory of the inference kernel: the weight image once, then for
// each warpgroup (one 128-edge tile in flight each) its input tile X and its
// hidden activations H
constexpr int I_WG = 4;                                      // tiles in flight per CTA
constexpr int I_TILE_BYTES = TILE * KIN * 2 + TILE * H * 2;  // X + H of one tile
constexpr int I_T = S_X;
constexpr int I_MISC = I_T + I_WG * I_TILE_BYTES;
constexpr int S_INFER = I_MISC + 64;
static_assert(S_INFER <= 227 * 1024, "the inference CTA exceeds the shared memory of a CTA");
static_assert(I_T % 128 == 0 && I_TILE_BYTES % 128 == 0, "operand tiles must stay 128-byte aligned");

// TMEM columns
constexpr uint32_t T_D = 0;      // layer output / backward dH  [128 x 128]
constexpr uint32_t T_G2 = 128;   // dW2 [o][k]
constexpr uint32_t T_G3 = 256;   // dW3
constexpr uint32_t T_G1 = 384;   // dW1 [o][k < 16]
constexpr uint32_t T_G4T = 400;  // dW4^T [k][o < 16]
constexpr uint32_t T_GB1 = 416;  // db1 (column 0 of the block)
constexpr uint32_t T_GB2 = 432;
constexpr uint32_t T_GB3 = 448;
constexpr uint32_t T_D4 = 464;   // layer-4 output [128 x 16]

constexpr uint32_t ID_F128 = tc::idesc_bf16(128, 128, false, false);
constexpr uint32_t ID_F16 = tc::idesc_bf16(128, 16, false, false);
constexpr uint32_t ID_G4T = tc::idesc_bf16(128, 16, true, true);
constexpr uint32_t ID_DH = tc::idesc_bf16(128, 128, false, true);
constexpr uint32_t ID_GW = tc::idesc_bf16(128, 128, true, true);
constexpr uint32_t ID_GB = tc::idesc_bf16(128, 16, true, false);
constexpr uint32_t ID_G1 = tc::idesc_bf16(128, 16, true, true);

// sigmoid(z) = (1 + tanh(z / 2)) / 2 with the hardware tanh approximation
// (relative error ~2^-11, below the BF16 rounding of every activation)
__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sigmoid(float z) { return fmaf(0.5f, tanh_approx(0.5f * z), 0.5f); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = sigmoid(z);
    return s * fmaf(z, 1.0f - s, 1.0f);
}
__device__ __forceinline__ uint32_t pack2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ float lo_bf(uint32_t p) { return __uint_as_float(p << 16); }

// SiLU in packed BF16 from the half pre-activation hz = z/2:
//   h = z * sigmoid(z) = z * (1 + tanh(z/2)) / 2 = hz + hz * tanh(hz),
// one special-function operation (the packed tanh) and one FMA per two
// activations; the forward passes of training and inference both use it.
__device__ __forceinline__ uint32_t silu_half2(uint32_t hz2) {
    uint32_t t, h;
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(hz2));
    asm("fma.rn.bf16x2 %0, %1, %2, %1;" : "=r"(h) : "r"(hz2), "r"(t));
    return h;
}
// The same from z (z/2 is exact in BF16).
__device__ __forceinline__ uint32_t silu2(uint32_t z2) {
    uint32_t hz;
    asm("mul.rn.bf16x2 %0, %1, %2;" : "=r"(hz) : "r"(z2), "r"(0x3F003F00u));
    return silu_half2(hz);
}
// Two FP32 values to BF16, rounded to nearest (ties away from zero: the
// conversion instruction rounds ties to even; they differ only on exact ties),
// with one integer add each and one byte permute: the conversion instruction
// shares its pipe with the packed tanh, which bounds the hidden-layer epilogues.
__device__ __forceinline__ uint32_t pack2_near(float a, float b) {
    return __byte_perm(__float_as_uint(a) + 0x8000u, __float_as_uint(b) + 0x8000u, 0x7632);
}
__device__ __forceinline__ float hi_bf(uint32_t p) { return __uint_as_float(p & 0xFFFF0000u); }

// 16 consecutive bf16 of row r, columns c0..c0+15 of a core-layout tile with C columns
__device__ __forceinline__ void st_row16(uint8_t* base, int r, int c0, int C, const uint32_t* p) {
    *reinterpret_cast<uint4*>(base + core_off(r, c0, C)) = make_uint4(p[0], p[1], p[2], p[3]);
    *reinterpret_cast<uint4*>(base + core_off(r, c0 + 8, C)) = make_uint4(p[4], p[5], p[6], p[7]);
}
__device__ __forceinline__ void ld_row16(const uint8_t* base, int r, int c0, int C, uint32_t* p) {
    const uint4 a = *reinterpret_cast<const uint4*>(base + core_off(r, c0, C));
    const uint4 b = *reinterpret_cast<const uint4*>(base + core_off(r, c0 + 8, C));
    p[0] = a.x; p[1] = a.y; p[2] = a.z; p[3] = a.w;
    p[4] = b.x; p[5] = b.y; p[6] = b.z; p[7] = b.w;
}

// the nine inputs of one sample, scaled; false when the row is padding
__device__ __forceinline__ bool sample_features(const float4* __restrict__ samples, long long s, const Scales& sc,
                                                float* f, float* t) {
    const float4 a = samples[3 * s], b = samples[3 * s + 1], c = samples[3 * s + 2];
    const int tt = (int)b.w;
    f[0] = a.x; f[1] = a.y; f[2] = a.z;
    f[3] = b.x * sc.inv_u; f[4] = b.y * sc.inv_u; f[5] = b.z * sc.inv_u;
    f[6] = a.w; f[7] = (float)(tt & 3); f[8] = (float)(tt >> 2);
    t[0] = c.x * sc.inv_f; t[1] = c.y * sc.inv_f; t[2] = c.z * sc.inv_f;
    return c.w != 0.0f;
}

__device__ __forceinline__ void store_x(uint8_t* sx, int e, const float* f) {
    uint32_t p[8];
    p[0] = pack2(f[0], f[1]); p[1] = pack2(f[2], f[3]); p[2] = pack2(f[4], f[5]); p[3] = pack2(f[6], f[7]);
    p[4] = pack2(f[8], 0.f); p[5] = 0u; p[6] = 0u; p[7] = 0u;
    st_row16(sx, e, 0, KIN, p);
}

// forward epilogue of a hidden layer, columns [16 c0, 16 c1) of row e:
// hz = (D + b) / 2 = D / 2 + bias_half (one FMA, exact scaling), rounded to BF16;
// H = silu(Z) -> hbuf and, for training, Z = 2 hz (exact) -> zbuf
__device__ __forceinline__ void epi_hidden(uint32_t trow, const float* bias_half, uint8_t* zbuf, uint8_t* hbuf,
                                           int e, int c0 = 0, int c1 = H / 16) {
#pragma unroll 1
    for (int c = c0; c < c1; ++c) {
        float v[16];
        tc::tmem_ld16(trow + T_D + 16 * c, v);
        uint32_t zp[8], hp[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint32_t hz = pack2_near(fmaf(v[2 * j], 0.5f, bias_half[16 * c + 2 * j]),
                                           fmaf(v[2 * j + 1], 0.5f, bias_half[16 * c + 2 * j + 1]));
            hp[j] = silu_half2(hz);
            if (zbuf) asm("add.rn.bf16x2 %0, %1, %1;" : "=r"(zp[j]) : "r"(hz));
        }
        if (zbuf) st_row16(zbuf, e, 16 * c, H, zp);
        st_row16(hbuf, e, 16 * c, H, hp);
    }
}

// The hidden layers' biases halved in place in a CTA's copy of the weight
// image (epi_hidden takes b/2); call between two CTA-wide barriers.
__device__ __forceinline__ void halve_hidden_biases(float* b1) {
    for (int k = threadIdx.x; k < 3 * H; k += blockDim.x) b1[k] *= 0.5f;
}

// backward epilogue: dZ = dH * silu'(Z) in place of Z; optionally H_prev = silu(Z_prev)
__device__ __forceinline__ void epi_back(uint32_t trow, uint8_t* zbuf, const uint8_t* zprev, uint8_t* hbuf, int e) {
#pragma unroll 1
    for (int c = 0; c < H / 16; ++c) {
        float v[16];
        tc::tmem_ld16(trow + T_D + 16 * c, v);
        uint32_t zp[8], dp[8];
        ld_row16(zbuf, e, 16 * c, H, zp);
#pragma unroll
        for (int j = 0; j < 8; ++j)
            dp[j] = pack2(v[2 * j] * dsilu(lo_bf(zp[j])), v[2 * j + 1] * dsilu(hi_bf(zp[j])));
        st_row16(zbuf, e, 16 * c, H, dp);
        if (zprev) {
            uint32_t qp[8], hp[8];
            ld_row16(zprev, e, 16 * c, H, qp);
#pragma unroll
            for (int j = 0; j < 8; ++j) hp[j] = silu2(qp[j]);
            st_row16(hbuf, e, 16 * c, H, hp);
        }
    }
}

__device__ __forceinline__ float warp_sum(float x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Training pass over `n` samples (rows order[g], or g when order is null).
// Writes this CTA's partial gradient (unscaled: dY = Y - T) and loss.
__global__ void __launch_bounds__(128, 1)
k_mlp_train(const uint8_t* __restrict__ image, const float4* __restrict__ samples,
            const long long* __restrict__ order, long long n, Scales sc, float* __restrict__ gpart,
            double* __restrict__ lossp, int* __restrict__ err, WaitCtl wc) {
    extern __shared__ __align__(128) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    {
        const uint4* src = reinterpret_cast<const uint4*>(image);
        uint4* dst = reinterpret_cast<uint4*>(sm + S_W);
        for (int k = tid; k < PK_BYTES / 16; k += 128) dst[k] = src[k];
        uint4* o = reinterpret_cast<uint4*>(sm + S_ONE);
        const uint32_t one2 = 0x3F803F80u;  // two bf16 ones
        for (int k = tid; k < KOUT * TILE * 2 / 16; k += 128) o[k] = make_uint4(one2, one2, one2, one2);
    }
    __syncthreads();  // the image is in shared memory
    halve_hidden_biases(reinterpret_cast<float*>(sm + S_W + PK_B));  // ordered by the barrier below
    const float* b1 = reinterpret_cast<const float*>(sm + S_W + PK_B);
    const float* b2 = b1 + H;
    const float* b3 = b2 + H;
    const float* b4 = b3 + H;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + S_MISC);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + S_MISC + 8);
    float* wpart = reinterpret_cast<float*>(sm + S_MISC + 16);  // [4 warps][4]
    const uint32_t mb = tc::smem_addr(mbar);
    if (tid == 0) tc::mbar_init(mb, 1);
    if (warp == 0) tc::tmem_alloc(tc::smem_addr(tslot), 512);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tb = *tslot;
    const uint32_t trow = tb + ((uint32_t)(warp * 32) << 16);

    const uint32_t aW1 = tc::smem_addr(sm + S_W + PK_W1), aW2 = tc::smem_addr(sm + S_W + PK_W2);
    const uint32_t aW3 = tc::smem_addr(sm + S_W + PK_W3), aW4 = tc::smem_addr(sm + S_W + PK_W4);
    const uint32_t aX = tc::smem_addr(sm + S_X), aDY = tc::smem_addr(sm + S_DY), aONE = tc::smem_addr(sm + S_ONE);
    const uint32_t aH = tc::smem_addr(sm + S_H), aZ1 = tc::smem_addr(sm + S_Z1);
    const uint32_t aZ2 = tc::smem_addr(sm + S_Z2), aZ3 = tc::smem_addr(sm + S_Z3);

    uint32_t phase = 0;
    bool ok = true;
    bool inflight = false;        // a committed MMA group whose completion was not seen
    uint32_t failed_parity = 0;
    auto run = [&](auto&& issue) {
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            if (wc.issue) {
                issue();
                tc::commit(mb);
            }
        }
        const bool done = tc::mbar_wait(mb, phase, wc.limit);
        tc::fence_after_sync();
        ok = __syncthreads_and(done) != 0;
        if (!ok) {
            inflight = wc.issue != 0;
            failed_parity = phase;
        }
        phase ^= 1u;
    };

    double acc_loss = 0.0;
    float acc_b4[3] = {0.f, 0.f, 0.f};
    const long long ntiles = (n + TILE - 1) / TILE;
    bool first = true;
    for (long long t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        // ---- inputs and targets of the tile
        const long long g = t * TILE + tid;
        float f[NIN] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, tg[3] = {0.f, 0.f, 0.f};
        bool valid = false;
        if (g < n) valid = sample_features(samples, order ? order[g] : g, sc, f, tg);
        if (!valid) {
#pragma unroll
            for (int k = 0; k < NIN; ++k) f[k] = 0.f;
        }
        store_x(sm + S_X, tid, f);
        // ---- forward
        run([&] { tc::mma_bf16(tb + T_D, tc::desc_k(aX, KIN), tc::desc_k(aW1, KIN), ID_F128, 0u); });
        if (!ok) break;
        epi_hidden(trow, b1, sm + S_Z1, sm + S_H, tid);
        run([&] {
            for (int s = 0; s < H / 16; ++s)
                tc::mma_bf16(tb + T_D, tc::desc_k(aH + 256 * s, H), tc::desc_k(aW2 + 256 * s, H), ID_F128, s > 0);
        });
        if (!ok) break;
        epi_hidden(trow, b2, sm + S_Z2, sm + S_H, tid);
        run([&] {
            for (int s = 0; s < H / 16; ++s)
                tc::mma_bf16(tb + T_D, tc::desc_k(aH + 256 * s, H), tc::desc_k(aW3 + 256 * s, H), ID_F128, s > 0);
        });
        if (!ok) break;
        epi_hidden(trow, b3, sm + S_Z3, sm + S_H, tid);
        run([&] {
            for (int s = 0; s < H / 16; ++s)
                tc::mma_bf16(tb + T_D4, tc::desc_k(aH + 256 * s, H), tc::desc_k(aW4 + 256 * s, H), ID_F16, s > 0);
        });
        if (!ok) break;
        {
            float v[16];
            tc::tmem_ld16(trow + T_D4, v);
            float dy[3], l = 0.f;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float d = (v[k] + b4[k]) - tg[k];
                dy[k] = valid ? d : 0.f;
                l += dy[k] * dy[k];
            }
            uint32_t p[8] = {pack2(dy[0], dy[1]), pack2(dy[2], 0.f), 0u, 0u, 0u, 0u, 0u, 0u};
            st_row16(sm + S_DY, tid, 0, KOUT, p);
            const float s0 = warp_sum(l), s1 = warp_sum(dy[0]), s2 = warp_sum(dy[1]), s3 = warp_sum(dy[2]);
            if (lane == 0) {
                wpart[4 * warp + 0] = s0;
                wpart[4 * warp + 1] = s1;
                wpart[4 * warp + 2] = s2;
                wpart[4 * warp + 3] = s3;
            }
        }
        // ---- backward, layer 4: dW4^T += H3^T dY ; dH3 = dY W4
        const uint32_t acc = first ? 0u : 1u;
        run([&] {
            for (int s = 0; s < TILE / 16; ++s)
                tc::mma_bf16(tb + T_G4T, tc::desc_mn(aH + 4096 * s, H), tc::desc_mn(aDY + 512 * s, KOUT), ID_G4T,
                             acc | (s > 0));
            tc::mma_bf16(tb + T_D, tc::desc_k(aDY, KOUT), tc::desc_mn(aW4, H), ID_DH, 0u);
        });
        if (!ok) break;
        if (tid == 0) {
            for (int w = 0; w < 4; ++w) {
                acc_loss += (double)wpart[4 * w];
                for (int k = 0; k < 3; ++k) acc_b4[k] += wpart[4 * w + 1 + k];
            }
        }
        epi_back(trow, sm + S_Z3, sm + S_Z2, sm + S_H, tid);  // dZ3 ; H2
        // ---- layer 3: dW3 += dZ3^T H2 ; db3 += dZ3^T 1 ; dH2 = dZ3 W3
        run([&] {
            for (int s = 0; s < TILE / 16; ++s) {
                tc::mma_bf16(tb + T_G3, tc::desc_mn(aZ3 + 4096 * s, H), tc::desc_mn(aH + 4096 * s, H), ID_GW,
                             acc | (s > 0));
                tc::mma_bf16(tb + T_GB3, tc::desc_mn(aZ3 + 4096 * s, H), tc::desc_k(aONE + 256 * s, TILE), ID_GB,
                             acc | (s > 0));
            }
            for (int s = 0; s < H / 16; ++s)
                tc::mma_bf16(tb + T_D, tc::desc_k(aZ3 + 256 * s, H), tc::desc_mn(aW3 + 4096 * s, H), ID_DH, s > 0);
        });
        if (!ok) break;
        epi_back(trow, sm + S_Z2, sm + S_Z1, sm + S_H, tid);  // dZ2 ; H1
        // ---- layer 2
        run([&] {
            for (int s = 0; s < TILE / 16; ++s) {
                tc::mma_bf16(tb + T_G2, tc::desc_mn(aZ2 + 4096 * s, H), tc::desc_mn(aH + 4096 * s, H), ID_GW,
                             acc | (s > 0));
                tc::mma_bf16(tb + T_GB2, tc::desc_mn(aZ2 + 4096 * s, H), tc::desc_k(aONE + 256 * s, TILE), ID_GB,
                             acc | (s > 0));
            }
            for (int s = 0; s < H / 16; ++s)
                tc::mma_bf16(tb + T_D, tc::desc_k(aZ2 + 256 * s, H), tc::desc_mn(aW2 + 4096 * s, H), ID_DH, s > 0);
        });
        if (!ok) break;
        epi_back(trow, sm + S_Z1, nullptr, nullptr, tid);  // dZ1
        // ---- layer 1: dW1 += dZ1^T X ; db1 += dZ1^T 1
        run([&] {
            for (int s = 0; s < TILE / 16; ++s) {
                tc::mma_bf16(tb + T_G1, tc::desc_mn(aZ1 + 4096 * s, H), tc::desc_mn(aX + 512 * s, KIN), ID_G1,
                             acc | (s > 0));
                tc::mma_bf16(tb + T_GB1, tc::desc_mn(aZ1 + 4096 * s, H), tc::desc_k(aONE + 256 * s, TILE), ID_GB,
                             acc | (s > 0));
            }
        });
        first = false;
    }
    if (!ok && tid == 0) atomicExch(err, 1);
    // ---- this CTA's partial gradient
    float* gp = gpart + (size_t)blockIdx.x * NPARAM;
    const int o = tid;
    if (first || !ok) {
        for (int p = tid; p < NPARAM; p += 128) gp[p] = 0.f;
    } else {
        float v[16];
        for (int c = 0; c < H / 16; ++c) {
            tc::tmem_ld16(trow + T_G2 + 16 * c, v);
            for (int k = 0; k < 16; ++k) gp[OFF_W2 + o * H + 16 * c + k] = v[k];
            tc::tmem_ld16(trow + T_G3 + 16 * c, v);
            for (int k = 0; k < 16; ++k) gp[OFF_W3 + o * H + 16 * c + k] = v[k];
        }
        tc::tmem_ld16(trow + T_G1, v);
        for (int k = 0; k < KIN; ++k) gp[OFF_W1 + o * KIN + k] = k < NIN ? v[k] : 0.f;
        tc::tmem_ld16(trow + T_G4T, v);
        for (int q = 0; q < KOUT; ++q) gp[OFF_W4 + q * H + o] = q < NOUT ? v[q] : 0.f;
        tc::tmem_ld16(trow + T_GB1, v);
        gp[OFF_B1 + o] = v[0];
        tc::tmem_ld16(trow + T_GB2, v);
        gp[OFF_B2 + o] = v[0];
        tc::tmem_ld16(trow + T_GB3, v);
        gp[OFF_B3 + o] = v[0];
        if (tid == 0)
            for (int q = 0; q < KOUT; ++q) gp[OFF_B4 + q] = q < NOUT ? acc_b4[q] : 0.f;
    }
    if (tid == 0) lossp[blockIdx.x] = acc_loss;
    // after a wait that ran out: wait, again within the limit, for the MMA
    // group still in flight before its TMEM is given back
    if (!ok && inflight) (void)tc::mbar_wait(mb, failed_parity, wc.limit);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tb, 512);
}


// Inference: the network on every row; SRC 0 takes the rows from training
// samples, SRC 1 builds them from the FP64 state along the CSR edges of the
// fluid particles.  out[g] = (fx, fy, fz, 0) in N, zero for masked rows.
// 256 threads: warpgroup 0 builds the rows and writes the outputs; the two
// warpgroups share each epilogue (columns 0-63 and 64-127 of the same rows:
// warps w and w+4 read the same TMEM lane quarter).
// Named barrier of one warpgroup (ids 1..4; 0 is __syncthreads), plain and
// with an AND reduction of a predicate.
__device__ __forceinline__ void wg_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }
__device__ __forceinline__ bool wg_sync_and(int id, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, %2, 128, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id)
        : "memory");
    return r != 0;
}

// Inference: Y = MLP(X) for rows of `samples` (SRC 0) or for the CSR edges of
// `es` (SRC 1, features computed from the FP64 state).  One CTA per SM, four
// warpgroups; each warpgroup owns one 128-edge tile at a time (its 128 TMEM
// columns, X and H buffers and mbarrier) and runs its own
// MMA -> epilogue chain, so four tiles are in flight per SM and one
// warpgroup's epilogue overlaps the others' MMAs.  The gathers of a
// warpgroup's next tile are issued during its current tile.
template <int SRC>
__global__ void __launch_bounds__(128 * I_WG, 1)
k_mlp_infer(const uint8_t* __restrict__ image, const float4* __restrict__ samples, long long n, EdgeSource es,
            Scales sc, float4* __restrict__ out, int* __restrict__ err, WaitCtl wc) {
    extern __shared__ __align__(128) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5, wg = tid >> 7, row = tid & 127;
    {
        const uint4* src = reinterpret_cast<const uint4*>(image);
        uint4* dst = reinterpret_cast<uint4*>(sm + S_W);
        for (int k = tid; k < PK_BYTES / 16; k += blockDim.x) dst[k] = src[k];
    }
    __syncthreads();  // the image is in shared memory
    halve_hidden_biases(reinterpret_cast<float*>(sm + S_W + PK_B));  // ordered by the barrier below
    const float* b1 = reinterpret_cast<const float*>(sm + S_W + PK_B);
    const float* b2 = b1 + H;
    const float* b3 = b2 + H;
    const float* b4 = b3 + H;
    uint64_t* mbars = reinterpret_cast<uint64_t*>(sm + I_MISC);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + I_MISC + 8 * I_WG);
    const uint32_t mb = tc::smem_addr(mbars + wg);
    if (row == 0) tc::mbar_init(mb, 1);
    if (warp == 0) tc::tmem_alloc(tc::smem_addr(tslot), 128 * I_WG);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tb = *tslot + 128u * (uint32_t)wg;  // this warpgroup's 128 TMEM columns
    const uint32_t trow = tb + ((uint32_t)((warp & 3) * 32) << 16);
    uint8_t* xs = sm + I_T + wg * I_TILE_BYTES;
    uint8_t* hs = xs + TILE * KIN * 2;
    const uint32_t aW1 = tc::smem_addr(sm + S_W + PK_W1), aW2 = tc::smem_addr(sm + S_W + PK_W2);
    const uint32_t aW3 = tc::smem_addr(sm + S_W + PK_W3), aW4 = tc::smem_addr(sm + S_W + PK_W4);
    const uint32_t aX = tc::smem_addr(xs), aH = tc::smem_addr(hs);
    const int bar = 1 + wg;

    uint32_t phase = 0;
    bool ok = true;
    bool inflight = false;        // a committed MMA group whose completion was not seen
    uint32_t failed_parity = 0;
    auto run = [&](auto&& issue) {
        tc::fence_async_smem();
        tc::fence_before_sync();
        wg_sync(bar);
        if (row == 0) {
            tc::fence_after_sync();
            if (wc.issue) {
                issue();
                tc::commit(mb);
            }
        }
        const bool done = tc::mbar_wait(mb, phase, wc.limit);
        tc::fence_after_sync();
        ok = wg_sync_and(bar, done);
        if (!ok) {
            inflight = wc.issue != 0;
            failed_parity = phase;
        }
        phase ^= 1u;
    };
    const long long rows = SRC == 0 ? n : es.ne;
    const long long ntiles = (rows + TILE - 1) / TILE;
    const long long stride = (long long)gridDim.x * I_WG;
    long long t = (long long)blockIdx.x * I_WG + wg;
    // this row's raw inputs, one tile ahead: ids, then the gathers
    int ni = 0, nj = 0;
    bool nin = false;
    double4 pi = make_double4(0, 0, 0, 0), pj = pi, vi = pi, vj = pi;
    float4 sa = make_float4(0.f, 0.f, 0.f, 0.f), sb = sa, scc = sa;
    auto load_ids = [&](long long tt) {
        const long long g = tt * TILE + row;
        nin = tt < ntiles && g < rows;
        if (SRC == 1 && nin) {
            ni = es.ei[g];
            nj = es.ej[g];
        }
    };
    auto load_raw = [&](long long tt) {
        if (!nin) return;
        if (SRC == 0) {
            const long long g = tt * TILE + row;
            sa = samples[3 * g];
            sb = samples[3 * g + 1];
            scc = samples[3 * g + 2];
        } else {
            pi = es.pos[ni];
            pj = es.pos[nj];
            vi = es.vel[ni];
            vj = es.vel[nj];
        }
    };
    load_ids(t);
    load_raw(t);
    for (; t < ntiles && ok; t += stride) {
        const long long g = t * TILE + row;
        const bool in = nin;
        float f[NIN] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        bool valid = false;
        if (in) {
            if (SRC == 0) {
                const int tt = (int)sb.w;
                f[0] = sa.x; f[1] = sa.y; f[2] = sa.z;
                f[3] = sb.x * sc.inv_u; f[4] = sb.y * sc.inv_u; f[5] = sb.z * sc.inv_u;
                f[6] = sa.w; f[7] = (float)(tt & 3); f[8] = (float)(tt >> 2);
                valid = scc.w != 0.0f;
            } else {
                double d[3] = {pj.x - pi.x, pj.y - pi.y, pj.z - pi.z};
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    if (d[k] > es.half_width[k]) d[k] -= es.width[k];
                    else if (d[k] < -es.half_width[k]) d[k] += es.width[k];
                }
                const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                valid = ni != nj && r2 < es.rv2;
                if (valid) {
                    f[0] = (float)(d[0] * es.inv_l0);
                    f[1] = (float)(d[1] * es.inv_l0);
                    f[2] = (float)(d[2] * es.inv_l0);
                    f[3] = (float)(vj.x - vi.x) * sc.inv_u;
                    f[4] = (float)(vj.y - vi.y) * sc.inv_u;
                    f[5] = (float)(vj.z - vi.z) * sc.inv_u;
                    f[6] = (float)(sqrt(r2) * es.inv_l0);
                    f[7] = (float)(int)pi.w;
                    f[8] = (float)(int)pj.w;
                }
            }
        }
        if (!valid) {
#pragma unroll
            for (int k = 0; k < NIN; ++k) f[k] = 0.f;
        }
        store_x(xs, row, f);
        load_ids(t + stride);
        run([&] { tc::mma_bf16(tb + T_D, tc::desc_k(aX, KIN), tc::desc_k(aW1, KIN), ID_F128, 0u); });
        if (!ok) break;
        load_raw(t + stride);  // the next tile's ids have arrived during the MMA
        epi_hidden(trow, b1, nullptr, hs, row);
        run([&] {
            for (int s = 0; s < H / 16; ++s)
                tc::mma_bf16(tb + T_D, tc::desc_k(aH + 256 * s, H), tc::desc_k(aW2 + 256 * s, H), ID_F128, s > 0);
        });
        if (!ok) break;
        epi_hidden(trow, b2, nullptr, hs, row);
        run([&] {
            for (int s = 0; s < H / 16; ++s)
                tc::mma_bf16(tb + T_D, tc::desc_k(aH + 256 * s, H), tc::desc_k(aW3 + 256 * s, H), ID_F128, s > 0);
        });
        if (!ok) break;
        epi_hidden(trow, b3, nullptr, hs, row);
        run([&] {  // the output layer reuses the first 16 columns
            for (int s = 0; s < H / 16; ++s)
                tc::mma_bf16(tb + T_D, tc::desc_k(aH + 256 * s, H), tc::desc_k(aW4 + 256 * s, H), ID_F16, s > 0);
        });
        if (!ok) break;
        float v[16];
        tc::tmem_ld16(trow + T_D, v);
        if (in) {
            out[g] = valid ? make_float4((v[0] + b4[0]) * sc.f_scale, (v[1] + b4[1]) * sc.f_scale,
                                         (v[2] + b4[2]) * sc.f_scale, 0.f)
                           : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
    if (!ok && row == 0) atomicExch(err, 1);
    // after a wait that ran out: wait, again within the limit, for this
    // warpgroup's MMA group still in flight before the TMEM is given back
    if (!ok && inflight) (void)tc::mbar_wait(mb, failed_parity, wc.limit);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(*tslot, 128 * I_WG);
}

// grad[p] = scale * sum of the CTA partials, in CTA order
__global__ void k_grad_reduce(const float* __restrict__ gpart, int ctas, float scale, float* __restrict__ grad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NPARAM) return;
    float s = 0.f;
    for (int c = 0; c < ctas; ++c) s += gpart[(size_t)c * NPARAM + p];
    grad[p] = s * scale;
}

// parameters that are padding (W1 inputs >= 9, W4 / b4 outputs >= 3)
__host__ __device__ inline bool is_padding(int p) {
    if (p < OFF_B1) return (p % KIN) >= NIN;
    if (p >= OFF_W4 && p < OFF_B4) return (p - OFF_W4) / H >= NOUT;
    if (p >= OFF_B4) return (p - OFF_B4) >= NOUT;
    return false;
}

__device__ inline void pack_param(int p, float w, uint8_t* image) {
    auto put = [&](int off, int r, int c, int C) {
        *reinterpret_cast<__nv_bfloat16*>(image + off + core_off(r, c, C)) = __float2bfloat16_rn(w);
    };
    float* bias = reinterpret_cast<float*>(image + PK_B);
    if (p < OFF_B1) put(PK_W1, p / KIN, p % KIN, KIN);
    else if (p < OFF_W2) bias[p - OFF_B1] = w;
    else if (p < OFF_B2) put(PK_W2, (p - OFF_W2) / H, (p - OFF_W2) % H, H);
    else if (p < OFF_W3) bias[H + p - OFF_B2] = w;
    else if (p < OFF_B3) put(PK_W3, (p - OFF_W3) / H, (p - OFF_W3) % H, H);
    else if (p < OFF_W4) bias[2 * H + p - OFF_B3] = w;
    else if (p < OFF_B4) put(PK_W4, (p - OFF_W4) / H, (p - OFF_W4) % H, H);
    else bias[3 * H + p - OFF_B4] = w;
}

__global__ void k_pack(const float* __restrict__ w, uint8_t* __restrict__ image) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NPARAM) return;
    pack_param(p, is_padding(p) ? 0.f : w[p], image);
}

// Adam (bias-corrected moments), then the BF16 image
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, float lr, float b1, float b2, float eps, float bc1, float bc2,
                       uint8_t* __restrict__ image) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NPARAM) return;
    float wp = w[p];
    if (is_padding(p)) {
        wp = 0.f;
    } else {
        const float gp = g[p];
        const float mp = b1 * m[p] + (1.f - b1) * gp;
        const float vp = b2 * v[p] + (1.f - b2) * gp * gp;
        m[p] = mp;
        v[p] = vp;
        wp -= lr * (mp / bc1) / (sqrtf(vp / bc2) + eps);
    }
    w[p] = wp;
    pack_param(p, wp, image);
}

}  // namespace

#define MTRY(x)                                         \
    do {                                                \
        cudaError_t e_ = (x);                           \
        if (e_ != cudaSuccess) {                        \
            if (err) *err = cudaGetErrorString(e_);     \
            return -3;                                  \
        }                                               \
    } while (0)

static int check_flag(Model* m, std::string* err) {
    int h = 0;
    MTRY(cudaMemcpyAsync(&h, m->err, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
    MTRY(cudaStreamSynchronize(m->stream));
    if (h) {
        if (err) *err = "tensor-core wait timed out in the edge-MLP kernel";
        return -5;
    }
    return 0;
}

int model_create(Model* m, unsigned long long seed, std::string* err) {
    MTRY(cudaGetDevice(&m->device));
    int sms = 0;
    MTRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device));
    m->ctas = sms;
    MTRY(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
    MTRY(cudaMalloc(&m->w, NPARAM * sizeof(float)));
    MTRY(cudaMalloc(&m->adam_m, NPARAM * sizeof(float)));
    MTRY(cudaMalloc(&m->adam_v, NPARAM * sizeof(float)));
    MTRY(cudaMalloc(&m->grad, NPARAM * sizeof(float)));
    MTRY(cudaMalloc(&m->gpart, (size_t)sms * NPARAM * sizeof(float)));
    MTRY(cudaMalloc(&m->lossp, (size_t)sms * sizeof(double)));
    MTRY(cudaMalloc(&m->image, PK_BYTES));
    MTRY(cudaMalloc(&m->err, sizeof(int)));
    MTRY(cudaMemset(m->adam_m, 0, NPARAM * sizeof(float)));
    MTRY(cudaMemset(m->adam_v, 0, NPARAM * sizeof(float)));
    MTRY(cudaMemset(m->image, 0, PK_BYTES));
    MTRY(cudaMemset(m->err, 0, sizeof(int)));
    MTRY(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, S_TRAIN));
    MTRY(cudaFuncSetAttribute(k_mlp_infer<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, S_INFER));
    MTRY(cudaFuncSetAttribute(k_mlp_infer<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, S_INFER));
    // uniform initialisation with variance 1 / fan_in (hidden) and a small output layer
    std::vector<float> w(NPARAM, 0.f);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<float> u(-1.f, 1.f);
    auto fill = [&](int off, int rows, int cols, int fan_in, float gain) {
        const float a = gain * std::sqrt(3.0f / (float)fan_in);
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c) w[off + r * cols + c] = a * u(rng);
    };
    fill(OFF_W1, H, KIN, NIN, 1.f);
    fill(OFF_W2, H, H, H, 1.f);
    fill(OFF_W3, H, H, H, 1.f);
    fill(OFF_W4, KOUT, H, H, 0.5f);
    for (int p = 0; p < NPARAM; ++p)
        if (is_padding(p)) w[p] = 0.f;
    m->adam_t = 0;
    return model_set_params(m, w.data(), err);
}

void model_destroy(Model* m) {
    cudaFree(m->w);
    cudaFree(m->adam_m);
    cudaFree(m->adam_v);
    cudaFree(m->grad);
    cudaFree(m->gpart);
    cudaFree(m->lossp);
    cudaFree(m->image);
    cudaFree(m->err);
    if (m->stream) cudaStreamDestroy(m->stream);
    *m = Model{};
}

int model_set_params(Model* m, const float* host, std::string* err) {
    MTRY(cudaMemcpyAsync(m->w, host, NPARAM * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    k_pack<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->w, m->image);
    MTRY(cudaGetLastError());
    MTRY(cudaStreamSynchronize(m->stream));
    return 0;
}

int model_get_params(Model* m, float* host, std::string* err) {
    MTRY(cudaMemcpyAsync(host, m->w, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MTRY(cudaStreamSynchronize(m->stream));
    return 0;
}

int model_grad(Model* m, const float4* samples, const long long* order, long long n, double* loss,
               std::string* err) {
    if (n <= 0) {
        if (err) *err = "no samples";
        return -1;
    }
    const long long ntiles = (n + TILE - 1) / TILE;
    const int ctas = (int)std::min<long long>(m->ctas, ntiles);
    k_mlp_train<<<ctas, 128, S_TRAIN, m->stream>>>(m->image, samples, order, n, m->sc, m->gpart, m->lossp, m->err,
                                                   WaitCtl{kWaitLimit, 1});
    MTRY(cudaGetLastError());
    k_grad_reduce<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->gpart, ctas, (float)(2.0 / (3.0 * (double)n)),
                                                               m->grad);
    MTRY(cudaGetLastError());
    if (loss) {
        std::vector<double> lp(ctas);
        MTRY(cudaMemcpyAsync(lp.data(), m->lossp, ctas * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
        const int rc = check_flag(m, err);
        if (rc) return rc;
        double s = 0.0;
        for (double x : lp) s += x;
        *loss = s / (3.0 * (double)n);
    }
    return 0;
}

int model_adam(Model* m, float lr, float beta1, float beta2, float eps, std::string* err) {
    ++m->adam_t;
    const float bc1 = 1.f - std::pow(beta1, (float)m->adam_t), bc2 = 1.f - std::pow(beta2, (float)m->adam_t);
    k_adam<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->w, m->adam_m, m->adam_v, m->grad, lr, beta1, beta2, eps,
                                                        bc1, bc2, m->image);
    MTRY(cudaGetLastError());
    return 0;
}

int model_predict(Model* m, const float4* samples, long long n, float4* out, std::string* err) {
    if (n <= 0) return 0;
    const long long ntiles = (n + TILE - 1) / TILE;
    const int ctas = (int)std::min<long long>(m->ctas, (ntiles + I_WG - 1) / I_WG);
    EdgeSource es{};
    k_mlp_infer<0><<<ctas, 128 * I_WG, S_INFER, m->stream>>>(m->image, samples, n, es, m->sc, out, m->err,
                                                              WaitCtl{kWaitLimit, 1});
    MTRY(cudaGetLastError());
    return check_flag(m, err);
}

int model_apply_edges(Model* m, const EdgeSource& src, float4* out, cudaStream_t s, int* launches,
                      std::string* err) {
    if (launches) *launches = 0;
    if (src.ne <= 0) return 0;
    const long long ntiles = (src.ne + TILE - 1) / TILE;
    const int ctas = (int)std::min<long long>(m->ctas, (ntiles + I_WG - 1) / I_WG);
    k_mlp_infer<1><<<ctas, 128 * I_WG, S_INFER, s>>>(m->image, nullptr, 0, src, m->sc, out, m->err,
                                                     WaitCtl{kWaitLimit, 1});
    MTRY(cudaGetLastError());
    if (launches) *launches = 1;
    return 0;
}

int model_error_flag(Model* m, std::string* err) { return check_flag(m, err); }

int model_check_wait(Model* m, int which, long long polls, std::string* err) {
    if (polls < 1 || polls > kWaitLimit || (which != 0 && which != 1)) {
        if (err) *err = "bad arguments";
        return -1;
    }
    // one tile of zero samples; the kernel's first wait runs out after `polls`
    // polls because no MMA group is issued, so nothing is in flight when it
    // sets the error flag and frees its TMEM
    float4* buf = nullptr;  // 3 float4 per sample (TILE samples), then TILE outputs
    const size_t bytes = (size_t)TILE * 4 * sizeof(float4);
    MTRY(cudaMalloc(&buf, bytes));
    float4* samples = buf;
    cudaError_t e = cudaMemsetAsync(buf, 0, bytes, m->stream);
    if (e == cudaSuccess) {
        if (which == 0)
            k_mlp_train<<<1, 128, S_TRAIN, m->stream>>>(m->image, samples, nullptr, TILE, m->sc, m->gpart, m->lossp,
                                                         m->err, WaitCtl{polls, 0});
        else
            k_mlp_infer<0><<<1, 128 * I_WG, S_INFER, m->stream>>>(m->image, samples, TILE, EdgeSource{}, m->sc,
                                                                   buf + 3 * TILE, m->err, WaitCtl{polls, 0});
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    cudaFree(buf);
    MTRY(e);
    const int rc = check_flag(m, err);
    // the model stays usable: clear the flag the self-test raised
    MTRY(cudaMemsetAsync(m->err, 0, sizeof(int), m->stream));
    MTRY(cudaStreamSynchronize(m->stream));
    return rc;
}

}  // namespace mlp
}  // namespace mph
