// Edge-MLP surrogate for the viscosity and surface-tension pair terms
// (the learned form of the step).  Host-side interface of k_mlp.cu.
//
// Network: 9 inputs (padded to 16) -> 128 -> 128 -> 128 -> 3 (padded to 16),
// SiLU after each hidden layer, BF16 weights and activations, FP32
// accumulation in tensor memory.  Inputs per edge (i, j): the displacement
// x_j - x_i over l0 (3), the relative velocity v_j - v_i over the model's
// velocity scale (3), the distance over l0, the particle types of i and j.
// Output: the pair's viscous + surface-tension force on i over the model's
// force scale.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

namespace mph {
namespace mlp {

constexpr int H = 128;     // hidden width
constexpr int NIN = 9;     // real inputs
constexpr int KIN = 16;    // padded input width
constexpr int NOUT = 3;    // real outputs
constexpr int KOUT = 16;   // padded output width
constexpr int TILE = 128;  // edges per tensor-core tile

// flat FP32 parameter vector: W1[H][KIN], b1[H], W2[H][H], b2[H], W3[H][H],
// b3[H], W4[KOUT][H], b4[KOUT]  (W[out][in]; padding entries stay zero)
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + H * KIN;
constexpr int OFF_W2 = OFF_B1 + H;
constexpr int OFF_B2 = OFF_W2 + H * H;
constexpr int OFF_W3 = OFF_B2 + H;
constexpr int OFF_B3 = OFF_W3 + H * H;
constexpr int OFF_W4 = OFF_B3 + H;
constexpr int OFF_B4 = OFF_W4 + KOUT * H;
constexpr int NPARAM = OFF_B4 + KOUT;

// packed image the kernels copy into shared memory as is: BF16 weights in the
// core-matrix layout, then FP32 biases b1, b2, b3, b4
constexpr int PK_W1 = 0;
constexpr int PK_W2 = PK_W1 + H * KIN * 2;
constexpr int PK_W3 = PK_W2 + H * H * 2;
constexpr int PK_W4 = PK_W3 + H * H * 2;
constexpr int PK_B = PK_W4 + KOUT * H * 2;
constexpr int PK_BYTES = PK_B + (3 * H + KOUT) * 4;

// one training sample = 3 float4:
//   s0 = (dx, dy, dz, r) / l0
//   s1 = (ux, uy, uz, type_i + 4 * type_j)      (u = v_j - v_i, m/s)
//   s2 = (fx, fy, fz, valid)                    (target pair force, N)
struct Scales {
    float inv_u;    // 1 / velocity scale
    float f_scale;  // force scale (N)
    float inv_f;    // 1 / force scale
    float pad;
};

struct Model {
    float* w = nullptr;       // FP32 master parameters [NPARAM]
    float* adam_m = nullptr;  // Adam moments
    float* adam_v = nullptr;
    float* grad = nullptr;    // reduced gradient [NPARAM]
    float* gpart = nullptr;   // per-CTA partial gradients [ctas][NPARAM]
    double* lossp = nullptr;  // per-CTA loss partials
    uint8_t* image = nullptr; // packed BF16 image [PK_BYTES]
    int* err = nullptr;       // device error flag (tensor-core wait timeout)
    int ctas = 0;
    long long adam_t = 0;
    Scales sc{1.f, 1.f, 1.f, 0.f};
    int device = 0;
    cudaStream_t stream = nullptr;
};

int model_create(Model* m, unsigned long long seed, std::string* err);
void model_destroy(Model* m);
// upload FP32 parameters (and repack), read them back
int model_set_params(Model* m, const float* host, std::string* err);
int model_get_params(Model* m, float* host, std::string* err);
// one pass of forward + backward over `n` device samples (indices `order`
// into `samples`, or 0..n-1 when order is null); the gradient of the mean
// squared error of the scaled outputs lands in m->grad, the loss in *loss
int model_grad(Model* m, const float4* samples, const long long* order, long long n, double* loss,
               std::string* err);
// Adam update from m->grad, then repack the BF16 image
int model_adam(Model* m, float lr, float beta1, float beta2, float eps, std::string* err);
// predictions for `n` device samples: out[e] = (fx, fy, fz, 0) in N (scaled back)
int model_predict(Model* m, const float4* samples, long long n, float4* out, std::string* err);

// The learned pair force of every edge of the fluid particles' neighbour
// lists (CSR edges ei/ej, `ne` of them) from the FP64 state, masked to
// j != i and r < rv: out[e] = (fx, fy, fz, 0) in N.  See k_mlp.cu.
struct EdgeSource {
    const double4* pos;   // {x, y, z, type}
    const double4* vel;   // {vx, vy, vz, PressureP}
    const int* ei;
    const int* ej;
    long long ne;
    double width[3], half_width[3], inv_l0, rv2;
};
int model_apply_edges(Model* m, const EdgeSource& src, float4* out, cudaStream_t s, int* launches,
                      std::string* err);
// nonzero (and *err set) when a tensor-core wait of an MLP kernel gave up
int model_error_flag(Model* m, std::string* err);
// Self-test of the bounded waits: the training (which 0) or inference
// (which 1) kernel on one tile with its MMA groups withheld and a wait limit
// of `polls`; returns what a timed-out wait returns (-5, *err set) once the
// kernel has freed its TMEM, and clears the model's error flag.
int model_check_wait(Model* m, int which, long long polls, std::string* err);

}  // namespace mlp
}  // namespace mph
