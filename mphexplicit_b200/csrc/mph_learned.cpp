// C ABI of the edge-MLP surrogate: models, sample datasets, training.
// The kernels are in k_mlp.cu; the learned step itself is in mph_host.cpp.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>
#include "mph_b200.h"
#include "mph_learned.h"

using mph::mlp::Model;

struct mph_model {
    Model m;
    std::string err;
};

namespace {

int set_err(std::string* dst, int rc, const std::string& msg) {
    if (dst) *dst = msg;
    return rc;
}

#define CU(x)                                                                  \
    do {                                                                       \
        cudaError_t e_ = (x);                                                  \
        if (e_ != cudaSuccess) return set_err(err, MPH_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)

// device scratch that lives for one call
struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

}  // namespace

extern "C" int mph_model_create(unsigned long long seed, mph_model** out) {
    if (!out) return MPH_ERR_ARG;
    *out = nullptr;
    mph_model* m = new mph_model();
    std::string e;
    const int rc = mph::mlp::model_create(&m->m, seed, &e);
    if (rc != 0) {
        mph::mlp::model_destroy(&m->m);
        delete m;
        mph::set_thread_error(MPH_ERR_CUDA, e);
        return rc == -3 ? MPH_ERR_CUDA : MPH_ERR_DEVICE;
    }
    *out = m;
    return MPH_OK;
}

extern "C" void mph_model_destroy(mph_model* m) {
    if (!m) return;
    mph::mlp::model_destroy(&m->m);
    delete m;
}

extern "C" int mph_model_param_count(void) { return mph::mlp::NPARAM; }

extern "C" int mph_model_get_params(mph_model* m, float* params) {
    if (!m || !params) return MPH_ERR_ARG;
    return mph::mlp::model_get_params(&m->m, params, &m->err) == 0 ? MPH_OK : MPH_ERR_CUDA;
}

extern "C" int mph_model_set_params(mph_model* m, const float* params) {
    if (!m || !params) return MPH_ERR_ARG;
    return mph::mlp::model_set_params(&m->m, params, &m->err) == 0 ? MPH_OK : MPH_ERR_CUDA;
}

extern "C" int mph_model_set_scales(mph_model* m, double velocity_scale, double force_scale) {
    if (!m || !(velocity_scale > 0.0) || !(force_scale > 0.0) || !std::isfinite(velocity_scale) ||
        !std::isfinite(force_scale))
        return MPH_ERR_ARG;
    m->m.sc.inv_u = (float)(1.0 / velocity_scale);
    m->m.sc.f_scale = (float)force_scale;
    m->m.sc.inv_f = (float)(1.0 / force_scale);
    return MPH_OK;
}

extern "C" int mph_model_get_scales(mph_model* m, double* velocity_scale, double* force_scale) {
    if (!m) return MPH_ERR_ARG;
    if (velocity_scale) *velocity_scale = 1.0 / (double)m->m.sc.inv_u;
    if (force_scale) *force_scale = (double)m->m.sc.f_scale;
    return MPH_OK;
}

static int map_rc(int rc) { return rc == 0 ? MPH_OK : rc == -1 ? MPH_ERR_ARG : rc == -5 ? MPH_ERR_DEVICE : MPH_ERR_CUDA; }

extern "C" int mph_model_gradient(mph_model* m, const float* samples, long long n, float* grad, double* loss) {
    if (!m || !samples || n <= 0 || !grad) return MPH_ERR_ARG;
    std::string* err = &m->err;
    DevBuf ds;
    const size_t bytes = (size_t)n * MPH_SAMPLE_FLOATS * sizeof(float);
    CU(cudaMalloc(&ds.p, bytes));
    CU(cudaMemcpyAsync(ds.p, samples, bytes, cudaMemcpyHostToDevice, m->m.stream));
    double l = 0.0;
    const int rc = mph::mlp::model_grad(&m->m, (const float4*)ds.p, nullptr, n, &l, err);
    if (rc) return map_rc(rc);
    CU(cudaMemcpyAsync(grad, m->m.grad, mph::mlp::NPARAM * sizeof(float), cudaMemcpyDeviceToHost, m->m.stream));
    CU(cudaStreamSynchronize(m->m.stream));
    if (loss) *loss = l;
    return MPH_OK;
}

extern "C" int mph_model_predict(mph_model* m, const float* samples, long long n, float* out) {
    if (!m || !samples || n <= 0 || !out) return MPH_ERR_ARG;
    std::string* err = &m->err;
    DevBuf ds, dout;
    const size_t bytes = (size_t)n * MPH_SAMPLE_FLOATS * sizeof(float);
    CU(cudaMalloc(&ds.p, bytes));
    CU(cudaMalloc(&dout.p, (size_t)n * sizeof(float4)));
    CU(cudaMemcpyAsync(ds.p, samples, bytes, cudaMemcpyHostToDevice, m->m.stream));
    const int rc = mph::mlp::model_predict(&m->m, (const float4*)ds.p, n, (float4*)dout.p, err);
    if (rc) return map_rc(rc);
    CU(cudaMemcpyAsync(out, dout.p, (size_t)n * sizeof(float4), cudaMemcpyDeviceToHost, m->m.stream));
    CU(cudaStreamSynchronize(m->m.stream));
    return MPH_OK;
}

extern "C" int mph_model_check_wait(mph_model* m, int kernel, long long polls) {
    if (!m || (kernel != 0 && kernel != 1) || polls < 1 || polls > (1ll << 22)) return MPH_ERR_ARG;
    return map_rc(mph::mlp::model_check_wait(&m->m, kernel, polls, &m->err));
}

extern "C" int mph_model_last_error(mph_model* m, char* buf, int len) {
    if (!m || !buf || len <= 0) return MPH_ERR_ARG;
    std::snprintf(buf, (size_t)len, "%s", m->err.c_str());
    return MPH_OK;
}

// ---- datasets ----------------------------------------------------------

struct mph_dataset {
    float4* s = nullptr;  // [capacity][3]
    long long cap = 0, n = 0;
    std::string err;
};

extern "C" int mph_dataset_create(long long capacity, mph_dataset** out) {
    if (!out || capacity <= 0) return MPH_ERR_ARG;
    *out = nullptr;
    mph_dataset* d = new mph_dataset();
    if (cudaMalloc(&d->s, (size_t)capacity * 3 * sizeof(float4)) != cudaSuccess) {
        cudaGetLastError();
        delete d;
        mph::set_thread_error(MPH_ERR_NOMEM, "dataset allocation failed");
        return MPH_ERR_NOMEM;
    }
    d->cap = capacity;
    *out = d;
    return MPH_OK;
}

extern "C" void mph_dataset_destroy(mph_dataset* d) {
    if (!d) return;
    cudaFree(d->s);
    delete d;
}

extern "C" long long mph_dataset_size(mph_dataset* d) { return d ? d->n : -1; }

extern "C" int mph_dataset_append(mph_dataset* d, const float* samples, long long n) {
    if (!d || !samples || n < 0) return MPH_ERR_ARG;
    if (d->n + n > d->cap) return MPH_ERR_CAPACITY;
    std::string* err = &d->err;
    CU(cudaMemcpy(d->s + 3 * d->n, samples, (size_t)n * 3 * sizeof(float4), cudaMemcpyHostToDevice));
    d->n += n;
    return MPH_OK;
}

extern "C" int mph_dataset_read(mph_dataset* d, long long first, long long n, float* samples) {
    if (!d || !samples || first < 0 || n < 0 || first + n > d->n) return MPH_ERR_ARG;
    std::string* err = &d->err;
    CU(cudaMemcpy(samples, d->s + 3 * first, (size_t)n * 3 * sizeof(float4), cudaMemcpyDeviceToHost));
    return MPH_OK;
}

namespace mph {
// internal: a dataset's device buffer and room (used by mph_collect_samples)
float4* dataset_reserve(mph_dataset* d, long long want, long long* got) {
    const long long room = d->cap - d->n;
    *got = std::min(room, want);
    return d->s + 3 * d->n;
}
void dataset_commit(mph_dataset* d, long long added) { d->n += added; }
Model* model_of(mph_model* m) { return &m->m; }
}  // namespace mph

extern "C" int mph_model_fit_scales(mph_model* m, mph_dataset* d) {
    if (!m || !d || d->n <= 0) return MPH_ERR_ARG;
    std::string* err = &m->err;
    // the RMS over the samples, on the host in blocks
    const long long blk = 1 << 20;
    std::vector<float> h((size_t)std::min(blk, d->n) * MPH_SAMPLE_FLOATS);
    double su = 0.0, sf = 0.0;
    long long cnt = 0;
    for (long long f = 0; f < d->n; f += blk) {
        const long long k = std::min(blk, d->n - f);
        CU(cudaMemcpy(h.data(), d->s + 3 * f, (size_t)k * 3 * sizeof(float4), cudaMemcpyDeviceToHost));
        for (long long q = 0; q < k; ++q) {
            const float* s = &h[(size_t)q * MPH_SAMPLE_FLOATS];
            if (s[11] == 0.f) continue;
            su += (double)s[4] * s[4] + (double)s[5] * s[5] + (double)s[6] * s[6];
            sf += (double)s[8] * s[8] + (double)s[9] * s[9] + (double)s[10] * s[10];
            ++cnt;
        }
    }
    if (cnt == 0 || !(su > 0.0) || !(sf > 0.0)) {
        m->err = "dataset has no non-zero samples";
        return MPH_ERR_ARG;
    }
    return mph_model_set_scales(m, std::sqrt(su / (3.0 * cnt)), std::sqrt(sf / (3.0 * cnt)));
}

extern "C" int mph_model_train(mph_model* m, mph_dataset* d, int epochs, int batch, double lr,
                               unsigned long long seed, double* loss) {
    if (!m || !d || d->n <= 0 || epochs <= 0 || batch <= 0 || !(lr > 0.0)) return MPH_ERR_ARG;
    std::string* err = &m->err;
    Model* md = &m->m;
    const long long n = d->n;
    std::vector<long long> idx((size_t)n);
    std::iota(idx.begin(), idx.end(), 0LL);
    std::mt19937_64 rng(seed);
    DevBuf order;
    CU(cudaMalloc(&order.p, (size_t)n * sizeof(long long)));
    const long long nb = (n + batch - 1) / batch;
    const long long total = nb * (long long)epochs;
    long long step = 0;
    double last = 0.0;
    for (int ep = 0; ep < epochs; ++ep) {
        std::shuffle(idx.begin(), idx.end(), rng);
        CU(cudaMemcpyAsync(order.p, idx.data(), (size_t)n * sizeof(long long), cudaMemcpyHostToDevice, md->stream));
        double sum = 0.0;
        for (long long b = 0; b < nb; ++b, ++step) {
            const long long first = b * batch, cnt = std::min<long long>(batch, n - first);
            double l = 0.0;
            int rc = mph::mlp::model_grad(md, d->s, (const long long*)order.p + first, cnt, &l, err);
            if (rc) return map_rc(rc);
            sum += l * (double)cnt;
            // cosine decay to 5 % of the initial rate
            const double frac = total > 1 ? (double)step / (double)(total - 1) : 1.0;
            const double rate = lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(3.14159265358979323846 * frac)));
            rc = mph::mlp::model_adam(md, (float)rate, 0.9f, 0.999f, 1e-8f, err);
            if (rc) return map_rc(rc);
        }
        last = sum / (double)n;
    }
    CU(cudaStreamSynchronize(md->stream));
    if (loss) *loss = last;
    return MPH_OK;
}
