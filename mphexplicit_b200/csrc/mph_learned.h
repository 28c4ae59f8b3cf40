// Internal glue between the learned-form C ABI (mph_learned.cpp), the step
// (mph_host.cpp) and the edge-MLP kernels (k_mlp.cu).
#pragma once
#include <string>
#include "mph_b200.h"
#include "mph_mlp.h"

namespace mph {
int set_thread_error(int code, const std::string& msg);
// room for up to `want` more samples at the end of a dataset
float4* dataset_reserve(mph_dataset* d, long long want, long long* got);
void dataset_commit(mph_dataset* d, long long added);
mlp::Model* model_of(mph_model* m);
}  // namespace mph
