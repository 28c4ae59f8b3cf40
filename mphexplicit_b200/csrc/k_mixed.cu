// k_mixed.cu — mixed-precision form (placeholder until the kernels land).
#include "mph_mixed.h"

namespace mph {

struct MixedState {
    long long rebuilds = 0;
};

int mixed_create(MixedState** out, const SimConst&, const mph_constants&, DevFP64&, cudaStream_t, std::string* err) {
    *out = nullptr;
    if (err) *err = "mixed form not built yet";
    return MPH_ERR_ARG;
}
int mixed_step(MixedState*, const SimConst&, DevFP64&, int, cudaStream_t, std::string* err) {
    if (err) *err = "mixed form not built yet";
    return MPH_ERR_STATE;
}
int mixed_export(MixedState*, const SimConst&, DevFP64&, cudaStream_t, std::string*) { return MPH_OK; }
int mixed_import(MixedState*, const SimConst&, DevFP64&, cudaStream_t, std::string*) { return MPH_OK; }
long long mixed_rebuilds(const MixedState* m) { return m ? m->rebuilds : 0; }
void mixed_destroy(MixedState* m) { delete m; }

}  // namespace mph
