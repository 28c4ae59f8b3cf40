// k_noalloc.cu — the cell sort as one entry point that allocates nothing.
//
// Some callers cannot call cudaMalloc: their device memory is owned by
// another allocator (a framework's caching allocator or a pool with a fixed
// budget, where an outside cudaMalloc can fail or fragment it), or they run a
// time-critical loop in which allocation and cudaFree (which synchronises the
// device) are not allowed.  mph_cell_sort_noalloc serves them: the caller
// passes device inputs and outputs, and the sort's scratch (keys and values
// padded to a power of two) lives in the file-scope array below instead of
// memory the library would allocate.
#include <cstring>
#include <string>
#include "mph_internal.h"

namespace mph {
namespace {

// Largest padded sort size the scratch holds: 2^20 keys + 2^20 values (8 MiB,
// resident on every GPU that loads this library until the process exits).
// n particles need the smallest power of two above n, so n <= 2^20 - 1.
constexpr int kNoAllocMaxPow2 = 1 << 20;
__device__ __align__(256) int g_sort_scratch[2 * kNoAllocMaxPow2];

// Device address of g_sort_scratch in the current context, looked up on
// every call (the array's name in host code is only a host-side stand-in).
// Once the module is loaded the lookup allocates nothing; not caching it
// keeps the address right after a device reset or with another context
// current on the same device.
int scratch_on_current_device(int** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
    if (e != cudaSuccess || !p)
        return set_thread_error(MPH_ERR_CUDA,
                                std::string("cudaGetSymbolAddress(sort scratch): ") + cudaGetErrorString(e));
    *out = static_cast<int*>(p);
    return MPH_OK;
}

// Cell index of main.cpp:1115-1133 from double[n][3] positions; pads get 2*Tot.
__global__ void k_cell_index_aos(SimConst c, const double* __restrict__ xyz, const int* __restrict__ type,
                                 int* __restrict__ keys, int* __restrict__ vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.pow2) return;
    if (i < c.n) {
        const double* p = xyz + 3 * (size_t)i;
        const int cx = ((int)floor((p[0] - c.dmin[0]) / c.cell_width[0])) % c.cc[0];
        const int cy = ((int)floor((p[1] - c.dmin[1]) / c.cell_width[1])) % c.cc[1];
        const int cz = ((int)floor((p[2] - c.dmin[2]) / c.cell_width[2])) % c.cc[2];
        int id = ((cx % c.cc[0] + c.cc[0]) % c.cc[0]) * c.cc[1] * c.cc[2] +
                 ((cy % c.cc[1] + c.cc[1]) % c.cc[1]) * c.cc[2] + ((cz % c.cc[2] + c.cc[2]) % c.cc[2]);
        const int t = type[i];
        if (t >= 2 && t < 4) id += c.tot;
        keys[i] = id;
        vals[i] = i;
    } else {
        keys[i] = 2 * c.tot;
        vals[i] = c.n;
    }
}

__global__ void k_copy_sorted(int n, const int* __restrict__ keys, const int* __restrict__ vals,
                              int* __restrict__ cell_index, int* __restrict__ cell_particle) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    cell_index[i] = keys[i];
    cell_particle[i] = vals[i];
}

}  // namespace
}  // namespace mph

extern "C" int mph_cell_sort_noalloc(const mph_constants* c, const mph_grid_header* h, int n, const double* xyz,
                                     const int* type, int* cell_index, int* cell_particle, int* cell_start,
                                     void* stream) {
    using namespace mph;
    if (!c || !h || !xyz || !type || !cell_index || !cell_particle || !cell_start || n <= 0)
        return set_thread_error(MPH_ERR_ARG, "mph_cell_sort_noalloc: bad arguments");
    if (c->total_cell_count < 1 || c->cell_count[0] < 1 || c->cell_count[1] < 1 || c->cell_count[2] < 1)
        return set_thread_error(MPH_ERR_GEOMETRY, "mph_cell_sort_noalloc: empty cell grid");
    int pe = 0;
    while ((n >> pe) != 0) ++pe;  // PowerParticleCount: smallest power of two above n (main.cpp:612-617)
    if (pe > 30 || (1 << pe) > kNoAllocMaxPow2)
        return set_thread_error(MPH_ERR_CAPACITY,
                                "mph_cell_sort_noalloc: " + std::to_string(n) +
                                    " particles exceed the static scratch (at most " +
                                    std::to_string(kNoAllocMaxPow2 - 1) + ")");
    int* scratch = nullptr;
    const int st = scratch_on_current_device(&scratch);
    if (st != MPH_OK) return st;
    SimConst sc;
    std::memset(&sc, 0, sizeof(sc));
    sc.n = n;
    sc.pow2 = 1 << pe;
    sc.tot = c->total_cell_count;
    for (int d = 0; d < 3; ++d) {
        sc.cc[d] = c->cell_count[d];
        sc.dmin[d] = h->domain_min[d];
        sc.cell_width[d] = c->cell_width[d];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int* keys = scratch;
    int* vals = scratch + sc.pow2;
    k_cell_index_aos<<<(sc.pow2 + 255) / 256, 256, 0, s>>>(sc, xyz, type, keys, vals);
    launch_bitonic_sort(sc, keys, vals, s);
    launch_cell_ranges(sc, keys, cell_start, s);
    k_copy_sorted<<<(n + 255) / 256, 256, 0, s>>>(n, keys, vals, cell_index, cell_particle);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return set_thread_error(MPH_ERR_CUDA, std::string("mph_cell_sort_noalloc: ") + cudaGetErrorString(e));
    return MPH_OK;
}
