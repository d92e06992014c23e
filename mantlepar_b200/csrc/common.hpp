// Shared host-side plumbing of the mantlepar_b200 C ABI: status strings,
// CUDA error mapping and the kernel launch counter.
#ifndef MP_COMMON_HPP
#define MP_COMMON_HPP

#include <cuda_runtime.h>

#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>

#include "../../include/mantlepar/mp.h"

namespace mp {

void set_error(const char* fmt, ...);
extern std::atomic<unsigned long long> g_launches;

// Set while this thread captures a CUDA graph: captured launches are counted
// when the graph runs, not when it is built.
inline thread_local bool g_capturing = false;

inline void count_launch(unsigned long long n = 1) {
    if (!g_capturing) g_launches.fetch_add(n, std::memory_order_relaxed);
}

// A named NVTX range over a scope of host work (stage launches, step loops,
// graph runs), for a profiler's timeline; without an attached tool the push
// and pop do nothing.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Map a CUDA error to MP_ERR_CUDA (or MP_ERR_NOMEM) and record its text.
inline mp_status cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return MP_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? MP_ERR_NOMEM : MP_ERR_CUDA;
}

// Kernels index cells and edges of one mesh with 32-bit unsigned arithmetic:
// meshes with 2^31 edges or more are rejected.
inline bool mesh_too_large(int nx, int ny) {
    const long long edges = (long long)nx * (ny + 1) + (long long)(nx + 1) * ny;
    return edges >= (1LL << 31);
}

}  // namespace mp

#define MP_CUDA(call)                                                        \
    do {                                                                     \
        cudaError_t mp_e_ = (call);                                          \
        if (mp_e_ != cudaSuccess) return ::mp::cuda_status(mp_e_, #call);   \
    } while (0)

#define MP_TRY(call)                                                         \
    do {                                                                     \
        mp_status mp_s_ = (call);                                            \
        if (mp_s_ != MP_OK) return mp_s_;                                    \
    } while (0)

#endif
