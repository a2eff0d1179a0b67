// Debug-build instrumentation.
//
// SIMP_CHECK_BOUNDS: device-side index checks.  A check that fails sets a bit
// of its translation unit's flag word (which index: SITE_*) and the access is
// skipped; nothing traps.  The host collects the words of every unit after
// each right-hand side or step (take_bounds_flags, abi.cu) and the entry
// point returns SIMP_ERR_BOUNDS.  Without the macro every check is `true` and
// the code is the production code.
//
// SIMP_NVTX: NVTX ranges around each pass launch, the re-sort and the entry
// points (host side; a captured step graph's replays fall under the range of
// the simp_gpu_step call that replays them).
#pragma once

#include <cuda_runtime.h>

namespace simp {

enum : unsigned {
    SITE_NEIGHBOUR = 1u,   // a neighbour index from a Verlet or pair list
    SITE_CELL = 2u,        // a cell key of the stencil walk
    SITE_SORT = 4u,        // a slot of the counting sort
    SITE_TILE = 8u,        // a shared-memory slot of the tiled passes
};

// Registers a reader of one translation unit's flag word (returns and
// clears it); every unit built with the checks registers one at load time.
int register_bounds_reader(unsigned (*take)());
// OR of every unit's flag word since the last call (0 without the checks).
unsigned take_bounds_flags();

}  // namespace simp

#ifdef SIMP_CHECK_BOUNDS
namespace {
__device__ unsigned g_simp_bounds = 0u;

__device__ __forceinline__ bool simp_in_range(long long v, long long lo, long long hi, unsigned site) {
    if (v >= lo && v < hi) return true;
    atomicOr(&g_simp_bounds, site);
    return false;
}

unsigned simp_take_bounds_word() {
    unsigned v = 0u, z = 0u;
    if (cudaMemcpyFromSymbol(&v, g_simp_bounds, sizeof(v)) != cudaSuccess) return ~0u;
    cudaMemcpyToSymbol(g_simp_bounds, &z, sizeof(z));
    return v;
}

const int g_simp_bounds_registered = simp::register_bounds_reader(&simp_take_bounds_word);
}  // namespace
#define SIMP_IN_RANGE(v, lo, hi, site) simp_in_range((long long)(v), (long long)(lo), (long long)(hi), (site))
#else
#define SIMP_IN_RANGE(v, lo, hi, site) true
#endif

#ifdef SIMP_NVTX
#include <nvtx3/nvToolsExt.h>
namespace simp {
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};
}  // namespace simp
#define SIMP_RANGE_CAT2(a, b) a##b
#define SIMP_RANGE_CAT(a, b) SIMP_RANGE_CAT2(a, b)
#define SIMP_RANGE(name) ::simp::NvtxRange SIMP_RANGE_CAT(simp_nvtx_range_, __LINE__)(name)
#else
#define SIMP_RANGE(name) ((void)0)
#endif
