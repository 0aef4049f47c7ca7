// Shared-memory pipeline primitives of the TMA-fed step kernels
// (stencil_tile.cu, stencil_slab.cu): mbarrier wrappers with bounded waits,
// the 4-D tiled tensor copy global -> shared (no multicast), the named
// barrier of the compute warps, and tensor-map encoding through the driver
// entry point.
#pragma once
#include "fitb_common.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdlib>
#include <cstring>

namespace fitb {
namespace tma {

constexpr unsigned kWaitLimit = 1u << 22;  // tries of one bounded mbarrier wait
constexpr int TK = 32;                      // cells per tile row: one warp

__device__ __forceinline__ unsigned saddr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void bar_expect(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(bar)) : "memory");
}

__device__ __forceinline__ bool bar_try(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false after kWaitLimit unsuccessful tries.
__device__ __forceinline__ bool bar_wait(unsigned long long* bar, unsigned parity) {
    for (unsigned n = 0; n < kWaitLimit; ++n)
        if (bar_try(bar, parity)) return true;
    return false;
}

// 4-D tiled tensor copy global -> shared completing on `bar`; c0 (the
// innermost coordinate) must keep the copy's start 16-byte aligned.
__device__ __forceinline__ void load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                        unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(saddr(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(saddr(bar))
        : "memory");
}

// Named barrier 1 among the CTA's `nthreads` compute threads.
__device__ __forceinline__ void compute_barrier(int nthreads) {
    asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

inline PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// L2 fill size of the tensor copies' misses: none (the sectors a box
// touches) unless the environment variable FITB_TMA_L2_PROMOTION says 64,
// 128 or 256 (read once per process; a tuning switch, every value computes
// the same bits).  Measured on the 256^3 slab step: 256-byte fills read
// 966 MB per step from DRAM in the CPML-free list against 901 MB without,
// and the step took 4 % longer.
inline CUtensorMapL2promotion l2_promotion() {
    static const CUtensorMapL2promotion v = [] {
        const char* e = std::getenv("FITB_TMA_L2_PROMOTION");
        if (!e) return CU_TENSOR_MAP_L2_PROMOTION_NONE;
        if (!std::strcmp(e, "64")) return CU_TENSOR_MAP_L2_PROMOTION_L2_64B;
        if (!std::strcmp(e, "128")) return CU_TENSOR_MAP_L2_PROMOTION_L2_128B;
        if (!std::strcmp(e, "256")) return CU_TENSOR_MAP_L2_PROMOTION_L2_256B;
        return CU_TENSOR_MAP_L2_PROMOTION_NONE;
    }();
    return v;
}

// 4-D tiled map: dims d0..d3 (d0 innermost), byte strides of d1..d3, box
// b0..b3; no interleave, no swizzle, zero fill outside the dims.
inline bool encode_4d(CUtensorMap* out, CUtensorMapDataType dt, const void* base, const unsigned long long dims[4],
                      const unsigned long long strides[3], const unsigned box[4]) {
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t d[4] = {dims[0], dims[1], dims[2], dims[3]};
    const cuuint64_t s[3] = {strides[0], strides[1], strides[2]};
    const cuuint32_t b[4] = {box[0], box[1], box[2], box[3]};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return fn(out, dt, 4, const_cast<void*>(base), d, s, b, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, l2_promotion(),
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// 4-D map over the padded field layout: (k, j, plane, component) with
// `ncomp` components of `vol` elements; box (bk, bj, 1, bc).
template <typename T>
bool encode_field_map(CUtensorMap* out, const void* base, const Geom& g, int ncomp, int bk, int bj, int bc = 3) {
    const unsigned long long dims[4] = {(unsigned long long)g.nkp, (unsigned long long)g.njp,
                                        (unsigned long long)(g.nx + 4), (unsigned long long)ncomp};
    const unsigned long long strides[3] = {(unsigned long long)g.sj * sizeof(T), (unsigned long long)g.si * sizeof(T),
                                           (unsigned long long)g.vol * sizeof(T)};
    const unsigned box[4] = {(unsigned)bk, (unsigned)bj, 1, (unsigned)bc};
    return encode_4d(out, sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, base,
                     dims, strides, box);
}

}  // namespace tma
}  // namespace fitb
