// Shared definitions for the REAPERS B200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace rp {

// ---------------------------------------------------------------------------
// Complex element types stored in HBM: interleaved (re, im), 8 or 16 bytes.
// ---------------------------------------------------------------------------
template <typename Real> struct Cplx;
template <> struct alignas(8) Cplx<float> { float x, y; };
template <> struct alignas(16) Cplx<double> { double x, y; };

// ---------------------------------------------------------------------------
// Host-side error handling.  Every C-ABI entry point returns an int status
// and records a message retrievable with rp_last_error().
// ---------------------------------------------------------------------------
struct Error {
    int code;
    std::string msg;
};

void set_error(int code, const std::string &msg);

#define RP_CUDA(call)                                                              \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            throw ::rp::Error{-3, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
        }                                                                          \
    } while (0)

#define RP_REQUIRE(cond, code, msg)                                               \
    do {                                                                           \
        if (!(cond)) throw ::rp::Error{(code), (msg)};                             \
    } while (0)

// Device error word bits (set by kernels, read by the host after a sync).
enum DeviceError : unsigned {
    DEV_ERR_WAIT_TIMEOUT = 1u,   // an mbarrier wait ran out of iterations
    DEV_ERR_BOUNDS = 2u,         // a debug bounds check failed
};

// Upper bound on polling iterations of any device-side wait.  A correct
// kernel completes a wait in far fewer; a wait that gives up sets
// DEV_ERR_WAIT_TIMEOUT in the error word and the kernel winds down.
constexpr uint32_t WAIT_LIMIT = 1u << 26;

// ---------------------------------------------------------------------------
// PTX helpers: mbarrier + bulk asynchronous copies (no multicast anywhere).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on an mbarrier phase.  Returns false (and records the timeout
// in *err, when given) if the phase did not complete within `limit` polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity,
                                                  unsigned *err, uint32_t limit = WAIT_LIMIT) {
    for (uint32_t it = 0; it < limit; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
    }
    if (err) atomicOr(err, DEV_ERR_WAIT_TIMEOUT);
    return false;
}

// 1-D bulk copy global -> shared completing on an mbarrier (transaction
// bytes).  Both addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *smem_dst, const void *gsrc, unsigned bytes,
                                         uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(smem_dst)),
        "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// The same copy with an L2 eviction-priority hint (a createpolicy value):
// source tiles that many CTAs re-read stay in L2 ahead of streaming data.
__device__ __forceinline__ void bulk_g2s_hint(void *smem_dst, const void *gsrc, unsigned bytes,
                                              uint64_t *bar, uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1], %2, [%3], %4;" ::"r"(smem_u32(smem_dst)),
        "l"(gsrc), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

__device__ __forceinline__ uint64_t l2_policy_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// ---------------------------------------------------------------------------
// Reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Error-free transformation a + b = s + e (Knuth TwoSum).
__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e) {
    s = a + b;
    double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

// Compensated accumulator (Neumaier): value = hi + lo.
struct CompSum {
    double hi = 0.0, lo = 0.0;
    __device__ __forceinline__ void add(double v) {
        double s, e;
        two_sum(hi, v, s, e);
        hi = s;
        lo += e;
    }
    __device__ __forceinline__ double value() const { return hi + lo; }
};

// Compensated sum of v[0], v[stride], ..., v[(n-1) stride] by one warp: lane
// l sums the indices congruent to l mod 32, then the 32 (hi, lo) pairs meet
// in a butterfly.  TwoSum's error term is exact whatever the operand order,
// so every lane ends with the same bits and the result is the same run to run.
__device__ __forceinline__ double warp_compsum(const double *v, int n, size_t stride) {
    const int lane = threadIdx.x & 31;
    CompSum c;
    for (int g = lane; g < n; g += 32) c.add(v[(size_t)g * stride]);
    double hi = c.hi, lo = c.lo;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ohi = __shfl_xor_sync(0xffffffffu, hi, o);
        const double olo = __shfl_xor_sync(0xffffffffu, lo, o);
        double sm, e;
        two_sum(hi, ohi, sm, e);
        hi = sm;
        lo = (lo + olo) + e;
    }
    return hi + lo;
}

}  // namespace rp
