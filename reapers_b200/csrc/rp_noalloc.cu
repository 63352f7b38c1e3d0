// Inner product <a|b> that allocates no device memory.
//
// rp_vec_dot keeps its per-block partial sums in a buffer it obtains with
// cudaMalloc on first use.  Some callers cannot let a library allocate: a
// host framework that owns all device memory through its own allocator and
// forbids foreign cudaMalloc calls, or a latency-critical loop in which
// cudaMalloc / cudaFree would implicitly synchronise the device.  This
// variant keeps its scratch in a fixed file-scope device array instead.
//
// Scratch: NOALLOC_MAX_BLOCKS per-block partial pairs (re, im) plus the
// reduced result, 16 KB + 16 B, resident on every device that loads the
// library until the process exits.  The grid is a few blocks per SM (at most
// NOALLOC_MAX_BLOCKS), each block reducing one contiguous span of a multiple
// of 256 elements; vectors longer than NOALLOC_MAX_ELEMS (2^28 elements: a
// 28-qubit state) are rejected.
//
// All calls share the one array and it keeps the previous call's contents;
// every slot a call reads is written by that same call first.  Calls that
// overlap on the GPU (other streams or host threads) race on the array.
#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/rpb200.h"
#include "rp_common.cuh"

namespace rp {

constexpr int NOALLOC_MAX_BLOCKS = 1024;
constexpr uint64_t NOALLOC_MAX_ELEMS = 1ull << 28;
constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_BLOCKS_PER_SM = 4;

// partials[2 * b + {0, 1}] for block b, result at [2 * NOALLOC_MAX_BLOCKS + {0, 1}]
static __device__ __align__(256) double g_noalloc_scratch[2 * NOALLOC_MAX_BLOCKS + 2];

template <typename Real>
__global__ void __launch_bounds__(NOALLOC_THREADS)
    k_dot_blocks(uint64_t n, uint64_t span, const Cplx<Real> *a, const Cplx<Real> *b,
                 double *scratch) {
    __shared__ double s_re[NOALLOC_THREADS / 32], s_im[NOALLOC_THREADS / 32];
    const uint64_t lo = (uint64_t)blockIdx.x * span;
    const uint64_t hi = lo + span < n ? lo + span : n;
    double sr = 0.0, si = 0.0;
    for (uint64_t k = lo + threadIdx.x; k < hi; k += NOALLOC_THREADS) {
        const Cplx<Real> x = a[k], y = b[k];
        sr = fma((double)x.x, (double)y.x, fma((double)x.y, (double)y.y, sr));
        si = fma((double)x.x, (double)y.y, fma(-(double)x.y, (double)y.x, si));
    }
    sr = warp_sum(sr);
    si = warp_sum(si);
    if ((threadIdx.x & 31) == 0) {
        s_re[threadIdx.x >> 5] = sr;
        s_im[threadIdx.x >> 5] = si;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        CompSum re, im;
        for (int w = 0; w < NOALLOC_THREADS / 32; w++) {
            re.add(s_re[w]);
            im.add(s_im[w]);
        }
        scratch[2 * blockIdx.x] = re.value();
        scratch[2 * blockIdx.x + 1] = im.value();
    }
}

// Fixed-order compensated sum of the first nblocks partial pairs.
__global__ void k_dot_finish(int nblocks, double *scratch) {
    if (threadIdx.x != 0) return;
    CompSum re, im;
    for (int b = 0; b < nblocks; b++) {
        re.add(scratch[2 * b]);
        im.add(scratch[2 * b + 1]);
    }
    scratch[2 * NOALLOC_MAX_BLOCKS] = re.value();
    scratch[2 * NOALLOC_MAX_BLOCKS + 1] = im.value();
}

void set_error(int code, const std::string &msg);

}  // namespace rp

using namespace rp;

extern "C" int rp_vec_dot_noalloc(int dtype, uint64_t n, const void *a, const void *b,
                                  double *out) {
    // Device address of the scratch array for each device, looked up once
    // per device with that device current.  In host code the symbol itself
    // only names a host-side stand-in, never a device address.
    static std::mutex mu;
    static double *addr[64] = {nullptr};
    static int sms[64] = {0};
    try {
        RP_REQUIRE(dtype == RP_C64 || dtype == RP_C128, RP_E_INVALID,
                   "dtype must be RP_C64 (1) or RP_C128 (2)");
        RP_REQUIRE(a && b && out, RP_E_INVALID, "null pointer");
        RP_REQUIRE((((uintptr_t)a | (uintptr_t)b) & 15) == 0, RP_E_INVALID,
                   "vectors must be 16-byte aligned");
        RP_REQUIRE(n <= NOALLOC_MAX_ELEMS, RP_E_INVALID,
                   "rp_vec_dot_noalloc: vector length " + std::to_string(n) +
                       " exceeds the fixed scratch limit of " + std::to_string(NOALLOC_MAX_ELEMS) +
                       " elements");
        int dev = 0;
        RP_CUDA(cudaGetDevice(&dev));
        RP_REQUIRE(dev >= 0 && dev < 64, RP_E_INVALID, "device ordinal out of range");
        double *scratch;
        int nsm;
        {
            std::lock_guard<std::mutex> lk(mu);
            if (!addr[dev]) {
                void *p = nullptr;
                RP_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
                RP_CUDA(cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev));
                addr[dev] = static_cast<double *>(p);
            }
            scratch = addr[dev];
            nsm = sms[dev];
        }
        if (n == 0) {
            out[0] = out[1] = 0.0;
            return RP_OK;
        }
        // a few blocks per SM, each over a span of whole 256-element steps
        uint64_t want = (n + NOALLOC_THREADS - 1) / NOALLOC_THREADS;
        want = std::min<uint64_t>(want, (uint64_t)NOALLOC_BLOCKS_PER_SM * std::max(1, nsm));
        want = std::min<uint64_t>(want, NOALLOC_MAX_BLOCKS);
        uint64_t span = (n + want - 1) / want;
        span = (span + NOALLOC_THREADS - 1) / NOALLOC_THREADS * NOALLOC_THREADS;
        const int nblocks = (int)((n + span - 1) / span);
        // Ordered on the legacy default stream, like a caller's own work.
        if (dtype == RP_C128)
            k_dot_blocks<double><<<nblocks, NOALLOC_THREADS>>>(
                n, span, static_cast<const Cplx<double> *>(a), static_cast<const Cplx<double> *>(b),
                scratch);
        else
            k_dot_blocks<float><<<nblocks, NOALLOC_THREADS>>>(
                n, span, static_cast<const Cplx<float> *>(a), static_cast<const Cplx<float> *>(b),
                scratch);
        RP_CUDA(cudaGetLastError());
        k_dot_finish<<<1, 32>>>(nblocks, scratch);
        RP_CUDA(cudaGetLastError());
        RP_CUDA(cudaMemcpy(out, scratch + 2 * NOALLOC_MAX_BLOCKS, 2 * sizeof(double),
                           cudaMemcpyDeviceToHost));
        return RP_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    }
}
