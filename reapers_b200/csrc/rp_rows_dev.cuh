// Device pieces of the row-layout H.psi kernel shared with the batched
// kernel: the 2-D TMA tile load and the per-term row update.
#pragma once

#include <cuda.h>

#include "rp_common.cuh"
#include "rp_apply_rows.cuh"

namespace rp {

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int c0, int c1,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
        : "memory");
}

// The 128-byte row at shared address rq, chunk p from rq ^ (p << 4).
__device__ __forceinline__ void load_row(float4 (&w)[8], uint32_t rq) {
#pragma unroll
    for (int p = 0; p < 8; p++) {
        asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                     : "=f"(w[p].x), "=f"(w[p].y), "=f"(w[p].z), "=f"(w[p].w)
                     : "r"(rq ^ ((uint32_t)p << 4)));
    }
}

// One term over a whole row already loaded by load_row.  w[p] holds source
// chunk p ^ xq (the permutation is in the load address); case K = x0 | z0 << 1 | kind << 2.
// Output element u = EPC p + e takes source element e ^ x0 of w[p] with sign
// (chunk sign p) * (-1)^(z0 & (e ^ x0)).
template <typename Real, int K>
__device__ __forceinline__ void row_case(Cplx<Real> (&acc)[128 / sizeof(Cplx<Real>)],
                                         const float4 (&w)[8], Real c0, uint32_t jc) {
    constexpr int EPC = 16 / (int)sizeof(Cplx<Real>);
    constexpr int X0 = K & 1, Z0 = (K >> 1) & 1, KIND = K >> 2;
    if constexpr (EPC == 1 && (X0 || Z0)) {
        return;
    } else {
        const Real cn = -c0;
#pragma unroll
        for (int p = 0; p < 8; p++) {
            const Real cp = ((jc >> p) & 1u) ? cn : c0;
#pragma unroll
            for (int e = 0; e < EPC; e++) {
                const int se = e ^ X0;
                Real vx, vy;
                if constexpr (EPC == 2) {
                    vx = se ? w[p].z : w[p].x;
                    vy = se ? w[p].w : w[p].y;
                } else {
                    vx = __hiloint2double(__float_as_int(w[p].y), __float_as_int(w[p].x));
                    vy = __hiloint2double(__float_as_int(w[p].w), __float_as_int(w[p].z));
                }
                const Real c = (Z0 & se) ? -cp : cp;
                Cplx<Real> &a = acc[EPC * p + e];
                if (KIND == 0) {
                    a.x = fma(c, vx, a.x);
                    a.y = fma(c, vy, a.y);
                } else {
                    a.x = fma(-c, vy, a.x);
                    a.y = fma(c, vx, a.y);
                }
            }
        }
    }
}

// One term over one 16-byte chunk p of the row: w holds source chunk p ^ xq.
template <typename Real, int K>
__device__ __forceinline__ void chunk_term(Cplx<Real> (&acc)[128 / sizeof(Cplx<Real>)],
                                           const float4 &w, int p, Real c0, uint32_t jc) {
    constexpr int EPC = 16 / (int)sizeof(Cplx<Real>);
    constexpr int X0 = K & 1, Z0 = (K >> 1) & 1, KIND = K >> 2;
    const Real cp = ((jc >> p) & 1u) ? -c0 : c0;
#pragma unroll
    for (int e = 0; e < EPC; e++) {
        const int se = e ^ X0;
        Real vx, vy;
        if constexpr (EPC == 2) {
            vx = se ? w.z : w.x;
            vy = se ? w.w : w.y;
        } else {
            vx = __hiloint2double(__float_as_int(w.y), __float_as_int(w.x));
            vy = __hiloint2double(__float_as_int(w.w), __float_as_int(w.z));
        }
        const Real c = (Z0 & se) ? -cp : cp;
        Cplx<Real> &a = acc[EPC * p + e];
        if (KIND == 0) {
            a.x = fma(c, vx, a.x);
            a.y = fma(c, vy, a.y);
        } else {
            a.x = fma(-c, vy, a.x);
            a.y = fma(c, vx, a.y);
        }
    }
}

// One term over a whole row, its source row read from rq (see load_row)
// one 16-byte chunk at a time, each applied as it arrives: 4 live load
// registers per thread instead of 32, which keeps the kernel within the
// register budget of two 288-thread CTAs per SM without spills.
template <typename Real, int K>
__device__ __forceinline__ void chunk_case(Cplx<Real> (&acc)[128 / sizeof(Cplx<Real>)],
                                           uint32_t rq, Real c0, uint32_t jc) {
    constexpr int EPC = 16 / (int)sizeof(Cplx<Real>);
    if constexpr (EPC == 1 && ((K & 1) || ((K >> 1) & 1))) {
        return;
    } else {
#pragma unroll
        for (int p = 0; p < 8; p++) {
            float4 w;
            asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                         : "=f"(w.x), "=f"(w.y), "=f"(w.z), "=f"(w.w)
                         : "r"(rq ^ ((uint32_t)p << 4)));
            chunk_term<Real, K>(acc, w, p, c0, jc);
        }
    }
}

}  // namespace rp
