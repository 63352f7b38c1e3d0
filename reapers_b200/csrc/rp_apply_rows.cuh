// Row-layout H.psi kernel (second generation): host-side table and launch.
#pragma once

#include <cuda.h>

#include <vector>

#include "rp_common.cuh"

namespace rp {

// A source/output tile is 256 rows of 128 bytes = 8 chunks of 16 bytes (16
// complex64 or 8 complex128 elements per row); consumer thread t owns output
// row t.  For a term with in-tile X part xl = (xr, xq, x0) -- row, chunk and
// element-in-chunk XOR -- output element (t, p, e) reads (t ^ xr, p ^ xq,
// e ^ x0).  cs packs xr (bits 0-7), xq (bits 8-10) and the code case
// x0 | z0 << 1 | kind << 2 (bits 11-13), z0 being the element-in-chunk bit of
// the Z mask.  js: bit p = parity(zq & (p ^ xq)), the chunk-dependent part of
// the sign (zq = chunk bits of z).  kind 0: real coefficient, 1: imaginary.
template <typename Real>
struct alignas(16) RowTerm {
    uint32_t cs, z, js;
    float cf;      // coefficient, FP32 kernels
    double cd;     // coefficient, FP64 kernels
    double pad;
};
static_assert(sizeof(RowTerm<float>) == 32, "layout");

struct alignas(16) RowGroup {
    uint32_t xh, first, count, pad;
};

// A real-coefficient Z string (X mask 0) folded into the per-row diagonal
// factor: zhi = z >> logC, the Z bits above the in-row element bits; the
// terms are bucketed by z & (C - 1), their in-row Z bits.
struct alignas(16) RowDiag {
    uint32_t zhi;
    float cf;      // coefficient, FP32 kernels
    double cd;     // coefficient, FP64 kernels
};
static_assert(sizeof(RowDiag) == 16, "layout");

struct RowPlan {
    bool ok = false;          // the row kernel applies to this Hamiltonian
    int B = 0, logC = 0;      // tile exponent, log2(elements per row)
    int ntiles = 0;
    int nterms = 0;           // after splitting complex coefficients
    std::vector<RowTerm<float>> terms;
    std::vector<RowGroup> groups;
    void *d_terms = nullptr;
    RowGroup *d_groups = nullptr;
    // fused diagonal: real Z strings summed per row (group 0 is then the
    // source tile x >> B == 0, the output's own tile)
    int ndiag = 0;
    std::vector<RowDiag> diag;          // by bucket z & (C - 1)
    std::vector<uint32_t> dstart;       // C + 1 bucket offsets into diag
    RowDiag *d_diag = nullptr;
    uint32_t *d_dstart = nullptr;
    int window = 0;           // CTAs of an aligned tile window (grid size)
    double alg_bytes_smem = 0;  // (G + 1) D s, G = distinct x >> B
    double alg_bytes_dram = 0;  // (G_w + 1) D s, G_w = distinct x >> (B + log2 window)
};

// Largest Hamiltonian (terms after splitting, groups) the row kernel stages
// in shared memory.
constexpr int ROW_MAX_TERMS = 2048;
constexpr int ROW_MAX_GROUPS = 1024;
// Fewest real Z strings worth the fused diagonal (below it they stay terms).
constexpr int ROW_DIAG_MIN = 4;
// RowTerm::cs bit (fused-diagonal plans): this term has the previous term's
// full X mask and case (bits 0-7 source row offset, 8-10 chunk permutation,
// 11-13 case), so it is applied to the row already loaded for that term.
constexpr uint32_t ROW_SAME_SRC = 1u << 14;

// any_len: build the table for any len >= the tile exponent (the batched
// kernel); otherwise only for states of at least 128 tiles.  fuse_diag: fold
// the real Z strings into the per-row diagonal factor (single-state kernel).
void rowplan_build(RowPlan &rp, int len, int dtype, const uint64_t *bits, const double *coeff,
                   int64_t nterms, bool any_len = false, bool fuse_diag = false);
void rowplan_upload(RowPlan &rp);
void rowplan_free(RowPlan &rp);

struct RowLaunch {
    const void *in = nullptr;
    void *out = nullptr;
    double alpha = 1.0;
    const double *alpha_dev = nullptr;
    int accumulate = 0;
    const int *active = nullptr;
    const void *const *dot_vecs = nullptr;
    int ndot = 0;
    double *partials = nullptr;   // [grid][ndot][2]
    unsigned *err = nullptr;
    // output tiles [tile0, tile0 + tile_count) only (tile_count 0: all);
    // every source tile stays readable
    uint32_t tile0 = 0, tile_count = 0;
    // sharded input (in unused): shards[i], i < 2^shard_bits, holds input
    // elements [i 2^(len-shard_bits), (i+1) 2^(len-shard_bits)); out is
    // output shard shard_rank
    const void *const *shards = nullptr;
    int shard_bits = 0, shard_rank = 0;
};

constexpr int ROW_MAX_SHARDS = 8;

void rows_launch(const RowPlan &rp, int len, int dtype, const RowLaunch &l, cudaStream_t st);

// Failure-path test hook: the next row-kernel launch withholds the tile copy
// of producer iteration `iteration` in CTA 0 and gives every pipeline wait
// `polls` polls, so that CTA's waits give up and it winds down (error word
// DEV_ERR_WAIT_TIMEOUT) while the other CTAs finish.  One launch only.
void rows_test_withhold(long iteration, uint32_t polls);

// 2-D TMA map of a state of 2^len elements at base (rows of 128 bytes, one
// 256-row tile per box, 128-byte swizzle).
CUtensorMap make_row_map(const void *base, int len, int dtype);

}  // namespace rp
