// H.psi for a sum of Pauli strings: host plan and launch interface.
#pragma once

#include <vector>

#include "rp_apply_rows.cuh"
#include "rp_common.cuh"

namespace rp {

// One Pauli term as the kernels read it.  The output tile exponent B splits an
// index n into a tile number (n >> B) and an in-tile offset; the consumer
// thread t in [0, P) owns offsets t + P*j, j in [0, E).
//   xl    : low B bits of the X mask (in-tile permutation)
//   z     : full Z mask
//   jsign : bit j = parity(z_j & (j ^ xl_j)), the j-dependent part of the sign,
//           z_j / xl_j being the bits of z / xl in the j field [log2 P, B)
//   kind  : 0 real coefficient, 1 imaginary coefficient, 2 general complex
// Records are 16-byte aligned (the kernel reads the four words as one uint4).
template <typename Real>
struct alignas(16) TermDesc {
    uint32_t xl, z, jsign, kind;
    Real cr, ci;
};
static_assert(sizeof(TermDesc<float>) == 32 && sizeof(TermDesc<double>) == 32, "layout");

// A group of terms sharing the same high X-mask part xh = x >> B: they all
// read the source tile (tile ^ xh).
struct alignas(16) GroupDesc {
    uint32_t xh, first, count, pad;
};

enum CoeffKind : uint32_t { COEFF_REAL = 0, COEFF_IMAG = 1, COEFF_COMPLEX = 2 };

// Kernel configuration chosen for a (length, precision) pair.
struct ApplyConfig {
    int B = 0;        // tile exponent
    int P = 0;        // consumer threads per CTA
    int stages = 0;   // shared-memory pipeline depth
    bool direct = false;   // tiny vectors: one thread per element, no tiling
    bool allow_rows = true;   // use the row-layout kernel when it applies
};

// Host copy of a grouped term table plus its device image.
struct ApplyPlan {
    int len = 0;
    int dtype = 0;
    ApplyConfig cfg;
    int ntiles = 0;
    int ngroups = 0;
    int nterms = 0;
    std::vector<GroupDesc> groups;
    std::vector<uint8_t> term_bytes;   // TermDesc<Real> records
    void *d_terms = nullptr;
    GroupDesc *d_groups = nullptr;
    // direct-kernel table: x, z, coefficient per term (list order)
    void *d_direct = nullptr;
    double alg_bytes = 0;   // (ngroups + 1) * D * sizeof(element): one read of
                            // every distinct source tile per output tile + the write
    RowPlan rows;           // row-layout kernel (used when rows.ok)
};

// Build the grouped table for the given configuration (host only; no GPU).
void plan_build(ApplyPlan &plan, int len, int dtype, const uint64_t *bits,
                const double *coeff, int64_t nterms, const ApplyConfig &cfg);

// Default configuration for a length and precision.
ApplyConfig default_config(int len, int dtype);

void plan_upload(ApplyPlan &plan);
void plan_free(ApplyPlan &plan);

// Arguments of one apply launch.
struct ApplyLaunch {
    const void *in = nullptr;
    void *out = nullptr;
    double alpha = 1.0;                 // out = alpha * (*alpha_dev) * H in
    const double *alpha_dev = nullptr;  // optional device scale factor
    int accumulate = 0;                 // out += ... instead of out = ...
    const int *active = nullptr;        // optional device flag: skip when 0
    // fused projections <u_i | out>, i < ndot (Krylov first pass)
    const void *const *dot_vecs = nullptr;   // device array of device pointers
    int ndot = 0;
    double *partials = nullptr;   // [grid][ndot][2] compensated-summed per CTA
    unsigned *err = nullptr;      // device error word
    // row kernel only: output tiles [tile0, tile0 + tile_count) of
    // 2^plan.rows.B elements (tile_count 0: the whole state)
    uint32_t tile0 = 0, tile_count = 0;
    // row kernel only: the input split into 2^shard_bits shards (in unused),
    // out = output shard shard_rank; see RowLaunch
    const void *const *shards = nullptr;
    int shard_bits = 0, shard_rank = 0;
};

// Grid size used for a plan (persistent CTAs); the partials buffer of a fused
// launch needs grid * ndot * 2 doubles.
int apply_grid(const ApplyPlan &plan);

void apply_launch(const ApplyPlan &plan, const ApplyLaunch &a, cudaStream_t stream);

int num_sms();

}  // namespace rp
