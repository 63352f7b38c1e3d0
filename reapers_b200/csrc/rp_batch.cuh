// Batched OTOC: many independent (disorder realisation, random state)
// problems, uneven qubit counts, one persistent launch per time step.
#pragma once

#include <vector>

#include "rp_apply.cuh"

namespace rp {

// One problem as the persistent kernel reads it (FP32 state, FP64 Krylov).
struct alignas(16) BatchProblem {
    const TermDesc<float> *terms;   // grouped by x >> B (tiled-kernel records)
    const GroupDesc *groups;
    const Cplx<float> *psi0;        // initial state (device)
    const RowTerm<float> *rterms;   // row-kernel records (rows != 0)
    const RowGroup *rgroups;
    int len, B, ntiles, ngroups;
    int rows, rnterms, rngroups, pad;   // H.psi by 2-D TMA row tiles when rows != 0
    uint32_t wx, wz, vx, vz;        // W and V Pauli strings (X, Z masks)
    float wcr, wci, vcr, vci;       // their coefficients
};

// Problems sharing a team size: one persistent launch per time step, teams
// (clusters of `team` CTAs) of which `nslots` are resident.
struct BatchClass {
    int team = 1, first = 0, count = 0, nslots = 0, maxB = 8, maxlen = 0;
    int maxrt = 0, maxrg = 0;                // largest row-kernel term / group lists
    bool any_rows = false, any_tiled = false;
    size_t smem = 0, ws_stride = 0, vec_stride = 0;
    int map_base = 0;                        // first TMA map of this class's slots
};

struct BatchPlan {
    int nprob = 0, krydim = 0, max_restarts = 0, hcap = 0;
    double tol = 0;
    std::vector<BatchClass> classes;         // in launch order
    std::vector<ApplyPlan> plans;            // per problem (host tables + device copies)
    std::vector<RowPlan> rplans;             // per problem: row-kernel tables (when used)
    CUtensorMap *maps = nullptr;             // [class slots][vector] 2-D TMA maps of the workspaces
    std::vector<BatchProblem> probs;         // device-pointer records, by class, largest first
    std::vector<int> order;                  // probs[i] is problem order[i]
    BatchProblem *d_probs = nullptr;
    void *ws = nullptr;                      // per-team workspaces (shared by the classes)
    int *counter = nullptr;                  // work queue heads [class][time index]
    double *F = nullptr;                     // [nprob][ntimes][2]
    int *applies = nullptr;                  // [nprob][ntimes]
    unsigned *err = nullptr;
    int ntimes_cap = 0;
    cudaGraphExec_t graph = nullptr;
    std::vector<double> graph_times;
};

// Problem p: len[p] qubits, nterms[p] terms (bits, coeff as for rp_ham_create),
// W and V single strings, psi0[p] a device complex64 vector, tile[p] the tile
// exponent (8..11, 0 = default) of the bulk-copy tile loop, team[p] the CTAs
// per problem (1, 2, 4, 8 or 16; 0 = default); tile and team may be null.
// Tile 12 selects the row-tile loop (2-D TMA, 4096-element swizzled tiles)
// for states of at least 2^12 elements.
void batch_build(BatchPlan &bp, int nprob, const int *len, const int64_t *nterms,
                 const uint64_t *const *bits, const double *const *coeff, const uint64_t *wbits,
                 const double *wcoeff, const uint64_t *vbits, const double *vcoeff,
                 const void *const *psi0, const int *tile, const int *team, int krydim,
                 double tol, int max_restarts, cudaStream_t st);
void batch_free(BatchPlan &bp);

// F[p][k] = <psi0| W(t_k) V W(t_k) V |psi0> for every problem; one persistent
// launch per time step and team size, captured once into a CUDA graph when
// use_graph.
void batch_otoc(BatchPlan &bp, int ntimes, const double *times, double *F_host,
                int *applies_host, int use_graph, cudaStream_t st);

// One launch of `napplies` H.psi products per problem (no Krylov); returns
// the device time in ms.  Used to tune the tile exponents.
double batch_probe(BatchPlan &bp, int napplies, cudaStream_t st);

}  // namespace rp
