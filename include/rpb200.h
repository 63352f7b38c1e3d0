/*
 * rpb200.h -- C ABI of the REAPERS B200 hot path (librpb200.so).
 *
 * Plain pointers and sizes only.  Every function returns 0 on success or a
 * negative status (RP_E_*); rp_last_error() returns the message of the last
 * failure on the calling thread.  Vectors are device pointers to interleaved
 * complex numbers (RP_C64: float re/im, 8 bytes; RP_C128: double re/im, 16
 * bytes), 16-byte aligned, of length 2^len.  All calls are ordered on the
 * library's stream (rp_stream()), a blocking stream and therefore ordered
 * with the legacy default stream both ways; calls that return a scalar or
 * copy to the host synchronise it, matching the synchronous semantics of the
 * reference's GPUImpl (inc/gpuimpl.h:628-638).
 *
 * Each entry point names the reference interface it replaces (paths inside
 * cl91/REAPERS).
 */
#ifndef RPB200_H
#define RPB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RP_C64 1  /* complex<float>  */
#define RP_C128 2 /* complex<double> */

#define RP_OK 0
#define RP_E_INTERNAL -1
#define RP_E_INVALID -2   /* InvalidArgument (inc/except.h:101-118) */
#define RP_E_CUDA -3      /* CudaError (inc/except.h:131-140) */
#define RP_E_NOMEM -4     /* DevOutOfMem (inc/except.h:162-170) */
#define RP_E_DEVICE -5    /* a device-side wait gave up (kernel error word) */
#define RP_E_NODEVICE -6  /* NoGpuDevice (inc/except.h:143-149) */

typedef struct rp_ham *rp_ham_t;

/* Per-Hamiltonian plan of the H.psi kernel. */
typedef struct {
    int len;             /* spin chain length */
    int dtype;           /* RP_C64 or RP_C128 */
    int nterms;          /* Pauli strings */
    int tile_exp;        /* B: output tile of 2^B elements (0: direct kernel) */
    int ngroups;         /* distinct high X-mask parts x >> B */
    int threads;         /* consumer threads per CTA */
    int stages;          /* shared-memory pipeline depth */
    int grid;            /* persistent CTAs */
    double alg_bytes;    /* (ngroups + 1) * 2^len * element size per apply */
    int kernel;          /* 0 direct, 1 tiled (bulk copies), 2 rows (TMA, swizzled) */
    int window;          /* CTAs in flight = aligned block of output tiles */
    double alg_bytes_dram; /* (G_w + 1) * 2^len * element size, G_w = distinct
                              x >> (tile_exp + log2 window): the compulsory DRAM
                              bytes when source blocks are served from L2 */
    double smem_bytes;   /* bytes moved through shared memory per apply: one
                            element per source-row load (a term after
                            splitting complex coefficients, less the terms
                            that reuse the previous term's row, the fused
                            diagonal counting as one) and output element,
                            plus every staged source tile */
    int nreads;          /* source-row loads per output element */
    int diag_terms;      /* real Z strings summed into the row kernel's per-row
                          * diagonal factor (0: none, or fewer than 4) */
} rp_ham_info_t;

/* Statistics of one evolve. */
typedef struct {
    int restarts;        /* Arnoldi cycles */
    int applies;         /* H.psi products */
    int passes;          /* orthogonalisation passes */
    int prods;           /* inner products the reference's MGS would take */
    int breakdown;       /* 1 if an invariant subspace ended the evolve */
    double last_err;     /* ||Hexp0|| of the final cycle */
} rp_evolve_stats_t;

/* --- context ------------------------------------------------------------ */
/* Select the device and create the stream.  Replaces the static-init
 * GPUContext (inc/gpuimpl.h:496-559); called lazily by every entry point.
 * A process stays bound to its first device: rp_init with another device
 * returns RP_E_INVALID, also after rp_shutdown. */
int rp_init(int device);
/* Release cached workspaces, scratch buffers and the stream (a later call
 * allocates them afresh on the same device). */
int rp_shutdown(void);
const char *rp_last_error(void);
/* GPUImpl::get_device_count (inc/gpuimpl.h:590-592). */
int rp_device_count(int *count);
/* The cudaStream_t all calls are ordered on. */
void *rp_stream(void);
/* Wait for the stream.  Like GPUImpl::sync_device's error peek
 * (inc/gpuimpl.h:634-638): returns RP_E_DEVICE if a pipeline wait of an
 * asynchronous rp_apply / rp_apply_shard gave up since the last check
 * (that product's output is incomplete), and clears the report. */
int rp_synchronize(void);

/* --- memory (DeviceVec, inc/gpuimpl.h:405-494) -------------------------- */
int rp_alloc(void **ptr, size_t bytes);
int rp_free(void *ptr);
/* kind: 0 host->device, 1 device->host, 2 device->device. */
int rp_memcpy(void *dst, const void *src, size_t bytes, int kind);

/* --- vector operations (GPUImpl BLAS-1, inc/gpuimpl.h:853-1002) -------- */
/* GPUImpl::zero_vec */
int rp_vec_zero(int dtype, uint64_t n, void *v);
/* GPUImpl::copy_vec, same precision and float<->double (rounds to nearest,
 * as CPUImpl::copy_vec does; the reference GPU kernel krnl_dtof_vec rounds
 * toward zero, src/krnl.cu:31-39) */
int rp_vec_copy(int dtype_dst, void *dst, int dtype_src, const void *src, uint64_t n);
/* GPUImpl::add_vec(v0, s, v1): y += (ar + i ai) x */
int rp_vec_axpy(int dtype, uint64_t n, void *y, double ar, double ai, const void *x);
/* GPUImpl::add_vec(res, v0, v1): res = a + b */
int rp_vec_add(int dtype, uint64_t n, void *res, const void *a, const void *b);
/* GPUImpl::scale_vec: v *= (ar + i ai) */
int rp_vec_scale(int dtype, uint64_t n, void *v, double ar, double ai);
/* GPUImpl::vec_prod: out[0] + i out[1] = <a|b> (conjugate-linear in a),
 * FP64 compensated accumulation */
int rp_vec_dot(int dtype, uint64_t n, const void *a, const void *b, double *out);
/* The same inner product as rp_vec_dot to FP64 rounding (the reduction
 * order differs, so the bits may too), but allocates no device memory: for
 * callers that cannot let a library call cudaMalloc (a framework that owns
 * all device memory through its own allocator, or a loop in which
 * cudaMalloc / cudaFree would implicitly synchronise the device).  No
 * counterpart in the reference.  Its scratch is a fixed 16 KB device array
 * (up to 1024 per-block partial sums); n may be at most 2^28 (larger n
 * returns RP_E_INVALID with a message); a and b 16-byte aligned, as for
 * every vector entry point.
 * The first call on each device looks up the array's device address; make
 * that first call before any stream capture.  All calls share the array:
 * calls that overlap on the GPU race.  Runs on the legacy default stream. */
int rp_vec_dot_noalloc(int dtype, uint64_t n, const void *a, const void *b, double *out);
/* GPUImpl::vec_norm */
int rp_vec_norm(int dtype, uint64_t n, const void *v, double *out);
/* GPUImpl::init_random without the normalisation: i.i.d. complex Gaussian
 * entries from a counter-based generator (deterministic per seed). */
int rp_vec_random(int dtype, uint64_t n, void *v, uint64_t seed);

/* --- Hamiltonian (DevSumOps, inc/gpuimpl.h:124-397, upload :1065-1085) -- */
/* terms: bits[k] in SpinOp's encoding (bit 2i = X on site i, bit 2i+1 = Z,
 * sigma_y stored as X|Z with the factor i in the coefficient, inc/ops.h:
 * 138-143, 285-288); coeff[2k], coeff[2k+1] = stored coefficient.  Equal
 * bit strings are summed by the caller (HostSumOps::operator+=,
 * inc/cpuimpl.h:233-253).  The table is grouped for the kernel here. */
int rp_ham_create(rp_ham_t *h, int len, int dtype, uint64_t nterms, const uint64_t *bits,
                  const double *coeff);
/* Same with an explicit tile exponent (5..12) for the tiled kernel, for
 * tuning and testing; 0 = default (the row kernel where it applies). */
int rp_ham_create_ex(rp_ham_t *h, int len, int dtype, uint64_t nterms, const uint64_t *bits,
                     const double *coeff, int tile_exp);
int rp_ham_destroy(rp_ham_t h);
int rp_ham_info(rp_ham_t h, rp_ham_info_t *info);

/* --- hot path ------------------------------------------------------------ */
/* GPUImpl::apply_ops (src/krnl.cu:220-257): out = H in, or out += H in when
 * accumulate != 0.  in and out must differ. */
int rp_apply(rp_ham_t h, void *out, const void *in, int accumulate);
/* Test hook of the failure path, no counterpart in the reference: the next
 * row-kernel launch (states of at least 2^19 complex64 / 2^18 complex128
 * elements) withholds the tile copy of producer iteration `iteration` in its
 * first CTA and gives every pipeline wait `wait_polls` polls (1024 to
 * 2^26).  That CTA's consumers wait on a barrier that nothing completes,
 * give up, let the copies in flight land and return; the other CTAs finish.
 * The next rp_synchronize returns RP_E_DEVICE and the context stays usable.
 * Applies to one launch. */
int rp_test_withhold_tile(int64_t iteration, uint32_t wait_polls);
/* out_host[i] = H in_host[i] for i < n: n states in HOST memory (2^len
 * elements of the Hamiltonian's precision each; pinned memory lets the
 * copies run asynchronously).  Pipelined over two device buffer pairs kept by
 * the library: the copy of state i+1 to the device and of result i-1 to the
 * host overlap H.psi on state i.  With the row kernel on large states
 * (two or more CTA windows of output tiles: 2^22 complex64 or 2^21
 * complex128 elements on a 148-SM B200) each product runs as up to 8
 * launches over consecutive output ranges, and each range is copied back as
 * soon as it is written.  Returns
 * when every result is on the host.
 * No reference counterpart: the reference applies one resident state. */
int rp_apply_host(rp_ham_t h, int n, const void *const *in_host, void *const *out_host);

/* The reference's multi-GPU apply (src/krnl.cu:96-114 with the split of
 * inc/gpuimpl.h:426-432): the state is split by its top shard_bits qubits
 * into 2^shard_bits shards of 2^(len-shard_bits) elements; shards[i] is a
 * device pointer to input shard i readable from this device (this GPU's
 * memory, or a peer's opened with rp_ipc_open), and out (2^(len-shard_bits)
 * elements) becomes output shard shard_rank of H in, or += with accumulate.
 * One launch of the row kernel: its TMA loads fetch every source tile from
 * the shard that holds it, over NVLink for a peer's.  1 <= shard_bits <= 3;
 * needs the row kernel (2^19+ complex64 or 2^18+ complex128 elements) with
 * at least one 2^12 (complex64) or 2^11 (complex128) element tile per shard.
 * The caller orders it: every shard final before the call (a barrier across
 * ranks), and no input shard rewritten until every rank's call has ended. */
int rp_apply_shard(rp_ham_t h, int shard_bits, int shard_rank, const void *const *shards,
                   void *out, int accumulate);

/* One process per GPU in place of the reference's in-process peer access
 * (inc/gpuimpl.h:524-538): a device pointer exported as the CUDA IPC handle
 * of its allocation plus its offset, opened in another process (peer access
 * enabled lazily) and closed there. */
typedef struct {
    unsigned char handle[64];
    uint64_t offset;
} rp_ipc_handle_t;
int rp_ipc_export(const void *ptr, rp_ipc_handle_t *out);
int rp_ipc_open(const rp_ipc_handle_t *h, void **ptr);
int rp_ipc_close(void *ptr);

/* Krylov<Impl>::evolve (inc/algo.h:267-365) as called by State::evolve
 * (inc/state.h:415-424): psi <- exp(-(beta + i t) H) psi in place, restarted
 * Arnoldi with krydim basis vectors, stop when ||Hexp0|| < tol, on breakdown,
 * or after max_iters restarts (0 = no limit).  t == 0 and beta == 0 returns
 * immediately, as State::evolve does.  stats may be NULL. */
int rp_evolve(rp_ham_t h, void *psi, double t, double beta, int krydim, double tol,
              int max_iters, rp_evolve_stats_t *stats);

/* Free the cached Krylov workspace (krydim + 2 vectors) and the device
 * buffers of rp_apply_host. */
int rp_workspace_release(void);

/* --- exact diagonalisation (the dense GPU path: DevSumOps::get_matrix,
 * get_eigensystem and _matexp, inc/gpuimpl.h:1180-1263, GPUImpl::mat_mul;
 * used by ExactDiagonalization, inc/algo.h:29-54) ------------------------- */
typedef struct rp_dense *rp_dense_t;
/* The dense matrix of a Hermitian Pauli sum on len <= 15 qubits (same term
 * arguments as rp_ham_create), built on the device from the term table, and
 * its eigensystem (library eigensolver, heevd, in the dtype's precision):
 * eigenvalues ascending, eigenvectors the columns of a dim x dim matrix. */
int rp_dense_create(rp_dense_t *d, int len, int dtype, uint64_t nterms, const uint64_t *bits,
                    const double *coeff);
/* evals: 2^len doubles, ascending. */
int rp_dense_eigenvalues(rp_dense_t d, double *evals);
/* *mat = the device eigenvector matrix (2^len x 2^len, column-major, the
 * dtype; owned by d, valid until rp_dense_destroy). */
int rp_dense_eigenvectors(rp_dense_t d, void **mat);
/* out (device vector, 2^len elements of the dtype) = eigenvector `index`:
 * the eigensystem column copy of ExactDiagonalization::ground_state. */
int rp_dense_eigenvector(rp_dense_t d, int64_t index, void *out);
/* out (device, 2^len x 2^len, column-major, the dtype) = exp((cr + i ci) H)
 * = V diag(exp((cr + i ci) lambda)) V^H (DevSumOps::_matexp). */
int rp_dense_expm(rp_dense_t d, double cr, double ci, void *out);
int rp_dense_destroy(rp_dense_t d);
/* res = mat vec for a dense dim x dim column-major device matrix
 * (GPUImpl::mat_mul, inc/gpuimpl.h:1012-1021): FP64 accumulation, fixed
 * summation order; res and vec distinct; dim at most 2^16. */
int rp_mat_vec(int dtype, uint64_t dim, const void *mat, const void *vec, void *res);

/* --- time-stepped Krylov primitives (no reference counterpart: the
 * reference only has the restarted evolve; these let a step controller
 * advance exp(-i dt H) psi one sub-step at a time) ------------------------ */
typedef struct {
    int m_eff;           /* basis size (m unless an invariant subspace was found) */
    int breakdown;
    int passes;          /* orthogonalisation passes taken (1 to 3 per basis vector) */
    int pad;
    double beta;         /* h_{m+1,m}: norm of the last orthogonalised vector */
    double beta0;        /* ||psi|| */
} rp_arnoldi_info_t;
/* One Arnoldi cycle of psi with m basis vectors (the reference's
 * orthogonalisation, inc/algo.h:77-173); the basis stays on the device until
 * the next call.  H receives the m x m Hessenberg matrix, complex interleaved,
 * column-major (2*m*m doubles). */
int rp_arnoldi(rp_ham_t h, const void *psi, int m, double *H, rp_arnoldi_info_t *info);
/* out = sum_{i < m_eff} coef_i v_i over the last rp_arnoldi basis
 * (coef: 2*m_eff doubles, complex interleaved). */
int rp_arnoldi_combine(const double *coef, void *out);
/* For c < ncand: col0[c] = first column of exp((fr[c] + i fi[c]) H), H m x m
 * complex column-major, m <= 1024, ncand <= 64; FP64 Pade-13 on the GPU,
 * one CTA per candidate (col0: 2*m*ncand doubles). */
int rp_expm_first_column(int m, const double *H, int ncand, const double *fr, const double *fi,
                         double *col0);

/* --- MLP of the learned step controller (no reference counterpart) -------
 * in -> 64 -> 64 -> out, tanh hidden layers, FP32; forward, backward and
 * Adam are CUDA kernels.  Arrays are host row-major [n][in] / [n][out]. */
typedef struct rp_mlp *rp_mlp_t;
int rp_mlp_create(rp_mlp_t *net, int in_dim, int out_dim, uint64_t seed);
int rp_mlp_num_params(rp_mlp_t net, int *n);
/* flat parameters [W1 (64 x in), b1, W2 (64 x 64), b2, W3 (out x 64), b3] */
int rp_mlp_get_params(rp_mlp_t net, float *p);
int rp_mlp_set_params(rp_mlp_t net, const float *p);
int rp_mlp_forward(rp_mlp_t net, const float *X, int n, float *Y);
/* mean loss (1/2 squared error) and its gradient over n samples */
int rp_mlp_grad(rp_mlp_t net, const float *X, const float *Y, int n, float *grad, float *loss);
/* Adam over shuffled mini-batches; *loss = mean loss of the last epoch */
int rp_mlp_train(rp_mlp_t net, const float *X, const float *Y, int n, int epochs, int batch,
                 float lr, uint64_t seed, float *loss);
int rp_mlp_destroy(rp_mlp_t net);

/* --- batched OTOC (the outer loops of examples/syk.cc:417-475 and
 * examples/simple-syk-krylov.cc:42-57 over many disorder realisations and
 * states, run as one persistent launch per time step and team size) ------- */
typedef struct rp_batch *rp_batch_t;
/* nprob problems; problem p has len[p] qubits (8..30), nterms[p] terms
 * (bits[p], coeff[p] as for rp_ham_create), W and V single Pauli strings
 * (wbits[p], wcoeff[2p..2p+1]; vbits[p], vcoeff[...]), an initial complex64
 * device state psi0[p] (kept, not modified), and a tile exponent tile[p]
 * (8..11, 0 = default; tile may be NULL).  FP32 vectors, FP64 Krylov
 * internals; krydim <= 32; every evolve stops after max_restarts restarts
 * (1..64) or when ||Hexp0|| < tol. */
int rp_batch_create(rp_batch_t *b, int nprob, const int *len, const int64_t *nterms,
                    const uint64_t *const *bits, const double *const *coeff,
                    const uint64_t *wbits, const double *wcoeff, const uint64_t *vbits,
                    const double *vcoeff, const void *const *psi0, const int *tile, int krydim,
                    double tol, int max_restarts);
/* As rp_batch_create, with team[p] the number of CTAs (a thread-block
 * cluster: 1, 2, 4, 8 or 16; 0 = the default for the qubit count) that share
 * problem p; problems of one team size form one launch per time step.  team
 * may be NULL. */
int rp_batch_create_ex(rp_batch_t *b, int nprob, const int *len, const int64_t *nterms,
                       const uint64_t *const *bits, const double *const *coeff,
                       const uint64_t *wbits, const double *wcoeff, const uint64_t *vbits,
                       const double *vcoeff, const void *const *psi0, const int *tile,
                       const int *team, int krydim, double tol, int max_restarts);
/* F[(p * ntimes + k) * 2 + {0,1}] = <psi0| W(t_k) V W(t_k) V |psi0> of problem
 * p (beta = 0), applies[p * ntimes + k] its H.psi count (either may be NULL).
 * One persistent launch per time step and team size; with use_graph the
 * launches are captured once into a CUDA graph and replayed. */
int rp_batch_otoc(rp_batch_t b, int ntimes, const double *times, double *F, int *applies,
                  int use_graph);
/* One persistent launch (per team size) doing only napplies H.psi products
 * per problem (no Krylov); *ms = the device time.  Used by the autotuner. */
int rp_batch_probe(rp_batch_t b, int napplies, double *ms);
int rp_batch_destroy(rp_batch_t b);

#ifdef __cplusplus
}
#endif

#endif /* RPB200_H */
