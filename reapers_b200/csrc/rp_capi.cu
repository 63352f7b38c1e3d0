// C ABI of librpb200.so: argument checking, error translation, context.
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "../../include/rpb200.h"
#include "rp_apply.cuh"
#include "rp_batch.cuh"
#include "rp_dense.cuh"
#include "rp_krylov.cuh"
#include "rp_mlp.cuh"
#include "rp_vec.cuh"

struct rp_ham {
    rp::ApplyPlan plan;
};

struct rp_batch {
    rp::BatchPlan plan;
};

struct rp_mlp {
    rp::Mlp net;
};

struct rp_dense {
    rp::DenseSystem sys;
};

namespace rp {

static thread_local std::string g_err = "no error";
static cudaStream_t g_stream = nullptr;
static int g_device = -1;
static KryWorkspace g_ws;
static ArnoldiResult g_arn;   // the basis of the last rp_arnoldi
static std::mutex g_mu;
// Error word of the asynchronous H.psi launches (rp_apply, rp_apply_shard,
// rp_apply_host): a pipeline wait that gave up sets a bit in it; the next
// synchronising call reads and clears it (RP_E_DEVICE).
static unsigned *g_dev_err = nullptr;

// g_err is per thread: entry points failing at once on several host threads
// each keep their own message.
void set_error(int code, const std::string &msg) {
    (void)code;
    g_err = msg;
}

static void ensure_init() {
    if (g_stream) return;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) throw Error{RP_E_NODEVICE, "no CUDA device available"};
    if (g_device < 0) g_device = 0;
    RP_CUDA(cudaSetDevice(g_device));
    // A blocking stream: work on it is ordered with the legacy default stream
    // in both directions, so buffers written by a caller on the default stream
    // (and reads of our results there) need no extra synchronisation.
    RP_CUDA(cudaStreamCreateWithFlags(&g_stream, cudaStreamDefault));
    if (!g_dev_err) {
        RP_CUDA(cudaMalloc((void **)&g_dev_err, sizeof(unsigned)));
        RP_CUDA(cudaMemset(g_dev_err, 0, sizeof(unsigned)));
    }
}

// After a stream synchronisation: report (and clear) a wait that gave up in
// an asynchronous H.psi launch since the last check.
static void check_device_error() {
    unsigned herr = 0;
    RP_CUDA(cudaMemcpy(&herr, g_dev_err, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (herr) {
        RP_CUDA(cudaMemset(g_dev_err, 0, sizeof(unsigned)));
        throw Error{RP_E_DEVICE, "a device-side wait gave up in an H.psi launch (error word " +
                                     std::to_string(herr) + "); its output is incomplete"};
    }
}

static size_t esize(int dtype) { return dtype == RP_C128 ? 16 : 8; }

static void check_dtype(int dtype) {
    RP_REQUIRE(dtype == RP_C64 || dtype == RP_C128, RP_E_INVALID,
               "dtype must be RP_C64 (1) or RP_C128 (2)");
}

static void check_vec(const void *p) {
    RP_REQUIRE(p != nullptr, RP_E_INVALID, "null vector pointer");
    RP_REQUIRE(((uintptr_t)p & 15) == 0, RP_E_INVALID, "vectors must be 16-byte aligned");
}

template <typename F>
static int guarded(F &&f) {
    try {
        std::lock_guard<std::mutex> lk(g_mu);
        ensure_init();
        f();
        return RP_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    } catch (const std::bad_alloc &) {
        set_error(RP_E_NOMEM, "host out of memory");
        return RP_E_NOMEM;
    } catch (const std::exception &e) {
        set_error(RP_E_INTERNAL, e.what());
        return RP_E_INTERNAL;
    }
}

}  // namespace rp

using namespace rp;

extern "C" {

int rp_init(int device) {
    try {
        std::lock_guard<std::mutex> lk(g_mu);
        // The kernels' shared-memory attributes and the SM count are set up
        // once for the first device; rp_shutdown frees the buffers, streams
        // and scratch, but the process stays bound to that device.
        if (g_device >= 0 && device != g_device) {
            throw Error{RP_E_INVALID, "rp_init: this process is bound to device " +
                                          std::to_string(g_device) +
                                          "; another device needs another process"};
        }
        g_device = device;
        ensure_init();
        return RP_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    }
}

static void pipe_release();

int rp_shutdown(void) {
    try {
        std::lock_guard<std::mutex> lk(g_mu);
        if (g_stream) cudaStreamSynchronize(g_stream);
        workspace_release(g_ws);
        pipe_release();
        scratch_release_all();
        dense_handles_release();
        if (g_dev_err) cudaFree(g_dev_err);
        g_dev_err = nullptr;
        if (g_stream) cudaStreamDestroy(g_stream);
        g_stream = nullptr;
        return RP_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    }
}

const char *rp_last_error(void) { return g_err.c_str(); }

int rp_device_count(int *count) {
    if (!count) {
        set_error(RP_E_INVALID, "null output pointer");
        return RP_E_INVALID;
    }
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
    *count = n;
    return RP_OK;
}

void *rp_stream(void) {
    void *s = nullptr;
    guarded([&] { s = (void *)g_stream; });
    return s;
}

int rp_synchronize(void) {
    return guarded([&] {
        RP_CUDA(cudaStreamSynchronize(g_stream));
        check_device_error();
    });
}

int rp_alloc(void **ptr, size_t bytes) {
    return guarded([&] {
        RP_REQUIRE(ptr, RP_E_INVALID, "null output pointer");
        *ptr = nullptr;
        cudaError_t e = cudaMalloc(ptr, bytes ? bytes : 16);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Error{RP_E_NOMEM, "failed to allocate " + std::to_string(bytes) +
                                        " bytes on the GPU device"};
        }
    });
}

int rp_free(void *ptr) {
    return guarded([&] {
        if (ptr) {
            RP_CUDA(cudaStreamSynchronize(g_stream));
            RP_CUDA(cudaFree(ptr));
        }
    });
}

int rp_memcpy(void *dst, const void *src, size_t bytes, int kind) {
    return guarded([&] {
        RP_REQUIRE(kind >= 0 && kind <= 2, RP_E_INVALID, "kind must be 0, 1 or 2");
        RP_REQUIRE(bytes == 0 || (dst && src), RP_E_INVALID, "null pointer");
        const cudaMemcpyKind k = kind == 0 ? cudaMemcpyHostToDevice
                                           : (kind == 1 ? cudaMemcpyDeviceToHost
                                                        : cudaMemcpyDeviceToDevice);
        RP_CUDA(cudaMemcpyAsync(dst, src, bytes, k, g_stream));
        if (kind != 2) RP_CUDA(cudaStreamSynchronize(g_stream));
    });
}

int rp_vec_zero(int dtype, uint64_t n, void *v) {
    return guarded([&] {
        check_dtype(dtype);
        check_vec(v);
        RP_CUDA(cudaMemsetAsync(v, 0, n * esize(dtype), g_stream));
    });
}

int rp_vec_copy(int dtype_dst, void *dst, int dtype_src, const void *src, uint64_t n) {
    return guarded([&] {
        check_dtype(dtype_dst);
        check_dtype(dtype_src);
        check_vec(dst);
        check_vec(src);
        vec_convert(dtype_dst, dst, dtype_src, src, n, g_stream);
    });
}

int rp_vec_axpy(int dtype, uint64_t n, void *y, double ar, double ai, const void *x) {
    return guarded([&] {
        check_dtype(dtype);
        check_vec(y);
        check_vec(x);
        vec_axpy(dtype, n, y, ar, ai, x, g_stream);
    });
}

int rp_vec_add(int dtype, uint64_t n, void *res, const void *a, const void *b) {
    return guarded([&] {
        check_dtype(dtype);
        check_vec(res);
        check_vec(a);
        check_vec(b);
        vec_add3(dtype, n, res, a, b, g_stream);
    });
}

int rp_vec_scale(int dtype, uint64_t n, void *v, double ar, double ai) {
    return guarded([&] {
        check_dtype(dtype);
        check_vec(v);
        vec_scale(dtype, n, v, ar, ai, g_stream);
    });
}

int rp_vec_dot(int dtype, uint64_t n, const void *a, const void *b, double *out) {
    return guarded([&] {
        check_dtype(dtype);
        check_vec(a);
        check_vec(b);
        RP_REQUIRE(out, RP_E_INVALID, "null output pointer");
        const int g = reduce_grid();
        // partials[g][2], then the reduced pair
        double *part = static_cast<double *>(
            scratch_get(SCR_DOT, ((size_t)g + 1) * 2 * sizeof(double), g_stream));
        double *red = part + (size_t)g * 2;
        VecTable tab{};
        tab.p[0] = a;
        multi_dot_partials(dtype, n, tab, 1, b, part, nullptr, nullptr, g_stream);
        reduce_partials(part, g, 1, red, g_stream);
        RP_CUDA(cudaMemcpyAsync(out, red, 2 * sizeof(double), cudaMemcpyDeviceToHost, g_stream));
        RP_CUDA(cudaStreamSynchronize(g_stream));
    });
}

int rp_vec_norm(int dtype, uint64_t n, const void *v, double *out) {
    return guarded([&] {
        check_dtype(dtype);
        check_vec(v);
        RP_REQUIRE(out, RP_E_INVALID, "null output pointer");
        *out = vec_norm_sync(dtype, n, v, nullptr, g_stream);
    });
}

int rp_vec_random(int dtype, uint64_t n, void *v, uint64_t seed) {
    return guarded([&] {
        check_dtype(dtype);
        check_vec(v);
        vec_random(dtype, n, v, seed, g_stream);
    });
}

int rp_ham_create_ex(rp_ham_t *h, int len, int dtype, uint64_t nterms, const uint64_t *bits,
                     const double *coeff, int tile_exp) {
    return guarded([&] {
        RP_REQUIRE(h, RP_E_INVALID, "null output pointer");
        RP_REQUIRE(nterms == 0 || (bits && coeff), RP_E_INVALID, "null term table");
        RP_REQUIRE(nterms < (1ull << 31), RP_E_INVALID, "too many terms");
        check_dtype(dtype);
        RP_REQUIRE(len >= 1 && len <= 32, RP_E_INVALID, "len must be in [1, 32]");
        ApplyConfig cfg = default_config(len, dtype);
        if (tile_exp) {
            RP_REQUIRE(tile_exp >= 5 && tile_exp <= 12 && tile_exp <= len, RP_E_INVALID,
                       "tile_exp must be in [5, min(12, len)]");
            cfg.direct = false;
            cfg.allow_rows = false;
            cfg.B = tile_exp;
            cfg.P = std::min(256, 1 << tile_exp);
        }
        rp_ham *H = new rp_ham;
        try {
            plan_build(H->plan, len, dtype, bits, coeff, (int64_t)nterms, cfg);
            plan_upload(H->plan);
        } catch (...) {
            plan_free(H->plan);
            delete H;
            throw;
        }
        *h = H;
    });
}

int rp_ham_create(rp_ham_t *h, int len, int dtype, uint64_t nterms, const uint64_t *bits,
                  const double *coeff) {
    return rp_ham_create_ex(h, len, dtype, nterms, bits, coeff, 0);
}

int rp_ham_destroy(rp_ham_t h) {
    return guarded([&] {
        if (!h) return;
        RP_CUDA(cudaStreamSynchronize(g_stream));
        plan_free(h->plan);
        delete h;
    });
}

int rp_ham_info(rp_ham_t h, rp_ham_info_t *info) {
    return guarded([&] {
        RP_REQUIRE(h && info, RP_E_INVALID, "null argument");
        const ApplyPlan &p = h->plan;
        info->len = p.len;
        info->dtype = p.dtype;
        info->nterms = p.nterms;
        info->tile_exp = p.cfg.direct ? 0 : p.cfg.B;
        info->ngroups = p.ngroups;
        info->threads = p.cfg.direct ? 32 : p.cfg.P;
        info->stages = p.cfg.direct ? 0 : p.cfg.stages;
        info->grid = apply_grid(p);
        info->alg_bytes = p.alg_bytes;
        info->kernel = p.cfg.direct ? 0 : (p.rows.ok ? 2 : 1);
        info->window = apply_grid(p);
        info->alg_bytes_dram = p.rows.ok ? p.rows.alg_bytes_dram : p.alg_bytes;
        const double vbytes = std::ldexp(1.0, p.len) * (p.dtype == RP_C128 ? 16.0 : 8.0);
        const int nt = p.rows.ok ? p.rows.nterms : p.nterms;
        const int ng = p.rows.ok ? (int)p.rows.groups.size() : p.ngroups;
        const int nd = p.rows.ok ? p.rows.ndiag : 0;
        // row loads per output element: terms that reuse the previous term's
        // row (ROW_SAME_SRC) load none; the fused diagonal loads the own row
        int shared = 0;
        if (p.rows.ok)
            for (const auto &t : p.rows.terms) shared += (t.cs & ROW_SAME_SRC) ? 1 : 0;
        info->nreads = nt - shared + (nd ? 1 : 0);
        info->smem_bytes = (double)(info->nreads + ng) * vbytes;
        info->diag_terms = nd;
        if (p.rows.ok) {
            info->tile_exp = p.rows.B;
            info->ngroups = (int)p.rows.groups.size();
            info->threads = 256;
            info->nterms = p.rows.nterms + p.rows.ndiag;
        }
    });
}

int rp_apply(rp_ham_t h, void *out, const void *in, int accumulate) {
    return guarded([&] {
        RP_REQUIRE(h, RP_E_INVALID, "null Hamiltonian");
        check_vec(out);
        check_vec(in);
        ApplyLaunch L;
        L.in = in;
        L.out = out;
        L.accumulate = accumulate;
        L.err = g_dev_err;
        apply_launch(h->plan, L, g_stream);
    });
}

int rp_test_withhold_tile(int64_t iteration, uint32_t wait_polls) {
    return guarded([&] { rows_test_withhold((long)iteration, wait_polls); });
}

int rp_apply_shard(rp_ham_t h, int shard_bits, int shard_rank, const void *const *shards, void *out,
                   int accumulate) {
    return guarded([&] {
        RP_REQUIRE(h && shards, RP_E_INVALID, "null argument");
        check_vec(out);
        ApplyLaunch L;
        L.out = out;
        L.accumulate = accumulate;
        L.shards = shards;
        L.shard_bits = shard_bits;
        L.shard_rank = shard_rank;
        L.err = g_dev_err;
        apply_launch(h->plan, L, g_stream);
    });
}

// CUDA IPC: a device pointer travels as the handle of its allocation plus
// its offset inside it (torch's caching allocator hands out interior
// pointers), and is opened with peer access enabled lazily.
static_assert(sizeof(cudaIpcMemHandle_t) == sizeof(((rp_ipc_handle_t *)0)->handle), "IPC handle size");

static PFN_cuMemGetAddressRange_v3020 get_address_range() {
    static PFN_cuMemGetAddressRange_v3020 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        RP_CUDA(cudaGetDriverEntryPoint("cuMemGetAddressRange", &p, cudaEnableDefault, &q));
        RP_REQUIRE(q == cudaDriverEntryPointSuccess && p, RP_E_CUDA, "cuMemGetAddressRange unavailable");
        fn = reinterpret_cast<PFN_cuMemGetAddressRange_v3020>(p);
    }
    return fn;
}

// Opened allocations by handle (an allocation may hold several exported
// tensors: it is mapped once and reference-counted), and the allocation of
// every pointer handed out.
static std::map<std::string, std::pair<void *, int>> g_ipc_bases;
static std::multimap<void *, std::string> g_ipc_ptrs;

int rp_ipc_export(const void *ptr, rp_ipc_handle_t *out) {
    return guarded([&] {
        RP_REQUIRE(ptr && out, RP_E_INVALID, "null argument");
        CUdeviceptr base = 0;
        size_t size = 0;
        const CUresult r = get_address_range()(&base, &size, (CUdeviceptr)(uintptr_t)ptr);
        RP_REQUIRE(r == CUDA_SUCCESS, RP_E_INVALID, "not a device allocation (cuMemGetAddressRange " +
                                                        std::to_string((int)r) + ")");
        cudaIpcMemHandle_t hd;
        RP_CUDA(cudaIpcGetMemHandle(&hd, reinterpret_cast<void *>(base)));
        std::memcpy(out->handle, &hd, sizeof(hd));
        out->offset = (uint64_t)((uintptr_t)ptr - (uintptr_t)base);
    });
}

int rp_ipc_open(const rp_ipc_handle_t *h, void **ptr) {
    return guarded([&] {
        RP_REQUIRE(h && ptr, RP_E_INVALID, "null argument");
        const std::string key(reinterpret_cast<const char *>(h->handle), sizeof(h->handle));
        auto it = g_ipc_bases.find(key);
        if (it == g_ipc_bases.end()) {
            cudaIpcMemHandle_t hd;
            std::memcpy(&hd, h->handle, sizeof(hd));
            void *base = nullptr;
            RP_CUDA(cudaIpcOpenMemHandle(&base, hd, cudaIpcMemLazyEnablePeerAccess));
            it = g_ipc_bases.emplace(key, std::make_pair(base, 0)).first;
        }
        it->second.second++;
        void *p = static_cast<char *>(it->second.first) + h->offset;
        g_ipc_ptrs.emplace(p, key);
        *ptr = p;
    });
}

int rp_ipc_close(void *ptr) {
    return guarded([&] {
        auto it = g_ipc_ptrs.find(ptr);
        RP_REQUIRE(it != g_ipc_ptrs.end(), RP_E_INVALID, "pointer was not opened by rp_ipc_open");
        const std::string key = it->second;
        g_ipc_ptrs.erase(it);
        auto b = g_ipc_bases.find(key);
        if (--b->second.second == 0) {
            void *base = b->second.first;
            g_ipc_bases.erase(b);
            RP_CUDA(cudaIpcCloseMemHandle(base));
        }
    });
}

// Output chunks of rp_apply_host with the row kernel: each chunk's
// device-to-host copy starts as soon as its output tiles are written, so
// only the last chunk's copy follows the final product.
constexpr int HOST_CHUNKS = 8;

// Device buffers and streams of rp_apply_host, kept between calls.
struct HostPipe {
    size_t bytes = 0;
    void *din[2] = {nullptr, nullptr}, *dout[2] = {nullptr, nullptr};
    cudaStream_t s_in = nullptr, s_out = nullptr;
    cudaEvent_t in_ready[2] = {}, comp_done[2] = {}, out_done[2] = {};
    cudaEvent_t part_done[HOST_CHUNKS] = {};
};
static HostPipe g_pipe;

static void pipe_release() {
    HostPipe &p = g_pipe;
    for (int b = 0; b < 2; b++) {
        if (p.din[b]) cudaFree(p.din[b]);
        if (p.dout[b]) cudaFree(p.dout[b]);
        if (p.in_ready[b]) cudaEventDestroy(p.in_ready[b]);
        if (p.comp_done[b]) cudaEventDestroy(p.comp_done[b]);
        if (p.out_done[b]) cudaEventDestroy(p.out_done[b]);
    }
    for (int c = 0; c < HOST_CHUNKS; c++)
        if (p.part_done[c]) cudaEventDestroy(p.part_done[c]);
    if (p.s_in) cudaStreamDestroy(p.s_in);
    if (p.s_out) cudaStreamDestroy(p.s_out);
    p = HostPipe{};
}

static void pipe_ensure(size_t bytes) {
    HostPipe &p = g_pipe;
    if (!p.s_in) {
        RP_CUDA(cudaStreamCreateWithFlags(&p.s_in, cudaStreamNonBlocking));
        RP_CUDA(cudaStreamCreateWithFlags(&p.s_out, cudaStreamNonBlocking));
        for (int b = 0; b < 2; b++) {
            RP_CUDA(cudaEventCreateWithFlags(&p.in_ready[b], cudaEventDisableTiming));
            RP_CUDA(cudaEventCreateWithFlags(&p.comp_done[b], cudaEventDisableTiming));
            RP_CUDA(cudaEventCreateWithFlags(&p.out_done[b], cudaEventDisableTiming));
        }
        for (int c = 0; c < HOST_CHUNKS; c++)
            RP_CUDA(cudaEventCreateWithFlags(&p.part_done[c], cudaEventDisableTiming));
    }
    if (p.bytes >= bytes) return;
    for (int b = 0; b < 2; b++) {
        if (p.din[b]) cudaFree(p.din[b]);
        if (p.dout[b]) cudaFree(p.dout[b]);
        p.din[b] = p.dout[b] = nullptr;
    }
    p.bytes = 0;
    for (int b = 0; b < 2; b++) {
        if (cudaMalloc(&p.din[b], bytes) != cudaSuccess || cudaMalloc(&p.dout[b], bytes) != cudaSuccess) {
            cudaGetLastError();
            throw Error{RP_E_NOMEM, "failed to allocate the host-apply device buffers"};
        }
    }
    p.bytes = bytes;
}

int rp_apply_host(rp_ham_t h, int n, const void *const *in_host, void *const *out_host) {
    return guarded([&] {
        RP_REQUIRE(h && n >= 0 && (n == 0 || (in_host && out_host)), RP_E_INVALID, "bad argument");
        if (n == 0) return;
        const size_t bytes = (size_t)esize(h->plan.dtype) << h->plan.len;
        pipe_ensure(bytes);
        HostPipe &p = g_pipe;
        // output chunks: whole multiples of the row kernel's CTA window (the
        // last chunk takes the rest); one chunk for the other kernels
        const RowPlan &rp = h->plan.rows;
        uint32_t per = 0;
        int nch = 1;
        if (rp.ok && rp.ntiles >= 2 * rp.window) {
            const uint32_t waves = (uint32_t)((rp.ntiles + rp.window - 1) / rp.window);
            per = (uint32_t)rp.window * ((waves + HOST_CHUNKS - 1) / HOST_CHUNKS);
            nch = (int)((rp.ntiles + per - 1) / per);
        }
        const size_t tile_bytes = rp.ok ? (size_t)esize(h->plan.dtype) << rp.B : bytes;
        for (int i = 0; i < n; i++) {
            RP_REQUIRE(in_host[i] && out_host[i], RP_E_INVALID, "null host vector");
            const int b = i & 1;
            // buffer b is free once H.psi i-2 has read it
            if (i >= 2) RP_CUDA(cudaStreamWaitEvent(p.s_in, p.comp_done[b], 0));
            RP_CUDA(cudaMemcpyAsync(p.din[b], in_host[i], bytes, cudaMemcpyHostToDevice, p.s_in));
            RP_CUDA(cudaEventRecord(p.in_ready[b], p.s_in));
            RP_CUDA(cudaStreamWaitEvent(g_stream, p.in_ready[b], 0));
            // the result buffer b is free once result i-2 reached the host
            if (i >= 2) RP_CUDA(cudaStreamWaitEvent(g_stream, p.out_done[b], 0));
            for (int c = 0; c < nch; c++) {
                ApplyLaunch L;
                L.in = p.din[b];
                L.out = p.dout[b];
                L.err = g_dev_err;
                size_t off = 0, len = bytes;
                if (nch > 1) {
                    L.tile0 = (uint32_t)c * per;
                    L.tile_count = std::min<uint32_t>(per, (uint32_t)rp.ntiles - L.tile0);
                    off = (size_t)L.tile0 * tile_bytes;
                    len = (size_t)L.tile_count * tile_bytes;
                }
                apply_launch(h->plan, L, g_stream);
                RP_CUDA(cudaEventRecord(p.part_done[c], g_stream));
                RP_CUDA(cudaStreamWaitEvent(p.s_out, p.part_done[c], 0));
                RP_CUDA(cudaMemcpyAsync(static_cast<char *>(out_host[i]) + off,
                                        static_cast<const char *>(p.dout[b]) + off, len,
                                        cudaMemcpyDeviceToHost, p.s_out));
            }
            RP_CUDA(cudaEventRecord(p.comp_done[b], g_stream));
            RP_CUDA(cudaEventRecord(p.out_done[b], p.s_out));
        }
        RP_CUDA(cudaStreamSynchronize(p.s_out));
        RP_CUDA(cudaStreamSynchronize(g_stream));
        check_device_error();
    });
}

int rp_evolve(rp_ham_t h, void *psi, double t, double beta, int krydim, double tol,
              int max_iters, rp_evolve_stats_t *stats) {
    return guarded([&] {
        RP_REQUIRE(h, RP_E_INVALID, "null Hamiltonian");
        check_vec(psi);
        RP_REQUIRE(max_iters >= 0, RP_E_INVALID, "max_iters must be non-negative");
        EvolveStats S{};
        krylov_evolve(h->plan, g_ws, psi, t, beta, krydim, tol, max_iters, &S, g_stream);
        if (stats) {
            stats->restarts = S.restarts;
            stats->applies = S.applies;
            stats->passes = S.passes;
            stats->prods = S.prods;
            stats->breakdown = S.breakdown;
            stats->last_err = S.last_err;
        }
    });
}

int rp_arnoldi(rp_ham_t h, const void *psi, int m, double *H, rp_arnoldi_info_t *info) {
    return guarded([&] {
        RP_REQUIRE(h && H && info, RP_E_INVALID, "null argument");
        check_vec(psi);
        krylov_arnoldi(h->plan, g_ws, psi, m, g_arn, g_stream);
        std::copy(g_arn.H.begin(), g_arn.H.end(), H);
        info->m_eff = g_arn.m_eff;
        info->breakdown = g_arn.breakdown;
        info->passes = g_arn.passes;
        info->pad = 0;
        info->beta = g_arn.beta;
        info->beta0 = g_arn.beta0;
    });
}

int rp_arnoldi_combine(const double *coef, void *out) {
    return guarded([&] {
        RP_REQUIRE(coef, RP_E_INVALID, "null argument");
        check_vec(out);
        krylov_combine(g_ws, g_arn, coef, out, g_stream);
    });
}

int rp_expm_first_column(int m, const double *H, int ncand, const double *fr, const double *fi,
                         double *col0) {
    return guarded([&] {
        RP_REQUIRE(H && fr && fi && col0, RP_E_INVALID, "null argument");
        expm_candidates(m, H, ncand, fr, fi, col0, g_stream);
    });
}

int rp_mlp_create(rp_mlp_t *net, int in_dim, int out_dim, uint64_t seed) {
    return guarded([&] {
        RP_REQUIRE(net, RP_E_INVALID, "null argument");
        rp_mlp *M = new rp_mlp;
        try {
            mlp_create(M->net, in_dim, out_dim, seed);
        } catch (...) {
            mlp_free(M->net);
            delete M;
            throw;
        }
        *net = M;
    });
}

int rp_mlp_num_params(rp_mlp_t net, int *n) {
    return guarded([&] {
        RP_REQUIRE(net && n, RP_E_INVALID, "null argument");
        *n = net->net.np;
    });
}

int rp_mlp_get_params(rp_mlp_t net, float *p) {
    return guarded([&] {
        RP_REQUIRE(net && p, RP_E_INVALID, "null argument");
        mlp_get(net->net, p);
    });
}

int rp_mlp_set_params(rp_mlp_t net, const float *p) {
    return guarded([&] {
        RP_REQUIRE(net && p, RP_E_INVALID, "null argument");
        mlp_set(net->net, p);
    });
}

int rp_mlp_forward(rp_mlp_t net, const float *X, int n, float *Y) {
    return guarded([&] {
        RP_REQUIRE(net && X && Y && n >= 0, RP_E_INVALID, "bad argument");
        if (n) mlp_forward(net->net, X, n, Y, g_stream);
    });
}

int rp_mlp_grad(rp_mlp_t net, const float *X, const float *Y, int n, float *grad, float *loss) {
    return guarded([&] {
        RP_REQUIRE(net && X && Y && grad && loss, RP_E_INVALID, "null argument");
        *loss = mlp_grad(net->net, X, Y, n, grad, g_stream);
    });
}

int rp_mlp_train(rp_mlp_t net, const float *X, const float *Y, int n, int epochs, int batch,
                 float lr, uint64_t seed, float *loss) {
    return guarded([&] {
        RP_REQUIRE(net && X && Y && loss, RP_E_INVALID, "null argument");
        *loss = mlp_train(net->net, X, Y, n, epochs, batch, lr, seed, g_stream);
    });
}

int rp_mlp_destroy(rp_mlp_t net) {
    return guarded([&] {
        if (!net) return;
        mlp_free(net->net);
        delete net;
    });
}

int rp_batch_create(rp_batch_t *b, int nprob, const int *len, const int64_t *nterms,
                    const uint64_t *const *bits, const double *const *coeff,
                    const uint64_t *wbits, const double *wcoeff, const uint64_t *vbits,
                    const double *vcoeff, const void *const *psi0, const int *tile, int krydim,
                    double tol, int max_restarts) {
    return rp_batch_create_ex(b, nprob, len, nterms, bits, coeff, wbits, wcoeff, vbits, vcoeff,
                              psi0, tile, nullptr, krydim, tol, max_restarts);
}

int rp_batch_create_ex(rp_batch_t *b, int nprob, const int *len, const int64_t *nterms,
                       const uint64_t *const *bits, const double *const *coeff,
                       const uint64_t *wbits, const double *wcoeff, const uint64_t *vbits,
                       const double *vcoeff, const void *const *psi0, const int *tile,
                       const int *team, int krydim, double tol, int max_restarts) {
    return guarded([&] {
        RP_REQUIRE(b && len && nterms && bits && coeff && wbits && wcoeff && vbits && vcoeff &&
                       psi0,
                   RP_E_INVALID, "null argument");
        rp_batch *B = new rp_batch;
        try {
            batch_build(B->plan, nprob, len, nterms, bits, coeff, wbits, wcoeff, vbits, vcoeff,
                        psi0, tile, team, krydim, tol, max_restarts, g_stream);
        } catch (...) {
            delete B;
            throw;
        }
        *b = B;
    });
}

int rp_batch_otoc(rp_batch_t b, int ntimes, const double *times, double *F, int *applies,
                  int use_graph) {
    return guarded([&] {
        RP_REQUIRE(b && times, RP_E_INVALID, "null argument");
        batch_otoc(b->plan, ntimes, times, F, applies, use_graph, g_stream);
    });
}

int rp_batch_probe(rp_batch_t b, int napplies, double *ms) {
    return guarded([&] {
        RP_REQUIRE(b && ms, RP_E_INVALID, "null argument");
        *ms = batch_probe(b->plan, napplies, g_stream);
    });
}

int rp_batch_destroy(rp_batch_t b) {
    return guarded([&] {
        if (!b) return;
        RP_CUDA(cudaStreamSynchronize(g_stream));
        batch_free(b->plan);
        delete b;
    });
}

int rp_dense_create(rp_dense_t *d, int len, int dtype, uint64_t nterms, const uint64_t *bits,
                    const double *coeff) {
    return guarded([&] {
        RP_REQUIRE(d, RP_E_INVALID, "null output pointer");
        RP_REQUIRE(nterms < (1ull << 31), RP_E_INVALID, "too many terms");
        rp_dense *D = new rp_dense;
        try {
            dense_build(D->sys, len, dtype, bits, coeff, (int64_t)nterms, g_stream);
        } catch (...) {
            delete D;
            throw;
        }
        *d = D;
    });
}

int rp_dense_eigenvalues(rp_dense_t d, double *evals) {
    return guarded([&] {
        RP_REQUIRE(d && evals, RP_E_INVALID, "null argument");
        std::copy(d->sys.evals.begin(), d->sys.evals.end(), evals);
    });
}

int rp_dense_eigenvectors(rp_dense_t d, void **mat) {
    return guarded([&] {
        RP_REQUIRE(d && mat, RP_E_INVALID, "null argument");
        *mat = d->sys.evecs;
    });
}

int rp_dense_eigenvector(rp_dense_t d, int64_t index, void *out) {
    return guarded([&] {
        RP_REQUIRE(d, RP_E_INVALID, "null argument");
        check_vec(out);
        dense_column(d->sys, index, out, g_stream);
    });
}

int rp_dense_expm(rp_dense_t d, double cr, double ci, void *out) {
    return guarded([&] {
        RP_REQUIRE(d, RP_E_INVALID, "null argument");
        check_vec(out);
        dense_expm(d->sys, cr, ci, out, g_stream);
    });
}

int rp_dense_destroy(rp_dense_t d) {
    return guarded([&] {
        if (!d) return;
        RP_CUDA(cudaStreamSynchronize(g_stream));
        dense_free(d->sys);
        delete d;
    });
}

int rp_mat_vec(int dtype, uint64_t dim, const void *mat, const void *vec, void *res) {
    return guarded([&] {
        check_dtype(dtype);
        check_vec(mat);
        check_vec(vec);
        check_vec(res);
        RP_REQUIRE(res != vec, RP_E_INVALID, "mat_vec needs distinct input and output vectors");
        RP_REQUIRE(dim <= (1ull << 16), RP_E_INVALID, "mat_vec takes matrices of at most 2^16 rows");
        dense_matvec(dtype, dim, mat, vec, res, g_stream);
    });
}

int rp_workspace_release(void) {
    return guarded([&] {
        RP_CUDA(cudaStreamSynchronize(g_stream));
        workspace_release(g_ws);
        pipe_release();
    });
}

}  // extern "C"
