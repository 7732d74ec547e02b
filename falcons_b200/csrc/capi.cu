// extern "C" boundary of libfalcons_b200.so (declared in include/falcons_b200.h).
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>

#include "../../include/falcons_b200.h"
#include "assemble.cuh"
#include "batch.cuh"
#include "context.cuh"
#include "interp.cuh"
#include "pipeline.cuh"
#include "static_scratch.cuh"

struct falcons_ctx {
    fb2::Context c;
    fb2::BatchPool batch;  // worker contexts of the batch entry points
};

namespace {
thread_local std::string g_last_error;

template <class F>
int guarded(F &&f) {
    try {
        f();
        return FALCONS_OK;
    } catch (const std::invalid_argument &e) {
        g_last_error = e.what();
        return FALCONS_EINVAL;
    } catch (const std::length_error &e) {
        g_last_error = e.what();
        return FALCONS_ELENGTH;
    } catch (const fb2::cuda_error &e) {
        g_last_error = e.what();
        return FALCONS_ECUDA;
    } catch (const std::bad_alloc &e) {
        g_last_error = "out of memory";
        return FALCONS_ENOMEM;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return FALCONS_ERUNTIME;
    } catch (...) {
        g_last_error = "unknown error";
        return FALCONS_ERUNTIME;
    }
}

fb2::InterpParams to_params(const falcons_interp_params *p) {
    if (!p) throw std::invalid_argument("null params");
    fb2::InterpParams q;
    q.eb = p->eb;
    q.cubic = p->interp_algo;
    q.direction = p->direction;
    q.anchor = p->anchor_stride;
    q.alpha = p->alpha;
    q.beta = p->beta;
    q.radius = p->radius;
    q.tuning = p->tuning;
    q.max_abs = p->max_abs;
    return q;
}

cudaStream_t pick(falcons_ctx *ctx, void *s) { return s ? static_cast<cudaStream_t>(s) : ctx->c.stream; }

// The largest |value| of a device field of dims[0..N) (fb2::InterpParams::max_abs).
double measured_max_abs(falcons_ctx *ctx, int dtype, const void *d_data, const long long *dims, int N, cudaStream_t st) {
    long long n = 1;
    for (int i = 0; i < N && i < 4; i++) n *= std::max<long long>(dims[i], 0);
    if (n <= 0) return 0;
    void *ws = ctx->c.work2.get(fb2::range_workspace_bytes());
    void *res = ctx->c.small.get(64);
    double h[3] = {0, 0, 0};
    if (dtype == FALCONS_DTYPE_F32) {
        fb2::device_range<float>(static_cast<const float *>(d_data), n, static_cast<float *>(res), ws, st);
        float f[3];
        FB2_CUDA(cudaMemcpyAsync(f, res, sizeof f, cudaMemcpyDeviceToHost, st));
        FB2_CUDA(cudaStreamSynchronize(st));
        for (int i = 0; i < 3; i++) h[i] = f[i];
    } else {
        fb2::device_range<double>(static_cast<const double *>(d_data), n, static_cast<double *>(res), ws, st);
        FB2_CUDA(cudaMemcpyAsync(h, res, sizeof h, cudaMemcpyDeviceToHost, st));
        FB2_CUDA(cudaStreamSynchronize(st));
    }
    return std::max(std::fabs(h[1]), std::fabs(h[2]));
}

void check_ctx(falcons_ctx *ctx) {
    if (!ctx) throw std::invalid_argument("null context");
    FB2_CUDA(cudaSetDevice(ctx->c.device));
}

void check_dtype(int dtype) {
    if (dtype != FALCONS_DTYPE_F32 && dtype != FALCONS_DTYPE_F64)
        throw std::invalid_argument("unsupported on GPU build: only float32 and float64 fields are supported");
}
}  // namespace

namespace fb2 {
static std::atomic<unsigned long long> g_launches{0};
unsigned long long count_launch() { return ++g_launches; }

static double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
Trace::Trace(const char *w) : what(w), t0(0), l0(0), on(std::getenv("FALCONS_TRACE") != nullptr) {
    if (on) {
        t0 = now_ms();
        l0 = g_launches.load();
    }
}
void Trace::mark(const char *label) {
    if (on)
        std::fprintf(stderr, "[falcons trace] %s %-28s +%8.3f ms  launches %llu\n", what, label, now_ms() - t0,
                     g_launches.load() - l0);
}
void Trace::gpu(const char *label, cudaStream_t s) {
    if (!on) return;
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    cudaEventRecord(e, s);
    events.emplace_back(label, e);
}
void Trace::gpu_dump() {
    if (!on || events.empty()) return;
    for (auto &p : events) cudaEventSynchronize(p.second);
    for (auto &p : events) {
        float ms = 0;
        cudaEventElapsedTime(&ms, events.front().second, p.second);
        std::fprintf(stderr, "[falcons trace] %s device: %-26s +%8.3f ms\n", what, p.first, ms);
    }
    for (auto &p : events) cudaEventDestroy(p.second);
    events.clear();
}
Trace::~Trace() {
    for (auto &p : events) cudaEventDestroy(p.second);
}
}  // namespace fb2

extern "C" {

const char *falcons_last_error(void) { return g_last_error.c_str(); }
uint64_t falcons_kernel_launches(void) { return fb2::g_launches.load(); }
const char *falcons_version(void) { return "falcons_b200 1.0.0 (stream format Falcons data version 1.0.0)"; }

int falcons_ctx_create(falcons_ctx **out, int device) {
    return guarded([&] {
        if (!out) throw std::invalid_argument("null output pointer");
        int n = 0;
        FB2_CUDA(cudaGetDeviceCount(&n));
        if (device < 0 || device >= n) throw std::invalid_argument("invalid CUDA device");
        FB2_CUDA(cudaSetDevice(device));
        auto *c = new falcons_ctx();
        c->c.device = device;
        c->batch.device = device;
        FB2_CUDA(cudaStreamCreateWithFlags(&c->c.stream, cudaStreamNonBlocking));
        fb2::stage_reserve(2);  // this context's share of the pinned read staging
        for (auto &e : c->c.ev) FB2_CUDA(cudaEventCreate(&e));
        *out = c;
    });
}

int falcons_ctx_destroy(falcons_ctx *ctx) {
    return guarded([&] {
        if (!ctx) return;
        cudaSetDevice(ctx->c.device);
        cudaStreamSynchronize(ctx->c.stream);
        delete ctx;
    });
}

int falcons_interp_compress(falcons_ctx *ctx, int dtype, const size_t *dims, int N, const falcons_interp_params *p,
                            void *d_data, int16_t *d_codes, void *d_unpred, size_t *n_codes, size_t *n_unpred,
                            void *stream) {
    return guarded([&] {
        check_ctx(ctx);
        check_dtype(dtype);
        if (!dims || !d_data || !d_codes || !d_unpred) throw std::invalid_argument("null pointer");
        std::lock_guard<std::mutex> lk(ctx->c.mu);
        long long d[4];
        for (int i = 0; i < N && i < 4; i++) d[i] = (long long)dims[i];
        fb2::InterpParams prm = to_params(p);
        cudaStream_t st = pick(ctx, stream);
        if (!(prm.max_abs >= 0)) prm.max_abs = measured_max_abs(ctx, dtype, d_data, d, N, st);
        const fb2::InterpPlan plan = fb2::make_plan(d, N, prm);
        const int es = dtype == FALCONS_DTYPE_F32 ? 4 : 8;
        void *ws = ctx->c.work.get(fb2::interp_workspace_bytes(plan, es));
        auto *cnt = static_cast<unsigned long long *>(ctx->c.small.get(64));
        fb2::LaunchTimes lt;
        fb2::LaunchTimes *ltp = ctx->c.time_levels ? &lt : nullptr;
        if (dtype == FALCONS_DTYPE_F32)
            fb2::interp_compress<float>(plan, static_cast<float *>(d_data), d_codes, static_cast<float *>(d_unpred),
                                        ws, cnt, st, ltp);
        else
            fb2::interp_compress<double>(plan, static_cast<double *>(d_data), d_codes,
                                         static_cast<double *>(d_unpred), ws, cnt, st, ltp);
        unsigned long long h = 0;
        FB2_CUDA(cudaMemcpyAsync(&h, cnt, 8, cudaMemcpyDeviceToHost, st));
        FB2_CUDA(cudaStreamSynchronize(st));
        if (ltp) {
            lt.read();
            ctx->c.lt_level.clear();
            ctx->c.lt_ms.clear();
            ctx->c.lt_codes.clear();
            // plan levels run from the first point and the coarsest level down to level 1
            for (const auto &x : lt.e) {
                ctx->c.lt_level.push_back(x.level);
                ctx->c.lt_ms.push_back(x.ms);
                ctx->c.lt_codes.push_back((unsigned long long)fb2::level_codes(plan, x.level));
            }
        }
        if (n_codes) *n_codes = (size_t)plan.n_codes;
        if (n_unpred) *n_unpred = (size_t)(plan.n_anchor + (long long)h);
    });
}

int falcons_time_levels(falcons_ctx *ctx, int on) {
    return guarded([&] {
        check_ctx(ctx);
        std::lock_guard<std::mutex> lk(ctx->c.mu);
        ctx->c.time_levels = on != 0;
    });
}

int falcons_level_times(falcons_ctx *ctx, int *level, float *ms, unsigned long long *codes, int cap, int *count) {
    return guarded([&] {
        check_ctx(ctx);
        std::lock_guard<std::mutex> lk(ctx->c.mu);
        const int n = (int)ctx->c.lt_ms.size();
        for (int i = 0; i < n && i < cap; i++) {
            if (level) level[i] = ctx->c.lt_level[i];
            if (ms) ms[i] = ctx->c.lt_ms[i];
            if (codes) codes[i] = ctx->c.lt_codes[i];
        }
        if (count) *count = n;
    });
}

int falcons_interp_decompress(falcons_ctx *ctx, int dtype, const size_t *dims, int N,
                              const falcons_interp_params *p, const int16_t *d_codes, size_t n_codes,
                              const void *d_unpred, size_t n_unpred, void *d_out, void *stream) {
    return guarded([&] {
        check_ctx(ctx);
        check_dtype(dtype);
        if (!dims || !d_out || !d_codes) throw std::invalid_argument("null pointer");
        std::lock_guard<std::mutex> lk(ctx->c.mu);
        long long d[4];
        for (int i = 0; i < N && i < 4; i++) d[i] = (long long)dims[i];
        const fb2::InterpPlan plan = fb2::make_plan(d, N, to_params(p));
        if ((long long)n_codes != plan.n_codes) throw std::invalid_argument("code count does not match the field");
        if ((long long)n_unpred < plan.n_anchor) throw std::invalid_argument("unpredictable list too short");
        const int es = dtype == FALCONS_DTYPE_F32 ? 4 : 8;
        void *ws = ctx->c.work.get(fb2::interp_workspace_bytes(plan, es));
        cudaStream_t st = pick(ctx, stream);
        if (dtype == FALCONS_DTYPE_F32)
            fb2::interp_decompress<float>(plan, d_codes, static_cast<const float *>(d_unpred), (long long)n_unpred,
                                          static_cast<float *>(d_out), ws, st);
        else
            fb2::interp_decompress<double>(plan, d_codes, static_cast<const double *>(d_unpred), (long long)n_unpred,
                                          static_cast<double *>(d_out), ws, st);
        fb2::interp_decompress_check(plan, es, ws, (long long)n_unpred, st);
    });
}

int falcons_interp_decompress_noalloc(int dtype, const size_t *dims, int N, const falcons_interp_params *p,
                                      const int16_t *d_codes, size_t n_codes, const void *d_unpred,
                                      size_t n_unpred, void *d_out, void *stream) {
    return guarded([&] {
        check_dtype(dtype);
        if (!dims || !d_out || !d_codes) throw std::invalid_argument("null pointer");
        long long d[4];
        for (int i = 0; i < N && i < 4; i++) d[i] = (long long)dims[i];
        const fb2::InterpPlan plan = fb2::make_plan(d, N, to_params(p));
        if ((long long)n_codes != plan.n_codes) throw std::invalid_argument("code count does not match the field");
        if ((long long)n_unpred < plan.n_anchor) throw std::invalid_argument("unpredictable list too short");
        const int es = dtype == FALCONS_DTYPE_F32 ? 4 : 8;
        const size_t need = fb2::interp_workspace_bytes(plan, es);
        if (need > (size_t)FALCONS_NOALLOC_SCRATCH_BYTES)
            throw std::invalid_argument("falcons_interp_decompress_noalloc: this field needs " + std::to_string(need) +
                                        " bytes of scratch, more than the " +
                                        std::to_string((size_t)FALCONS_NOALLOC_SCRATCH_BYTES) +
                                        " static bytes (FALCONS_NOALLOC_SCRATCH_BYTES); use "
                                        "falcons_interp_decompress for fields this large");
        void *ws = fb2::static_scratch_current_device();
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        if (dtype == FALCONS_DTYPE_F32)
            fb2::interp_decompress<float>(plan, d_codes, static_cast<const float *>(d_unpred), (long long)n_unpred,
                                          static_cast<float *>(d_out), ws, st);
        else
            fb2::interp_decompress<double>(plan, d_codes, static_cast<const double *>(d_unpred), (long long)n_unpred,
                                          static_cast<double *>(d_out), ws, st);
        fb2::interp_decompress_check(plan, es, ws, (long long)n_unpred, st);
    });
}

int falcons_device_range(falcons_ctx *ctx, int dtype, const void *d_data, size_t n, double *range_out, void *stream) {
    return guarded([&] {
        check_ctx(ctx);
        check_dtype(dtype);
        if (!d_data || n == 0) throw std::invalid_argument("empty input");
        std::lock_guard<std::mutex> lk(ctx->c.mu);
        cudaStream_t st = pick(ctx, stream);
        void *ws = ctx->c.work2.get(fb2::range_workspace_bytes());
        void *res = ctx->c.small.get(64);
        double h[3];
        if (dtype == FALCONS_DTYPE_F32) {
            fb2::device_range<float>(static_cast<const float *>(d_data), (long long)n, static_cast<float *>(res), ws, st);
            float f[3];
            FB2_CUDA(cudaMemcpyAsync(f, res, sizeof(f), cudaMemcpyDeviceToHost, st));
            FB2_CUDA(cudaStreamSynchronize(st));
            h[0] = f[0];
        } else {
            fb2::device_range<double>(static_cast<const double *>(d_data), (long long)n, static_cast<double *>(res), ws,
                                      st);
            FB2_CUDA(cudaMemcpyAsync(h, res, sizeof(h), cudaMemcpyDeviceToHost, st));
            FB2_CUDA(cudaStreamSynchronize(st));
        }
        if (range_out) *range_out = h[0];
    });
}

// ---- full pipeline (pipeline.cu) ----
size_t falcons_compress_size_bound(int dtype, const falcons_config *conf) {
    size_t r = 0;
    if (guarded([&] { r = fb2::compress_size_bound(dtype == FALCONS_DTYPE_F64 ? 8 : 4, conf); }) != FALCONS_OK) return 0;
    return r;
}

int falcons_compress(falcons_ctx *ctx, int dtype, const falcons_config *conf, void *data, uint32_t flags, void *out,
                     size_t cap, size_t *out_len, falcons_config *conf_out) {
    return guarded([&] {
        check_ctx(ctx);
        check_dtype(dtype);
        std::lock_guard<std::mutex> lk(ctx->c.mu);
        fb2::compress_host(ctx->c, dtype == FALCONS_DTYPE_F64 ? 8 : 4, conf, data, flags, out, cap, out_len, conf_out);
    });
}

int falcons_read_config(const void *stream_bytes, size_t len, falcons_config *conf_out) {
    return guarded([&] { fb2::read_config(stream_bytes, len, conf_out); });
}

int falcons_decompress(falcons_ctx *ctx, int dtype, const void *stream_bytes, size_t len, void *out, size_t cap_elems,
                       falcons_config *conf_out) {
    return guarded([&] {
        check_ctx(ctx);
        check_dtype(dtype);
        std::lock_guard<std::mutex> lk(ctx->c.mu);
        fb2::decompress_host(ctx->c, dtype == FALCONS_DTYPE_F64 ? 8 : 4, stream_bytes, len, out, cap_elems, conf_out);
    });
}

int falcons_compress_device(falcons_ctx *ctx, int dtype, const falcons_config *conf, void *d_data, void *d_out,
                            size_t cap, size_t *out_len, falcons_config *conf_out, void *stream) {
    return guarded([&] {
        check_ctx(ctx);
        check_dtype(dtype);
        std::lock_guard<std::mutex> lk(ctx->c.mu);
        fb2::compress_device(ctx->c, dtype == FALCONS_DTYPE_F64 ? 8 : 4, conf, d_data, d_out, cap, out_len, conf_out,
                             pick(ctx, stream));
    });
}

int falcons_decompress_device(falcons_ctx *ctx, int dtype, const void *d_stream, size_t len, void *d_out,
                              size_t cap_elems, falcons_config *conf_out, void *stream) {
    return guarded([&] {
        check_ctx(ctx);
        check_dtype(dtype);
        std::lock_guard<std::mutex> lk(ctx->c.mu);
        fb2::decompress_device(ctx->c, dtype == FALCONS_DTYPE_F64 ? 8 : 4, d_stream, len, d_out, cap_elems, conf_out,
                               pick(ctx, stream));
    });
}

int falcons_compress_batch(falcons_ctx *ctx, falcons_batch_item *items, size_t n, int workers) {
    return guarded([&] {
        check_ctx(ctx);
        fb2::run_batch(ctx->batch, true, items, n, workers);
    });
}

int falcons_decompress_batch(falcons_ctx *ctx, falcons_batch_item *items, size_t n, int workers) {
    return guarded([&] {
        check_ctx(ctx);
        fb2::run_batch(ctx->batch, false, items, n, workers);
    });
}

int falcons_batch_workers(falcons_ctx *ctx, size_t field_bytes) {
    int w = 0;
    if (guarded([&] {
            check_ctx(ctx);
            w = fb2::batch_tuned_workers(ctx->batch, field_bytes);
        }) != FALCONS_OK)
        return 0;
    return w;
}

int falcons_encode_codes(falcons_ctx *ctx, const int16_t *d_codes, size_t n, void *d_out, size_t cap, size_t *out_len,
                         void *stream) {
    return guarded([&] {
        check_ctx(ctx);
        std::lock_guard<std::mutex> lk(ctx->c.mu);
        cudaStream_t st = pick(ctx, stream);
        size_t len = fb2::encode_codes(ctx->c, d_codes, n, static_cast<uint8_t *>(d_out), cap, st);
        FB2_CUDA(cudaStreamSynchronize(st));
        if (out_len) *out_len = len;
    });
}

int falcons_decode_codes(falcons_ctx *ctx, const void *d_in, size_t len, size_t n, int16_t *d_codes, void *stream) {
    return guarded([&] {
        check_ctx(ctx);
        std::lock_guard<std::mutex> lk(ctx->c.mu);
        cudaStream_t st = pick(ctx, stream);
        fb2::decode_codes(ctx->c, static_cast<const uint8_t *>(d_in), len, n, d_codes, st);
        FB2_CUDA(cudaStreamSynchronize(st));
    });
}

}  // extern "C"
