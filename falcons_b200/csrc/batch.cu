// Batches of fields (batch.cuh): a worker per host thread, each with its own context, fields
// handed out largest first; the worker count per direction and field-size class is tuned on the
// first batch of that class (successive slices of the batch run with 2, 4, 8 and 16 workers, then,
// where the batch has the fields, with 16, 8, 4 and 2 again, and the count with the highest field
// bytes per second in either pass is kept).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>

#include "assemble.cuh"
#include "batch.cuh"
#include "pipeline.cuh"

namespace fb2 {
namespace {

constexpr int kMaxWorkers = 32;

size_t item_bytes(const falcons_batch_item &it, bool compress) {
    const size_t elem = it.dtype == FALCONS_DTYPE_F64 ? 8 : 4;
    if (!compress) return it.cap * elem;  // the caller's output capacity stands for the field size
    size_t num = 1;
    if (it.conf.N < 1 || it.conf.N > 4) return 0;
    for (int i = 0; i < it.conf.N; i++) num *= (size_t)it.conf.dims[i];
    return num * elem;
}

int size_class(size_t bytes) {
    int c = 0;
    while (bytes > 1) {
        bytes >>= 1;
        c++;
    }
    return c;
}

void init_worker(Context &c, int device) {
    c.device = device;
    FB2_CUDA(cudaSetDevice(device));
    FB2_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    stage_reserve(2);  // this worker's share of the pinned read staging
    for (auto &e : c.ev) FB2_CUDA(cudaEventCreate(&e));
}

// One field on one worker; its status (and, on failure, its message) go into the item.
void run_item(Context &c, bool compress, falcons_batch_item &it, std::string &err) {
    int status = FALCONS_OK;
    try {
        if (it.dtype != FALCONS_DTYPE_F32 && it.dtype != FALCONS_DTYPE_F64)
            throw std::invalid_argument("unsupported on GPU build: only float32 and float64 fields are supported");
        const int elem = it.dtype == FALCONS_DTYPE_F64 ? 8 : 4;
        if (compress) {
            const falcons_config in = it.conf;
            size_t len = 0;
            compress_device(c, elem, &in, it.d_data, it.d_stream, it.cap, &len, &it.conf, c.stream);
            it.len = len;
        } else {
            decompress_device(c, elem, it.d_stream, it.len, it.d_data, it.cap, &it.conf, c.stream);
        }
    } catch (const std::invalid_argument &e) {
        status = FALCONS_EINVAL;
        err = e.what();
    } catch (const std::length_error &e) {
        status = FALCONS_ELENGTH;
        err = e.what();
    } catch (const cuda_error &e) {
        status = FALCONS_ECUDA;
        err = e.what();
    } catch (const std::bad_alloc &) {
        status = FALCONS_ENOMEM;
        err = "out of memory";
    } catch (const std::exception &e) {
        status = FALCONS_ERUNTIME;
        err = e.what();
    }
    it.status = status;
}

void ensure_workers(BatchPool &bp, int w) {
    while ((int)bp.workers.size() < w) {
        auto c = std::make_unique<Context>();
        init_worker(*c, bp.device);
        bp.workers.push_back(std::move(c));
    }
}

// Items order[lo, hi) on W workers; returns the wall time in seconds.
double run_range(BatchPool &bp, bool compress, falcons_batch_item *items, const std::vector<size_t> &order, size_t lo,
                 size_t hi, int W, std::vector<std::string> &errs) {
    const auto t0 = std::chrono::steady_clock::now();
    std::atomic<size_t> next{lo};
    auto body = [&](int w) {
        cudaSetDevice(bp.device);
        Context &c = *bp.workers[w];
        for (;;) {
            const size_t k = next.fetch_add(1);
            if (k >= hi) break;
            run_item(c, compress, items[order[k]], errs[order[k]]);
        }
    };
    std::vector<std::thread> th;
    th.reserve(W);
    for (int w = 1; w < W; w++) th.emplace_back(body, w);
    body(0);
    for (auto &t : th) t.join();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

int batch_tuned_workers(BatchPool &bp, size_t bytes) {
    std::lock_guard<std::mutex> lk(bp.mu);
    auto it = bp.best.find(2 * size_class(bytes) + 1);
    return it == bp.best.end() ? 0 : it->second;
}

void run_batch(BatchPool &bp, bool compress, falcons_batch_item *items, size_t n, int workers) {
    if (n == 0) return;
    if (!items) throw std::invalid_argument("null batch");
    std::lock_guard<std::mutex> lk(bp.mu);
    FB2_CUDA(cudaSetDevice(bp.device));
    std::vector<std::string> errs(n);
    std::vector<size_t> bytes(n);
    size_t total = 0;
    for (size_t i = 0; i < n; i++) {
        bytes[i] = item_bytes(items[i], compress);
        total += bytes[i];
        items[i].status = FALCONS_ERUNTIME;  // until the item has run
    }
    std::vector<size_t> order(n);
    std::iota(order.begin(), order.end(), 0);
    size_t pos = 0;
    int W = workers > 0 ? std::min(workers, kMaxWorkers) : 0;
    if (W == 0) {
        const int key = 2 * size_class(total / n) + (compress ? 1 : 0);  // tuned per direction
        auto found = bp.best.find(key);
        if (found != bp.best.end()) {
            W = found->second;
        } else {
            // tune on the batch's own fields, in their given order (a mix of sizes): per candidate
            // count, a slice of w fields that is not timed (the workers' first calls size their
            // scratch), then a timed slice of 6 w fields; where the batch has the fields, the
            // candidates run a second time in the reverse order and each keeps its better rate (a
            // slice that met a stall of the device or the driver does not decide alone)
            const int cand[4] = {2, 4, 8, 16};
            double rate_of[4] = {0, 0, 0, 0};
            int measured = 0;
            for (int pass = 0; pass < 2; pass++) {
                for (int c = 0; c < 4; c++) {
                    const int ci = pass == 0 ? c : 3 - c;
                    const int w = cand[ci];
                    if (pass == 1 && rate_of[ci] == 0) continue;  // not measured in the first pass
                    if (n - pos < (size_t)(7 * w)) {
                        if (pass == 0) break;
                        continue;
                    }
                    ensure_workers(bp, w);
                    run_range(bp, compress, items, order, pos, pos + w, w, errs);
                    pos += w;
                    const double s = run_range(bp, compress, items, order, pos, pos + 6 * w, w, errs);
                    size_t b = 0;
                    for (size_t k = pos; k < pos + 6 * w; k++) b += bytes[order[k]];
                    const double rate = s > 0 ? (double)b / s : 0;
                    if (pass == 0) measured++;
                    rate_of[ci] = std::max(rate_of[ci], rate);
                    pos += 6 * w;
                }
            }
            int best_w = 0;
            double best_rate = 0;
            for (int c = 0; c < 4; c++)
                if (rate_of[c] > best_rate) {
                    best_rate = rate_of[c];
                    best_w = cand[c];
                }
            W = best_w ? best_w : 8;
            if (measured >= 2) bp.best[key] = W;
        }
    }
    // the rest, largest first
    std::sort(order.begin() + pos, order.end(), [&](size_t a, size_t b) { return bytes[a] > bytes[b]; });
    W = std::max(1, std::min<int>(W, (int)std::max<size_t>(1, n - pos)));
    ensure_workers(bp, W);
    if (pos < n) run_range(bp, compress, items, order, pos, n, W, errs);
    for (size_t i = 0; i < n; i++)
        if (items[i].status != FALCONS_OK) {
            const std::string m = "batch item " + std::to_string(i) + ": " + errs[i];
            switch (items[i].status) {
                case FALCONS_EINVAL: throw std::invalid_argument(m);
                case FALCONS_ELENGTH: throw std::length_error(m);
                case FALCONS_ECUDA: throw cuda_error(m);
                default: throw std::runtime_error(m);
            }
        }
}

}  // namespace fb2
