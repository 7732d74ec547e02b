// Batches of fields: many independent compress or decompress calls run concurrently, each on a
// worker of its own (a host thread with a context: a stream and its scratch), so that the
// small kernels and host steps of many fields overlap on the GPU.  Every field goes through the
// same per-field path (pipeline.cu) as a single call, so its stream and reconstruction are the
// same bits as that call's.
#pragma once
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/falcons_b200.h"
#include "context.cuh"

namespace fb2 {

struct BatchPool {
    int device = 0;
    std::mutex mu;                                  // one batch at a time per pool
    std::vector<std::unique_ptr<Context>> workers;  // created on first use, kept for reuse
    std::map<int, int> best;                        // tuned worker count per (field-size class, direction)
};

// Runs items[0, n): compress (d_data -> d_stream) or decompress (d_stream -> d_data).  `workers`
// <= 0 picks the worker count per field-size class with the autotuner.  Per-item errors go to
// the items' status; the call itself fails only on argument or set-up errors.
void run_batch(BatchPool &bp, bool compress, falcons_batch_item *items, size_t n, int workers);

// The worker count the autotuner settled on for compressing fields of about `bytes` bytes (0: not
// tuned).
int batch_tuned_workers(BatchPool &bp, size_t bytes);

}  // namespace fb2
