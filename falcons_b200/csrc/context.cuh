// Per-device library context: grow-only device/host scratch buffers and a private stream.
#pragma once
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "common.cuh"

namespace fb2 {

// A grow-only device allocation (never shrinks; freed with the context).
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    void *get(size_t need) {
        if (need > bytes) {
            if (ptr) FB2_CUDA(cudaFree(ptr));
            ptr = nullptr;
            bytes = 0;
            size_t cap = need + need / 8 + 4096;
            FB2_CUDA(cudaMalloc(&ptr, cap));
            bytes = cap;
        }
        return ptr;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

struct PinnedBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    void *get(size_t need) {
        if (need > bytes) {
            if (ptr) FB2_CUDA(cudaFreeHost(ptr));
            ptr = nullptr;
            bytes = 0;
            size_t cap = need + need / 8 + 4096;
            FB2_CUDA(cudaMallocHost(&ptr, cap));
            bytes = cap;
        }
        return ptr;
    }
    void release() {
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

struct Context {
    int device = 0;
    cudaStream_t stream = nullptr;
    // measurement of falcons_interp_compress (falcons_time_levels): the last call's launches
    bool time_levels = false;
    std::vector<int> lt_level;
    std::vector<float> lt_ms;
    std::vector<unsigned long long> lt_codes;
    std::mutex mu;                 // one call at a time per context
    DevBuf field, codes, unpred, work, work2, out, small;
    PinnedBuf host_small;
    cudaEvent_t ev[8] = {};
    // a second stream for work that overlaps the calling stream, with its fork/join events
    // (created on first use by side_stream())
    cudaStream_t side = nullptr;
    cudaEvent_t side_ev[3] = {};
    ~Context() {
        field.release();
        codes.release();
        unpred.release();
        work.release();
        work2.release();
        out.release();
        small.release();
        host_small.release();
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
        for (auto &e : side_ev)
            if (e) cudaEventDestroy(e);
        if (side) cudaStreamDestroy(side);
        if (stream) cudaStreamDestroy(stream);
    }
};

// The context's second stream (non-blocking), created on first use on the current device.  (At
// the highest stream priority it let the large encoders of one field start a few percent sooner,
// but under many concurrent requests it held back the other workers' kernels: serving latency
// several times higher.)
inline cudaStream_t side_stream(Context &ctx) {
    if (!ctx.side) FB2_CUDA(cudaStreamCreateWithFlags(&ctx.side, cudaStreamNonBlocking));
    for (auto &e : ctx.side_ev)
        if (!e) FB2_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return ctx.side;
}

// Work issued on `side` after construction is ordered after the work already issued on `st`;
// work issued on `st` after join() (or after destruction) is ordered after all of it.
struct SideFork {
    cudaStream_t st, side;
    cudaEvent_t fork_ev, join_ev;
    bool joined = false;
    SideFork(Context &ctx, cudaStream_t s) : st(s), side(side_stream(ctx)), fork_ev(ctx.side_ev[0]),
                                             join_ev(ctx.side_ev[1]) {
        FB2_CUDA(cudaEventRecord(fork_ev, st));
        FB2_CUDA(cudaStreamWaitEvent(side, fork_ev, 0));
    }
    void join() {
        FB2_CUDA(cudaEventRecord(join_ev, side));
        FB2_CUDA(cudaStreamWaitEvent(st, join_ev, 0));
        joined = true;
    }
    ~SideFork() {
        if (!joined) {  // error paths: the calling stream must not free what `side` still uses
            cudaEventRecord(join_ev, side);
            cudaStreamWaitEvent(st, join_ev, 0);
        }
    }
};

}  // namespace fb2
