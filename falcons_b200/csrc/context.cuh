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
    std::mutex mu;                 // one call at a time per context
    DevBuf field, codes, unpred, work, work2, out, small;
    PinnedBuf host_small;
    cudaEvent_t ev[8] = {};
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
        if (stream) cudaStreamDestroy(stream);
    }
};

}  // namespace fb2
