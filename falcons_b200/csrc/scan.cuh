// Device-wide exclusive prefix sums (tile reduce -> single-block scan of tile sums -> tile
// downsweep), and warp/block scan helpers shared by the entropy kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace fb2 {

template <class T>
__device__ __forceinline__ T warp_incl_scan(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
    }
    return v;
}

// Block-wide exclusive scan; returns the exclusive prefix and writes the block total.
// `sh` must hold 32 elements.  All threads of the block must call it.
template <class T>
__device__ __forceinline__ T block_excl_scan(T v, T *sh, T &total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    T incl = warp_incl_scan(v);
    if (lane == 31) sh[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        T w = lane < nw ? sh[lane] : T(0);
        w = warp_incl_scan(w);
        sh[lane] = w;
    }
    __syncthreads();
    const T before = wid ? sh[wid - 1] : T(0);
    total = sh[nw - 1];
    __syncthreads();
    return before + incl - v;
}

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

template <class TIn, class TOut>
__global__ void __launch_bounds__(kScanThreads) k_tile_reduce(const TIn *__restrict__ in, long long n,
                                                             TOut *__restrict__ tile_sum) {
    const long long base = (long long)blockIdx.x * kScanTile;
    TOut s = 0;
    for (int j = 0; j < kScanItems; j++) {
        const long long i = base + (long long)j * kScanThreads + threadIdx.x;
        if (i < n) s += (TOut)in[i];
    }
    __shared__ TOut sh[32];
    TOut tot;
    block_excl_scan<TOut>(s, sh, tot);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = tot;
}

// In-place exclusive scan of n values with one block; writes data[n] = total.
template <class T>
__global__ void __launch_bounds__(1024) k_scan_small(T *__restrict__ data, long long n) {
    __shared__ T sh[32];
    __shared__ T carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long long base = 0; base < n; base += blockDim.x) {
        const long long i = base + threadIdx.x;
        const T v = i < n ? data[i] : T(0);
        T tot;
        const T ex = block_excl_scan<T>(v, sh, tot);
        if (i < n) data[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) data[n] = carry;
}

template <class TIn, class TOut>
__global__ void __launch_bounds__(kScanThreads) k_tile_downsweep(const TIn *__restrict__ in, long long n,
                                                                const TOut *__restrict__ tile_off,
                                                                TOut *__restrict__ out) {
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    TOut v[kScanItems];
    TOut s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const long long i = base + j;
        v[j] = i < n ? (TOut)in[i] : TOut(0);
        s += v[j];
    }
    __shared__ TOut sh[32];
    TOut tot;
    TOut run = block_excl_scan<TOut>(s, sh, tot) + tile_off[blockIdx.x];
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const long long i = base + j;
        if (i < n) out[i] = run;
        run += v[j];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) out[n] = run;
}

// Scratch for exclusive_scan: (tiles + 1) * sizeof(TOut)
inline size_t scan_scratch_bytes(long long n, int out_size) {
    const long long tiles = (n + kScanTile - 1) / kScanTile;
    return (size_t)(tiles + 2) * out_size + 256;
}

// out[0..n] = exclusive prefix sums of in[0..n), out[n] = total.  Note: the reduce phase
// sums in a strided order and the downsweep in a contiguous order; both are exact for integers.
template <class TIn, class TOut>
void exclusive_scan(const TIn *in, long long n, TOut *out, void *scratch, cudaStream_t st) {
    if (n <= 0) {
        FB2_CUDA(cudaMemsetAsync(out, 0, sizeof(TOut), st));
        return;
    }
    const long long tiles = (n + kScanTile - 1) / kScanTile;
    TOut *ts = static_cast<TOut *>(scratch);
    k_tile_reduce<TIn, TOut><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, ts);
    FB2_CHECK_LAUNCH();
    k_scan_small<TOut><<<1, 1024, 0, st>>>(ts, tiles);
    FB2_CHECK_LAUNCH();
    k_tile_downsweep<TIn, TOut><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, ts, out);
    FB2_CHECK_LAUNCH();
}

}  // namespace fb2
