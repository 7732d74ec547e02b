// Entries of the 1-D blockwise Lorenzo + Huffman path (lorenzo.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../include/falcons_b200.h"
#include "assemble.cuh"

namespace fb2 {

// Whether a stream's Config selects the Lorenzo path decoded here: a 1-D field, Lorenzo
// order 1 and / or 2 (composed per block when both are on), no regression predictor.
bool lorenzo_stream_supported(const falcons_config &c);

// Writes [u64 payload bytes][zstd raw-block frame of the payload] of field d_x (c.num values, not
// modified) to d_pay; returns the bytes written; throws std::length_error past pcap.
template <class T>
size_t lorenzo_compress(const falcons_config &c, const T *d_x, uint8_t *d_pay, size_t pcap, cudaStream_t st);

// The interpolation tuner's Lorenzo trial (lorenzo_compress_test, FalconsAlgoInterp.hpp:229-262)
// over B sample blocks of V points (device, contiguous): the compression ratio of their
// blockwise Lorenzo codes (orders 1 and 2, block 5) with quantbin / 2 as radius, zstd level 3.
template <class T>
double lorenzo_trial_ratio(const T *d_blocks, long long B, long long V, double eb, int quantbin, cudaStream_t st);

// Decodes the logical payload (host view `view` for its headers, device copy d_flat for its bulk)
// into d_out (c.num values); throws std::invalid_argument on a malformed payload.
template <class T>
void lorenzo_decompress(const falcons_config &c, const ByteView &view, const uint8_t *d_flat, T *d_out,
                        cudaStream_t st);

}  // namespace fb2
