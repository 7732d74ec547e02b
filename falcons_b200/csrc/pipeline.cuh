// Full compress / decompress pipeline (stream format of the reference's serial build).
#pragma once
#include <stdint.h>

#include "../../include/falcons_b200.h"
#include "context.cuh"

namespace fb2 {

size_t compress_size_bound(int elem, const falcons_config *conf);
void compress_host(Context &ctx, int elem, const falcons_config *conf, void *data, uint32_t flags, void *out,
                   size_t cap, size_t *out_len, falcons_config *conf_out);
void read_config(const void *bytes, size_t len, falcons_config *conf_out);
void decompress_host(Context &ctx, int elem, const void *bytes, size_t len, void *out, size_t cap_elems,
                     falcons_config *conf_out);
void compress_device(Context &ctx, int elem, const falcons_config *conf, void *d_data, void *d_out, size_t cap,
                     size_t *out_len, falcons_config *conf_out, cudaStream_t st);
void decompress_device(Context &ctx, int elem, const void *d_stream, size_t len, void *d_out, size_t cap_elems,
                       falcons_config *conf_out, cudaStream_t st);

// Entropy stage (RleFseEncoder format): returns bytes written to d_out.
size_t encode_codes(Context &ctx, const int16_t *d_codes, size_t n, uint8_t *d_out, size_t cap, cudaStream_t st);
void decode_codes(Context &ctx, const uint8_t *d_in, size_t len, size_t n, int16_t *d_codes, cudaStream_t st);

}  // namespace fb2
