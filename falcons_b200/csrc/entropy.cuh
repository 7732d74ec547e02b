// Entropy stage in the RleFseEncoder<int16_t> stream format (reference encoder/RleFseEncoder.hpp).
//
// Encoder header (save/load, :1072-1079): [u8 method | use_delta << 7][u16 lo][u16 mode].
// method 0 (:897-982):  6 x u64 [nr nv s_rcl s_vcl rbp vbp] | FSE(run classes) | FSE(value classes)
//                       | run mantissas | value mantissas   (Elias-gamma classes + MSB-first raw bits)
// method 1 (:582-843):  u64 S, then S segments, each: u64 N, u64 K, K x u64 blen, K x u64 nvk,
//                       15 x 256 x u16 normalized counts, K tANS streams, escape block (:483-575).
// FSE class streams (fse_enc/fse_dec, :150-187) are 64 Ki-symbol blocks [u8 flag][...].
//
// The device encoder chooses method and delta exactly as preprocess_encode (:850-895) does, so the
// method byte matches the reference.  Within method 1 it chooses its own segment count S (the
// decoder reads S from the stream) to expose 16 x S independent tANS chains; K = 16 (the reference
// decoder's limit).  Every table, count and stream it writes is decodable by the reference.
#pragma once
#include <stdint.h>

#include <vector>

#include "assemble.cuh"
#include "context.cuh"

namespace fb2 {

struct EntropyChoice {
    int method;        // 0 = RLE + gamma + FSE, 1 = order-1 tANS
    bool delta;        // forward difference before coding
};

// Encoder-side tunables (chosen by the autotuner; defaults give ~2% table overhead).
struct EntropyTuning {
    long long o1_segment = 0;          // symbols per method-1 segment (0 = automatic)
    int o1_streams = 16;               // K, 1..16
    bool per_segment_tables = false;   // one table set per segment (the reference's choice)
    std::vector<long long> regions;    // code positions where the statistics change (level starts);
                                       // segments of one region share a table set
};

EntropyChoice choose_entropy(Context &ctx, const int16_t *d_codes, size_t n, cudaStream_t st);

// Encodes n codes (device) into d_out (device); returns the encoder header + payload size.
// The code array is not modified.
size_t entropy_encode(Context &ctx, const int16_t *d_codes, size_t n, const EntropyChoice &ch, uint8_t *d_out,
                      size_t cap, cudaStream_t st, const EntropyTuning &tune = EntropyTuning());

// Appends the encoder header + payload pieces to `as` (pieces reference scratch owned by `pool`).
void entropy_encode_into(Pool &pool, Assembler &as, const int16_t *d_codes, size_t n, const EntropyChoice &ch,
                         cudaStream_t st, const EntropyTuning &tune = EntropyTuning());

// Decodes the encoder header + payload into n codes.  d_in: the bytes on the device (flat);
// h: the same bytes readable on the host (used to parse the block structure).  Returns the
// number of bytes consumed.
size_t entropy_decode(Context &ctx, const uint8_t *d_in, const ByteView &h, size_t n, int16_t *d_codes,
                      cudaStream_t st);

}  // namespace fb2
