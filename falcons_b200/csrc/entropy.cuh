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

// Decode checkpoints (the "FB2C" skippable frame written after the header index).  The tANS chains
// of method 1 and the FSE class blocks are sequential bit streams; at every `part` symbols the
// encoder records where the decoder will be (bit position, state(s), context, escape count), so
// the decoder runs every part of every stream at once instead of one thread per stream.  Frame
// content: u32 tag "FB2C", u32 version 1, u32 o1_part, u32 fse_part, u64 n_o1, u64 n_fse, then
// n_o1 chain checkpoints of 12 bytes and n_fse block checkpoints of 8 bytes, in stream order.
// Decoders that do not know the frame (the reference's included) skip it.
constexpr uint32_t kCkptTag = 0x43324246u;  // "FB2C"
constexpr uint32_t kCkptVersion = 1;
constexpr size_t kCkptHeader = 32;          // content bytes before the arrays

struct DecodeCheckpoints {
    const uint8_t *d_o1 = nullptr;   // device address of the chain checkpoints (any alignment)
    unsigned long long n_o1 = 0;
    uint32_t o1_part = 0;
    const uint8_t *d_fse = nullptr;  // device address of the block checkpoints
    unsigned long long n_fse = 0;
    uint32_t fse_part = 0;
};

// Reads an FB2C frame content header (kCkptHeader bytes); d_content is the device address of the
// content and avail the content size.  Returns false when it is not a usable checkpoint frame.
bool parse_ckpt_header(const uint8_t *h, const uint8_t *d_content, size_t avail, DecodeCheckpoints &out);

// Encoder-side tunables.
struct EntropyTuning {
    long long o1_segment = 0;          // symbols per method-1 segment (0: the reference's count, N / 8 Mi in [1, 16])
    int o1_streams = 16;               // K, 1..16
    bool per_segment_tables = false;   // one table set per segment (the reference's choice)
    std::vector<long long> regions;    // code positions where the statistics change (level starts);
                                       // segments of one region share a table set
    uint32_t ckpt_part = 1024;         // symbols per decode part (power of two, 0 = no checkpoints)
    // a second stream (and two events) on which the escape side stream runs next to the chain
    // encoder; none: everything runs on the calling stream
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    // recorded on `side` when the escape class blocks are next in line; the chain encoder waits
    // for it, so that the blocks, launched first, take their SMs before the encoder's CTAs fill
    // the rest
    cudaEvent_t queued_ev = nullptr;
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
                      cudaStream_t st, const DecodeCheckpoints *ck = nullptr);

}  // namespace fb2
