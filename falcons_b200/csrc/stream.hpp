// Host-side serialisation of the reference's serial stream format.
//
//   [Config header]   utils/Config.hpp:316-360 (save), :372-454 (load)
//   [u64 srcLen][zstd frame(buffer)]                lossless/Lossless_zstd.hpp:29-46
//   buffer = decomposition header ‖ u64 n_codes ‖ encoder header ‖ encoder payload
//            compressor/FalconsGenericCompressor.hpp:73-89
//   decomposition header  InterpolationDecomposition.hpp:241-251 + LinearQuantizer.hpp:142-152
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/falcons_b200.h"

namespace fb2 {

constexpr uint32_t kMagic = 0xF342F310u;        // Falcons_MAGIC_NUMBER
constexpr uint32_t kDataVersion = 1u << 24;     // versionInt("1.0.0")
enum { ALGO_LORENZO_REG = 0, ALGO_INTERP_LORENZO, ALGO_INTERP, ALGO_NOPRED, ALGO_LOSSLESS };
enum { EB_ABS = 0, EB_REL, EB_PSNR, EB_L2NORM, EB_ABS_AND_REL, EB_ABS_OR_REL };

// Normalises dims the way Config::setDims does (drops dims <= 1; all ones -> {1}).
void normalize_dims(falcons_config &c);
void default_config(falcons_config &c);

// Config::save; returns the header size (byte 0 holds it).
size_t config_save(const falcons_config &c, uint8_t *out);
size_t config_size(const falcons_config &c);
// Config::load + the checks of Falcons_read_config (magic, data version, payload presence).
size_t config_load(const uint8_t *in, size_t avail, falcons_config &c);

struct DecompHeader {
    int N;
    uint64_t dims[4];
    uint32_t blocksize;
    int32_t interp_id, direction;
    uint64_t anchor;
    double alpha, beta;
    uint8_t quant_uid;
    double eb;
    int32_t radius;
    int32_t n_unpred;
};
size_t decomp_header_size(int N);
void decomp_header_write(const DecompHeader &h, std::vector<uint8_t> &out);

// libzstd (runtime-loaded) for frames with compressed blocks and for the dispatcher's
// lossless comparison; throws std::runtime_error when the library is unavailable.
bool zstd_available();
size_t zstd_compress_bound(size_t n);
size_t zstd_compress(const void *src, size_t n, void *dst, size_t cap, int level);
// ZSTD_compress of src[0, n) at `level` into `out` when its size is below `limit` (returns true);
// false when it is not.  Fields whose frame is far larger than `limit` stop early: the streaming
// API codes the input a chunk at a time and the call gives up once its frame so far exceeds
// limit by 2 % + 4 KiB (the streaming frame's size can differ from ZSTD_compress's by a few bytes,
// never by that much); otherwise the answer is ZSTD_compress's own frame.
bool zstd_compress_if_below(const void *src, size_t n, int level, size_t limit, std::vector<uint8_t> &out);
size_t zstd_decompress(const void *src, size_t n, void *dst, size_t cap);
unsigned long long zstd_frame_content_size(const void *src, size_t n);

// True when [src, src+n) is one zstd frame of raw blocks with a content size (and optional
// trailing skippable frames); sets the offset of the first block header and the content size.
bool parse_raw_frame(const uint8_t *src, size_t n, size_t &first_block, size_t &content);

}  // namespace fb2
