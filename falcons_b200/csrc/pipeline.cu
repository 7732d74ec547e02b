#include <stdexcept>

#include "entropy.cuh"
#include "pipeline.cuh"

namespace fb2 {
size_t compress_size_bound(int, const falcons_config *) { throw std::runtime_error("not implemented"); }
void compress_host(Context &, int, const falcons_config *, void *, uint32_t, void *, size_t, size_t *, falcons_config *) {
    throw std::runtime_error("not implemented");
}
void read_config(const void *, size_t, falcons_config *) { throw std::runtime_error("not implemented"); }
void decompress_host(Context &, int, const void *, size_t, void *, size_t, falcons_config *) {
    throw std::runtime_error("not implemented");
}
void compress_device(Context &, int, const falcons_config *, void *, void *, size_t, size_t *, falcons_config *,
                     cudaStream_t) {
    throw std::runtime_error("not implemented");
}
void decompress_device(Context &, int, const void *, size_t, void *, size_t, falcons_config *, cudaStream_t) {
    throw std::runtime_error("not implemented");
}
size_t encode_codes(Context &ctx, const int16_t *d_codes, size_t n, uint8_t *d_out, size_t cap, cudaStream_t st) {
    const EntropyChoice ch = choose_entropy(ctx, d_codes, n, st);
    return entropy_encode(ctx, d_codes, n, ch, d_out, cap, st);
}
void decode_codes(Context &ctx, const uint8_t *d_in, size_t len, size_t n, int16_t *d_codes, cudaStream_t st) {
    entropy_decode(ctx, d_in, nullptr, len, n, d_codes, st);
}
}  // namespace fb2
