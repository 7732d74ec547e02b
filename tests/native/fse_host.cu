// Test build of the FSE block coder of falcons_b200/csrc/fse.cuh for the host: the same
// __host__ __device__ functions the GPU entropy kernels run (NCount header, count normalization,
// tables, 2-state coding), called on the CPU so that tests/test_fse_host.py checks them against
// the reference's zfse FSE_compress / FSE_decompress without a GPU.  Test infrastructure; the
// product never loads it.
#include <cstring>

#include "../../falcons_b200/csrc/fse.cuh"

using namespace fb2::fse;

extern "C" {
// One block as the entropy coder writes it: returns 0 (store raw), 1 (single symbol) or the size.
long long fseh_compress(const uint8_t *src, size_t n, uint8_t *dst, size_t cap) {
    static BlockScratch w;
    return (long long)compress_block(dst, cap, src, n, w);
}

// Decodes n symbols of a block written by fseh_compress or FSE_compress; 0 on success.
int fseh_decompress(const uint8_t *src, size_t size, uint8_t *out, size_t n) {
    static DEntry dt[1 << kMaxTableLog];
    static uint8_t sym[1 << kMaxTableLog];
    return decompress_block(out, n, src, size, dt, sym) ? 0 : -1;
}

// Normalized counts of a histogram: returns tableLog, 1 or 0 as normalize_count does.
int fseh_normalize(const uint32_t *count, unsigned maxSV, unsigned long long total, unsigned tableLog, int16_t *norm) {
    return (int)normalize_count(norm, tableLog, count, total, maxSV);
}

long long fseh_write_ncount(const int16_t *norm, unsigned maxSV, unsigned tableLog, uint8_t *out) {
    return (long long)write_ncount(out, norm, maxSV, tableLog);
}

// Returns the header size (0 when malformed); maxSV in: the largest symbol accepted, out: the last.
long long fseh_read_ncount(const uint8_t *in, size_t size, int16_t *norm, unsigned *maxSV, unsigned *tableLog) {
    return (long long)read_ncount(norm, maxSV, tableLog, in, size);
}

unsigned fseh_choose_table_log(size_t n, unsigned present) { return choose_table_log(kDefaultTableLog, n, present); }
}
