/*
 * Minimal declarations of the public libzstd entry points that the reference's
 * lossless stage (include/Falcons/lossless/Lossless_zstd.hpp) and the tuner call.
 *
 * Test infrastructure only: this header lets the oracle recipe compile the
 * reference sources against the runtime libzstd.so.1 present in the image, which
 * ships without development headers.  The prototypes are the documented public
 * libzstd API (stable since v1.3); nothing here is product code.
 */
#ifndef ORACLE_ZSTD_DECL_H
#define ORACLE_ZSTD_DECL_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ZSTD_CONTENTSIZE_UNKNOWN (0ULL - 1)
#define ZSTD_CONTENTSIZE_ERROR (0ULL - 2)

size_t ZSTD_compress(void *dst, size_t dstCapacity, const void *src, size_t srcSize, int compressionLevel);
size_t ZSTD_decompress(void *dst, size_t dstCapacity, const void *src, size_t compressedSize);
size_t ZSTD_compressBound(size_t srcSize);
unsigned ZSTD_isError(size_t code);
const char *ZSTD_getErrorName(size_t code);
unsigned long long ZSTD_getFrameContentSize(const void *src, size_t srcSize);

#ifdef __cplusplus
}
#endif
#endif
