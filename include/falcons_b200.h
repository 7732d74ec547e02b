/*
 * falcons_b200.h — C ABI of the B200-native Falcons compression path (libfalcons_b200.so).
 *
 * Plain pointers and sizes only.  Host pointers are ordinary (pageable or pinned) memory;
 * device pointers are CUDA global memory on the context's device.  `stream` is a cudaStream_t
 * passed as void* (NULL = the context's private stream).  Every function returns a status
 * (FALCONS_OK = 0) and leaves a message for falcons_last_error() on failure.  Status codes map
 * onto the reference's exception types in include/Falcons/api/falcons.hpp:
 *   FALCONS_EINVAL  -> std::invalid_argument
 *   FALCONS_ELENGTH -> std::length_error
 *   FALCONS_ERUNTIME, FALCONS_ECUDA, FALCONS_ENOMEM -> std::runtime_error
 *
 * Reference interfaces each entry point replaces (JLiu-1/Falcons, include/Falcons/...):
 *   falcons_compress             api/falcons.hpp:54      Falcons_compress<T>(conf, data, cmpData, cmpCap)
 *   falcons_compress_size_bound  api/impl/FalconsImpl.hpp:44  Falcons_compress_size_bound<T>(conf)
 *   falcons_read_config          api/falcons.hpp:122     Falcons_read_config(conf, cmpData, cmpSize)
 *   falcons_decompress           api/falcons.hpp:158,184 Falcons_decompress<T>(conf, cmpData, cmpSize, decData[, cap])
 *   falcons_compress_device      api/falcons.hpp:54      same, with the field already in device memory
 *   falcons_decompress_device    api/falcons.hpp:158     same, reconstructing into device memory
 *   falcons_interp_compress      decomposition/InterpolationDecomposition.hpp:131  compress() -> codes, unpred
 *   falcons_interp_decompress    decomposition/InterpolationDecomposition.hpp:48   decompress()
 *   falcons_device_range         utils/Statistic.hpp:160  data_range()
 *   falcons_encode_codes         encoder/RleFseEncoder.hpp:850-982,1072  preprocess_encode + save + encode
 *   falcons_decode_codes         encoder/RleFseEncoder.hpp:984-1079      load + decode
 */
#ifndef FALCONS_B200_H
#define FALCONS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    FALCONS_OK = 0,
    FALCONS_EINVAL = 1,
    FALCONS_ELENGTH = 2,
    FALCONS_ERUNTIME = 3,
    FALCONS_ECUDA = 4,
    FALCONS_ENOMEM = 5
};

enum { FALCONS_DTYPE_F32 = 0, FALCONS_DTYPE_F64 = 1 };

typedef struct falcons_ctx falcons_ctx;

/* Parameters of the interpolation decomposition (InterpolationDecomposition.hpp:131-146). */
typedef struct {
    double eb;               /* absolute error bound, already resolved */
    int32_t interp_algo;     /* 0 linear, 1 cubic (Config::interpAlgo) */
    int32_t direction;       /* Config::interpDirection: 0 or N!-1 */
    int64_t anchor_stride;   /* Config::interpAnchorStride, resolved (>= 0, power of two) */
    double alpha;            /* Config::interpAlpha */
    double beta;             /* Config::interpBeta */
    int32_t radius;          /* Config::quantbinCnt / 2 */
    int32_t tuning;          /* 1: the auto-tuner's trial sweeps (TUNING::ENABLED), N >= 3 */
    double max_abs;          /* compress: the field's largest |value| when the caller knows it (>= 0);
                                negative or NaN: falcons_interp_compress measures it (one read of the
                                field).  It selects the fused kernels; the output does not depend on it.
                                Ignored by decompress. */
} falcons_interp_params;

/* The fields of Falcons::Config (utils/Config.hpp:482-511) that the path reads or writes. */
typedef struct {
    int32_t N;
    uint64_t dims[4];        /* slowest first, C order */
    uint64_t num;
    int32_t cmprAlgo;        /* ALGO_LORENZO_REG=0, ALGO_INTERP_LORENZO=1, ALGO_INTERP=2, ALGO_NOPRED=3, ALGO_LOSSLESS=4 */
    int32_t errorBoundMode;  /* EB_ABS=0, EB_REL, EB_PSNR, EB_L2NORM, EB_ABS_AND_REL, EB_ABS_OR_REL */
    double absErrorBound;
    double relErrorBound;
    double psnrErrorBound;
    double l2normErrorBound;
    int32_t lorenzo, lorenzo2, regression, regression2, openmp;
    int32_t quantbinCnt;
    int32_t blockSize;
    int32_t predDim;
    int32_t dataType;
    int32_t interpAlgo;
    int32_t interpDirection;
    int32_t interpAnchorStride;  /* -1: default {4096, 128, 32, 16}[N-1] */
    double interpAlpha;
    double interpBeta;
} falcons_config;

/* falcons_compress flags */
#define FALCONS_FLAG_WRITEBACK 1u  /* copy the partially reconstructed field back into the caller's
                                      buffer, as the reference's in-place compressor leaves it */

/* ---- context ---- */
int falcons_ctx_create(falcons_ctx **out, int device);
int falcons_ctx_destroy(falcons_ctx *ctx);
const char *falcons_last_error(void);
const char *falcons_version(void);
/* Number of CUDA kernels this library has launched in the process (all contexts). */
uint64_t falcons_kernel_launches(void);

/* ---- drop-in API (host buffers) ---- */
size_t falcons_compress_size_bound(int dtype, const falcons_config *conf);
int falcons_compress(falcons_ctx *ctx, int dtype, const falcons_config *conf, void *data, uint32_t flags,
                     void *out, size_t cap, size_t *out_len, falcons_config *conf_out);
int falcons_read_config(const void *stream_bytes, size_t len, falcons_config *conf_out);
int falcons_decompress(falcons_ctx *ctx, int dtype, const void *stream_bytes, size_t len, void *out,
                       size_t cap_elems, falcons_config *conf_out);

/* ---- device-resident variants (field in HBM; compressed stream in host or device memory) ---- */
int falcons_compress_device(falcons_ctx *ctx, int dtype, const falcons_config *conf, void *d_data,
                            void *d_out, size_t cap, size_t *out_len, falcons_config *conf_out, void *stream);
int falcons_decompress_device(falcons_ctx *ctx, int dtype, const void *d_stream, size_t len, void *d_out,
                              size_t cap_elems, falcons_config *conf_out, void *stream);

/* ---- stage-level entry points (device pointers) ---- */
int falcons_interp_compress(falcons_ctx *ctx, int dtype, const size_t *dims, int N, const falcons_interp_params *p,
                            void *d_data, int16_t *d_codes, void *d_unpred, size_t *n_codes, size_t *n_unpred,
                            void *stream);
/* Per-launch device times of falcons_interp_compress on this context, for measurement (off by
 * default).  With timing on, every call records a CUDA event pair on its stream around each pass
 * launch (a fused level is one launch); falcons_level_times returns the last call's launches: the
 * level each codes (levels in coding order, the coarsest first and the unit-step level last), its
 * time in ms and the codes of that level, up to `cap` entries, and their number in *count. */
int falcons_time_levels(falcons_ctx *ctx, int on);
int falcons_level_times(falcons_ctx *ctx, int *level, float *ms, unsigned long long *codes, int cap, int *count);
/* falcons_interp_decompress: d_unpred holds n_unpred values (the anchors, then one value per escape
 * code in stream order).  Codes that name more escapes than the list holds return FALCONS_EINVAL
 * without reading past the list.  The call waits for `stream` before it returns. */
int falcons_interp_decompress(falcons_ctx *ctx, int dtype, const size_t *dims, int N,
                              const falcons_interp_params *p, const int16_t *d_codes, size_t n_codes,
                              const void *d_unpred, size_t n_unpred, void *d_out, void *stream);
int falcons_device_range(falcons_ctx *ctx, int dtype, const void *d_data, size_t n, double *range_out, void *stream);
int falcons_encode_codes(falcons_ctx *ctx, const int16_t *d_codes, size_t n, void *d_out, size_t cap,
                         size_t *out_len, void *stream);
int falcons_decode_codes(falcons_ctx *ctx, const void *d_in, size_t len, size_t n, int16_t *d_codes, void *stream);

/* ---- batches of fields (device memory) ----
 *
 * Many independent fields in one call: every item is one Falcons_compress or Falcons_decompress
 * of a field in device memory (api/falcons.hpp:54,158; the reference's per-field driver is
 * api/impl/FalconsAlgoInterp.hpp:33-69, one call per field).  The items run concurrently on
 * worker threads of the context, each with its own stream and scratch, largest first, so the
 * small kernels and host steps of many fields overlap on the GPU; every item's stream and
 * reconstruction are the bits a single falcons_compress_device / falcons_decompress_device call
 * gives.  `workers` <= 0 lets the context's autotuner choose the worker count for the batch's
 * field-size class (tuned on the first batch of that class, kept for the next ones).
 *
 * Per item: compress reads conf, d_data (the field, overwritten with the partial reconstruction),
 * d_stream and cap (its capacity in bytes) and writes len and conf (as stored in the stream);
 * decompress reads d_stream and len and writes d_data (cap: its capacity in elements) and conf.
 * status is FALCONS_OK or the item's own error; the call returns FALCONS_OK when every item
 * succeeded, else the first failed item's status (its message names the item). */
typedef struct {
    int32_t dtype;          /* FALCONS_DTYPE_F32 or FALCONS_DTYPE_F64 */
    int32_t status;         /* out */
    falcons_config conf;
    void *d_data;
    void *d_stream;
    size_t cap;
    size_t len;
} falcons_batch_item;
int falcons_compress_batch(falcons_ctx *ctx, falcons_batch_item *items, size_t n, int workers);
int falcons_decompress_batch(falcons_ctx *ctx, falcons_batch_item *items, size_t n, int workers);
/* The worker count the autotuner chose for compressing fields of about field_bytes bytes (0: not
 * tuned yet).  Compress and decompress are tuned apart. */
int falcons_batch_workers(falcons_ctx *ctx, size_t field_bytes);

/* ---- allocation-free decompress (no counterpart in the reference) ----
 *
 * falcons_interp_decompress without a context and without any device allocation: the same
 * kernels, with their scratch in a static device region of FALCONS_NOALLOC_SCRATCH_BYTES per
 * device instead of the context's work buffers.  It is for callers that cannot let a library
 * allocate device memory: an application that hands nearly all of HBM to its own pool at
 * start-up leaves cudaMalloc nothing to give, and a latency-bound decode thread cannot absorb
 * cudaFree's implicit device-wide synchronisation or a work buffer's first-use growth.
 *
 * - Limit: the field's scratch (about 4 bytes per code for float, 8 for double, plus 12 bytes per
 *   4096 codes) must fit in FALCONS_NOALLOC_SCRATCH_BYTES (64 MiB: about 16.7 million float or
 *   8.3 million double codes).  Larger fields are rejected with FALCONS_EINVAL and a message
 *   giving the size needed; use falcons_interp_decompress for them.
 * - Device and stream: works on the CURRENT device; `stream` is a cudaStream_t of that device
 *   (NULL: the default stream).  The call returns once the stream's work up to and including it
 *   has finished (it reads back the number of escape codes, 8 bytes, to check it against
 *   n_unpred), so d_out is complete on return.
 * - Set-up: the first call on a device (with that device current) resolves the scratch address
 *   and loads the decompress kernels there, which reserves the region; make that first call
 *   before any stream capture begins.  Later calls allocate nothing.  The resolved address is kept
 *   for the life of the process: a device reset (cudaDeviceReset) after the first call is not
 *   supported.
 * - Nothing in the scratch has to start at zero: every word the call reads, it wrote earlier in
 *   the same call.
 * - Overlapping calls race: all calls on a device share the one region, so two calls whose work
 *   overlaps in time (on different streams, or from different threads) corrupt each other's
 *   scratch.  Issue them on one stream, or make each call's stream wait for the previous call.
 * Arguments and results are those of falcons_interp_decompress. */
#define FALCONS_NOALLOC_SCRATCH_BYTES (64u << 20)
int falcons_interp_decompress_noalloc(int dtype, const size_t *dims, int N, const falcons_interp_params *p,
                                      const int16_t *d_codes, size_t n_codes, const void *d_unpred,
                                      size_t n_unpred, void *d_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* FALCONS_B200_H */
