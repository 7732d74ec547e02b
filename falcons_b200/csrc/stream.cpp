#include "stream.hpp"

#include <dlfcn.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <stdexcept>

namespace fb2 {

namespace {
template <class T>
void put(uint8_t *&p, T v) {
    memcpy(p, &v, sizeof(T));
    p += sizeof(T);
}
template <class T>
T get(const uint8_t *&p, const uint8_t *end) {
    if ((size_t)(end - p) < sizeof(T)) throw std::invalid_argument("Truncated Falcons configuration field");
    T v;
    memcpy(&v, p, sizeof(T));
    p += sizeof(T);
    return v;
}
}  // namespace

void default_config(falcons_config &c) {
    memset(&c, 0, sizeof(c));
    c.N = 1;
    c.dims[0] = 1;
    c.num = 1;
    c.cmprAlgo = ALGO_INTERP_LORENZO;
    c.errorBoundMode = EB_ABS;
    c.absErrorBound = 1e-3;
    c.lorenzo = 1;
    c.regression = 1;
    c.quantbinCnt = 65536;
    c.interpAlgo = 1;
    c.interpAnchorStride = -1;
    c.interpAlpha = 1.25;
    c.interpBeta = 2.0;
}

void normalize_dims(falcons_config &c) {
    uint64_t d[4];
    int n = 0;
    if (c.N < 0 || c.N > 4) throw std::invalid_argument("Data dimension higher than 4 is not supported.");
    for (int i = 0; i < c.N; i++)
        if (c.dims[i] > 1) d[n++] = c.dims[i];
    if (n == 0) {
        d[0] = 1;
        n = 1;
    }
    c.N = n;
    c.num = 1;
    for (int i = 0; i < 4; i++) c.dims[i] = i < n ? d[i] : 0;
    for (int i = 0; i < n; i++) c.num *= d[i];
    c.predDim = n;
    if (c.blockSize == 0) c.blockSize = (n == 1 ? 128 : (n == 2 ? 16 : 6));
}

size_t config_save(const falcons_config &c, uint8_t *out) {
    uint8_t *p = out + 1;
    put<uint32_t>(p, kMagic);
    put<uint32_t>(p, kDataVersion);
    put<char>(p, (char)c.N);
    // utils/ByteUtil.hpp vector_bit_width / vector2bytes: LSB-first packing of the dims
    uint64_t mx = 0;
    for (int i = 0; i < c.N; i++) mx = std::max<uint64_t>(mx, c.dims[i]);
    uint8_t bw = 0;
    while (mx > 0) {
        mx >>= 1;
        bw++;
    }
    put<uint8_t>(p, bw);
    const size_t nbytes = ((size_t)c.N * bw + 7) / 8;
    memset(p, 0, nbytes);
    size_t bit = 0;
    for (int i = 0; i < c.N; i++)
        for (int b = 0; b < bw; b++, bit++)
            if ((c.dims[i] >> b) & 1) p[bit / 8] |= (uint8_t)(1u << (bit % 8));
    p += nbytes;
    put<uint64_t>(p, c.num);
    put<uint8_t>(p, (uint8_t)c.cmprAlgo);
    put<uint8_t>(p, (uint8_t)c.errorBoundMode);
    switch (c.errorBoundMode) {
        case EB_ABS: put<double>(p, c.absErrorBound); break;
        case EB_REL: put<double>(p, c.relErrorBound); break;
        case EB_PSNR: put<double>(p, c.psnrErrorBound); break;
        case EB_L2NORM: put<double>(p, c.l2normErrorBound); break;
        case EB_ABS_OR_REL:
        case EB_ABS_AND_REL:
            put<double>(p, c.absErrorBound);
            put<double>(p, c.relErrorBound);
            break;
        default: break;
    }
    const uint8_t boolvals = (uint8_t)(((c.lorenzo & 1) << 7) | ((c.lorenzo2 & 1) << 6) | ((c.regression & 1) << 5) |
                                       ((c.regression2 & 1) << 4) | ((c.openmp & 1) << 3));
    put<uint8_t>(p, boolvals);
    put<uint8_t>(p, (uint8_t)c.dataType);
    put<int32_t>(p, c.quantbinCnt);
    put<int32_t>(p, c.blockSize);
    put<uint8_t>(p, (uint8_t)c.predDim);
    const size_t sz = (size_t)(p - out);
    if (sz > 255) throw std::length_error("configuration header too large");
    out[0] = (uint8_t)sz;
    return sz;
}

size_t config_size(const falcons_config &c) {
    uint8_t tmp[512];
    return config_save(c, tmp);
}

size_t config_load(const uint8_t *in, size_t avail, falcons_config &c) {
    if (!in || avail < 1) throw std::invalid_argument("Truncated Falcons configuration");
    const size_t hs = in[0];
    if (hs < 1 || hs > avail) throw std::invalid_argument("Truncated Falcons configuration");
    const uint8_t *p = in + 1, *end = in + hs;
    default_config(c);
    const uint32_t magic = get<uint32_t>(p, end);
    const uint32_t ver = get<uint32_t>(p, end);
    const int N = get<char>(p, end);
    const uint8_t bw = get<uint8_t>(p, end);
    if (N < 1 || N > 4 || bw < 1 || bw > 64) throw std::invalid_argument("Invalid Falcons dimensions");
    const size_t nbytes = ((size_t)N * bw + 7) / 8;
    if ((size_t)(end - p) < nbytes) throw std::invalid_argument("Truncated Falcons dimensions");
    c.N = N;
    size_t bit = 0;
    for (int i = 0; i < N; i++) {
        uint64_t v = 0;
        for (int b = 0; b < bw; b++, bit++) v |= (uint64_t)((p[bit / 8] >> (bit % 8)) & 1) << b;
        c.dims[i] = v;
    }
    p += nbytes;
    c.num = get<uint64_t>(p, end);
    uint64_t expected = 1;
    for (int i = 0; i < N; i++) {
        if (c.dims[i] == 0 || c.dims[i] > ~0ULL / expected) throw std::invalid_argument("Invalid Falcons element count");
        expected *= c.dims[i];
    }
    if (c.num != expected) throw std::invalid_argument("Falcons dimensions do not match element count");
    c.cmprAlgo = get<uint8_t>(p, end);
    c.errorBoundMode = get<uint8_t>(p, end);
    if (c.errorBoundMode > EB_ABS_OR_REL || c.cmprAlgo > ALGO_LOSSLESS)
        throw std::invalid_argument("Invalid Falcons algorithm or error mode");
    switch (c.errorBoundMode) {
        case EB_ABS: c.absErrorBound = get<double>(p, end); break;
        case EB_REL: c.relErrorBound = get<double>(p, end); break;
        case EB_PSNR: c.psnrErrorBound = get<double>(p, end); break;
        case EB_L2NORM: c.l2normErrorBound = get<double>(p, end); break;
        default:
            c.absErrorBound = get<double>(p, end);
            c.relErrorBound = get<double>(p, end);
            break;
    }
    if (p < end) {
        const uint8_t b = get<uint8_t>(p, end);
        c.lorenzo = (b >> 7) & 1;
        c.lorenzo2 = (b >> 6) & 1;
        c.regression = (b >> 5) & 1;
        c.regression2 = (b >> 4) & 1;
        c.openmp = (b >> 3) & 1;
    }
    if (p < end) c.dataType = get<uint8_t>(p, end);
    if (p < end) c.quantbinCnt = get<int32_t>(p, end);
    if (p < end) c.blockSize = get<int32_t>(p, end);
    if (p < end) c.predDim = get<uint8_t>(p, end);
    if (magic != kMagic)
        throw std::invalid_argument("magic number mismatch, the input data is not compressed by Falcons");
    if (ver != kDataVersion) throw std::invalid_argument("Please use the Falcons version that wrote this stream");
    if (avail <= hs) throw std::invalid_argument("Missing Falcons compressed payload");
    return hs;
}

size_t decomp_header_size(int N) { return (size_t)N * 8 + 4 + 4 + 4 + 8 + 8 + 8 + 1 + 8 + 4 + 4; }

void decomp_header_write(const DecompHeader &h, std::vector<uint8_t> &out) {
    const size_t o = out.size();
    out.resize(o + decomp_header_size(h.N));
    uint8_t *p = out.data() + o;
    for (int i = 0; i < h.N; i++) put<uint64_t>(p, h.dims[i]);
    put<uint32_t>(p, h.blocksize);
    put<int32_t>(p, h.interp_id);
    put<int32_t>(p, h.direction);
    put<uint64_t>(p, h.anchor);
    put<double>(p, h.alpha);
    put<double>(p, h.beta);
    put<uint8_t>(p, h.quant_uid);
    put<double>(p, h.eb);
    put<int32_t>(p, h.radius);
    put<int32_t>(p, h.n_unpred);
}

// ------------------------------------------------------------------ libzstd (runtime-loaded)
namespace {
// The streaming entry points of the stable zstd API (zstd.h, 1.4.0 on): ZSTD_inBuffer /
// ZSTD_outBuffer, ZSTD_c_compressionLevel = 100, ZSTD_e_continue = 0, ZSTD_e_end = 2.
struct ZInBuf {
    const void *src;
    size_t size, pos;
};
struct ZOutBuf {
    void *dst;
    size_t size, pos;
};
struct Zstd {
    void *h = nullptr;
    size_t (*compress)(void *, size_t, const void *, size_t, int) = nullptr;
    size_t (*decompress)(void *, size_t, const void *, size_t) = nullptr;
    size_t (*bound)(size_t) = nullptr;
    unsigned (*is_error)(size_t) = nullptr;
    unsigned long long (*fcs)(const void *, size_t) = nullptr;
    // optional (streaming)
    void *(*create_cctx)() = nullptr;
    size_t (*free_cctx)(void *) = nullptr;
    size_t (*set_param)(void *, int, int) = nullptr;
    size_t (*set_pledged)(void *, unsigned long long) = nullptr;
    size_t (*stream2)(void *, ZOutBuf *, ZInBuf *, int) = nullptr;
    Zstd() {
        const char *names[] = {"libzstd.so.1", "libzstd.so"};
        for (const char *n : names) {
            h = dlopen(n, RTLD_NOW | RTLD_LOCAL);
            if (h) break;
        }
        if (!h) return;
        compress = (decltype(compress))dlsym(h, "ZSTD_compress");
        decompress = (decltype(decompress))dlsym(h, "ZSTD_decompress");
        bound = (decltype(bound))dlsym(h, "ZSTD_compressBound");
        is_error = (decltype(is_error))dlsym(h, "ZSTD_isError");
        fcs = (decltype(fcs))dlsym(h, "ZSTD_getFrameContentSize");
        if (!compress || !decompress || !bound || !is_error || !fcs) h = nullptr;
        if (!h) return;
        create_cctx = (decltype(create_cctx))dlsym(h, "ZSTD_createCCtx");
        free_cctx = (decltype(free_cctx))dlsym(h, "ZSTD_freeCCtx");
        set_param = (decltype(set_param))dlsym(h, "ZSTD_CCtx_setParameter");
        set_pledged = (decltype(set_pledged))dlsym(h, "ZSTD_CCtx_setPledgedSrcSize");
        stream2 = (decltype(stream2))dlsym(h, "ZSTD_compressStream2");
    }
    bool streaming() const { return create_cctx && free_cctx && set_param && set_pledged && stream2; }
};
Zstd &zs() {
    static Zstd z;
    return z;
}
}  // namespace

bool zstd_available() { return zs().h != nullptr; }

size_t zstd_compress_bound(size_t n) {
    // ZSTD_COMPRESSBOUND of the zstd public API
    return n + (n >> 8) + ((n < (128 << 10)) ? (((128 << 10) - n) >> 11) : 0);
}

size_t zstd_compress(const void *src, size_t n, void *dst, size_t cap, int level) {
    if (!zstd_available()) throw std::runtime_error("libzstd is not available");
    const size_t r = zs().compress(dst, cap, src, n, level);
    if (zs().is_error(r)) throw std::runtime_error("Zstd compression failed");
    return r;
}

bool zstd_compress_if_below(const void *src, size_t n, int level, size_t limit, std::vector<uint8_t> &out) {
    if (!zstd_available()) throw std::runtime_error("libzstd is not available");
    Zstd &z = zs();
    const size_t stop = limit + limit / 50 + 4096;
    if (z.streaming()) {
        void *cc = z.create_cctx();
        if (!cc) throw std::bad_alloc();
        bool past = false;
        try {
            if (z.is_error(z.set_param(cc, 100 /* ZSTD_c_compressionLevel */, level)) ||
                z.is_error(z.set_pledged(cc, (unsigned long long)n)))
                throw std::runtime_error("Zstd compression failed");
            std::vector<uint8_t> buf(1 << 18);
            size_t produced = 0;
            constexpr size_t kChunk = 1 << 20;
            for (size_t at = 0; at < n && !past; at += kChunk) {
                ZInBuf in{static_cast<const uint8_t *>(src) + at, std::min(kChunk, n - at), 0};
                while (in.pos < in.size) {
                    ZOutBuf o{buf.data(), buf.size(), 0};
                    const size_t r = z.stream2(cc, &o, &in, 0 /* ZSTD_e_continue */);
                    if (z.is_error(r)) throw std::runtime_error("Zstd compression failed");
                    produced += o.pos;
                }
                past = produced >= stop;
            }
        } catch (...) {
            z.free_cctx(cc);
            throw;
        }
        z.free_cctx(cc);
        if (past) return false;
    }
    out.resize(zstd_compress_bound(n) + 16);
    out.resize(zstd_compress(src, n, out.data(), out.size(), level));
    return out.size() < limit;
}

size_t zstd_decompress(const void *src, size_t n, void *dst, size_t cap) {
    if (!zstd_available()) throw std::runtime_error("libzstd is not available to decode a compressed zstd frame");
    const size_t r = zs().decompress(dst, cap, src, n);
    if (zs().is_error(r)) throw std::invalid_argument("Invalid or truncated Falcons Zstd payload");
    return r;
}

unsigned long long zstd_frame_content_size(const void *src, size_t n) {
    size_t fb = 0, content = 0;
    if (parse_raw_frame(static_cast<const uint8_t *>(src), n, fb, content)) return content;
    if (!zstd_available()) throw std::runtime_error("libzstd is not available");
    return zs().fcs(src, n);
}

bool parse_raw_frame(const uint8_t *src, size_t n, size_t &first_block, size_t &content) {
    if (n < 6) return false;
    uint32_t magic;
    memcpy(&magic, src, 4);
    if (magic != 0xFD2FB528u) return false;
    const uint8_t fhd = src[4];
    const int fcs_flag = fhd >> 6;
    const bool single = (fhd >> 5) & 1;
    const int did_flag = fhd & 3;
    const bool checksum = (fhd >> 2) & 1;
    if (((fhd >> 3) & 1) || checksum || did_flag) return false;
    size_t p = 5;
    if (!single) p += 1;  // window descriptor
    static const int fcs_sizes[4] = {0, 2, 4, 8};
    int fcs_bytes = fcs_sizes[fcs_flag];
    if (fcs_flag == 0 && single) fcs_bytes = 1;
    if (fcs_bytes == 0) return false;
    if (p + fcs_bytes > n) return false;
    uint64_t v = 0;
    for (int i = 0; i < fcs_bytes; i++) v |= (uint64_t)src[p + i] << (8 * i);
    if (fcs_flag == 1) v += 256;
    p += fcs_bytes;
    first_block = p;
    content = (size_t)v;
    // every block must be raw, full-size except the last
    size_t done = 0;
    while (true) {
        if (p + 3 > n) return false;
        const uint32_t bh = (uint32_t)src[p] | ((uint32_t)src[p + 1] << 8) | ((uint32_t)src[p + 2] << 16);
        const bool last = bh & 1;
        const int type = (bh >> 1) & 3;
        const size_t bs = bh >> 3;
        if (type != 0) return false;
        p += 3;
        if (p + bs > n) return false;
        done += bs;
        p += bs;
        if (last) break;
        if (bs != 128 * 1024) return false;
    }
    if (done != content) return false;
    // trailing bytes may only be skippable frames
    while (p < n) {
        if (p + 8 > n) return false;
        uint32_t m, sz;
        memcpy(&m, src + p, 4);
        memcpy(&sz, src + p + 4, 4);
        if ((m & 0xFFFFFFF0u) != 0x184D2A50u) return false;
        p += 8 + (size_t)sz;
        if (p > n) return false;
    }
    return true;
}

}  // namespace fb2
