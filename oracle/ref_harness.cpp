// Test-infrastructure harness around the UNMODIFIED reference (JLiu-1/Falcons) headers.
//
// oracle/Makefile compiles this file against the reference's own include tree and its
// vendored FSE sources, producing oracle/_ref/libfalcons_ref.so.  Only the tests, the
// fixture generator under tests/golden/ and bench.py's reference arm load it, and only
// as a reference for the tests or a timed CPU baseline.  Nothing in the product links it.
//
// Entry points (all extern "C", plain pointers):
//   ref_compress_<t>            include/Falcons/api/falcons.hpp:54       (Falcons_compress into a buffer)
//   ref_decompress_<t>          include/Falcons/api/falcons.hpp:184      (capacity-checked Falcons_decompress)
//   ref_size_bound_<t>          include/Falcons/api/impl/FalconsImpl.hpp:44
//   ref_interp_compress_<t>     decomposition/InterpolationDecomposition.hpp:131 (codes + unpred, in stream order)
//   ref_interp_decompress_<t>   decomposition/InterpolationDecomposition.hpp:48
//   ref_rlefse_encode/decode    encoder/RleFseEncoder.hpp:850-1079
//   ref_zstd_compress/decompress lossless/Lossless_zstd.hpp:29-78
//   ref_fse_compress/decompress  encoder/zfse FSE_compress / FSE_decompress (one FSE block)
//   ref_lorenzo_payload_<t>     the pre-zstd payload of the 1-D blockwise Lorenzo path as the
//                               tuner configures it (api/impl/FalconsAlgoInterp.hpp:229-262,
//                               479-490; compressor/FalconsGenericCompressor.hpp:64-81), without
//                               the dispatcher's choice between it and a lossless stream
//   ref_lorenzo_decode_<t>      its decoder (FalconsGenericCompressor.hpp decompress steps)
//   ref_lorenzo_trial_<t>       the interpolation tuner's Lorenzo trial over sample blocks
//                               (lorenzo_compress_test, FalconsAlgoInterp.hpp:229-262): its buffer
//                               before zstd, rebuilt stage by stage, and its own ratio
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "Falcons/api/falcons.hpp"

using namespace Falcons;

extern "C" {
struct ref_conf {
    int32_t cmprAlgo;
    int32_t errorBoundMode;
    double absErrorBound;
    double relErrorBound;
    double psnrErrorBound;
    double l2normErrorBound;
    int32_t interpAlgo;
    int32_t interpDirection;
    int32_t interpAnchorStride;
    int32_t openmp;
    double interpAlpha;
    double interpBeta;
    int32_t quantbinCnt;
    int32_t lorenzo;
    int32_t lorenzo2;
    int32_t regression;
    int32_t regression2;
    int32_t blockSize;
};
}

static thread_local std::string g_err;

static Config make_conf(const size_t *dims, int N, const ref_conf *c) {
    Config conf;
    conf.setDims(dims, dims + N);
    conf.cmprAlgo = static_cast<uint8_t>(c->cmprAlgo);
    conf.errorBoundMode = static_cast<uint8_t>(c->errorBoundMode);
    conf.absErrorBound = c->absErrorBound;
    conf.relErrorBound = c->relErrorBound;
    conf.psnrErrorBound = c->psnrErrorBound;
    conf.l2normErrorBound = c->l2normErrorBound;
    conf.interpAlgo = static_cast<uint8_t>(c->interpAlgo);
    conf.interpDirection = static_cast<uint8_t>(c->interpDirection);
    conf.interpAnchorStride = c->interpAnchorStride;
    conf.openmp = c->openmp != 0;
    conf.interpAlpha = c->interpAlpha;
    conf.interpBeta = c->interpBeta;
    if (c->quantbinCnt > 0) conf.quantbinCnt = c->quantbinCnt;
    conf.lorenzo = c->lorenzo != 0;
    conf.lorenzo2 = c->lorenzo2 != 0;
    conf.regression = c->regression != 0;
    conf.regression2 = c->regression2 != 0;
    if (c->blockSize > 0) conf.blockSize = c->blockSize;
    return conf;
}

template <class T>
static long long do_compress(const size_t *dims, int N, const ref_conf *c, T *data, char *out, size_t cap) {
    try {
        Config conf = make_conf(dims, N, c);
        return static_cast<long long>(Falcons_compress<T>(conf, data, out, cap));
    } catch (std::exception &e) {
        g_err = e.what();
        return -1;
    }
}

template <class T>
static long long do_size_bound(const size_t *dims, int N, const ref_conf *c) {
    Config conf = make_conf(dims, N, c);
    return static_cast<long long>(Falcons_compress_size_bound<T>(conf));
}

template <class T>
static int do_decompress(const char *cmp, size_t size, T *out, size_t cap, size_t *dims_out, int *N_out) {
    try {
        Config conf;
        T *dst = out;
        Falcons_decompress<T>(conf, cmp, size, dst, cap);
        *N_out = conf.N;
        for (int i = 0; i < conf.N; i++) dims_out[i] = conf.dims[i];
        return 0;
    } catch (std::exception &e) {
        g_err = e.what();
        return -1;
    }
}

template <class T, uint N>
static int interp_compress_n(const size_t *dims, const ref_conf *c, int tuning, T *data, int16_t *codes,
                             size_t *ncodes, T *unpred, size_t *nunpred) {
    Config conf = make_conf(dims, N, c);
    conf.cmprAlgo = ALGO_INTERP;
    if (conf.interpAnchorStride < 0) {
        std::array<size_t, 4> anchor_strides = {4096, 128, 32, 16};
        conf.interpAnchorStride = anchor_strides[N - 1];
    }
    int16_t *q = nullptr;
    uint64_t nq = 0;
    std::vector<T> up;
    if (tuning) {
        auto dec = make_decomposition_interpolation<TUNING::ENABLED, T, N>(
            conf, LinearQuantizer<T>(conf.absErrorBound, conf.quantbinCnt / 2));
        std::tie(q, nq) = dec.compress(conf, data);
        up = dec.test_unpred();
    } else {
        auto dec = make_decomposition_interpolation<TUNING::DISABLED, T, N>(
            conf, LinearQuantizer<T>(conf.absErrorBound, conf.quantbinCnt / 2));
        std::tie(q, nq) = dec.compress(conf, data);
        up = dec.test_unpred();
    }
    if (nq > *ncodes || up.size() > *nunpred) {
        delete[] q;
        g_err = "output arrays too small";
        return -1;
    }
    memcpy(codes, q, nq * sizeof(int16_t));
    memcpy(unpred, up.data(), up.size() * sizeof(T));
    *ncodes = nq;
    *nunpred = up.size();
    delete[] q;
    return 0;
}

template <class T, uint N>
static int interp_decompress_n(const size_t *dims, const ref_conf *c, const int16_t *codes, size_t ncodes,
                               const T *unpred, size_t nunpred, T *out) {
    Config conf = make_conf(dims, N, c);
    conf.cmprAlgo = ALGO_INTERP;
    if (conf.interpAnchorStride < 0) {
        std::array<size_t, 4> anchor_strides = {4096, 128, 32, 16};
        conf.interpAnchorStride = anchor_strides[N - 1];
    }
    // Serialise the decomposition header exactly as InterpolationDecomposition::save does
    // (InterpolationDecomposition.hpp:241-251 + LinearQuantizer.hpp:142-152), then load it.
    std::vector<uchar> buf(256 + nunpred * sizeof(T));
    uchar *p = buf.data();
    size_t max_dim = 1;
    for (uint i = 0; i < N; i++) max_dim = std::max(max_dim, dims[i]);
    for (uint i = 0; i < N; i++) write(static_cast<size_t>(dims[i]), p);
    write(static_cast<uint>(max_dim), p);
    write(static_cast<int>(conf.interpAlgo), p);
    write(static_cast<int>(conf.interpDirection), p);
    write(static_cast<size_t>(conf.interpAnchorStride), p);
    write(conf.interpAlpha, p);
    write(conf.interpBeta, p);
    write(static_cast<uchar>(0b10), p);
    write(conf.absErrorBound, p);
    write(static_cast<int>(conf.quantbinCnt / 2), p);
    write(static_cast<int>(nunpred), p);
    write(unpred, nunpred, p);
    const uchar *rp = buf.data();
    size_t remaining = p - buf.data();
    auto dec = make_decomposition_interpolation<TUNING::DISABLED, T, N>(
        conf, LinearQuantizer<T>(conf.absErrorBound, conf.quantbinCnt / 2));
    dec.load(rp, remaining);
    std::vector<int16_t> q(codes, codes + ncodes);
    q.resize(ncodes + 64);
    dec.decompress(conf, q.data(), out);
    return 0;
}

template <class T>
static int do_interp_compress(const size_t *dims, int N, const ref_conf *c, int tuning, T *data, int16_t *codes,
                              size_t *ncodes, T *unpred, size_t *nunpred) {
    try {
        switch (N) {
            case 1: return interp_compress_n<T, 1>(dims, c, tuning, data, codes, ncodes, unpred, nunpred);
            case 2: return interp_compress_n<T, 2>(dims, c, tuning, data, codes, ncodes, unpred, nunpred);
            case 3: return interp_compress_n<T, 3>(dims, c, tuning, data, codes, ncodes, unpred, nunpred);
            case 4: return interp_compress_n<T, 4>(dims, c, tuning, data, codes, ncodes, unpred, nunpred);
        }
    } catch (std::exception &e) {
        g_err = e.what();
    }
    return -1;
}

template <class T>
static int do_interp_decompress(const size_t *dims, int N, const ref_conf *c, const int16_t *codes, size_t ncodes,
                                const T *unpred, size_t nunpred, T *out) {
    try {
        switch (N) {
            case 1: return interp_decompress_n<T, 1>(dims, c, codes, ncodes, unpred, nunpred, out);
            case 2: return interp_decompress_n<T, 2>(dims, c, codes, ncodes, unpred, nunpred, out);
            case 3: return interp_decompress_n<T, 3>(dims, c, codes, ncodes, unpred, nunpred, out);
            case 4: return interp_decompress_n<T, 4>(dims, c, codes, ncodes, unpred, nunpred, out);
        }
    } catch (std::exception &e) {
        g_err = e.what();
    }
    return -1;
}

extern "C" {
const char *ref_last_error() { return g_err.c_str(); }

long long ref_compress_f32(const size_t *d, int N, const ref_conf *c, float *x, char *o, size_t cap) {
    return do_compress<float>(d, N, c, x, o, cap);
}
long long ref_compress_f64(const size_t *d, int N, const ref_conf *c, double *x, char *o, size_t cap) {
    return do_compress<double>(d, N, c, x, o, cap);
}
long long ref_size_bound_f32(const size_t *d, int N, const ref_conf *c) { return do_size_bound<float>(d, N, c); }
long long ref_size_bound_f64(const size_t *d, int N, const ref_conf *c) { return do_size_bound<double>(d, N, c); }
int ref_decompress_f32(const char *s, size_t n, float *o, size_t cap, size_t *dims, int *N) {
    return do_decompress<float>(s, n, o, cap, dims, N);
}
int ref_decompress_f64(const char *s, size_t n, double *o, size_t cap, size_t *dims, int *N) {
    return do_decompress<double>(s, n, o, cap, dims, N);
}
int ref_interp_compress_f32(const size_t *d, int N, const ref_conf *c, int tuning, float *x, int16_t *q, size_t *nq,
                            float *u, size_t *nu) {
    return do_interp_compress<float>(d, N, c, tuning, x, q, nq, u, nu);
}
int ref_interp_compress_f64(const size_t *d, int N, const ref_conf *c, int tuning, double *x, int16_t *q, size_t *nq,
                            double *u, size_t *nu) {
    return do_interp_compress<double>(d, N, c, tuning, x, q, nq, u, nu);
}
int ref_interp_decompress_f32(const size_t *d, int N, const ref_conf *c, const int16_t *q, size_t nq, const float *u,
                              size_t nu, float *o) {
    return do_interp_decompress<float>(d, N, c, q, nq, u, nu, o);
}
int ref_interp_decompress_f64(const size_t *d, int N, const ref_conf *c, const int16_t *q, size_t nq, const double *u,
                              size_t nu, double *o) {
    return do_interp_decompress<double>(d, N, c, q, nq, u, nu, o);
}

// RleFseEncoder<int16_t>: [u8 method|delta<<7][u16 lo][u16 mode] + payload, as FalconsGenericCompressor writes it.
long long ref_rlefse_encode(const int16_t *codes, size_t n, uint8_t *out, size_t cap) {
    try {
        std::vector<int16_t> tmp(codes, codes + n);
        tmp.resize(n + 16);
        RleFseEncoder<int16_t> enc;
        enc.preprocess_encode(tmp.data(), n, 65536);
        std::vector<uchar> buf(std::max<size_t>(cap, 8 * n + 65536));
        uchar *p = buf.data();
        enc.save(p);
        enc.encode(tmp.data(), n, p);
        size_t len = p - buf.data();
        if (len > cap) {
            g_err = "capacity";
            return -1;
        }
        memcpy(out, buf.data(), len);
        return static_cast<long long>(len);
    } catch (std::exception &e) {
        g_err = e.what();
        return -1;
    }
}

long long ref_rlefse_decode(const uint8_t *in, size_t n_in, size_t n_codes, int16_t *out) {
    try {
        RleFseEncoder<int16_t> enc;
        const uchar *p = in;
        size_t rem = n_in;
        enc.load(p, rem);
        int16_t *q = enc.decode(p, n_codes);
        memcpy(out, q, n_codes * sizeof(int16_t));
        delete[] q;
        return static_cast<long long>(p - in);
    } catch (std::exception &e) {
        g_err = e.what();
        return -1;
    }
}

// zfse FSE_compress / FSE_decompress (encoder/zfse/fse_compress.c, fse_decompress.c), the block
// coder RleFseEncoder calls (RleFseEncoder.hpp:155,184).  Returns the size, or -1 on an error code.
long long ref_fse_compress(const uint8_t *src, size_t n, uint8_t *dst, size_t cap) {
    const size_t r = FSE_compress(dst, cap, src, n);
    if (FSE_isError(r)) {
        g_err = "FSE_compress error";
        return -1;
    }
    return static_cast<long long>(r);
}

long long ref_fse_decompress(const uint8_t *src, size_t n, uint8_t *dst, size_t cap) {
    const size_t r = FSE_decompress(dst, cap, src, n);
    if (FSE_isError(r)) {
        g_err = "FSE_decompress error";
        return -1;
    }
    return static_cast<long long>(r);
}

long long ref_zstd_compress(const uint8_t *src, size_t n, uint8_t *dst, size_t cap) {
    try {
        Lossless_zstd z;
        return static_cast<long long>(z.compress(src, n, dst, cap));
    } catch (std::exception &e) {
        g_err = e.what();
        return -1;
    }
}

long long ref_zstd_decompress(const uint8_t *src, size_t n, uint8_t *dst, size_t cap) {
    try {
        Lossless_zstd z;
        uchar *d = nullptr;
        size_t dl = 0;
        z.decompress(src, n, d, dl);
        if (dl > cap) {
            free(d);
            g_err = "capacity";
            return -1;
        }
        memcpy(dst, d, dl);
        free(d);
        return static_cast<long long>(dl);
    } catch (std::exception &e) {
        g_err = e.what();
        return -1;
    }
}
}

// ---- the 1-D blockwise Lorenzo path, stage by stage
template <class T>
static auto lorenzo_decomposition(const Config &conf) {
    std::vector<std::shared_ptr<concepts::PredictorInterface<T, 1>>> predictors;
    predictors.push_back(std::make_shared<LorenzoPredictor<T, 1, 1>>(conf.absErrorBound));
    predictors.push_back(std::make_shared<LorenzoPredictor<T, 1, 2>>(conf.absErrorBound));
    return make_decomposition_blockwise<T, 1>(conf, ComposedPredictor<T, 1>(predictors),
                                              LinearQuantizer<T>(conf.absErrorBound, conf.quantbinCnt / 2));
}

template <class T>
static Config lorenzo_conf(size_t n, double eb, int quantbin) {
    Config conf(n);
    conf.cmprAlgo = ALGO_LORENZO_REG;
    conf.errorBoundMode = EB_ABS;
    conf.absErrorBound = eb;
    conf.lorenzo = true;
    conf.lorenzo2 = true;
    conf.regression = false;
    conf.regression2 = false;
    conf.openmp = false;
    conf.blockSize = 5;
    conf.quantbinCnt = quantbin;
    return conf;
}

template <class T>
static long long do_lorenzo_payload(const T *x, size_t n, double eb, int quantbin, uint8_t *out, size_t cap,
                                    T *after) {
    try {
        Config conf = lorenzo_conf<T>(n, eb, quantbin);
        auto dec = lorenzo_decomposition<T>(conf);
        std::vector<T> work(x, x + n);
        auto [q, nq] = dec.compress(conf, work.data());
        std::vector<uchar> buf(std::max<size_t>(4096, 64 + nq * (sizeof(T) + 8) + 2 * 65540));
        uchar *p = buf.data();
        dec.save(p);
        write<uint64_t>(nq, p);
        HuffmanEncoder<int> enc;
        enc.preprocess_encode(q, nq, dec.get_out_range().second);
        enc.save(p);
        enc.encode(q, nq, p);
        enc.postprocess_encode();
        delete[] q;
        const size_t len = p - buf.data();
        if (len > cap) {
            g_err = "capacity";
            return -1;
        }
        memcpy(out, buf.data(), len);
        if (after) memcpy(after, work.data(), n * sizeof(T));  // the input buffer after compress
        return static_cast<long long>(len);
    } catch (std::exception &e) {
        g_err = e.what();
        return -1;
    }
}

template <class T>
static long long do_lorenzo_decode(const uint8_t *in, size_t len, size_t n, T *out) {
    try {
        Config conf = lorenzo_conf<T>(n, 0.0, 65536);
        LinearQuantizer<T> quantizer;
        std::vector<std::shared_ptr<concepts::PredictorInterface<T, 1>>> predictors;
        predictors.push_back(std::make_shared<LorenzoPredictor<T, 1, 1>>());
        predictors.push_back(std::make_shared<LorenzoPredictor<T, 1, 2>>());
        auto dec = make_decomposition_blockwise<T, 1>(conf, ComposedPredictor<T, 1>(predictors), quantizer);
        const uchar *p = in;
        size_t rem = len;
        dec.load(p, rem);
        uint64_t nq = 0;
        read(nq, p, rem);
        if (nq != n) throw std::invalid_argument("code count");
        HuffmanEncoder<int> enc;
        enc.load(p, rem);
        int *q = enc.decode(p, nq);
        enc.postprocess_decode();
        dec.decompress(conf, q, out);
        delete[] q;
        return static_cast<long long>(p - in);
    } catch (std::exception &e) {
        g_err = e.what();
        return -1;
    }
}

extern "C" {
long long ref_lorenzo_payload_f32(const float *x, size_t n, double eb, int qb, uint8_t *o, size_t cap, float *r) {
    return do_lorenzo_payload<float>(x, n, eb, qb, o, cap, r);
}
long long ref_lorenzo_payload_f64(const double *x, size_t n, double eb, int qb, uint8_t *o, size_t cap, double *r) {
    return do_lorenzo_payload<double>(x, n, eb, qb, o, cap, r);
}
long long ref_lorenzo_decode_f32(const uint8_t *in, size_t len, size_t n, float *out) {
    return do_lorenzo_decode<float>(in, len, n, out);
}
long long ref_lorenzo_decode_f64(const uint8_t *in, size_t len, size_t n, double *out) {
    return do_lorenzo_decode<double>(in, len, n, out);
}
}

template <class T>
static double do_lorenzo_trial(const T *blocks, size_t B, size_t V, double eb, int quantbin, uint8_t *out, size_t cap,
                               long long *out_len) {
    try {
        Config conf = lorenzo_conf<T>(V, eb, quantbin);
        // the trial's buffer, stage by stage as lorenzo_compress_test writes it
        auto dec = lorenzo_decomposition<T>(conf);
        std::vector<int> total;
        std::vector<std::vector<T>> sampled;
        for (size_t b = 0; b < B; b++) {
            std::vector<T> blk(blocks + b * V, blocks + (b + 1) * V);
            sampled.push_back(blk);
            auto [q, nq] = dec.compress(conf, blk.data());
            total.insert(total.end(), q, q + nq);
            delete[] q;
        }
        HuffmanEncoder<int> enc;
        enc.preprocess_encode(total, conf.quantbinCnt);
        std::vector<uchar> buf(std::max<size_t>(4096, 64 + total.size() * (sizeof(T) + 8) + 2 * 65540));
        uchar *p = buf.data();
        dec.save(p);
        enc.save(p);
        write<size_t>(total.size(), p);
        enc.encode(total, p);
        enc.postprocess_encode();
        const size_t len = p - buf.data();
        if (len > cap) {
            g_err = "capacity";
            return -1;
        }
        memcpy(out, buf.data(), len);
        *out_len = (long long)len;
        // and the reference's own ratio
        std::vector<uchar> zbuf(std::max<size_t>(1 << 20, 4 * len + 65536));
        return lorenzo_compress_test<T, 1>(sampled, conf, zbuf.data(), zbuf.size());
    } catch (std::exception &e) {
        g_err = e.what();
        return -1;
    }
}

extern "C" {
double ref_lorenzo_trial_f32(const float *b, size_t B, size_t V, double eb, int qb, uint8_t *o, size_t cap,
                             long long *len) {
    return do_lorenzo_trial<float>(b, B, V, eb, qb, o, cap, len);
}
double ref_lorenzo_trial_f64(const double *b, size_t B, size_t V, double eb, int qb, uint8_t *o, size_t cap,
                             long long *len) {
    return do_lorenzo_trial<double>(b, B, V, eb, qb, o, cap, len);
}
}
