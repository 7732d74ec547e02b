/*
 * falcons_gpu.hpp — the reference's C++ API (Falcons_compress / Falcons_decompress<T> /
 * Falcons_read_config / Falcons::Falcons_compress_size_bound over Falcons::Config) with bodies that
 * call the B200 library's C ABI (include/falcons_b200.h, libfalcons_b200.so).
 *
 * It replaces include/Falcons/api/falcons.hpp of the reference (JLiu-1/Falcons):
 *   Falcons_compress(conf, data, cmpData, cmpCap)     api/falcons.hpp:54
 *   Falcons_compress(conf, data, cmpSize)             api/falcons.hpp:111   (new[]; caller delete[]s)
 *   Falcons_read_config(conf, cmpData, cmpSize)       api/falcons.hpp:122
 *   Falcons_decompress(conf, cmpData, cmpSize, dec)   api/falcons.hpp:158   (new T[num] when dec == nullptr)
 *   Falcons_decompress(conf, ..., dec, decCapacity)   api/falcons.hpp:184
 *   Falcons_decompress<T>(conf, cmpData, cmpSize)     api/falcons.hpp:208   (new[]; caller delete[]s)
 *   Falcons::Falcons_compress_size_bound<T>(conf)     api/impl/FalconsImpl.hpp:44
 * with the same semantics: the input field is overwritten with the partial reconstruction, the
 * Config is overwritten from the stream on decompress, and failures throw std::invalid_argument,
 * std::length_error or std::runtime_error as the reference does.  Integral element types compile
 * and throw std::invalid_argument("unsupported on GPU build").
 *
 * It includes the reference's own Falcons::Config (utils/Config.hpp) and the header-only utilities
 * its falcons.hpp made visible to callers (FileUtil, Timer, Statistic, version), so that callers
 * such as the falcons CLI build unchanged against it: put include/dropin (whose
 * Falcons/api/falcons.hpp includes this file) and this directory ahead of the reference's include
 * directory, and link libfalcons_b200.so.
 *
 * Each calling thread gets its own library context on device 0 (FALCONS_GPU_DEVICE overrides the
 * device ordinal), created at its first call and destroyed at thread exit.
 */
#ifndef FALCONS_GPU_HPP
#define FALCONS_GPU_HPP

#include <cstdlib>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "Falcons/utils/Config.hpp"
#include "Falcons/utils/FileUtil.hpp"
#include "Falcons/utils/Statistic.hpp"
#include "Falcons/utils/Timer.hpp"
#include "Falcons/version.hpp"
#include "falcons_b200.h"

namespace falcons_gpu {

// Status -> the reference's exception types.
inline void check(int rc) {
    if (rc == FALCONS_OK) return;
    const std::string m = falcons_last_error();
    if (rc == FALCONS_EINVAL) throw std::invalid_argument(m);
    if (rc == FALCONS_ELENGTH) throw std::length_error(m);
    throw std::runtime_error(m);
}

inline falcons_ctx *ctx() {
    struct Holder {
        falcons_ctx *p = nullptr;
        Holder() {
            const char *d = std::getenv("FALCONS_GPU_DEVICE");
            check(falcons_ctx_create(&p, d ? std::atoi(d) : 0));
        }
        ~Holder() {
            if (p) falcons_ctx_destroy(p);
        }
    };
    thread_local Holder h;
    return h.p;
}

template <class T>
constexpr bool supported() {
    return std::is_same<T, float>::value || std::is_same<T, double>::value;
}

template <class T>
constexpr int dtype() {
    return std::is_same<T, float>::value ? FALCONS_DTYPE_F32 : FALCONS_DTYPE_F64;
}

template <class T>
inline void require_supported() {
    if (!supported<T>()) throw std::invalid_argument("unsupported on GPU build");
}

// Falcons::Config -> the C ABI's configuration record (the fields the path reads).
inline falcons_config to_c(const Falcons::Config &c) {
    falcons_config o{};
    if (c.dims.size() > 4 || c.N < 1 || c.N > 4)
        throw std::invalid_argument("Data dimension higher than 4 is not supported.");
    o.N = c.N;
    for (size_t i = 0; i < c.dims.size(); i++) o.dims[i] = c.dims[i];
    o.num = c.num;
    o.cmprAlgo = c.cmprAlgo;
    o.errorBoundMode = c.errorBoundMode;
    o.absErrorBound = c.absErrorBound;
    o.relErrorBound = c.relErrorBound;
    o.psnrErrorBound = c.psnrErrorBound;
    o.l2normErrorBound = c.l2normErrorBound;
    o.lorenzo = c.lorenzo;
    o.lorenzo2 = c.lorenzo2;
    o.regression = c.regression;
    o.regression2 = c.regression2;
    o.openmp = c.openmp;
    o.quantbinCnt = c.quantbinCnt;
    o.blockSize = c.blockSize;
    o.predDim = c.predDim;
    o.dataType = c.dataType;
    o.interpAlgo = c.interpAlgo;
    o.interpDirection = c.interpDirection;
    o.interpAnchorStride = c.interpAnchorStride;
    o.interpAlpha = c.interpAlpha;
    o.interpBeta = c.interpBeta;
    return o;
}

// The record read from a stream -> Falcons::Config (dims through setDims, as Config::load sets them).
inline void from_c(const falcons_config &o, Falcons::Config &c) {
    std::vector<size_t> d(o.dims, o.dims + (o.N >= 1 && o.N <= 4 ? o.N : 0));
    c.setDims(d.begin(), d.end());
    c.cmprAlgo = (uint8_t)o.cmprAlgo;
    c.errorBoundMode = (uint8_t)o.errorBoundMode;
    c.absErrorBound = o.absErrorBound;
    c.relErrorBound = o.relErrorBound;
    c.psnrErrorBound = o.psnrErrorBound;
    c.l2normErrorBound = o.l2normErrorBound;
    c.lorenzo = o.lorenzo != 0;
    c.lorenzo2 = o.lorenzo2 != 0;
    c.regression = o.regression != 0;
    c.regression2 = o.regression2 != 0;
    c.openmp = o.openmp != 0;
    c.quantbinCnt = o.quantbinCnt;
    c.blockSize = o.blockSize;
    c.predDim = (uint8_t)o.predDim;
    c.dataType = (uint8_t)o.dataType;
    c.interpAlgo = (uint8_t)o.interpAlgo;
    c.interpDirection = (uint8_t)o.interpDirection;
    c.interpAnchorStride = o.interpAnchorStride;
    c.interpAlpha = o.interpAlpha;
    c.interpBeta = o.interpBeta;
}

}  // namespace falcons_gpu

namespace Falcons {
template <class T>
size_t Falcons_compress_size_bound(const Config &config) {
    falcons_gpu::require_supported<T>();
    const falcons_config c = falcons_gpu::to_c(config);
    return falcons_compress_size_bound(falcons_gpu::dtype<T>(), &c);
}
}  // namespace Falcons

template <class T>
size_t Falcons_compress(const Falcons::Config &config, const T *data, char *cmpData, size_t cmpCap) {
    falcons_gpu::require_supported<T>();
    const falcons_config c = falcons_gpu::to_c(config);
    falcons_config used;
    size_t len = 0;
    falcons_gpu::check(falcons_compress(falcons_gpu::ctx(), falcons_gpu::dtype<T>(), &c, const_cast<T *>(data),
                                        FALCONS_FLAG_WRITEBACK, cmpData, cmpCap, &len, &used));
    return len;
}

template <class T>
char *Falcons_compress(const Falcons::Config &config, const T *data, size_t &cmpSize) {
    const size_t cap = Falcons::Falcons_compress_size_bound<T>(config);
    char *buffer = new char[cap];
    try {
        cmpSize = Falcons_compress(config, data, buffer, cap);
    } catch (...) {
        delete[] buffer;
        throw;
    }
    return buffer;
}

inline void Falcons_read_config(Falcons::Config &config, const char *cmpData, size_t cmpSize) {
    falcons_config o;
    falcons_gpu::check(falcons_read_config(cmpData, cmpSize, &o));
    falcons_gpu::from_c(o, config);
}

template <class T>
void Falcons_decompress(Falcons::Config &config, const char *cmpData, size_t cmpSize, T *&decData,
                        size_t decCapacity) {
    falcons_gpu::require_supported<T>();
    Falcons_read_config(config, cmpData, cmpSize);
    if (decData == nullptr || config.num > decCapacity)
        throw std::invalid_argument("The decompression buffer is too small");
    falcons_config o;
    falcons_gpu::check(falcons_decompress(falcons_gpu::ctx(), falcons_gpu::dtype<T>(), cmpData, cmpSize, decData,
                                          decCapacity, &o));
    falcons_gpu::from_c(o, config);
}

template <class T>
void Falcons_decompress(Falcons::Config &config, const char *cmpData, size_t cmpSize, T *&decData) {
    falcons_gpu::require_supported<T>();
    Falcons_read_config(config, cmpData, cmpSize);
    const bool owned = decData == nullptr;
    if (owned) decData = new T[config.num];
    try {
        Falcons_decompress(config, cmpData, cmpSize, decData, (size_t)config.num);
    } catch (...) {
        if (owned) {
            delete[] decData;
            decData = nullptr;
        }
        throw;
    }
}

template <class T>
T *Falcons_decompress(Falcons::Config &config, const char *cmpData, size_t cmpSize) {
    T *decData = nullptr;
    Falcons_decompress<T>(config, cmpData, cmpSize, decData);
    return decData;
}

#endif  // FALCONS_GPU_HPP
