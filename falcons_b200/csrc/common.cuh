// Shared device/host definitions of the B200 Falcons path.
//
// Bit-exactness contract: every floating-point operation on the prediction/quantization path is
// written with an explicit round-to-nearest intrinsic (no contraction is possible), in the
// operation order of the reference's scalar build:
//   interpolation formulas   include/Falcons/utils/Interpolators.hpp:49-117
//   linear quantizer         include/Falcons/quantizer/LinearQuantizer.hpp:49-133
#pragma once
#include <cmath>
#include <limits>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace fb2 {

// ---------------------------------------------------------------- error handling
struct cuda_error : std::runtime_error {
    explicit cuda_error(const std::string &s) : std::runtime_error(s) {}
};

#define FB2_CUDA(call)                                                                                  \
    do {                                                                                                \
        cudaError_t e__ = (call);                                                                       \
        if (e__ != cudaSuccess)                                                                         \
            throw ::fb2::cuda_error(std::string("CUDA error ") + cudaGetErrorString(e__) + " at " +    \
                                    __FILE__ + ":" + std::to_string(__LINE__));                         \
    } while (0)

// Every kernel launch of the library is followed by FB2_CHECK_LAUNCH(), which also counts it.
unsigned long long count_launch();

// Host-side phase trace, on when the environment variable FALCONS_TRACE is set: each mark()
// prints to stderr the host time since the traced call began and the kernel launches so far.
// A long gap between two marks with few launches is host work the GPU waited for.
// gpu() records a CUDA event on a stream; gpu_dump() waits for them and prints each one's device
// time since the first, which shows what ran when across the streams of one call.
struct Trace {
    const char *what;
    double t0;
    unsigned long long l0;
    bool on;
    std::vector<std::pair<const char *, cudaEvent_t>> events;
    explicit Trace(const char *w);
    Trace(const Trace &) = delete;
    Trace &operator=(const Trace &) = delete;
    ~Trace();
    void mark(const char *label);
    void gpu(const char *label, cudaStream_t s);
    void gpu_dump();
};
#define FB2_CHECK_LAUNCH()      \
    do {                        \
        ::fb2::count_launch();  \
        FB2_CUDA(cudaGetLastError()); \
    } while (0)

// ---------------------------------------------------------------- predictor formulas
enum Formula : int { F_EQUAL = 0, F_LINEAR, F_LINEAR1, F_QUAD1, F_QUAD2, F_QUAD3, F_CUBIC };

// A predictor: formula plus up to four operand indices along the pass line (grid units).
struct Rule {
    int f;
    int o0, o1, o2, o3;
};

__host__ __device__ __forceinline__ Rule mk_rule(int f, long long a, long long b = 0, long long c = 0,
                                                 long long d = 0) {
    Rule r;
    r.f = f;
    r.o0 = (int)a;
    r.o1 = (int)b;
    r.o2 = (int)c;
    r.o3 = (int)d;
    return r;
}

// Predictor of target t on a line of n grid points whose targets are visited by the
// 1-D line routines (reference: Interpolation_quantizer.inl:2623-2700).
__host__ __device__ __forceinline__ Rule line_rule(bool cubic, int t, int n) {
    const int odd = n / 2, even = n - odd;
    if (!cubic) {
        if (t < 2 * odd - 1) return mk_rule(F_LINEAR, t - 1, t + 1);
        if (n < 3) return mk_rule(F_EQUAL, 2 * (even - 1));
        return mk_rule(F_LINEAR1, 2 * (even - 2), 2 * (even - 1));
    }
    if (t == 1) {
        if (even < 2) return mk_rule(F_EQUAL, 0);
        if (even < 3) return mk_rule(F_LINEAR, 0, 2);
        return mk_rule(F_QUAD1, 0, 2, 4);
    }
    if (odd < even) {
        if (t == 2 * odd - 1) return mk_rule(F_QUAD2, 2 * (even - 3), 2 * (even - 2), 2 * (even - 1));
    } else {
        if (t == 2 * odd - 1) return mk_rule(F_LINEAR1, 2 * (even - 2), 2 * (even - 1));
        if (odd > 2 && t == 2 * odd - 3) return mk_rule(F_QUAD2, 2 * (even - 3), 2 * (even - 2), 2 * (even - 1));
    }
    return mk_rule(F_CUBIC, t - 3, t - 1, t + 1, t + 3);
}

// Predictor of target row/plane t for the row-buffer passes (2-D y, 3-D z and y sweeps,
// reference InterpolationDecomposition.hpp:602-721, 819-1135, 1136-1375).  `skip` marks the
// final pass of level 1, whose linear edge reads three grid units back instead of two.
__host__ __device__ __forceinline__ Rule row_rule(bool cubic, int t, int n, bool skip) {
    if (!cubic) {
        if (t < n - 1) return mk_rule(F_LINEAR, t - 1, t + 1);
        if (n < 3) return mk_rule(F_EQUAL, n - 2);
        return mk_rule(F_LINEAR1, n - 1 - (skip ? 3 : 2), n - 2);
    }
    if (t == 1) {
        if (n >= 5) return mk_rule(F_QUAD1, 0, 2, 4);
        if (n >= 3) return mk_rule(F_LINEAR, 0, 2);
        return mk_rule(F_EQUAL, 0);
    }
    if (n & 1) {
        if (t == n - 2) return mk_rule(F_QUAD2, n - 5, n - 3, n - 1);
    } else {
        if (t == n - 1) return mk_rule(F_LINEAR1, n - 4, n - 2);
        if (t == n - 3 && n > 4) return mk_rule(F_QUAD2, n - 6, n - 4, n - 2);
    }
    return mk_rule(F_CUBIC, t - 3, t - 1, t + 1, t + 3);
}

// ---------------------------------------------------------------- exact arithmetic per type
template <class T> struct Arith;

template <> struct Arith<float> {
    __device__ __forceinline__ static float add(float a, float b) { return __fadd_rn(a, b); }
    __device__ __forceinline__ static float sub(float a, float b) { return __fsub_rn(a, b); }
    __device__ __forceinline__ static float mul(float a, float b) { return __fmul_rn(a, b); }
    __device__ __forceinline__ static float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    __device__ __forceinline__ static float from_double(double v) { return __double2float_rn(v); }
};

template <> struct Arith<double> {
    __device__ __forceinline__ static double add(double a, double b) { return __dadd_rn(a, b); }
    __device__ __forceinline__ static double sub(double a, double b) { return __dsub_rn(a, b); }
    __device__ __forceinline__ static double mul(double a, double b) { return __dmul_rn(a, b); }
    __device__ __forceinline__ static double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
    __device__ __forceinline__ static double from_double(double v) { return v; }
};

// Interpolators.hpp:49-117 (floating branches).  Division by 2, 8 and 16 is exact, so it is
// written as the equivalent exact multiplication.
template <class T>
__device__ __forceinline__ T apply_formula(int f, T a, T b, T c, T d) {
    using A = Arith<T>;
    T t;
    switch (f) {
        case F_EQUAL: return a;
        case F_LINEAR: return A::mul(A::add(a, b), T(0.5));
        case F_LINEAR1: return A::fma(T(-0.5), a, A::mul(T(1.5), b));
        case F_QUAD1: t = A::fma(T(6), b, -c); t = A::fma(T(3), a, t); return A::mul(t, T(0.125));
        case F_QUAD2: t = A::fma(T(6), b, -a); t = A::fma(T(3), c, t); return A::mul(t, T(0.125));
        case F_QUAD3:
            t = A::sub(A::mul(T(3), a), A::mul(T(10), b));
            t = A::add(t, A::mul(T(15), c));
            return A::mul(t, T(0.125));
        default:
            t = A::mul(A::add(b, c), T(9));
            t = A::sub(t, a);
            t = A::sub(t, d);
            return A::mul(t, T(0.0625));
    }
}

// Per-level quantizer parameters (LinearQuantizer::set_eb: ebx2 = 2 eb, ebx2_r = 1 / ebx2).
struct QParams {
    double eb, ebx2, ebx2_r;
    int radius;
    float ebf;  // the largest float <= eb: for a float e, |e| <= eb exactly when |e| <= ebf
};

// The largest float not above v (v >= 0).
inline float float_at_most(double v) {
    float f = (float)v;
    if ((double)f > v) f = std::nextafter(f, -std::numeric_limits<float>::infinity());
    return f;
}

// LinearQuantizer::quantize_and_overwrite / quantize_without_overwrite.  Returns the code;
// `recon` receives the reconstructed value (the input itself for an unpredictable value).
template <class T>
__device__ __forceinline__ bool within_eb(T err, const QParams &qp) {
    return (double)err >= -qp.eb && (double)err <= qp.eb;
}
template <>
__device__ __forceinline__ bool within_eb<float>(float err, const QParams &qp) {
    return fabsf(err) <= qp.ebf;  // the same test in float (NaN fails both)
}

template <class T>
__device__ __forceinline__ int quantize(T x, T pred, const QParams &qp, T &recon) {
    using A = Arith<T>;
    const T diff = A::sub(x, pred);
    const int q = __double2int_rn(__dmul_rn((double)diff, qp.ebx2_r));
    if (q > -qp.radius && q < qp.radius) {
        const T dq = A::from_double(__fma_rn((double)q, qp.ebx2, (double)pred));
        if (within_eb<T>(A::sub(dq, x), qp)) {
            recon = dq;
            return q;
        }
    }
    recon = x;
    return -qp.radius;
}

// LinearQuantizer::recover_pred
template <class T>
__device__ __forceinline__ T dequantize(int q, T pred, const QParams &qp) {
    return Arith<T>::from_double(__fma_rn((double)q, qp.ebx2, (double)pred));
}

}  // namespace fb2
