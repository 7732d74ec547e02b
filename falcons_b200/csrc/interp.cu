// Interpolation decomposition kernels (prediction + linear quantization) for sm_100a.
//
// Plan construction mirrors the reference's level loop and pass order:
//   levels / anchors / per-level eb   InterpolationDecomposition.hpp:131-239, 286-359
//   non-tuning pass order             InterpolationDecomposition.hpp:2294-2527
//   tuning / 4-D generic sweeps       InterpolationDecomposition.hpp:436-528 (fastest_dim_first)
//   legacy 1-D line (tuning N<=2)     InterpolationDecomposition.hpp:371-419
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <type_traits>

#include "interp.cuh"
#include "assemble.cuh"

namespace fb2 {

static long long count_of(long long dim, long long st) { return (dim - 1) / st + 1; }

// ------------------------------------------------------------------------------------------ plan
namespace {

struct Builder {
    InterpPlan &P;
    const InterpParams &prm;
    long long pos = 0;  // next code position

    Builder(InterpPlan &p, const InterpParams &q) : P(p), prm(q) {}

    static PassLaunch blank() {
        PassLaunch L{};
        for (int i = 0; i < 4; i++) { L.cnt[i] = 1; L.est[i] = 0; }
        return L;
    }

    // Row-buffer pass along dim pd; `outer` (may be -1) and `inner` are the other dims.
    void rows(int level, long long s, int pd, int outer, long long so, int inner, long long sk, bool skip) {
        const long long n = (P.dims[pd] - 1) / s + 1;
        if (n <= 1) return;
        const long long co = outer >= 0 ? count_of(P.dims[outer], so) : 1;
        const long long C = count_of(P.dims[inner], sk);
        const long long m = n / 2;
        const bool cubic = prm.cubic != 0;
        const bool late = cubic && (n % 2 == 0) && n > 2 && P.N == 3;
        const bool lin_tail = !cubic && (n % 2 == 0) && n >= 3 && !skip;
        const long long mr = late ? m - 1 : m;
        PassLaunch L = blank();
        L.kind = KIND_ROW;
        L.cubic = cubic;
        L.skip = skip;
        L.n = (int)n;
        L.step = s * P.off[pd];
        L.A = co;
        L.C = C;
        L.sa = outer >= 0 ? so * P.off[outer] : 0;
        L.sc = sk * P.off[inner];
        L.t0 = 1;
        L.rows_in_group = mr;
        L.b_off = 0;
        L.p_base = pos;
        L.level = level;
        L.B = lin_tail ? mr - 1 : mr;
        if (L.B > 0) P.passes.push_back(L);
        if (lin_tail) {
            PassLaunch T = L;
            T.B = 1;
            T.t0 = (int)(n - 1);
            T.b_off = mr - 1;
            P.passes.push_back(T);
        }
        if (late) {
            PassLaunch E = L;
            E.B = 1;
            E.t0 = (int)(n - 1);
            E.rows_in_group = 1;
            E.b_off = 0;
            E.p_base = pos + co * mr * C;
            P.passes.push_back(E);
        }
        pos += co * m * C;
    }

    // 1-D line pass along the last dim; lines enumerated by (a over dim0, b over dim1) as given.
    void lines(int level, long long s, int pd, long long A, long long sa, long long B, long long sb, bool skip) {
        const long long n = (P.dims[pd] - 1) / s + 1;
        if (n <= 1) return;
        PassLaunch L = blank();
        L.kind = KIND_LINE;
        L.cubic = prm.cubic != 0;
        L.skip = skip;
        L.n = (int)n;
        L.step = s * P.off[pd];
        L.A = A;
        L.B = B;
        L.C = n / 2;
        L.sa = sa;
        L.sb = sb;
        L.p_base = pos;
        L.level = level;
        P.passes.push_back(L);
        pos += A * B * (n / 2);
    }

    void disabled_level(int level, long long s, bool last) {
        const long long s2 = 2 * s;
        const int N = P.N;
        if (N == 1) {
            lines(level, s, 0, 1, 0, 1, 0, last);
        } else if (N == 2) {
            if (prm.direction == 0) {
                rows(level, s, 0, -1, 0, 1, s2, false);
                lines(level, s, 1, 1, 0, count_of(P.dims[0], s), s * P.off[0], last);
            } else {
                lines(level, s, 1, 1, 0, count_of(P.dims[0], s2), s2 * P.off[0], false);
                rows(level, s, 0, -1, 0, 1, s, last);
            }
        } else {
            if (prm.direction == 0) {
                rows(level, s, 0, 1, s2, 2, s2, false);
                rows(level, s, 1, 0, s, 2, s2, false);
                lines(level, s, 2, count_of(P.dims[0], s), s * P.off[0], count_of(P.dims[1], s), s * P.off[1], last);
            } else {
                lines(level, s, 2, count_of(P.dims[0], s2), s2 * P.off[0], count_of(P.dims[1], s2), s2 * P.off[1],
                      false);
                rows(level, s, 1, 0, s2, 2, s, false);
                rows(level, s, 0, 1, s, 2, s, last);
            }
        }
    }

    // One foreach sweep of interpolation_1d_fastest_dim_first with the pass dim restricted to
    // t in [t0, t1) step 2.
    void generic_sweep(int level, long long s, int pd, const long long *st, long long t0, long long t1, int mode) {
        const long long n = (P.dims[pd] - 1) / s + 1;
        PassLaunch L = blank();
        L.kind = KIND_GENERIC;
        L.cubic = prm.cubic != 0;
        L.n = (int)n;
        L.step = s * P.off[pd];
        L.N = P.N;
        L.pd = pd;
        L.g_t0 = (int)t0;
        L.g_mode = mode;
        long long total = 1;
        for (int d = 0; d < P.N; d++) {
            if (d == pd) {
                L.cnt[d] = t1 > t0 ? (t1 - t0 + 1) / 2 : 0;
                L.est[d] = 2 * L.step;
            } else {
                L.cnt[d] = count_of(P.dims[d], st[d]);
                L.est[d] = st[d] * P.off[d];
            }
            total *= L.cnt[d];
        }
        L.A = 1;
        L.B = 1;
        L.C = total;
        L.p_base = pos;
        L.level = level;
        if (total > 0) P.passes.push_back(L);
        pos += total;
    }

    void generic_pass(int level, long long s, int pd, const long long *st) {
        const long long n = (P.dims[pd] - 1) / s + 1;
        if (n <= 1) return;
        if (!prm.cubic) {
            generic_sweep(level, s, pd, st, 1, n - 1, 0);
            if (n % 2 == 0) generic_sweep(level, s, pd, st, n - 1, n, 2);
        } else {
            generic_sweep(level, s, pd, st, 3, n >= 3 ? n - 3 : 0, 0);
            long long b[4];
            int nb = 0;
            b[nb++] = 1;
            if (n % 2 == 1 && n > 3) b[nb++] = n - 2;
            if (n % 2 == 0 && n > 4) b[nb++] = n - 3;
            if (n % 2 == 0 && n > 2) b[nb++] = n - 1;
            for (int i = 0; i < nb; i++) generic_sweep(level, s, pd, st, b[i], b[i] + 1, 1);
        }
    }

    void tuning_level(int level, long long s) {
        int seq[4];
        {
            int a[4] = {0, 1, 2, 3};
            for (int it = 0; it < prm.direction; it++) {
                int i = P.N - 2;
                while (i >= 0 && a[i] >= a[i + 1]) i--;
                if (i < 0) break;
                int j = P.N - 1;
                while (a[j] <= a[i]) j--;
                std::swap(a[i], a[j]);
                std::reverse(a + i + 1, a + P.N);
            }
            for (int i = 0; i < 4; i++) seq[i] = a[i];
        }
        const long long s2 = 2 * s;
        if (P.N >= 3) {
            long long st[4] = {s2, s2, s2, s2};
            generic_pass(level, s, seq[0], st);
            for (int i = 1; i < P.N; i++) {
                st[seq[i - 1]] = s;
                generic_pass(level, s, seq[i], st);
            }
        } else if (P.N == 2) {
            const int d0 = seq[0], d1 = seq[1];
            legacy_lines(level, s, d0, count_of(P.dims[d1], s2), s2 * P.off[d1]);
            legacy_lines(level, s, d1, count_of(P.dims[d0], s), s * P.off[d0]);
        } else {
            legacy_lines(level, s, 0, 1, 0);
        }
    }

    // Legacy 1-D routine interpolation_1d (InterpolationDecomposition.hpp:371-419) on A lines.
    void legacy_lines(int level, long long s, int pd, long long A, long long sa) {
        const long long n = (P.dims[pd] - 1) / s + 1;
        if (n <= 1) return;
        PassLaunch L = blank();
        L.kind = KIND_LEGACY;
        L.cubic = prm.cubic != 0;
        L.n = (int)n;
        L.step = s * P.off[pd];
        L.A = A;
        L.sa = sa;
        L.B = 1;
        L.C = n / 2;
        L.p_base = pos;
        L.level = level;
        P.passes.push_back(L);
        pos += A * (n / 2);
    }
};

}  // namespace

InterpPlan make_plan(const long long *dims, int N, const InterpParams &p) {
    if (N < 1 || N > 4) throw std::invalid_argument("Data dimension higher than 4 is not supported.");
    if (!(p.eb > 0) || !std::isfinite(p.eb)) throw std::invalid_argument("error bound must be positive and finite");
    if (p.radius < 1 || p.radius > 32768) throw std::invalid_argument("quantization radius must be in [1, 32768]");
    if (p.anchor < 0 || (p.anchor & (p.anchor - 1)) != 0)
        throw std::invalid_argument("Anchor stride should be 0 or 2's exponentials");
    if (p.cubic != 0 && p.cubic != 1) throw std::invalid_argument("interpAlgo must be linear (0) or cubic (1)");
    int fact = 1;
    for (int i = 2; i <= N; i++) fact *= i;
    if (p.direction < 0 || p.direction >= fact) throw std::invalid_argument("interpDirection out of range");
    if (!p.tuning && N >= 2 && N <= 3 && p.direction != 0 && p.direction != fact - 1)
        throw std::invalid_argument("interpDirection must be 0 or N!-1 for 2-D and 3-D fields");

    InterpPlan P;
    P.N = N;
    P.max_abs = p.max_abs;
    P.num = 1;
    for (int d = 0; d < N; d++) {
        if (dims[d] < 1) throw std::invalid_argument("zero-sized dimension");
        P.dims[d] = dims[d];
        P.num *= dims[d];
    }
    for (int d = N; d < 4; d++) { P.dims[d] = 1; }
    P.off[N - 1] = 1;
    for (int d = N - 2; d >= 0; d--) P.off[d] = P.off[d + 1] * P.dims[d + 1];
    for (int d = N; d < 4; d++) P.off[d] = 0;
    if (P.num > (1LL << 40)) throw std::invalid_argument("field too large");

    int level_count = -1;
    bool use_anchor = false;
    for (int d = 0; d < N; d++) {
        int lv = (int)std::ceil(std::log2((double)P.dims[d]));
        if (level_count < lv) level_count = lv;
        if (P.dims[d] > p.anchor) use_anchor = true;
    }
    P.anchor = use_anchor ? p.anchor : 0;
    if (P.anchor > 0) {
        int maxl = (int)std::log2((double)P.anchor) + 1;
        if (maxl <= level_count) level_count = maxl;
    }
    // index 0: the constructor's reciprocal 0.5/eb (used only by the anchor-free first point)
    P.levels.push_back(QParams{p.eb, 2 * p.eb, 0.5 / p.eb, p.radius, float_at_most(p.eb)});
    Builder b(P, p);
    P.first_point = 0;
    P.n_anchor = 0;
    if (P.anchor == 0) {
        P.first_point = 1;
        b.pos = 1;
    } else {
        P.n_anchor = 1;
        for (int d = 0; d < N; d++) P.n_anchor *= count_of(P.dims[d], P.anchor);
        level_count--;
    }
    for (int level = level_count; level > 0; level--) {
        double cur = p.eb;
        if (p.alpha < 0) {
            cur = level >= 3 ? p.eb * 0.5 : p.eb;
        } else if (p.alpha >= 1) {
            double ratio = std::pow(p.alpha, level - 1);
            if (ratio > p.beta) ratio = p.beta;
            cur = p.eb / ratio;
        }
        const int li = (int)P.levels.size();
        P.levels.push_back(QParams{cur, 2 * cur, 1.0 / (2 * cur), p.radius, float_at_most(cur)});
        P.level_starts.push_back(b.pos);
        const long long s = 1LL << (level - 1);
        if (p.tuning || N == 4) b.tuning_level(li, s);
        else b.disabled_level(li, s, level == 1);
    }
    P.n_codes = b.pos;
    if (P.n_codes + P.n_anchor != P.num) throw std::logic_error("interpolation plan does not cover the field");
    return P;
}

// ------------------------------------------------------------------------------------------ kernels
namespace {

constexpr int kTile = 4096;         // codes per escape-scan tile
constexpr int kTileThreads = 256;   // 16 codes per thread
constexpr int kPassThreads = 256;

// Compress: one more escape in the tile of kTile codes holding code position p (the escape scan's
// tile counts, gathered while the passes code).
__device__ __forceinline__ void count_escape(unsigned *etile, long long p) {
    if (etile) atomicAdd(etile + p / kTile, 1u);
}

template <class T, int KIND, bool DECOMP>
__global__ void __launch_bounds__(kPassThreads) k_pass(const PassLaunch L, T *__restrict__ x,
                                                      int16_t *__restrict__ codes, T *__restrict__ esc,
                                                      const QParams qp, unsigned *__restrict__ etile) {
    const long long cstride = (long long)gridDim.x * blockDim.x;
    for (long long a = blockIdx.z; a < L.A; a += gridDim.z) {
        for (long long b = blockIdx.y; b < L.B; b += gridDim.y) {
            for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < L.C; c += cstride) {
                long long line, p;
                int t;
                Rule r;
                if (KIND == KIND_ROW) {
                    t = L.t0 + 2 * (int)b;
                    line = a * L.sa + c * L.sc;
                    p = L.p_base + (a * L.rows_in_group + b + L.b_off) * L.C + c;
                    r = row_rule(L.cubic, t, L.n, L.skip);
                } else if (KIND == KIND_LINE) {
                    t = 1 + 2 * (int)c;
                    line = a * L.sa + b * L.sb;
                    p = L.p_base + (a * L.B + b) * L.C + c;
                    r = line_rule(L.cubic, t, L.n);
                } else if (KIND == KIND_GENERIC) {
                    long long rem = c, off = 0;
                    int tg = 0;
#pragma unroll
                    for (int d = 3; d >= 0; d--) {
                        if (d >= L.N) continue;
                        const long long i = rem % L.cnt[d];
                        rem /= L.cnt[d];
                        if (d == L.pd) tg = L.g_t0 + 2 * (int)i;
                        else off += i * L.est[d];
                    }
                    t = tg;
                    line = off;
                    p = L.p_base + c;
                    if (L.g_mode == 2) {
                        r = L.n < 3 ? mk_rule(F_EQUAL, L.n - 2) : mk_rule(F_LINEAR1, L.n - 3, L.n - 2);
                    } else if (L.g_mode == 1) {
                        const int bb = t, n = L.n;
                        if (bb >= 3) {
                            if (bb + 3 < n) r = mk_rule(F_CUBIC, bb - 3, bb - 1, bb + 1, bb + 3);
                            else if (bb + 1 < n) r = mk_rule(F_QUAD2, bb - 3, bb - 1, bb + 1);
                            else r = mk_rule(F_LINEAR1, bb - 3, bb - 1);
                        } else {
                            if (bb + 3 < n) r = mk_rule(F_QUAD1, bb - 1, bb + 1, bb + 3);
                            else if (bb + 1 < n) r = mk_rule(F_LINEAR, bb - 1, bb + 1);
                            else r = mk_rule(F_EQUAL, bb - 1);
                        }
                    } else if (L.cubic) {
                        r = mk_rule(F_CUBIC, t - 3, t - 1, t + 1, t + 3);
                    } else {
                        r = mk_rule(F_LINEAR, t - 1, t + 1);
                    }
                } else {  // KIND_LEGACY: interpolation_1d on line a; its own visiting order
                    t = 1 + 2 * (int)c;
                    line = a * L.sa;
                    const int n = L.n;
                    int rank = (int)c;
                    if (!L.cubic || n < 5) {
                        if (t + 1 < n) r = mk_rule(F_LINEAR, t - 1, t + 1);
                        else r = n < 4 ? mk_rule(F_EQUAL, n - 2) : mk_rule(F_LINEAR1, n - 4, n - 2);
                    } else {
                        const int tf = (n & 1) ? n - 2 : n - 3;  // first odd t with t + 3 >= n
                        const int mid = (tf - 3) / 2;
                        if (t == 1) {
                            r = mk_rule(F_QUAD1, 0, 2, 4);
                            rank = mid;
                        } else if (t == tf) {
                            r = mk_rule(F_QUAD2, t - 3, t - 1, t + 1);
                            rank = mid + 1;
                        } else if (t > tf) {
                            r = mk_rule(F_QUAD3, n - 6, n - 4, n - 2);
                            rank = mid + 2;
                        } else {
                            r = mk_rule(F_CUBIC, t - 3, t - 1, t + 1, t + 3);
                            rank = (t - 3) / 2;
                        }
                    }
                    p = L.p_base + a * L.C + rank;
                }
                const long long st = L.step;
                // Operands are never written by this launch: read them through the read-only path.
                const T o0 = __ldg(x + line + (long long)r.o0 * st);
                const T o1 = r.f != F_EQUAL ? __ldg(x + line + (long long)r.o1 * st) : o0;
                const T o2 = r.f >= F_QUAD1 ? __ldg(x + line + (long long)r.o2 * st) : o0;
                const T o3 = r.f == F_CUBIC ? __ldg(x + line + (long long)r.o3 * st) : o0;
                const T pred = apply_formula<T>(r.f, o0, o1, o2, o3);
                T *xp = x + line + (long long)t * st;
                if (!DECOMP) {
                    const T v = *xp;
                    T recon;
                    const int q = quantize<T>(v, pred, qp, recon);
                    codes[p] = (int16_t)q;
                    if (q == -qp.radius) {
                        esc[p] = v;
                        count_escape(etile, p);
                    } else if (!L.skip) {
                        *xp = recon;
                    }
                } else {
                    const int q = codes[p];
                    *xp = (q != -qp.radius) ? dequantize<T>(q, pred, qp) : esc[p];
                }
            }
        }
    }
}

template <class T, bool DECOMP>
__global__ void k_first_point(T *x, int16_t *codes, T *esc, const QParams qp, unsigned *etile) {
    if (!DECOMP) {
        T recon;
        const T v = x[0];
        const int q = quantize<T>(v, T(0), qp, recon);
        codes[0] = (int16_t)q;
        if (q == -qp.radius) {
            esc[0] = v;
            count_escape(etile, 0);
        } else {
            x[0] = recon;
        }
    } else {
        const int q = codes[0];
        x[0] = q != -qp.radius ? dequantize<T>(q, T(0), qp) : esc[0];
    }
}

struct AnchorGrid {
    int N;
    long long cnt[4], est[4];
    long long total;
};

template <class T, bool DECOMP>
__global__ void k_anchors(const AnchorGrid G, T *x, T *unpred) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < G.total;
         i += (long long)gridDim.x * blockDim.x) {
        long long rem = i, off = 0;
        for (int d = G.N - 1; d >= 0; d--) {
            off += (rem % G.cnt[d]) * G.est[d];
            rem /= G.cnt[d];
        }
        if (!DECOMP) unpred[i] = x[off];
        else x[off] = unpred[i];
    }
}

// Escape counting per tile of kTile codes.
__global__ void __launch_bounds__(kTileThreads) k_esc_count(const int16_t *__restrict__ codes, long long n, int esc,
                                                            unsigned *__restrict__ tile_count) {
    const long long base = (long long)blockIdx.x * kTile + threadIdx.x * 16;
    int cnt = 0;
    // 16-byte vectors when the code array is 16-byte aligned (tile starts are multiples of 16 codes)
    if (base + 16 <= n && (reinterpret_cast<uintptr_t>(codes) & 15) == 0) {
        const int4 *v = reinterpret_cast<const int4 *>(codes + base);
        int4 w[2] = {__ldg(v), __ldg(v + 1)};
        const int16_t *h = reinterpret_cast<const int16_t *>(w);
#pragma unroll
        for (int j = 0; j < 16; j++) cnt += (h[j] == esc);
    } else {
        for (long long j = base; j < n && j < base + 16; j++) cnt += (codes[j] == esc);
    }
    // block reduction
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    __shared__ int ws[kTileThreads / 32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x < 32) {
        int v2 = threadIdx.x < kTileThreads / 32 ? ws[threadIdx.x] : 0;
        v2 = __reduce_add_sync(0xffffffffu, v2);
        if (threadIdx.x == 0) tile_count[blockIdx.x] = v2;
    }
}

// Exclusive scan of tile counts (single block; every thread scans kScanRun consecutive counts per
// round); writes offsets[0..ntiles] and the total.
constexpr int kScanRun = 16;
__global__ void __launch_bounds__(1024) k_scan_u32(const unsigned *__restrict__ in, unsigned long long *__restrict__ out,
                                                   long long n, unsigned long long *total) {
    __shared__ unsigned long long warp_sums[32];
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long long base = 0; base < n; base += 1024LL * kScanRun) {
        const long long i0 = base + (long long)threadIdx.x * kScanRun;
        const bool whole = i0 + kScanRun <= n;  // 16-byte vectors (both arrays are 256-byte aligned)
        unsigned v[kScanRun];
        unsigned long long sum = 0;
        if (whole) {
#pragma unroll
            for (int j = 0; j < kScanRun / 4; j++) {
                const uint4 u = __ldg(reinterpret_cast<const uint4 *>(in + i0) + j);
                v[4 * j] = u.x;
                v[4 * j + 1] = u.y;
                v[4 * j + 2] = u.z;
                v[4 * j + 3] = u.w;
            }
        } else {
#pragma unroll
            for (int j = 0; j < kScanRun; j++) v[j] = i0 + j < n ? __ldg(in + i0 + j) : 0u;
        }
#pragma unroll
        for (int j = 0; j < kScanRun; j++) sum += v[j];
        // inclusive warp scan of the run sums, then across warps
        unsigned long long s = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, s, o);
            if ((threadIdx.x & 31) >= (unsigned)o) s += y;
        }
        if ((threadIdx.x & 31) == 31) warp_sums[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x < 32) {
            unsigned long long w = warp_sums[threadIdx.x];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
                if (threadIdx.x >= (unsigned)o) w += y;
            }
            warp_sums[threadIdx.x] = w;  // inclusive over warps
        }
        __syncthreads();
        const unsigned long long wprev = (threadIdx.x >> 5) ? warp_sums[(threadIdx.x >> 5) - 1] : 0;
        unsigned long long e = carry + wprev + s - sum;
        if (whole) {
#pragma unroll
            for (int j = 0; j < kScanRun; j += 2) {
                const unsigned long long e1 = e + v[j];
                reinterpret_cast<ulonglong2 *>(out + i0)[j / 2] = make_ulonglong2(e, e1);
                e = e1 + v[j + 1];
            }
        } else {
#pragma unroll
            for (int j = 0; j < kScanRun; j++) {
                if (i0 + j < n) out[i0 + j] = e;
                e += v[j];
            }
        }
        __syncthreads();
        if (threadIdx.x == 1023) carry += wprev + s;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[n] = carry;
        if (total) *total = carry;
    }
}

// Per tile: rank the escapes in stream order and move their values between the scattered
// per-position array `esc` and the compact unpredictable list (after the anchors).
template <class T, bool DECOMP>
__global__ void __launch_bounds__(kTileThreads) k_esc_scatter(const int16_t *__restrict__ codes, long long n, int esc_code,
                                                              const unsigned long long *__restrict__ tile_off,
                                                              T *__restrict__ esc, T *__restrict__ unpred,
                                                              long long n_anchor, unsigned long long n_esc_max) {
    const unsigned long long t0 = tile_off[blockIdx.x], t1 = tile_off[blockIdx.x + 1];
    if (t0 == t1) return;
    const long long base = (long long)blockIdx.x * kTile + threadIdx.x * 16;
    unsigned mask = 0;
    for (int j = 0; j < 16; j++) {
        const long long i = base + j;
        if (i < n && codes[i] == esc_code) mask |= 1u << j;
    }
    const int cnt = __popc(mask);
    // block exclusive scan of cnt
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int s = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
    }
    __shared__ int wsum[kTileThreads / 32];
    if (lane == 31) wsum[wid] = s;
    __syncthreads();
    int before = 0;
    for (int w = 0; w < wid; w++) before += wsum[w];
    unsigned long long r = t0 + before + s - cnt;
    while (mask) {
        const int j = __ffs(mask) - 1;
        mask &= mask - 1;
        const long long i = base + j;
        if (!DECOMP) unpred[n_anchor + r] = esc[i];
        else if (r < n_esc_max) esc[i] = unpred[n_anchor + r];  // a list too short is reported by the host
        r++;
    }
}

// Cubic interior predictor (Interpolators.hpp cubic: (9 (b + c) - a - d) / 16) and linear.
template <class T>
__device__ __forceinline__ T cubic_pred(T a, T b, T c, T d) {
    using A = Arith<T>;
    T t = A::mul(A::add(b, c), T(9));
    t = A::sub(t, a);
    t = A::sub(t, d);
    return A::mul(t, T(0.0625));
}
template <class T>
__device__ __forceinline__ T linear_pred(T a, T b) {
    return Arith<T>::mul(Arith<T>::add(a, b), T(0.5));
}

// Quantizes (compress: v is the target's value, recon goes back to *xp unless `skip`) or
// reconstructs (decompress) one target; p is its position in the code stream.
template <class T, bool DECOMP>
__device__ __forceinline__ void pass_target(T *__restrict__ xp, T v, T pred, int16_t *__restrict__ cp,
                                            T *__restrict__ ep, const QParams &qp, bool skip, unsigned *etile,
                                            long long p) {
    if (!DECOMP) {
        T recon;
        const int q = quantize<T>(v, pred, qp, recon);
        *cp = (int16_t)q;
        if (q == -qp.radius) {
            *ep = v;
            count_escape(etile, p);
        } else if (!skip) {
            *xp = recon;
        }
    } else {
        const int q = *cp;
        *xp = (q != -qp.radius) ? dequantize<T>(q, pred, qp) : *ep;
    }
}

// Row-buffer passes (KIND_ROW): one thread per column, kRowsPerBlock consecutive target rows per
// block (their operand rows overlap, so most operand loads hit L1), grid (columns, row groups,
// outer).  Interior targets take the cubic (or linear) formula without evaluating the edge rules.
constexpr int kRowsPerBlock = 8;
template <class T, bool DECOMP>
__global__ void __launch_bounds__(kPassThreads) k_row_fast(const PassLaunch L, T *__restrict__ x,
                                                          int16_t *__restrict__ codes, T *__restrict__ esc,
                                                          const QParams qp, unsigned *__restrict__ etile) {
    const long long cstride = (long long)gridDim.x * blockDim.x;
    const long long st = L.step;
    for (long long a = blockIdx.z; a < L.A; a += gridDim.z) {
        for (long long bg = blockIdx.y; bg * kRowsPerBlock < L.B; bg += gridDim.y)
        for (long long b = bg * kRowsPerBlock; b < min(L.B, (bg + 1) * kRowsPerBlock); b++) {
            const int t = L.t0 + 2 * (int)b;
            const bool interior = L.cubic ? (t >= 3 && t <= L.n - 5) : (t < L.n - 1);
            const Rule r = row_rule(L.cubic, t, L.n, L.skip);
            const long long prow = L.p_base + (a * L.rows_in_group + b + L.b_off) * L.C;
            for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < L.C; c += cstride) {
                T *xl = x + a * L.sa + c * L.sc;
                T pred;
                if (interior) {
                    pred = L.cubic ? cubic_pred<T>(__ldg(xl + (t - 3) * st), __ldg(xl + (t - 1) * st),
                                                   __ldg(xl + (t + 1) * st), __ldg(xl + (t + 3) * st))
                                   : linear_pred<T>(__ldg(xl + (t - 1) * st), __ldg(xl + (t + 1) * st));
                } else {
                    const T o0 = __ldg(xl + (long long)r.o0 * st);
                    const T o1 = r.f != F_EQUAL ? __ldg(xl + (long long)r.o1 * st) : o0;
                    const T o2 = r.f >= F_QUAD1 ? __ldg(xl + (long long)r.o2 * st) : o0;
                    const T o3 = r.f == F_CUBIC ? __ldg(xl + (long long)r.o3 * st) : o0;
                    pred = apply_formula<T>(r.f, o0, o1, o2, o3);
                }
                T *xp = xl + (long long)t * st;
                pass_target<T, DECOMP>(xp, DECOMP ? T(0) : *xp, pred, codes + prow + c, esc + prow + c, qp, L.skip, etile,
                                       prow + c);
            }
        }
    }
}

// Line passes (KIND_LINE) whose line fits kLineMax bytes: one warp per line; the warp stages the
// line in shared memory with coalesced loads (every value read once), then predicts its targets
// (odd positions; their operands are the even positions, which this pass never writes).
// Interior targets take the cubic (or linear) formula without evaluating the edge rules.
constexpr int kLineThreads = 256;
constexpr int kLineMax = 4096;
template <class T, bool DECOMP>
__global__ void __launch_bounds__(kLineThreads) k_line_smem(const PassLaunch L, T *__restrict__ x,
                                                           int16_t *__restrict__ codes, T *__restrict__ esc,
                                                           const QParams qp, unsigned *__restrict__ etile) {
    __shared__ T buf[kLineThreads / 32][kLineMax / sizeof(T)];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    T *bw = buf[wid];
    const long long nlines = L.A * L.B;
    const long long st = L.step;
    const int n = L.n, C = (int)L.C, odd = n / 2;
    // cubic interior: 3 <= t <= 2 * odd - 5; linear interior: t < 2 * odd - 1
    const int tlo = L.cubic ? 3 : 1, thi = L.cubic ? 2 * odd - 5 : 2 * odd - 3;
    for (long long l = (long long)blockIdx.x * (kLineThreads / 32) + wid; l < nlines;
         l += (long long)gridDim.x * (kLineThreads / 32)) {
        const long long a = l / L.B, b = l - a * L.B;
        T *xl = x + a * L.sa + b * L.sb;
        __syncwarp();
        if (st == 1) {
            for (int i = lane; i < n; i += 32) bw[i] = xl[i];
        } else {
            for (int i = lane; i < n; i += 32) bw[i] = xl[(long long)i * st];
        }
        __syncwarp();
        int16_t *cl = codes + L.p_base + l * L.C;
        T *el = esc + L.p_base + l * L.C;
        for (int cc = lane; cc < C; cc += 32) {
            const int t = 1 + 2 * cc;
            T pred;
            if (t >= tlo && t <= thi) {
                pred = L.cubic ? cubic_pred<T>(bw[t - 3], bw[t - 1], bw[t + 1], bw[t + 3]) : linear_pred<T>(bw[t - 1], bw[t + 1]);
            } else {
                const Rule r = line_rule(L.cubic, t, n);
                const T o0 = bw[r.o0];
                const T o1 = r.f != F_EQUAL ? bw[r.o1] : o0;
                const T o2 = r.f >= F_QUAD1 ? bw[r.o2] : o0;
                const T o3 = r.f == F_CUBIC ? bw[r.o3] : o0;
                pred = apply_formula<T>(r.f, o0, o1, o2, o3);
            }
            pass_target<T, DECOMP>(xl + (long long)t * st, bw[t], pred, cl + cc, el + cc, qp, L.skip, etile,
                                   L.p_base + l * L.C + cc);
        }
    }
}

template <class T, bool DECOMP>
void launch_pass(const PassLaunch &L, T *x, int16_t *codes, T *esc, const QParams &qp, unsigned *etile,
                 cudaStream_t st) {
    if (L.kind == KIND_ROW) {
        dim3 grid((unsigned)std::max<long long>(1, std::min<long long>((L.C + kPassThreads - 1) / kPassThreads, 1 << 20)),
                  (unsigned)std::min<long long>((L.B + kRowsPerBlock - 1) / kRowsPerBlock, 65535),
                  (unsigned)std::min<long long>(L.A, 65535));
        k_row_fast<T, DECOMP><<<grid, kPassThreads, 0, st>>>(L, x, codes, esc, qp, etile);
        FB2_CHECK_LAUNCH();
        return;
    }
    if (L.kind == KIND_LINE && (long long)L.n * (long long)sizeof(T) <= kLineMax) {
        const long long nlines = L.A * L.B;
        const long long blocks = std::min<long long>((nlines + kLineThreads / 32 - 1) / (kLineThreads / 32), 148LL * 64);
        k_line_smem<T, DECOMP><<<(unsigned)std::max<long long>(blocks, 1), kLineThreads, 0, st>>>(L, x, codes, esc, qp, etile);
        FB2_CHECK_LAUNCH();
        return;
    }
    dim3 block(kPassThreads);
    const long long gx = std::min<long long>((L.C + kPassThreads - 1) / kPassThreads, 1 << 20);
    dim3 grid((unsigned)std::max<long long>(gx, 1), (unsigned)std::min<long long>(L.B, 65535),
              (unsigned)std::min<long long>(L.A, 65535));
    switch (L.kind) {
        case KIND_ROW: k_pass<T, KIND_ROW, DECOMP><<<grid, block, 0, st>>>(L, x, codes, esc, qp, etile); break;
        case KIND_LINE: k_pass<T, KIND_LINE, DECOMP><<<grid, block, 0, st>>>(L, x, codes, esc, qp, etile); break;
        case KIND_GENERIC: k_pass<T, KIND_GENERIC, DECOMP><<<grid, block, 0, st>>>(L, x, codes, esc, qp, etile); break;
        default: k_pass<T, KIND_LEGACY, DECOMP><<<grid, block, 0, st>>>(L, x, codes, esc, qp, etile); break;
    }
    FB2_CHECK_LAUNCH();
}

// The y pass and the x pass of one level of a field (direction 0; any grid step), fused: one
// CTA per (z plane, tile of kFuseR rows x kFuseW columns) stages its tile plus a halo of kFuseHalo
// rows and columns (every rule operand lies within 3 grid units of its target) in shared memory,
// runs the y pass (ROW: odd rows, even columns; the halo columns' targets are recomputed so that
// the x pass can read them) and then the x pass (LINE: odd columns) on the staged tile, and
// writes the tile back once.  When the level's z pass precedes them (3-D), a CTA of an odd plane
// first predicts that plane's z-pass targets (even rows, even columns of the staged tile, halo
// included) from the four even planes around it, read from global memory (this level never
// writes those points).  Codes and escape slots go to the positions the passes have in the code
// stream (InterpolationDecomposition.hpp:2294-2527 visiting order).
struct FusedYX {
    PassLaunch y;     // ROW pass along y: rows t = 1 + 2 b (b < y.B), columns at even x
    PassLaunch late;  // its last-row pass (t = n - 1), when has_late
    PassLaunch x;     // LINE pass along x: lines (z, y)
    PassLaunch z;     // ROW pass along z: planes t = 1 + 2 b (b < z.B) at even y and x, when has_z
    PassLaunch zlate; // its last-plane pass (t = nz - 1), when has_zlate
    int has_late, has_z, has_zlate;
};
constexpr int kFuseW = 64, kFuseR = 64, kFuseHalo = 4;
constexpr int kFusePW = kFuseW + 2 * kFuseHalo, kFusePR = kFuseR + 2 * kFuseHalo;
constexpr int kFuseThreads = 256;

template <class T, bool DECOMP>
__global__ void __launch_bounds__(kFuseThreads, sizeof(T) == 4 ? 8 : 6) k_yx_fused(const FusedYX F, T *__restrict__ xf,
                                                           int16_t *__restrict__ codes, T *__restrict__ esc,
                                                           const QParams qp, unsigned *__restrict__ etile) {
    __shared__ __align__(16) T tile[kFusePR * kFusePW];
    constexpr int P = kFusePW, H = kFuseHalo;
    const int ny = F.y.n, nx = F.x.n;
    const long long a = blockIdx.z;
    const int x0 = (int)blockIdx.x * kFuseW, x1 = min(nx, x0 + kFuseW);
    const int y0 = (int)blockIdx.y * kFuseR, y1 = min(ny, y0 + kFuseR);
    const int xl = max(0, x0 - H), xr = min(nx, x1 + H), TW = xr - xl;
    const int yl = max(0, y0 - H), yr = min(ny, y1 + H), TR = yr - yl;
    T *plane = xf + a * F.x.sa;
    const long long sy = F.x.sb, sx = F.x.step;  // element steps of one grid unit in y and x
    // stage rows [yl, yr) x columns [xl, xr) (tile row r, column c: y = yl + r, x = xl + c)
    constexpr int V = 16 / sizeof(T);
    const bool vec = sx == 1 && ((reinterpret_cast<uintptr_t>(plane + xl) & 15) == 0) && (sy % V == 0) && (TW % V == 0);
    if (vec) {
        // thread (vector slot qq of a row, row group); kFusePW / V slots per row at most
        constexpr int NQ = kFusePW / V, NG = kFuseThreads / NQ;
        const int nq = TW / V, qq = threadIdx.x % NQ, g = threadIdx.x / NQ;
        if (qq < nq && g < NG) {
            const T *src = plane + (long long)(yl + g) * sy + xl + qq * V;
            T *dstp = tile + g * P + qq * V;
            for (int rr = g; rr < TR; rr += NG, src += NG * sy, dstp += NG * P) {
                const unsigned sa = (unsigned)__cvta_generic_to_shared(dstp);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(src) : "memory");
            }
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
    } else {
        for (int i = threadIdx.x; i < TR * TW; i += blockDim.x) {
            const int rr = i / TW, cc = i - rr * TW;
            tile[rr * P + cc] = plane[(yl + rr) * sy + (xl + cc) * sx];
        }
    }
    __syncthreads();
    // z pass of an odd plane: even rows x even columns of the staged tile
    const bool zplane = F.has_z && (a & 1);
    if (zplane) {
        const int nz = F.z.n, t = (int)a;
        const bool zl = F.has_zlate && t == nz - 1;
        const long long sz = F.x.sa;  // element step of one plane
        const int re0 = (yl + 1) & ~1, ce0 = (xl + 1) & ~1;
        const int nre = (yr - re0 + 1) / 2, nce = (xr - ce0 + 1) / 2;
        const Rule r = row_rule(true, t, nz, F.z.skip);
        const bool inner = t >= 3 && t <= nz - 5;
        constexpr int NCZ = kFusePW / 2, NGZ = kFuseThreads / NCZ;  // thread (column, row group)
        const int czi = threadIdx.x % NCZ, gz = threadIdx.x / NCZ;
        for (int ri = gz; ri < nre && czi < nce && gz < NGZ; ri += NGZ) {
            const int yg = re0 + 2 * ri, xg = ce0 + 2 * czi;
            const T *col = xf + (long long)yg * sy + (long long)xg * sx;  // col[z * sz] is (z, yg, xg)
            T pred;
            if (inner) {
                pred = cubic_pred<T>(col[(t - 3) * sz], col[(t - 1) * sz], col[(t + 1) * sz], col[(t + 3) * sz]);
            } else {
                const T o0 = col[r.o0 * sz];
                const T o1 = r.f != F_EQUAL ? col[r.o1 * sz] : o0;
                const T o2 = r.f >= F_QUAD1 ? col[r.o2 * sz] : o0;
                const T o3 = r.f == F_CUBIC ? col[r.o3 * sz] : o0;
                pred = apply_formula<T>(r.f, o0, o1, o2, o3);
            }
            const long long ay = yg >> 1, c = xg >> 1;
            const long long p = zl ? F.zlate.p_base + ay * F.zlate.C + c
                                   : F.z.p_base + (ay * F.z.rows_in_group + ((t - 1) >> 1) + F.z.b_off) * F.z.C + c;
            T *xp = tile + (yg - yl) * P + (xg - xl);
            if (!DECOMP) {
                const bool own = yg >= y0 && yg < y1 && xg >= x0 && xg < x1;
                T recon;
                const T v = *xp;
                const int q = quantize<T>(v, pred, qp, recon);
                if (own) codes[p] = (int16_t)q;
                if (q == -qp.radius) {
                    if (own) {
                        esc[p] = v;
                        count_escape(etile, p);
                    }
                } else if (!F.z.skip) {
                    *xp = recon;
                }
            } else {
                const int q = codes[p];
                *xp = (q != -qp.radius) ? dequantize<T>(q, pred, qp) : esc[p];
            }
        }
        __syncthreads();
    }
    // y pass: odd rows of [y0, y1) x even columns of [xl, xr); thread (column tc, row group g)
    {
        constexpr int NC = kFusePW / 2, NG = kFuseThreads / NC;
        const int ce0 = (xl + 1) & ~1;
        const int tc = threadIdx.x % NC, g = threadIdx.x / NC;
        const int xg = ce0 + 2 * tc;
        // code position of (row t, column xg): main rows p0 + ((t - 1) / 2 - y0 / 2) * C
        const long long c = xg >> 1;
        const long long p0 = F.y.p_base + ((long long)a * F.y.rows_in_group + (y0 >> 1) + F.y.b_off) * F.y.C + c;
        for (int tr = g; tr < kFuseR / 2 && g < NG && xg < xr; tr += NG) {
            const int t = y0 + 1 + 2 * tr;
            if (t >= y1) break;
            const bool late = F.has_late && t == ny - 1;
            const T *col = tile + (xg - xl) - yl * P;  // col[y * P] is (y, xg)
            T pred;
            if (t >= 3 && t <= ny - 5) {
                pred = cubic_pred<T>(col[(t - 3) * P], col[(t - 1) * P], col[(t + 1) * P], col[(t + 3) * P]);
            } else {
                const Rule r = row_rule(true, t, ny, F.y.skip);
                const T o0 = col[r.o0 * P];
                const T o1 = r.f != F_EQUAL ? col[r.o1 * P] : o0;
                const T o2 = r.f >= F_QUAD1 ? col[r.o2 * P] : o0;
                const T o3 = r.f == F_CUBIC ? col[r.o3 * P] : o0;
                pred = apply_formula<T>(r.f, o0, o1, o2, o3);
            }
            const long long p = late ? F.late.p_base + a * F.late.C + c : p0 + (long long)tr * F.y.C;
            T *xp = tile + (t - yl) * P + (xg - xl);
            if (!DECOMP) {
                const bool own = xg >= x0 && xg < x1;
                T recon;
                const T v = *xp;
                const int q = quantize<T>(v, pred, qp, recon);
                if (own) codes[p] = (int16_t)q;
                if (q == -qp.radius) {
                    if (own) {
                        esc[p] = v;
                        count_escape(etile, p);
                    }
                } else if (!F.y.skip) {
                    *xp = recon;
                }
            } else {
                const int q = codes[p];
                *xp = (q != -qp.radius) ? dequantize<T>(q, pred, qp) : esc[p];
            }
        }
    }
    __syncthreads();
    // x pass: rows [y0, y1) x odd columns of [x0, x1); thread (column k, row group g)
    {
        constexpr int NO = kFuseW / 2, NG = kFuseThreads / NO;
        static_assert(kFuseThreads % NO == 0, "whole row groups");
        const int odd = nx / 2, tlo = 3, thi = 2 * odd - 5;
        const int k = threadIdx.x % NO, g = threadIdx.x / NO;
        const int t = x0 + 1 + 2 * k;
        const long long px0 = F.x.p_base + ((long long)a * F.x.B + y0) * F.x.C + ((t - 1) >> 1);
        for (int yy = y0 + g; yy < y1 && t < x1; yy += NG) {
            const T *row = tile + (yy - yl) * P - xl;  // row[x]
            T pred;
            if (t >= tlo && t <= thi) {
                pred = cubic_pred<T>(row[t - 3], row[t - 1], row[t + 1], row[t + 3]);
            } else {
                const Rule r = line_rule(true, t, nx);
                const T o0 = row[r.o0];
                const T o1 = r.f != F_EQUAL ? row[r.o1] : o0;
                const T o2 = r.f >= F_QUAD1 ? row[r.o2] : o0;
                const T o3 = r.f == F_CUBIC ? row[r.o3] : o0;
                pred = apply_formula<T>(r.f, o0, o1, o2, o3);
            }
            const long long p = px0 + (long long)(yy - y0) * F.x.C;
            T *xp = tile + (yy - yl) * P + (t - xl);
            if (!DECOMP) {
                T recon;
                const T v = *xp;
                const int q = quantize<T>(v, pred, qp, recon);
                codes[p] = (int16_t)q;
                if (q == -qp.radius) {
                    esc[p] = v;
                    count_escape(etile, p);
                } else if (!F.x.skip) {
                    *xp = recon;
                }
            } else {
                const int q = codes[p];
                *xp = (q != -qp.radius) ? dequantize<T>(q, pred, qp) : esc[p];
            }
        }
    }
    __syncthreads();
    // write the tile back: every row, or (compress with a final x pass, no z targets in this plane)
    // the y pass's target rows
    {
        const bool odd_rows = !DECOMP && F.x.skip && !zplane;
        constexpr int NG = kFuseThreads / kFuseW;
        static_assert(kFuseThreads % kFuseW == 0, "whole row groups");
        const int cc = threadIdx.x % kFuseW, g = threadIdx.x / kFuseW;
        const int ys = odd_rows ? 2 : 1;
        if (x0 + cc < x1)
            for (int yy = y0 + (odd_rows ? 1 : 0) + ys * g; yy < y1; yy += ys * NG)
                plane[yy * sy + (x0 + cc) * sx] = tile[(yy - yl) * P + (x0 - xl) + cc];
    }
}

// The levels whose grid step is one element (the finest level, 7/8 of the codes) or two (the next,
// 7/64) of a float field whose rows are 16-byte aligned: the passes, tiles and code positions of
// k_yx_fused, with the tile's even and odd grid columns kept apart in shared memory so that a
// thread takes four consecutive targets of a row at a time (16-byte shared-memory loads and
// stores, one 8-byte code store).  Grid coordinates below; a grid column is STEP elements:
//   tile column c <-> x = x0 - 4 + c; row r <-> y = y0 - 4 + r (72 x 72: 64 + a halo of 4)
//   E[r * 40 + e]      even column c = 2e        (e in [0, 36))
//   O[r * 40 + m + 2]  odd column c = 2m + 1     (own odd columns: m in [2, 34))
// Every pass covers whole groups of four, the halo included, so that the lanes of a warp run the
// same code: the z pass (odd planes) the even rows y0 - 2 .. y0 + 66 x the 36 even columns
// x0 - 4 .. x0 + 66, the y pass the odd rows of the tile x the same columns, the x pass the rows
// of the tile x its 32 odd columns.  Targets outside the tile (the halo; their codes belong to the
// neighbouring tiles, but the y and x passes read their values) are recomputed and not stored,
// and targets outside the field are computed from don't-care values and not stored either.
// A plane's z rule is the same for the whole CTA; the y and x rules leave the interior cubic one
// only in the tiles at the field's edges.
constexpr int kL1Rows = 72, kL1S = 40, kL1Groups = 9;
constexpr int kL1Threads = 256;

__device__ __forceinline__ float *l1_e(float *E, int r, int e) { return E + r * kL1S + e; }
__device__ __forceinline__ float *l1_o(float *O, int r, int m) { return O + r * kL1S + m + 2; }
// the value at tile column c of row r
__device__ __forceinline__ float l1_at(float *E, float *O, int r, int c) {
    return (c & 1) ? *l1_o(O, r, (c - 1) >> 1) : *l1_e(E, r, c >> 1);
}

// Quantizes (compress) or reconstructs (decompress) four targets at consecutive code positions
// p .. p + 3, of values v and predictions pred.  `valid` (bit k: target k lies in the field) and
// `own` (bit k: its code belongs to this tile) select the code and escape slots read
// (decompress) and written (compress); compress leaves the reconstructions in v when `keep` (the
// reference overwrites in every pass but the last of level 1).
template <bool DECOMP>
__device__ __forceinline__ void l1_quad(float (&v)[4], const float (&pred)[4], int16_t *__restrict__ codes,
                                        float *__restrict__ esc, long long p, unsigned valid, unsigned own, bool keep,
                                        const QParams &qp, unsigned *__restrict__ etile) {
    int16_t *cp = codes + p;
    const bool vec = (reinterpret_cast<uintptr_t>(cp) & 7u) == 0;
    int q[4];
    if (!DECOMP) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            float recon;
            q[k] = quantize<float>(v[k], pred[k], qp, recon);
            if (q[k] == -qp.radius && ((own >> k) & 1u)) {
                esc[p + k] = v[k];
                count_escape(etile, p + k);
            }
            if (keep) v[k] = recon;  // the value itself when it escaped
        }
        if (own == 0xFu && vec) {
            *reinterpret_cast<uint2 *>(cp) = make_uint2((uint32_t)(q[0] & 0xFFFF) | ((uint32_t)q[1] << 16),
                                                        (uint32_t)(q[2] & 0xFFFF) | ((uint32_t)q[3] << 16));
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++)
                if ((own >> k) & 1u) cp[k] = (int16_t)q[k];
        }
    } else {
        if (valid == 0xFu && vec) {
            const uint2 w = *reinterpret_cast<const uint2 *>(cp);
            q[0] = (int16_t)(w.x & 0xFFFF);
            q[1] = (int16_t)(w.x >> 16);
            q[2] = (int16_t)(w.y & 0xFFFF);
            q[3] = (int16_t)(w.y >> 16);
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) q[k] = ((valid >> k) & 1u) ? (int)cp[k] : 0;
        }
#pragma unroll
        for (int k = 0; k < 4; k++)
            v[k] = (q[k] != -qp.radius) ? dequantize<float>(q[k], pred[k], qp) : ((valid >> k) & 1u) ? esc[p + k] : 0.f;
    }
}

// bit k set when a + 2 k lies in [lo, hi)
__device__ __forceinline__ unsigned l1_mask(int a, int lo, int hi) {
    if (a >= lo && a + 6 < hi) return 0xFu;
    unsigned m = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) m |= (a + 2 * k >= lo && a + 2 * k < hi) ? (1u << k) : 0u;
    return m;
}

template <bool DECOMP, int STEP>
__global__ void __launch_bounds__(kL1Threads, 6) k_l1_fused(const FusedYX F, float *__restrict__ xf,
                                                            int16_t *__restrict__ codes, float *__restrict__ esc,
                                                            const QParams qp, unsigned *__restrict__ etile) {
    __shared__ __align__(16) float E[kL1Rows * kL1S];
    __shared__ __align__(16) float O[kL1Rows * kL1S];
    const int ny = F.y.n, nx = F.x.n;
    const int a = (int)blockIdx.z;
    const int x0 = (int)blockIdx.x * kFuseW, x1 = min(nx, x0 + kFuseW);
    const int y0 = (int)blockIdx.y * kFuseR, y1 = min(ny, y0 + kFuseR);
    const int xo = x0 - 4, yo = y0 - 4;
    const long long sy = F.x.sb, sz = F.x.sa;
    float *plane = xf + (long long)a * sz;
    const int tid = threadIdx.x;
    // ---- stage rows [yo, yo + 72) x grid columns [xo, xo + 72), 16 bytes at a time: four grid
    // columns per vector at a grid step of one element, two (at element offsets 0 and 2) at two
    constexpr int VPR = 72 / (4 / STEP);  // vectors per row
    constexpr int NV = kL1Rows * VPR;
    constexpr int ITER = 3;               // loads in flight per thread before their stores
    for (int base = 0; base < NV; base += ITER * kL1Threads) {
        float4 v[ITER];
#pragma unroll
        for (int k = 0; k < ITER; k++) {
            const int idx = base + tid + k * kL1Threads;
            const int r = idx / VPR, i = idx - r * VPR;
            const int y = yo + r, x = xo + (4 / STEP) * i;  // the vector's first grid column
            v[k] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (idx < NV && y >= 0 && y < ny) {
                const float *src = plane + (long long)y * sy + (long long)x * STEP;
                if (STEP == 1 ? (x >= 0 && x + 3 < nx) : (x >= 0 && x + 2 < nx)) {
                    v[k] = __ldg(reinterpret_cast<const float4 *>(src));
                } else if (STEP == 1) {
                    if (x >= 0 && x < nx) v[k].x = src[0];
                    if (x + 1 >= 0 && x + 1 < nx) v[k].y = src[1];
                    if (x + 2 >= 0 && x + 2 < nx) v[k].z = src[2];
                    if (x + 3 >= 0 && x + 3 < nx) v[k].w = src[3];
                } else {
                    if (x >= 0 && x < nx) v[k].x = src[0];
                    if (x + 1 >= 0 && x + 1 < nx) v[k].z = src[2];
                }
            }
        }
#pragma unroll
        for (int k = 0; k < ITER; k++) {
            const int idx = base + tid + k * kL1Threads;
            if (idx >= NV) break;
            const int r = idx / VPR, i = idx - r * VPR;
            if (STEP == 1) {
                *reinterpret_cast<float2 *>(l1_e(E, r, 2 * i)) = make_float2(v[k].x, v[k].z);
                *reinterpret_cast<float2 *>(l1_o(O, r, 2 * i)) = make_float2(v[k].y, v[k].w);
            } else {
                *l1_e(E, r, i) = v[k].x;
                *l1_o(O, r, i) = v[k].z;
            }
        }
    }
    __syncthreads();
    // ---- z pass of an odd plane t = a: even rows x even columns, operands in the even planes
    // around it (points of coarser levels, which this level never writes)
    const bool zplane = F.has_z && (a & 1);
    if (zplane) {
        const int nz = F.z.n, t = a;
        const bool zl = F.has_zlate && t == nz - 1;
        const long long zb = zl ? F.zlate.p_base : F.z.p_base + ((long long)((t - 1) >> 1) + F.z.b_off) * F.z.C;
        const long long zr = zl ? F.zlate.C : F.z.rows_in_group * F.z.C;
        const bool inner = t >= 3 && t <= nz - 5;
        const Rule rz = row_rule(true, t, nz, F.z.skip);
        const float *q0 = xf + (long long)rz.o0 * sz;
        const float *q1 = xf + (long long)(rz.f != F_EQUAL ? rz.o1 : rz.o0) * sz;
        const float *q2 = xf + (long long)(rz.f >= F_QUAD1 ? rz.o2 : rz.o0) * sz;
        const float *q3 = xf + (long long)(rz.f == F_CUBIC ? rz.o3 : rz.o0) * sz;
        for (int i = tid; i < 35 * kL1Groups; i += kL1Threads) {
            const int rr = i / kL1Groups, g = i - kL1Groups * rr;
            const int r = 2 + 2 * rr, y = yo + r;
            if (y < 0 || y >= ny) continue;
            const int xg = xo + 8 * g;  // targets xg, xg + 2, xg + 4, xg + 6
            const unsigned valid = l1_mask(xg, 0, nx);
            const unsigned own = (y >= y0 && y < y1) ? l1_mask(xg, x0, x1) : 0u;
            float *slot = l1_e(E, r, 4 * g);
            const float4 cur = *reinterpret_cast<const float4 *>(slot);
            float v[4] = {cur.x, cur.y, cur.z, cur.w}, pred[4];
            const long long off = (long long)y * sy + (long long)xg * STEP;
            if (xg >= 0 && xg + 7 < nx) {
                float o[4][4];
                const float *qs[4] = {q0, q1, q2, q3};
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    if (STEP == 1) {
                        const float4 *src = reinterpret_cast<const float4 *>(qs[j] + off);
                        const float4 lo = __ldg(src), hi = __ldg(src + 1);
                        o[j][0] = lo.x;
                        o[j][1] = lo.z;
                        o[j][2] = hi.x;
                        o[j][3] = hi.z;
                    } else {
#pragma unroll
                        for (int k = 0; k < 4; k++) o[j][k] = __ldg(qs[j] + off + 4 * k);
                    }
                }
#pragma unroll
                for (int k = 0; k < 4; k++)
                    pred[k] = inner ? cubic_pred<float>(o[0][k], o[1][k], o[2][k], o[3][k])
                                    : apply_formula<float>(rz.f, o[0][k], o[1][k], o[2][k], o[3][k]);
            } else {
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    pred[k] = 0.f;
                    if (!((valid >> k) & 1u)) continue;
                    const long long ok = off + 2 * k * STEP;
                    pred[k] = apply_formula<float>(rz.f, __ldg(q0 + ok), __ldg(q1 + ok), __ldg(q2 + ok), __ldg(q3 + ok));
                }
            }
            l1_quad<DECOMP>(v, pred, codes, esc, zb + (long long)(y >> 1) * zr + (xg >> 1), valid, own, !F.z.skip, qp, etile);
            *reinterpret_cast<float4 *>(slot) = make_float4(v[0], v[1], v[2], v[3]);
        }
        __syncthreads();
    }
    // ---- y pass: odd rows of [y0, y1) x even columns (halo included)
    {
        const int nyr = (y1 - y0) >> 1;  // odd rows y0 + 1, y0 + 3, ... below y1
        const long long ya = (long long)a * F.y.rows_in_group + F.y.b_off;
        for (int i = tid; i < nyr * kL1Groups; i += kL1Threads) {
            const int k2 = i / kL1Groups, g = i - kL1Groups * k2;
            const int t = y0 + 1 + 2 * k2, r = t - yo;
            const int xg = xo + 8 * g;
            const unsigned valid = l1_mask(xg, 0, nx);
            const unsigned own = l1_mask(xg, x0, x1);
            const bool late = F.has_late && t == ny - 1;
            const long long p =
                (late ? F.late.p_base + (long long)a * F.late.C : F.y.p_base + (ya + ((t - 1) >> 1)) * F.y.C) + (xg >> 1);
            float *slot = l1_e(E, r, 4 * g);
            const float4 cur = *reinterpret_cast<const float4 *>(slot);
            float v[4] = {cur.x, cur.y, cur.z, cur.w}, pred[4];
            if (t >= 3 && t <= ny - 5) {
                const float4 u0 = *reinterpret_cast<const float4 *>(l1_e(E, r - 3, 4 * g));
                const float4 u1 = *reinterpret_cast<const float4 *>(l1_e(E, r - 1, 4 * g));
                const float4 u2 = *reinterpret_cast<const float4 *>(l1_e(E, r + 1, 4 * g));
                const float4 u3 = *reinterpret_cast<const float4 *>(l1_e(E, r + 3, 4 * g));
                pred[0] = cubic_pred<float>(u0.x, u1.x, u2.x, u3.x);
                pred[1] = cubic_pred<float>(u0.y, u1.y, u2.y, u3.y);
                pred[2] = cubic_pred<float>(u0.z, u1.z, u2.z, u3.z);
                pred[3] = cubic_pred<float>(u0.w, u1.w, u2.w, u3.w);
            } else {
                const Rule ry = row_rule(true, t, ny, F.y.skip);
                const int r0 = ry.o0 - yo, r1 = (ry.f != F_EQUAL ? ry.o1 : ry.o0) - yo;
                const int r2 = (ry.f >= F_QUAD1 ? ry.o2 : ry.o0) - yo, r3 = (ry.f == F_CUBIC ? ry.o3 : ry.o0) - yo;
#pragma unroll
                for (int k = 0; k < 4; k++)
                    pred[k] = apply_formula<float>(ry.f, *l1_e(E, r0, 4 * g + k), *l1_e(E, r1, 4 * g + k),
                                                   *l1_e(E, r2, 4 * g + k), *l1_e(E, r3, 4 * g + k));
            }
            l1_quad<DECOMP>(v, pred, codes, esc, p, valid, own, !F.y.skip, qp, etile);
            *reinterpret_cast<float4 *>(slot) = make_float4(v[0], v[1], v[2], v[3]);
        }
    }
    __syncthreads();
    // ---- x pass: rows [y0, y1) x odd columns of [x0, x1), eight groups of four per row
    {
        const int nrows = y1 - y0;
        const int thi = 2 * (nx / 2) - 5;  // odd columns up to here take the interior cubic rule
        const long long xb = F.x.p_base + (long long)a * F.x.B * F.x.C + (x0 >> 1);
        for (int i = tid; i < nrows * 8; i += kL1Threads) {
            const int yy = i >> 3, g = i & 7;
            const int r = yy + 4;
            const int ta = x0 + 1 + 8 * g;  // targets ta, ta + 2, ta + 4, ta + 6
            const unsigned valid = l1_mask(ta, 0, x1);
            if (!valid) continue;
            float *slot = l1_o(O, r, 4 * g + 2);
            const float4 cur = *reinterpret_cast<const float4 *>(slot);
            float v[4] = {cur.x, cur.y, cur.z, cur.w}, pred[4];
            if (ta >= 3 && ta + 6 <= thi) {
                const float4 A = *reinterpret_cast<const float4 *>(l1_e(E, r, 4 * g));
                const float4 B = *reinterpret_cast<const float4 *>(l1_e(E, r, 4 * g + 4));
                pred[0] = cubic_pred<float>(A.y, A.z, A.w, B.x);
                pred[1] = cubic_pred<float>(A.z, A.w, B.x, B.y);
                pred[2] = cubic_pred<float>(A.w, B.x, B.y, B.z);
                pred[3] = cubic_pred<float>(B.x, B.y, B.z, B.w);
            } else {
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const int t = ta + 2 * k;
                    pred[k] = 0.f;
                    if (!((valid >> k) & 1u)) continue;
                    if (t >= 3 && t <= thi) {
                        pred[k] = cubic_pred<float>(l1_at(E, O, r, t - 3 - xo), l1_at(E, O, r, t - 1 - xo),
                                                    l1_at(E, O, r, t + 1 - xo), l1_at(E, O, r, t + 3 - xo));
                    } else {
                        const Rule rx = line_rule(true, t, nx);
                        const float o0 = l1_at(E, O, r, rx.o0 - xo);
                        const float o1 = rx.f != F_EQUAL ? l1_at(E, O, r, rx.o1 - xo) : o0;
                        const float o2 = rx.f >= F_QUAD1 ? l1_at(E, O, r, rx.o2 - xo) : o0;
                        const float o3 = rx.f == F_CUBIC ? l1_at(E, O, r, rx.o3 - xo) : o0;
                        pred[k] = apply_formula<float>(rx.f, o0, o1, o2, o3);
                    }
                }
            }
            l1_quad<DECOMP>(v, pred, codes, esc, xb + (long long)(y0 + yy) * F.x.C + 4 * g, valid, valid, !F.x.skip, qp, etile);
            if (DECOMP || !F.x.skip) *reinterpret_cast<float4 *>(slot) = make_float4(v[0], v[1], v[2], v[3]);
        }
    }
    __syncthreads();
    // ---- write the tile back: every row, or (compress with a final x pass, no z targets in this
    // plane) the y pass's target rows; columns [x0, x1), re-interleaved 16 bytes at a time
    {
        const bool odd_rows = !DECOMP && F.x.skip && !zplane;
        const int nrows = y1 - y0;
        for (int task = tid; task < nrows * 16; task += kL1Threads) {
            const int yy = task >> 4, i = task & 15;
            const int y = y0 + yy;
            if (odd_rows && !(y & 1)) continue;
            const int r = yy + 4, x = x0 + 4 * i;
            if (x >= x1) continue;
            const float2 e = *reinterpret_cast<const float2 *>(l1_e(E, r, 2 + 2 * i));
            const float2 o = *reinterpret_cast<const float2 *>(l1_o(O, r, 2 + 2 * i));
            float *dst = plane + (long long)y * sy + (long long)x * STEP;
            if (STEP == 1 && x + 3 < x1) {
                *reinterpret_cast<float4 *>(dst) = make_float4(e.x, o.x, e.y, o.y);
            } else {  // at a step of two the finer level's points lie between: one value at a time
                dst[0] = e.x;
                if (x + 1 < x1) dst[STEP] = o.x;
                if (x + 2 < x1) dst[2 * STEP] = e.y;
                if (x + 3 < x1) dst[3 * STEP] = o.y;
            }
        }
    }
}

// Whether passes i (and i + 1, i + 2) form a fusable y + x pair; fills F.
bool fusable_yx(const std::vector<PassLaunch> &ps, size_t i, size_t elem, FusedYX &F, size_t &used) {
    if (i + 1 >= ps.size()) return false;
    const PassLaunch &y = ps[i];
    if (y.kind != KIND_ROW || !y.cubic || y.skip || y.t0 != 1 || y.b_off != 0 || y.B != y.rows_in_group) return false;
    size_t j = i + 1;
    F.has_late = 0;
    if (ps[j].kind == KIND_ROW) {
        const PassLaunch &e = ps[j];
        if (e.t0 != y.n - 1 || e.B != 1 || e.rows_in_group != 1 || e.b_off != 0 || e.A != y.A || e.C != y.C ||
            e.sa != y.sa || e.sc != y.sc || e.step != y.step || e.level != y.level || e.n != y.n || e.skip != y.skip ||
            e.p_base != y.p_base + y.A * y.B * y.C)
            return false;
        F.late = e;
        F.has_late = 1;
        j++;
        if (j >= ps.size()) return false;
    }
    if (y.B != y.n / 2 - (F.has_late ? 1 : 0)) return false;  // the passes cover every odd row
    const PassLaunch &x = ps[j];
    if (x.kind != KIND_LINE || !x.cubic || x.level != y.level || x.step < 1 || x.A != y.A || x.sa != y.sa ||
        x.sb != y.step || x.B != y.n || x.C != x.n / 2 || y.sc != 2 * x.step || y.C != (x.n - 1) / 2 + 1 ||
        y.A > 65535 ||
        x.n < 2 || y.n < 2)
        return false;
    (void)elem;
    if (y.A > 65535 || (y.n + kFuseR - 1) / kFuseR > 65535) return false;
    F.y = y;
    F.x = x;
    used = j - i + 1;
    return true;
}

template <class T, bool DECOMP>
void launch_fused_yx(const FusedYX &F, T *x, int16_t *codes, T *esc, const QParams &qp, unsigned *etile,
                     cudaStream_t st) {
    dim3 grid((unsigned)((F.x.n + kFuseW - 1) / kFuseW), (unsigned)((F.y.n + kFuseR - 1) / kFuseR), (unsigned)F.y.A);
    if constexpr (std::is_same<T, float>::value) {
        // a grid step of one or two elements with 16-byte aligned rows and planes: the
        // split-column kernel
        const bool rows16 = F.x.sb % 4 == 0 && (F.y.A == 1 || F.x.sa % 4 == 0);
        if ((F.x.step == 1 || F.x.step == 2) && rows16 && (reinterpret_cast<uintptr_t>(x) & 15) == 0) {
            if (F.x.step == 1) k_l1_fused<DECOMP, 1><<<grid, kL1Threads, 0, st>>>(F, x, codes, esc, qp, etile);
            else k_l1_fused<DECOMP, 2><<<grid, kL1Threads, 0, st>>>(F, x, codes, esc, qp, etile);
            FB2_CHECK_LAUNCH();
            return;
        }
    }
    k_yx_fused<T, DECOMP><<<grid, kFuseThreads, 0, st>>>(F, x, codes, esc, qp, etile);
    FB2_CHECK_LAUNCH();
}

// Whether passes i (and i + 1) are the z pass that precedes the fusable y + x passes starting
// right after it; fills F (z, zlate, y, late, x) and `used` (all of them).
bool fusable_zyx(const std::vector<PassLaunch> &ps, size_t i, size_t elem, FusedYX &F, size_t &used) {
    if (i >= ps.size()) return false;
    const PassLaunch &z = ps[i];
    if (z.kind != KIND_ROW || !z.cubic || z.skip || z.t0 != 1 || z.b_off != 0 || z.B != z.rows_in_group) return false;
    size_t j = i + 1, u = 0;
    PassLaunch zl{};
    int has_zl = 0;
    if (j < ps.size() && ps[j].kind == KIND_ROW && ps[j].t0 == z.n - 1 && ps[j].B == 1 && ps[j].rows_in_group == 1 &&
        ps[j].p_base == z.p_base + z.A * z.B * z.C) {
        zl = ps[j];
        if (zl.b_off != 0 || zl.A != z.A || zl.C != z.C || zl.sa != z.sa || zl.sc != z.sc || zl.step != z.step ||
            zl.level != z.level || zl.n != z.n || zl.skip != z.skip)
            return false;
        has_zl = 1;
        j++;
    }
    if (z.B != z.n / 2 - has_zl) return false;
    if (!fusable_yx(ps, j, elem, F, u)) return false;
    if (z.level != F.y.level || z.n != F.y.A || z.step != F.y.sa || z.A != (F.y.n - 1) / 2 + 1 ||
        z.sa != 2 * F.y.step || z.C != (F.x.n - 1) / 2 + 1 || z.sc != 2 * F.x.step || z.n < 2)
        return false;
    F.z = z;
    F.zlate = zl;
    F.has_z = 1;
    F.has_zlate = has_zl;
    used = j - i + u;
    return true;
}

// Whether quantizing a reconstruction again gives it back, for every field value of magnitude up
// to max_abs at error bound eb.  The fused kernels need this when they compress: a CTA recomputes
// the targets in its halo from the values it stages, and the CTA owning those targets may already
// have written their reconstructions back, so the value staged there is the original or the
// reconstruction r = fl(q 2eb + pred).  Re-quantizing r gives q again when
// |fl(r - pred) / 2eb - q| < 1/2.  With u the unit roundoff of T (2^-24 float, 2^-53 double),
// |q| < 2^15 and |pred| <= 7 (max_abs + eb) (the largest weight sum of the interpolation
// formulas), that error is at most u (2 |q| + |pred| / 2eb) + (double-rounding terms)
// <= u 2^16 + 3.5 u (max_abs / eb + 1), below 1/4 when eb >= 2^-20 max_abs (float) or
// 2^-49 max_abs (double).  Below that bound (error bounds near the type's precision) the plan
// runs its passes one kernel each, which recompute nothing.
template <class T>
bool requant_exact(double eb, double max_abs) {
    const double tol = sizeof(T) == 4 ? 0x1p-20 : 0x1p-49;
    return max_abs >= 0 && std::isfinite(max_abs) && eb >= tol * max_abs;
}

// Runs the plan's passes in order, the fusable z + y + x and y + x passes as one kernel.
template <class T, bool DECOMP>
void run_passes(const InterpPlan &plan, T *x, int16_t *codes, T *esc, unsigned *etile, cudaStream_t st,
                LaunchTimes *lt = nullptr) {
    const std::vector<PassLaunch> &ps = plan.passes;
    for (size_t i = 0; i < ps.size();) {
        FusedYX F{};
        size_t used = 0;
        if ((fusable_zyx(ps, i, sizeof(T), F, used) || fusable_yx(ps, i, sizeof(T), F, used)) &&
            (DECOMP || requant_exact<T>(plan.levels[F.y.level].eb, plan.max_abs))) {
            if (lt) lt->begin(F.y.level, st);
            launch_fused_yx<T, DECOMP>(F, x, codes, esc, plan.levels[F.y.level], etile, st);
            if (lt) lt->end(st);
            i += used;
        } else {
            if (lt) lt->begin(ps[i].level, st);
            launch_pass<T, DECOMP>(ps[i], x, codes, esc, plan.levels[ps[i].level], etile, st);
            if (lt) lt->end(st);
            i++;
        }
    }
}

struct WsLayout {
    size_t esc_off, tiles_off, scan_off, total_off, bytes;
    long long ntiles;
};

WsLayout ws_layout(const InterpPlan &plan, int elem) {
    WsLayout w;
    auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
    w.ntiles = (plan.n_codes + kTile - 1) / kTile;
    w.esc_off = 0;
    w.tiles_off = al(w.esc_off + (size_t)std::max<long long>(plan.n_codes, 1) * elem);
    w.scan_off = al(w.tiles_off + (size_t)(w.ntiles + 1) * 4);
    w.total_off = al(w.scan_off + (size_t)(w.ntiles + 1) * 8);
    w.bytes = al(w.total_off + 8);
    return w;
}

AnchorGrid anchor_grid(const InterpPlan &plan) {
    AnchorGrid G;
    G.N = plan.N;
    G.total = plan.n_anchor;
    for (int d = 0; d < 4; d++) {
        G.cnt[d] = d < plan.N ? count_of(plan.dims[d], plan.anchor) : 1;
        G.est[d] = d < plan.N ? plan.anchor * plan.off[d] : 0;
    }
    return G;
}

}  // namespace

size_t interp_workspace_bytes(const InterpPlan &plan, int elem_size) { return ws_layout(plan, elem_size).bytes; }

void interp_decompress_check(const InterpPlan &plan, int elem_size, const void *d_ws, long long n_unpred,
                             cudaStream_t st) {
    const WsLayout w = ws_layout(plan, elem_size);
    unsigned long long total = 0;
    if (w.ntiles > 0)
        total = d2h(reinterpret_cast<const unsigned long long *>(static_cast<const char *>(d_ws) + w.total_off), 1, st)[0];
    if ((long long)total > n_unpred - plan.n_anchor)
        throw std::invalid_argument("the codes name " + std::to_string(total) + " unpredictable values but the list holds " +
                                    std::to_string(n_unpred - plan.n_anchor) + " after the anchors");
}

template <class T>
void interp_compress_passes(const InterpPlan &plan, T *d_x, int16_t *d_codes, void *d_ws, unsigned long long *d_n_esc,
                            cudaStream_t st, LaunchTimes *lt) {
    const WsLayout w = ws_layout(plan, sizeof(T));
    char *ws = static_cast<char *>(d_ws);
    T *esc = reinterpret_cast<T *>(ws + w.esc_off);
    unsigned *tiles = reinterpret_cast<unsigned *>(ws + w.tiles_off);
    unsigned long long *scan = reinterpret_cast<unsigned long long *>(ws + w.scan_off);
    // the passes count their escapes per tile of kTile codes as they code them
    if (w.ntiles > 0) FB2_CUDA(cudaMemsetAsync(tiles, 0, (size_t)w.ntiles * sizeof(unsigned), st));
    unsigned *etile = w.ntiles > 0 ? tiles : nullptr;
    if (plan.first_point) {
        k_first_point<T, false><<<1, 1, 0, st>>>(d_x, d_codes, esc, plan.levels[0], etile);
        FB2_CHECK_LAUNCH();
    }
    run_passes<T, false>(plan, d_x, d_codes, esc, etile, st, lt);
    if (w.ntiles > 0) {
        k_scan_u32<<<1, 1024, 0, st>>>(tiles, scan, w.ntiles, d_n_esc);
        FB2_CHECK_LAUNCH();
    } else if (d_n_esc) {
        FB2_CUDA(cudaMemsetAsync(d_n_esc, 0, 8, st));
    }
}

template <class T>
void interp_compress_finish(const InterpPlan &plan, const T *d_x, const int16_t *d_codes, T *d_unpred, void *d_ws,
                            cudaStream_t st) {
    const WsLayout w = ws_layout(plan, sizeof(T));
    char *ws = static_cast<char *>(d_ws);
    T *esc = reinterpret_cast<T *>(ws + w.esc_off);
    unsigned long long *scan = reinterpret_cast<unsigned long long *>(ws + w.scan_off);
    if (plan.n_anchor > 0) {
        // the anchors are never targets, so the field still holds them after the passes
        const AnchorGrid G = anchor_grid(plan);
        const int blocks = (int)std::min<long long>((G.total + 255) / 256, 4096);
        k_anchors<T, false><<<blocks, 256, 0, st>>>(G, const_cast<T *>(d_x), d_unpred);
        FB2_CHECK_LAUNCH();
    }
    if (w.ntiles > 0) {
        k_esc_scatter<T, false><<<(unsigned)w.ntiles, kTileThreads, 0, st>>>(
            d_codes, plan.n_codes, -plan.levels[0].radius, scan, esc, d_unpred, plan.n_anchor, ~0ull);
        FB2_CHECK_LAUNCH();
    }
}

template <class T>
void interp_compress(const InterpPlan &plan, T *d_x, int16_t *d_codes, T *d_unpred, void *d_ws,
                     unsigned long long *d_n_esc, cudaStream_t st, LaunchTimes *lt) {
    interp_compress_passes<T>(plan, d_x, d_codes, d_ws, d_n_esc, st, lt);
    interp_compress_finish<T>(plan, d_x, d_codes, d_unpred, d_ws, st);
}

template <class T>
void interp_decompress(const InterpPlan &plan, const int16_t *d_codes, const T *d_unpred, long long n_unpred, T *d_x,
                       void *d_ws, cudaStream_t st) {
    if (n_unpred < plan.n_anchor) throw std::invalid_argument("unpredictable list too short");
    const WsLayout w = ws_layout(plan, sizeof(T));
    char *ws = static_cast<char *>(d_ws);
    T *esc = reinterpret_cast<T *>(ws + w.esc_off);
    unsigned *tiles = reinterpret_cast<unsigned *>(ws + w.tiles_off);
    unsigned long long *scan = reinterpret_cast<unsigned long long *>(ws + w.scan_off);
    unsigned long long *total = reinterpret_cast<unsigned long long *>(ws + w.total_off);
    int16_t *codes = const_cast<int16_t *>(d_codes);
    T *unpred = const_cast<T *>(d_unpred);
    if (plan.n_anchor > 0) {
        const AnchorGrid G = anchor_grid(plan);
        const int blocks = (int)std::min<long long>((G.total + 255) / 256, 4096);
        k_anchors<T, true><<<blocks, 256, 0, st>>>(G, d_x, unpred);
        FB2_CHECK_LAUNCH();
    }
    const int escc = -plan.levels[0].radius;
    if (w.ntiles > 0) {
        k_esc_count<<<(unsigned)w.ntiles, kTileThreads, 0, st>>>(codes, plan.n_codes, escc, tiles);
        FB2_CHECK_LAUNCH();
        k_scan_u32<<<1, 1024, 0, st>>>(tiles, scan, w.ntiles, total);
        FB2_CHECK_LAUNCH();
        k_esc_scatter<T, true><<<(unsigned)w.ntiles, kTileThreads, 0, st>>>(
            codes, plan.n_codes, escc, scan, esc, unpred, plan.n_anchor,
            (unsigned long long)(n_unpred - plan.n_anchor));
        FB2_CHECK_LAUNCH();
    }
    if (plan.first_point) {
        k_first_point<T, true><<<1, 1, 0, st>>>(d_x, codes, esc, plan.levels[0], nullptr);
        FB2_CHECK_LAUNCH();
    }
    run_passes<T, true>(plan, d_x, codes, esc, nullptr, st);
}

// ------------------------------------------------------------------------------------------ range
namespace {
constexpr int kRangeBlocks = 1184;  // 8 x 148 SMs

template <class T>
__global__ void __launch_bounds__(256) k_minmax(const T *__restrict__ x, long long n, T *__restrict__ part) {
    T lo = x[0], hi = x[0];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const T v = __ldg(x + i);
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
    }
    __shared__ T slo[256], shi[256];
    slo[threadIdx.x] = lo;
    shi[threadIdx.x] = hi;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            slo[threadIdx.x] = slo[threadIdx.x + s] < slo[threadIdx.x] ? slo[threadIdx.x + s] : slo[threadIdx.x];
            shi[threadIdx.x] = shi[threadIdx.x + s] > shi[threadIdx.x] ? shi[threadIdx.x + s] : shi[threadIdx.x];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = slo[0];
        part[2 * blockIdx.x + 1] = shi[0];
    }
}

template <class T>
__global__ void k_minmax_final(const T *__restrict__ part, int nb, T *out) {
    __shared__ T slo[256], shi[256];
    T lo = part[0], hi = part[1];
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        lo = part[2 * i] < lo ? part[2 * i] : lo;
        hi = part[2 * i + 1] > hi ? part[2 * i + 1] : hi;
    }
    slo[threadIdx.x] = lo;
    shi[threadIdx.x] = hi;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            slo[threadIdx.x] = slo[threadIdx.x + s] < slo[threadIdx.x] ? slo[threadIdx.x + s] : slo[threadIdx.x];
            shi[threadIdx.x] = shi[threadIdx.x + s] > shi[threadIdx.x] ? shi[threadIdx.x + s] : shi[threadIdx.x];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = Arith<T>::sub(shi[0], slo[0]);
        out[1] = slo[0];
        out[2] = shi[0];
    }
}
}  // namespace

size_t range_workspace_bytes() { return (size_t)kRangeBlocks * 2 * sizeof(double); }

template <class T>
void device_range(const T *d_x, long long n, T *d_out, void *d_ws, cudaStream_t st) {
    T *part = static_cast<T *>(d_ws);
    const int nb = (int)std::max<long long>(1, std::min<long long>(kRangeBlocks, (n + 255) / 256));
    k_minmax<T><<<nb, 256, 0, st>>>(d_x, n, part);
    FB2_CHECK_LAUNCH();
    k_minmax_final<T><<<1, 256, 0, st>>>(part, nb, d_out);
    FB2_CHECK_LAUNCH();
}

namespace {
template <class T>
cudaError_t preload_decompress_kernels() {
    const void *fns[] = {
        reinterpret_cast<const void *>(&k_anchors<T, true>),
        reinterpret_cast<const void *>(&k_esc_scatter<T, true>),
        reinterpret_cast<const void *>(&k_first_point<T, true>),
        reinterpret_cast<const void *>(&k_pass<T, KIND_ROW, true>),
        reinterpret_cast<const void *>(&k_pass<T, KIND_LINE, true>),
        reinterpret_cast<const void *>(&k_pass<T, KIND_GENERIC, true>),
        reinterpret_cast<const void *>(&k_pass<T, KIND_LEGACY, true>),
        reinterpret_cast<const void *>(&k_row_fast<T, true>),
        reinterpret_cast<const void *>(&k_line_smem<T, true>),
        reinterpret_cast<const void *>(&k_yx_fused<T, true>),
        reinterpret_cast<const void *>(&k_l1_fused<true, 1>),
        reinterpret_cast<const void *>(&k_l1_fused<true, 2>),
    };
    for (const void *f : fns) {
        cudaFuncAttributes a;
        const cudaError_t e = cudaFuncGetAttributes(&a, f);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}
}  // namespace

cudaError_t interp_decompress_preload() {
    for (const void *f : {reinterpret_cast<const void *>(&k_esc_count), reinterpret_cast<const void *>(&k_scan_u32)}) {
        cudaFuncAttributes a;
        const cudaError_t e = cudaFuncGetAttributes(&a, f);
        if (e != cudaSuccess) return e;
    }
    const cudaError_t e = preload_decompress_kernels<float>();
    return e != cudaSuccess ? e : preload_decompress_kernels<double>();
}

void LaunchTimes::begin(int level, cudaStream_t st) {
    Entry x{level, nullptr, nullptr, 0.f};
    FB2_CUDA(cudaEventCreate(&x.a));
    FB2_CUDA(cudaEventCreate(&x.b));
    e.push_back(x);
    FB2_CUDA(cudaEventRecord(x.a, st));
}
void LaunchTimes::end(cudaStream_t st) { FB2_CUDA(cudaEventRecord(e.back().b, st)); }
void LaunchTimes::read() {
    for (Entry &x : e) {
        FB2_CUDA(cudaEventSynchronize(x.b));
        FB2_CUDA(cudaEventElapsedTime(&x.ms, x.a, x.b));
    }
}
LaunchTimes::~LaunchTimes() {
    for (Entry &x : e) {
        if (x.a) cudaEventDestroy(x.a);
        if (x.b) cudaEventDestroy(x.b);
    }
}

long long level_codes(const InterpPlan &plan, int li) {
    const long long off = (long long)plan.levels.size() - (long long)plan.level_starts.size();
    const long long k = li - off;
    if (k < 0 || k >= (long long)plan.level_starts.size()) return 0;
    const long long end = k + 1 < (long long)plan.level_starts.size() ? plan.level_starts[k + 1] : plan.n_codes;
    return end - plan.level_starts[k];
}

template void interp_compress<float>(const InterpPlan &, float *, int16_t *, float *, void *, unsigned long long *,
                                     cudaStream_t, LaunchTimes *);
template void interp_compress_passes<float>(const InterpPlan &, float *, int16_t *, void *, unsigned long long *,
                                            cudaStream_t, LaunchTimes *);
template void interp_compress_passes<double>(const InterpPlan &, double *, int16_t *, void *, unsigned long long *,
                                             cudaStream_t, LaunchTimes *);
template void interp_compress_finish<float>(const InterpPlan &, const float *, const int16_t *, float *, void *,
                                            cudaStream_t);
template void interp_compress_finish<double>(const InterpPlan &, const double *, const int16_t *, double *, void *,
                                             cudaStream_t);
template void interp_compress<double>(const InterpPlan &, double *, int16_t *, double *, void *,
                                      unsigned long long *, cudaStream_t, LaunchTimes *);
template void interp_decompress<float>(const InterpPlan &, const int16_t *, const float *, long long, float *,
                                       void *, cudaStream_t);
template void interp_decompress<double>(const InterpPlan &, const int16_t *, const double *, long long, double *,
                                        void *, cudaStream_t);
template void device_range<float>(const float *, long long, float *, void *, cudaStream_t);
template void device_range<double>(const double *, long long, double *, void *, cudaStream_t);

}  // namespace fb2
