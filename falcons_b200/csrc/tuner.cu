// Device auto-tuner for ALGO_INTERP_LORENZO.
//
// Reference (JLiu-1/Falcons include/Falcons/...):
//   api/impl/FalconsAlgoInterp.hpp:273-544  sample sizing, candidate sets, ranking, final choice
//   api/impl/FalconsAlgoInterp.hpp:100-226  trial compression of the sampled blocks + zstd ratio
//   utils/Sample.hpp:6-159                  profiling_block: drop near-constant blocks
//   utils/Sample.hpp:234-345                sampleBlocks: strided block selection
// The profile pass and the trial decompositions run on the GPU; the zstd ranking of the trial
// codes (a few hundred KB) uses the runtime libzstd, as the reference does.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "assemble.cuh"
#include "interp.cuh"
#include "lorenzo_path.cuh"
#include "stream.hpp"
#include "tuner.cuh"

namespace fb2 {
namespace {

struct Geo {
    int N;
    long long dims[4], off[4];
};

// One thread per candidate block (reference loop order: first dim outermost).
template <class T>
__global__ void k_profile(const T *__restrict__ x, const Geo g, long long bs, long long stride, double eb,
                          const long long *__restrict__ cnt, long long total, uint8_t *__restrict__ keep) {
    const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= total) return;
    long long rem = b, start = 0;
    for (int d = g.N - 1; d >= 0; d--) {
        start += (rem % cnt[d]) * bs * g.off[d];
        rem /= cnt[d];
    }
    T mn = x[start], mx = x[start];
    const long long per = bs / stride + 1;
    long long tot = 1;
    for (int d = 0; d < g.N; d++) tot *= per;
    for (long long it = 0; it < tot; it++) {
        long long r = it, o = start;
        for (int d = g.N - 1; d >= 0; d--) {
            o += (r % per) * stride * g.off[d];
            r /= per;
        }
        const T v = x[o];
        if (v < mn) mn = v;
        else if (v > mx) mx = v;
    }
    keep[b] = (double)(mx - mn) > eb;
}

template <class T>
__global__ void k_cut_block(const T *__restrict__ x, const Geo g, const long long *__restrict__ starts, long long side,
                            long long V, T *__restrict__ out) {
    const long long blk = blockIdx.y;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < V; i += (long long)gridDim.x * blockDim.x) {
        long long rem = i, o = 0;
        for (int d = g.N - 1; d >= 0; d--) {
            o += (starts[blk * 4 + d] + rem % side) * g.off[d];
            rem /= side;
        }
        out[blk * V + i] = x[o];
    }
}

// interp_compress_test[_batch] ratio of one candidate over all sampled blocks.
template <class T>
double trial_ratio(Pool &pool, const T *d_blocks, long long B, long long side, int N, const InterpParams &prm,
                   cudaStream_t st) {
    long long dims[4];
    for (int d = 0; d < N; d++) dims[d] = side;
    const InterpPlan plan = make_plan(dims, N, prm);
    const long long V = plan.num;
    T *work = pool.get<T>((size_t)(B * V));
    FB2_CUDA(cudaMemcpyAsync(work, d_blocks, (size_t)(B * V) * sizeof(T), cudaMemcpyDeviceToDevice, st));
    // every block's codes start on a 32-byte boundary (the escape scan reads them as vectors)
    const long long cstride = (plan.n_codes + 15) & ~15LL;
    int16_t *codes = pool.get<int16_t>((size_t)(B * cstride) + 16);
    T *unpred = pool.get<T>((size_t)(B * V) + 16);
    void *ws = pool.get<uint8_t>(interp_workspace_bytes(plan, sizeof(T)));
    unsigned long long *nesc = pool.get<unsigned long long>((size_t)B);
    for (long long b = 0; b < B; b++)
        interp_compress<T>(plan, work + b * V, codes + b * cstride, unpred + b * V, ws, nesc + b, st);
    std::vector<unsigned long long> ne = d2h(nesc, (size_t)B, st);
    std::vector<int16_t> hs = d2h(codes, (size_t)(B * cstride), st);
    std::vector<int16_t> hc((size_t)(B * plan.n_codes));
    for (long long b = 0; b < B; b++)
        std::copy(hs.begin() + b * cstride, hs.begin() + b * cstride + plan.n_codes, hc.begin() + b * plan.n_codes);
    std::vector<T> hu = d2h(unpred, (size_t)(B * V), st);
    std::vector<uint8_t> buf;
    for (long long b = 0; b < B; b++) {
        const size_t nu = (size_t)(plan.n_anchor + (long long)ne[b]);
        const uint8_t *p = reinterpret_cast<const uint8_t *>(hu.data() + b * V);
        buf.insert(buf.end(), p, p + nu * sizeof(T));
    }
    const uint8_t *pc = reinterpret_cast<const uint8_t *>(hc.data());
    buf.insert(buf.end(), pc, pc + hc.size() * 2);
    std::vector<uint8_t> z(zstd_compress_bound(buf.size()) + 16);
    const size_t zs = zstd_compress(buf.data(), buf.size(), z.data(), z.size(), 3) + sizeof(size_t);
    return (double)((size_t)V * (size_t)B * sizeof(T)) * 1.0 / (double)zs;
}

}  // namespace

template <class T>
void tune_interp(Context &ctx, falcons_config &c, const T *d_x, cudaStream_t st, double max_abs) {
    (void)ctx;
    const int N = c.N;
    const double num = (double)c.num;
    const double sampleRate = 0.005;
    static const size_t sbs_default[4] = {4096, 128, 32, 16};
    size_t sbs = sbs_default[N - 1];
    size_t shortest = c.dims[0];
    for (int i = 0; i < N; i++) shortest = std::min<size_t>(shortest, c.dims[i]);
    while (sbs >= shortest) sbs /= 2;
    while (sbs >= 16 && (std::pow((double)(sbs + 1), N) / num) > 1.5 * sampleRate) sbs /= 2;
    if (sbs < 8) sbs = 8;
    bool to_tune = std::pow((double)(sbs + 1), N) <= 0.05 * num;
    for (int i = 0; i < N; i++)
        if (c.dims[i] < sbs) to_tune = false;
    if (!to_tune || !zstd_available()) {
        c.cmprAlgo = ALGO_INTERP;
        return;
    }
    Pool pool(st);
    Geo g;
    g.N = N;
    for (int d = 0; d < 4; d++) {
        g.dims[d] = d < N ? (long long)c.dims[d] : 1;
    }
    g.off[N - 1] = 1;
    for (int d = N - 2; d >= 0; d--) g.off[d] = g.off[d + 1] * g.dims[d + 1];
    const long long bs = (long long)sbs;
    // profiling_block (Sample.hpp:6-159): candidate starts at multiples of bs, strictly below dim - bs
    std::vector<long long> cnt(4, 1);
    long long total = 1;
    bool any = true;
    for (int d = 0; d < N; d++) {
        if (g.dims[d] < bs) any = false;
        cnt[d] = g.dims[d] > bs ? (g.dims[d] - bs + bs - 1) / bs : 0;
        total *= cnt[d];
    }
    std::vector<std::vector<long long>> starts;
    if (any && total > 0) {
        long long *d_cnt = h2d(pool, cnt, st);
        uint8_t *keep = pool.get<uint8_t>((size_t)total);
        const long long stride = std::max<long long>(1, bs / 4);
        k_profile<T><<<(unsigned)((total + 127) / 128), 128, 0, st>>>(d_x, g, bs, stride, c.absErrorBound, d_cnt,
                                                                      total, keep);
        FB2_CHECK_LAUNCH();
        std::vector<uint8_t> hk = d2h(keep, (size_t)total, st);
        for (long long b = 0; b < total; b++) {
            if (!hk[b]) continue;
            std::vector<long long> s(N);
            long long rem = b;
            for (int d = N - 1; d >= 0; d--) {
                s[d] = (rem % cnt[d]) * bs;
                rem /= cnt[d];
            }
            starts.push_back(s);
        }
    }
    const double per_block = std::pow((double)(sbs + 1), N);
    const bool profiling = (double)starts.size() * per_block >= 0.5 * sampleRate * num;
    // sampleBlocks (Sample.hpp:234-345)
    std::vector<std::vector<long long>> sel;
    {
        size_t totalblock_num = 1;
        for (int i = 0; i < N; i++) totalblock_num *= (size_t)(int)((c.dims[i] - 1) / sbs);
        bool ok = true;
        for (int i = 0; i < N; i++)
            if (c.dims[i] < sbs) ok = false;
        if (ok) {
            if (profiling) {
                const size_t nf = starts.size();
                size_t stride = (size_t)(nf / (totalblock_num * sampleRate));
                if (stride <= 0) stride = 1;
                const size_t n_sel = (nf + stride - 1) / stride;
                for (size_t si = 0; si < n_sel; si++) sel.push_back(starts[si * stride]);
            } else {
                size_t stride = (size_t)(1.0 / sampleRate);
                if (stride <= 0) stride = 1;
                size_t idx = 0;
                std::vector<long long> cur(N, 0);
                // nested loops over block starts < dim - sbs, first dim outermost
                std::vector<long long> lim(N);
                long long tot2 = 1;
                for (int d = 0; d < N; d++) {
                    lim[d] = (long long)c.dims[d] > bs ? ((long long)c.dims[d] - bs + bs - 1) / bs : 0;
                    tot2 *= lim[d];
                }
                for (long long b = 0; b < tot2; b++) {
                    long long rem = b;
                    for (int d = N - 1; d >= 0; d--) {
                        cur[d] = (rem % lim[d]) * bs;
                        rem /= lim[d];
                    }
                    if (idx % stride == 0) sel.push_back(cur);
                    idx++;
                }
            }
        }
    }
    // sample_blocks (Sample.hpp:162-231) with block side sbs + 1
    for (int d = 0; d < N; d++)
        if ((long long)c.dims[d] < bs + 1) sel.clear();
    const double sampling_num = (double)sel.size() * per_block;
    if (sampling_num == 0 || sampling_num >= num * 0.2) {
        c.cmprAlgo = ALGO_INTERP;
        return;
    }
    const long long B = (long long)sel.size();
    const long long side = bs + 1;
    const long long V = (long long)std::llround(per_block);
    std::vector<long long> hst((size_t)B * 4, 0);
    for (long long b = 0; b < B; b++)
        for (int d = 0; d < N; d++) hst[b * 4 + d] = sel[b][d];
    long long *d_st = h2d(pool, hst, st);
    T *blocks = pool.get<T>((size_t)(B * V));
    dim3 grid((unsigned)std::min<long long>((V + 255) / 256, 4096), (unsigned)B);
    k_cut_block<T><<<grid, 256, 0, st>>>(d_x, g, d_st, side, V, blocks);
    FB2_CHECK_LAUNCH();
    const falcons_config lorenzo_base = c;  // FalconsAlgoInterp.hpp:340 (before the interpolation trials)

    InterpParams base;
    base.eb = c.absErrorBound;
    base.anchor = c.interpAnchorStride;
    base.radius = c.quantbinCnt / 2;
    base.tuning = 1;
    base.max_abs = max_abs;  // the blocks' values are the field's
    int fact = 1;
    for (int i = 2; i <= N; i++) fact *= i;
    const int reverse = fact - 1;
    c.interpDirection = 0;
    if (N <= 2) {
        c.interpAlpha = 1.0;
        c.interpBeta = 1.0;
    } else {
        c.interpAlpha = 1.25;
        c.interpBeta = 2.0;
    }
    double best = 0;
    int best_algo = c.interpAlgo, best_dir = 0;
    for (int i = 0; i < 4; i++) {
        InterpParams p = base;
        p.cubic = (i / 2 == 0) ? 0 : 1;
        p.direction = (i % 2 == 0) ? 0 : reverse;
        p.alpha = c.interpAlpha;
        p.beta = c.interpBeta;
        const double r = trial_ratio<T>(pool, blocks, B, side, N, p, st);
        if (r > best) {
            best = r;
            best_algo = p.cubic;
            best_dir = p.direction;
        }
    }
    c.interpAlgo = best_algo;
    c.interpDirection = best_dir;
    if (N <= 2) {
        // two-step search of the serial build (omp_get_max_threads() == 1): alpha/beta on top
        static const double alphas[3] = {1.0, 1.25, 1.5};
        static const double betas[3] = {1.0, 2.0, 2.5};
        double ab[3] = {0, 0, 0};
        for (int i = 1; i < 3; i++) {
            InterpParams p = base;
            p.cubic = c.interpAlgo;
            p.direction = c.interpDirection;
            p.alpha = alphas[i];
            p.beta = betas[i];
            ab[i] = trial_ratio<T>(pool, blocks, B, side, N, p, st);
        }
        for (int i = 1; i < 3; i++) {
            if (ab[i] > best * 1.02) {
                best = ab[i];
                c.interpAlpha = alphas[i];
                c.interpBeta = betas[i];
            }
        }
    }
    // N == 1 also trials the blockwise Lorenzo predictor (FalconsAlgoInterp.hpp:479-498) and keeps
    // it when it beats interpolation by 10 % (both ratios below 50); below relErrorBound 1.01e-6 a
    // ratio above 5 is retried with 16384 quantization bins, kept when 2 % better (:524-533).
    if (N == 1 && best < 50) {
        double lr = lorenzo_trial_ratio<T>(blocks, B, V, c.absErrorBound, c.quantbinCnt, st);
        if (lr >= best * 1.1 && lr < 50) {
            int qb = c.quantbinCnt;
            if (c.relErrorBound < 1.01e-6 && lr > 5 && qb != 16384) {
                const double r2 = lorenzo_trial_ratio<T>(blocks, B, V, c.absErrorBound, 16384, st);
                if (r2 > lr * 1.02) {
                    lr = r2;
                    qb = 16384;
                }
            }
            // the trial's Config (Lorenzo orders 1 and 2, no regression, serial) with the field's
            // dims set back: Config::setDims resets the block size to 128 for 1-D and predDim to N
            // (utils/Config.hpp:165-181), so the field is coded in blocks of 128, the trial's 5 not kept
            c = lorenzo_base;
            c.cmprAlgo = ALGO_LORENZO_REG;
            c.lorenzo = 1;
            c.lorenzo2 = 1;
            c.regression = 0;
            c.regression2 = 0;
            c.openmp = 0;
            c.quantbinCnt = qb;
            c.blockSize = 128;
            c.predDim = 1;
            return;
        }
    }
    c.cmprAlgo = ALGO_INTERP;
}

template void tune_interp<float>(Context &, falcons_config &, const float *, cudaStream_t, double);
template void tune_interp<double>(Context &, falcons_config &, const double *, cudaStream_t, double);

}  // namespace fb2
