// The 1-D blockwise Lorenzo + Huffman path (ALGO_LORENZO_REG; lorenzo.cuh has the format and the
// reference lines).
//
// Decode: the payload is on the device (d_flat, logical bytes); the host reads its small headers,
// then one single-thread CTA per Huffman record decodes the selection and the codes, and one
// single-thread CTA walks the reconstruction (each a sequential chain, see lorenzo.cuh).
//
// Encode (FalconsGenericCompressor.hpp:64-81 with the blockwise decomposition): one thread walks
// the quantization; the histograms of the selection and of the codes are counted by the grid; one
// thread per record builds the Huffman code book (the reference's heap order, canonical codes);
// the grid packs the bits (chunk bit counts, their scan, then every thread packs 16 symbols from
// its start bit); the payload pieces then go through the Assembler like the interpolation path's.
#include <stdexcept>
#include <vector>

#include "assemble.cuh"
#include "common.cuh"
#include "lorenzo.cuh"
#include "lorenzo_path.cuh"
#include "stream.hpp"

namespace fb2 {
namespace {

struct HuffJob {
    const uint8_t *lens;
    const uint8_t *bits;
    unsigned long long nbytes;
    uint32_t offset, nstates;
    unsigned long long n;
    int32_t *out;
    uint32_t *order;  // nstates entries of scratch
};

__global__ void k_lz_huff_decode(const HuffJob *__restrict__ jobs, int njobs, int *__restrict__ err) {
    if (threadIdx.x != 0 || (int)blockIdx.x >= njobs) return;
    const HuffJob j = jobs[blockIdx.x];
    lz::HuffTables h;
    int e = lz::huff_tables(j.lens, j.nstates, j.offset, j.order, h);
    if (!e) e = lz::huff_decode(j.bits, j.nbytes, h, j.order, (size_t)j.n, j.out);
    if (e) atomicExch(err, e);
}

template <class T>
__global__ void k_lz_reconstruct(const int32_t *__restrict__ codes, unsigned long long n, const int32_t *sel,
                                 int sel_all, int block, const T *__restrict__ unpred, uint32_t n_unpred, double eb,
                                 int radius, T *__restrict__ out, int *__restrict__ err) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int e = lz::reconstruct<T>(codes, (size_t)n, sel, sel_all, block, unpred, n_unpred, eb, radius, out);
    if (e) atomicExch(err, 16 + e);
}

template <class T>
__global__ void k_lz_quantize(const T *__restrict__ x, unsigned long long n, double eb, int radius, int block,
                              int composed, int sel_all, int32_t *__restrict__ codes, int32_t *__restrict__ sel,
                              T *__restrict__ unpred, uint32_t *__restrict__ n_unpred, int *__restrict__ err) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int e = lz::quantize_blocks<T>(x, (size_t)n, eb, radius, block, composed, sel_all, codes, sel, unpred,
                                         (uint32_t)n, n_unpred);
    if (e) atomicExch(err, 32 + e);
}

// The tuner's trial: B independent sample blocks of V points, one thread each (every block starts
// from the two zero values before it, as each of the reference's per-block compress calls does).
template <class T>
__global__ void k_lz_quantize_many(const T *__restrict__ x, long long B, long long V, double eb, int radius,
                                   int block, int32_t *__restrict__ codes, int32_t *__restrict__ sel,
                                   T *__restrict__ unpred, uint32_t *__restrict__ n_unpred, int *__restrict__ err) {
    const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const long long nblk = (V + block - 1) / block;
    const int e = lz::quantize_blocks<T>(x + b * V, (size_t)V, eb, radius, block, 1, 0, codes + b * V, sel + b * nblk,
                                         unpred + b * V, (uint32_t)V, n_unpred + b);
    if (e) atomicExch(err, 32 + e);
}

// hist[v] += 1 for every symbol v of sym[0, n) (symbols are in [0, 65536): biased codes, selections)
__global__ void k_lz_hist(const int32_t *__restrict__ sym, unsigned long long n, unsigned long long *__restrict__ hist,
                          int *__restrict__ err) {
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const int32_t v = sym[i];
        if (v < 0 || v > 65535) {
            atomicExch(err, 40);
            continue;
        }
        atomicAdd(&hist[v], 1ULL);
    }
}

// The code book of one record, built by one thread from its histogram (65537 counts, the last 0).
struct BookJob {
    const unsigned long long *hist;
    unsigned long long total;
    lz::HuffNode *nodes;  // 2 * 65538 entries
    int *heap;            // 2 * 65538 + 1 entries
    uint8_t *lens;        // 65538 entries
    uint32_t *codes;      // 65538 entries
    unsigned long long *info;  // out: offset, state count, table flag, code bits
};

__global__ void k_lz_book(const BookJob *__restrict__ jobs, int njobs, int *__restrict__ err) {
    if (threadIdx.x != 0 || (int)blockIdx.x >= njobs) return;
    const BookJob j = jobs[blockIdx.x];
    uint32_t lo = 0, hi = 65535;
    while (lo < 65535 && !j.hist[lo]) lo++;
    while (hi > lo && !j.hist[hi]) hi--;
    if (!j.hist[lo]) {  // an empty record is never built
        atomicExch(err, 41);
        return;
    }
    const uint32_t ns = hi - lo + 2;
    const unsigned long long *freq = j.hist + lo;  // freq[ns - 1] = hist[hi + 1] = 0
    if (lz::huff_lengths(freq, ns, j.nodes, j.heap, j.lens) < 0) {
        atomicExch(err, 42);
        return;
    }
    const int table = lz::huff_codes(j.lens, freq, ns, j.total, j.codes);
    unsigned long long bits = 0;
    for (uint32_t s = 0; s < ns; s++) bits += freq[s] * j.lens[s];
    j.info[0] = lo;
    j.info[1] = ns;
    j.info[2] = (unsigned long long)table;
    j.info[3] = bits;
}

// Bit packing of one Huffman record in parallel (the layout of lz::huff_pack: code bit b of a
// symbol at stream bit start + b, stream bits little-endian within bytes): the grid takes chunks
// of kPackChunk symbols; each chunk's bit count, an exclusive scan of those, then every thread
// packs 16 consecutive symbols from its start bit (a block scan of the threads' counts), OR-ing
// each code into the one or two 32-bit words it spans.
constexpr int kPackThreads = 256, kPackPer = 16, kPackChunk = kPackThreads * kPackPer;

__global__ void __launch_bounds__(kPackThreads) k_lz_chunk_bits(const int32_t *__restrict__ sym, unsigned long long n,
                                                                uint32_t offset, const uint8_t *__restrict__ lens,
                                                                unsigned long long *__restrict__ chunk_bits) {
    const unsigned long long c0 = (unsigned long long)blockIdx.x * kPackChunk;
    const unsigned long long c1 = min(n, c0 + kPackChunk);
    unsigned b = 0;
    for (unsigned long long i = c0 + threadIdx.x; i < c1; i += kPackThreads) b += lens[(uint32_t)sym[i] - offset];
    b = __reduce_add_sync(0xffffffffu, b);
    __shared__ unsigned ws[kPackThreads / 32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kPackThreads / 32; w++) t += ws[w];
        chunk_bits[blockIdx.x] = t;
    }
}

// In-place exclusive scan of v[0, n) (one CTA).
__global__ void __launch_bounds__(1024) k_lz_scan(unsigned long long *__restrict__ v, unsigned long long n) {
    __shared__ unsigned long long wsum[32];
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (unsigned long long base = 0; base < n; base += 1024) {
        const unsigned long long i = base + threadIdx.x;
        const unsigned long long x = i < n ? v[i] : 0;
        unsigned long long s = x;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= (unsigned)o) s += y;
        }
        if (lane == 31) wsum[wid] = s;
        __syncthreads();
        if (wid == 0) {
            unsigned long long w = wsum[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= (unsigned)o) w += y;
            }
            wsum[lane] = w;
        }
        __syncthreads();
        const unsigned long long excl = carry + (wid ? wsum[wid - 1] : 0) + s - x;
        if (i < n) v[i] = excl;
        __syncthreads();
        if (threadIdx.x == 1023) carry = excl + x;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kPackThreads) k_lz_pack_chunks(const int32_t *__restrict__ sym, unsigned long long n,
                                                                 uint32_t offset, const uint8_t *__restrict__ lens,
                                                                 const uint32_t *__restrict__ codes,
                                                                 const unsigned long long *__restrict__ chunk_off,
                                                                 uint32_t *__restrict__ out) {
    const unsigned long long i0 = (unsigned long long)blockIdx.x * kPackChunk + threadIdx.x * kPackPer;
    const unsigned long long i1 = min(n, i0 + kPackPer);
    unsigned b = 0;
    for (unsigned long long i = i0; i < i1; i++) b += lens[(uint32_t)sym[i] - offset];
    // block exclusive scan of b
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned s = b;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= (unsigned)o) s += y;
    }
    __shared__ unsigned ws[kPackThreads / 32];
    if (lane == 31) ws[wid] = s;
    __syncthreads();
    unsigned before = 0;
    for (unsigned w = 0; w < wid; w++) before += ws[w];
    unsigned long long bit = chunk_off[blockIdx.x] + before + s - b;
    for (unsigned long long i = i0; i < i1; i++) {
        const uint32_t k = (uint32_t)sym[i] - offset;
        const unsigned l = lens[k];
        const uint32_t c = codes[k];
        // bits of the code beyond its 32-bit word are zero
        const unsigned sh = (unsigned)(bit & 31);
        const unsigned long long w = bit >> 5;
        if (c) {
            atomicOr(out + w, c << sh);
            if (sh && (l > 32 - sh)) {
                const uint32_t hi = c >> (32 - sh);
                if (hi) atomicOr(out + w + 1, hi);
            }
        }
        bit += l;
    }
}

}  // namespace

bool lorenzo_stream_supported(const falcons_config &c) {
    const int methods = (c.lorenzo ? 1 : 0) + (c.lorenzo2 ? 1 : 0) + (c.regression ? 1 : 0);
    return c.N == 1 && methods >= 1 && !c.regression && !c.regression2 && c.blockSize >= 1;
}

template <class T>
void lorenzo_decompress(const falcons_config &c, const ByteView &view, const uint8_t *d_flat, T *d_out,
                        cudaStream_t st) {
    if (!lorenzo_stream_supported(c))
        throw std::invalid_argument(
            "unsupported on GPU build: ALGO_LORENZO_REG streams other than 1-D Lorenzo (orders 1 and 2)");
    Trace tr("lorenzo decode");
    const size_t n = (size_t)c.num, block = (size_t)c.blockSize;
    const size_t nblocks = (n + block - 1) / block;
    const bool composed = c.lorenzo && c.lorenzo2;  // ComposedPredictor: a selection record
    const lz::Layout l = lz::parse_payload(view, n, nblocks, composed, sizeof(T));
    Pool pool(st);
    int32_t *codes = pool.get<int32_t>(n + 1);
    int32_t *sel = composed ? pool.get<int32_t>(nblocks + 1) : nullptr;
    std::vector<HuffJob> jobs;
    auto job = [&](const lz::Record &r, size_t count, int32_t *out) {
        jobs.push_back(HuffJob{d_flat + r.lens_off, d_flat + r.bits_off, r.nbytes, r.offset, r.nstates,
                               (unsigned long long)count, out, pool.get<uint32_t>(r.nstates)});
    };
    if (composed && nblocks) job(l.sel, nblocks, sel);
    job(l.codes, n, codes);
    T *unpred = pool.get<T>((size_t)l.n_unpred + 1);
    if (l.n_unpred)
        launch_gather(pool, {Piece{d_flat + l.unpred_off, 0, (unsigned long long)l.n_unpred * sizeof(T)}},
                      reinterpret_cast<uint8_t *>(unpred), st);
    int *d_err = pool.get<int>(1);
    FB2_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    HuffJob *d_jobs = h2d(pool, jobs, st);
    k_lz_huff_decode<<<(unsigned)jobs.size(), 32, 0, st>>>(d_jobs, (int)jobs.size(), d_err);
    FB2_CHECK_LAUNCH();
    k_lz_reconstruct<T><<<1, 32, 0, st>>>(codes, (unsigned long long)n, sel, c.lorenzo2 && !c.lorenzo ? 1 : 0,
                                          (int)block, unpred, l.n_unpred, l.eb, l.radius, d_out, d_err);
    FB2_CHECK_LAUNCH();
    const std::vector<int> e = d2h(d_err, 1, st);
    tr.mark("reconstructed");
    if (e[0]) throw std::invalid_argument("Invalid or corrupted Falcons Lorenzo payload");
}

namespace {

// A Huffman record built on the device: its code lengths (device), packed bits (device) and the
// header values the host writes.
struct BuiltRecord {
    const uint8_t *lens;
    const uint8_t *packed;
    uint32_t lo, ns;
    int table;
    unsigned long long nbytes;
};

// Builds the records of the symbol arrays syms[k] (device, counts[k] symbols each): histograms on
// the grid, one code book per CTA, one packing thread per record.  Synchronizes the stream.
std::vector<BuiltRecord> build_records(Pool &pool, const std::vector<const int32_t *> &syms,
                                       const std::vector<size_t> &counts, int *d_err, cudaStream_t st) {
    constexpr size_t kStates = 65538;
    std::vector<BookJob> jobs;
    for (size_t k = 0; k < syms.size(); k++) {
        unsigned long long *hist = pool.get<unsigned long long>(65537);
        FB2_CUDA(cudaMemsetAsync(hist, 0, 65537 * sizeof(unsigned long long), st));
        k_lz_hist<<<grid_for((long long)counts[k], 256, 148 * 8), 256, 0, st>>>(
            syms[k], (unsigned long long)counts[k], hist, d_err);
        FB2_CHECK_LAUNCH();
        jobs.push_back(BookJob{hist, (unsigned long long)counts[k], pool.get<lz::HuffNode>(2 * kStates),
                               pool.get<int>(2 * kStates + 1), pool.get<uint8_t>(kStates),
                               pool.get<uint32_t>(kStates), pool.get<unsigned long long>(4)});
    }
    BookJob *d_jobs = h2d(pool, jobs, st);
    k_lz_book<<<(unsigned)jobs.size(), 32, 0, st>>>(d_jobs, (int)jobs.size(), d_err);
    FB2_CHECK_LAUNCH();
    std::vector<BuiltRecord> out;
    for (size_t k = 0; k < jobs.size(); k++) {
        const std::vector<unsigned long long> info = d2h(jobs[k].info, 4, st);
        if (d2h(d_err, 1, st)[0]) throw std::runtime_error("Lorenzo encoding failed");
        BuiltRecord r{jobs[k].lens, nullptr, (uint32_t)info[0], (uint32_t)info[1], (int)info[2], (info[3] + 7) / 8};
        uint8_t *packed = pool.get<uint8_t>((size_t)r.nbytes + 16);
        FB2_CUDA(cudaMemsetAsync(packed, 0, (size_t)r.nbytes + 16, st));
        const unsigned long long nsym = (unsigned long long)counts[k];
        if (nsym > 0) {
            const unsigned long long nchunks = (nsym + kPackChunk - 1) / kPackChunk;
            unsigned long long *coff = pool.get<unsigned long long>(nchunks + 1);
            k_lz_chunk_bits<<<(unsigned)nchunks, kPackThreads, 0, st>>>(syms[k], nsym, r.lo, jobs[k].lens, coff);
            FB2_CHECK_LAUNCH();
            k_lz_scan<<<1, 1024, 0, st>>>(coff, nchunks);
            FB2_CHECK_LAUNCH();
            k_lz_pack_chunks<<<(unsigned)nchunks, kPackThreads, 0, st>>>(syms[k], nsym, r.lo, jobs[k].lens,
                                                                         jobs[k].codes, coff,
                                                                         reinterpret_cast<uint32_t *>(packed));
            FB2_CHECK_LAUNCH();
        }
        r.packed = packed;
        out.push_back(r);
    }
    return out;
}

// A record's header (HuffmanEncoder::save) and its bits (HuffmanEncoder::encode).
void record_header(Assembler &as, const BuiltRecord &r) {
    as.val<int32_t>((int32_t)(((uint32_t)r.table << 31) | r.lo));
    const uint8_t be[4] = {(uint8_t)(r.ns >> 24), (uint8_t)(r.ns >> 16), (uint8_t)(r.ns >> 8), (uint8_t)r.ns};
    as.bytes(be, 4);
    as.dev(r.lens, r.ns);
}
void record_bits(Assembler &as, const BuiltRecord &r) {
    as.val<uint64_t>(r.nbytes);
    as.dev(r.packed, (size_t)r.nbytes);
}

}  // namespace

template <class T>
size_t lorenzo_compress(const falcons_config &c, const T *d_x, uint8_t *d_pay, size_t pcap, cudaStream_t st) {
    if (!lorenzo_stream_supported(c))
        throw std::invalid_argument(
            "unsupported on GPU build: ALGO_LORENZO_REG other than 1-D Lorenzo (orders 1 and / or 2, no regression)");
    Trace tr("lorenzo encode");
    const size_t n = (size_t)c.num, block = (size_t)c.blockSize;
    const size_t nblocks = (n + block - 1) / block;
    const bool composed = c.lorenzo && c.lorenzo2;
    const int radius = c.quantbinCnt / 2;
    const double eb = c.absErrorBound;
    Pool pool(st);
    int32_t *codes = pool.get<int32_t>(n + 1);
    int32_t *sel = pool.get<int32_t>(nblocks + 1);
    T *unpred = pool.get<T>(n + 1);
    uint32_t *d_nu = pool.get<uint32_t>(1);
    int *d_err = pool.get<int>(1);
    FB2_CUDA(cudaMemsetAsync(d_nu, 0, sizeof(uint32_t), st));
    FB2_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    k_lz_quantize<T><<<1, 32, 0, st>>>(d_x, (unsigned long long)n, eb, radius, (int)block, composed ? 1 : 0,
                                       c.lorenzo2 && !c.lorenzo ? 1 : 0, codes, sel, unpred, d_nu, d_err);
    FB2_CHECK_LAUNCH();
    // the records: the selection (composed predictors only), then the codes
    std::vector<const int32_t *> syms;
    std::vector<size_t> counts;
    if (composed && nblocks) {
        syms.push_back(sel);
        counts.push_back(nblocks);
    }
    syms.push_back(codes);
    counts.push_back(n);
    const std::vector<BuiltRecord> rec = build_records(pool, syms, counts, d_err, st);
    const uint32_t nu = d2h(d_nu, 1, st)[0];
    tr.mark("code books built");
    // FalconsGenericCompressor.hpp:64-81: decomposition (selection, quantizer), code count, codes
    Assembler as;
    as.with_index = false;
    if (composed) {
        as.val<uint64_t>((uint64_t)nblocks);
        if (nblocks) {
            record_header(as, rec[0]);
            record_bits(as, rec[0]);
        }
    }
    as.val<uint8_t>(0b10);  // LinearQuantizer::save
    as.val<double>(eb);
    as.val<int32_t>(radius);
    as.val<int32_t>((int32_t)nu);
    as.dev(unpred, (size_t)nu * sizeof(T));
    as.val<uint64_t>((uint64_t)n);
    record_header(as, rec.back());
    record_bits(as, rec.back());
    if (as.framed_size() > pcap) throw std::length_error("The buffer for compressed data is not large enough.");
    const size_t out = as.run_framed(pool, d_pay, st);
    tr.mark("payload assembled");
    return out;
}

template <class T>
double lorenzo_trial_ratio(const T *d_blocks, long long B, long long V, double eb, int quantbin, cudaStream_t st) {
    Trace tr("lorenzo trial");
    constexpr int kBlock = 5;
    const long long nblk = (V + kBlock - 1) / kBlock;
    const int radius = quantbin / 2;
    Pool pool(st);
    int32_t *codes = pool.get<int32_t>((size_t)(B * V) + 1);
    int32_t *sel = pool.get<int32_t>((size_t)(B * nblk) + 1);
    T *unpred = pool.get<T>((size_t)(B * V) + 1);
    uint32_t *d_nu = pool.get<uint32_t>((size_t)B);
    int *d_err = pool.get<int>(1);
    FB2_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    k_lz_quantize_many<T><<<(unsigned)((B + 31) / 32), 32, 0, st>>>(d_blocks, B, V, eb, radius, kBlock, codes, sel,
                                                                    unpred, d_nu, d_err);
    FB2_CHECK_LAUNCH();
    const std::vector<BuiltRecord> rec =
        build_records(pool, {sel, codes}, {(size_t)(B * nblk), (size_t)(B * V)}, d_err, st);
    const std::vector<uint32_t> nu = d2h(d_nu, (size_t)B, st);
    unsigned long long nu_all = 0;
    for (uint32_t u : nu) nu_all += u;
    // lorenzo_compress_test (FalconsAlgoInterp.hpp:229-262): the decomposition's save (the
    // selection of all blocks, the quantizer with the unpredictable values of all blocks), the
    // encoder's save, the code count, the encoder's bits; then zstd
    Assembler as;
    as.with_index = false;
    as.val<uint64_t>((uint64_t)(B * nblk));
    record_header(as, rec[0]);
    record_bits(as, rec[0]);
    as.val<uint8_t>(0b10);
    as.val<double>(eb);
    as.val<int32_t>(radius);
    as.val<int32_t>((int32_t)nu_all);
    for (long long b = 0; b < B; b++) as.dev(unpred + b * V, (size_t)nu[b] * sizeof(T));
    record_header(as, rec[1]);
    as.val<uint64_t>((uint64_t)(B * V));
    record_bits(as, rec[1]);
    uint8_t *d_buf = pool.get<uint8_t>((size_t)as.pos + 16);
    as.run(pool, d_buf, st);
    const std::vector<uint8_t> h = d2h(d_buf, (size_t)as.pos, st);
    std::vector<uint8_t> z(zstd_compress_bound(h.size()) + 16);
    const size_t zs = zstd_compress(h.data(), h.size(), z.data(), z.size(), 3) + sizeof(size_t);
    tr.mark("trial compressed");
    return (double)((size_t)V * (size_t)B * sizeof(T)) / (double)zs;
}

template double lorenzo_trial_ratio<float>(const float *, long long, long long, double, int, cudaStream_t);
template double lorenzo_trial_ratio<double>(const double *, long long, long long, double, int, cudaStream_t);

template size_t lorenzo_compress<float>(const falcons_config &, const float *, uint8_t *, size_t, cudaStream_t);
template size_t lorenzo_compress<double>(const falcons_config &, const double *, uint8_t *, size_t, cudaStream_t);

template void lorenzo_decompress<float>(const falcons_config &, const ByteView &, const uint8_t *, float *,
                                        cudaStream_t);
template void lorenzo_decompress<double>(const falcons_config &, const ByteView &, const uint8_t *, double *,
                                         cudaStream_t);

}  // namespace fb2
