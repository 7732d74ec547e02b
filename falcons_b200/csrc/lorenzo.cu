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
// one thread per record packs the bits; the payload pieces then go through the Assembler like the
// interpolation path's.
#include <stdexcept>
#include <vector>

#include "assemble.cuh"
#include "common.cuh"
#include "lorenzo.cuh"
#include "lorenzo_path.cuh"

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

__global__ void k_lz_pack(const int32_t *__restrict__ sym, unsigned long long n, uint32_t offset,
                          const uint8_t *__restrict__ lens, const uint32_t *__restrict__ codes, uint8_t *__restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    lz::huff_pack(sym, 0, (size_t)n, offset, lens, codes, 0, out);
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
    struct Rec {
        const int32_t *sym;
        size_t count;
        BookJob job;
    };
    std::vector<Rec> recs;
    auto add = [&](const int32_t *sym, size_t count) {
        constexpr size_t kStates = 65538;
        Rec r{sym, count, {}};
        unsigned long long *hist = pool.get<unsigned long long>(65537);
        FB2_CUDA(cudaMemsetAsync(hist, 0, 65537 * sizeof(unsigned long long), st));
        k_lz_hist<<<grid_for((long long)count, 256, 148 * 8), 256, 0, st>>>(sym, (unsigned long long)count, hist,
                                                                            d_err);
        FB2_CHECK_LAUNCH();
        r.job = BookJob{hist, (unsigned long long)count, pool.get<lz::HuffNode>(2 * kStates),
                        pool.get<int>(2 * kStates + 1), pool.get<uint8_t>(kStates), pool.get<uint32_t>(kStates),
                        pool.get<unsigned long long>(4)};
        recs.push_back(r);
    };
    if (composed && nblocks) add(sel, nblocks);
    add(codes, n);
    std::vector<BookJob> jobs;
    for (const Rec &r : recs) jobs.push_back(r.job);
    BookJob *d_jobs = h2d(pool, jobs, st);
    k_lz_book<<<(unsigned)jobs.size(), 32, 0, st>>>(d_jobs, (int)jobs.size(), d_err);
    FB2_CHECK_LAUNCH();
    std::vector<std::vector<unsigned long long>> info;
    for (const Rec &r : recs) info.push_back(d2h(r.job.info, 4, st));
    const std::vector<uint32_t> h_nu = d2h(d_nu, 1, st);
    const std::vector<int> h_err = d2h(d_err, 1, st);
    if (h_err[0]) throw std::runtime_error("Lorenzo encoding failed");
    tr.mark("code books built");
    // payload pieces
    Assembler as;
    as.with_index = false;
    auto record = [&](size_t k) {
        const Rec &r = recs[k];
        const unsigned long long lo = info[k][0], ns = info[k][1], table = info[k][2], bits = info[k][3];
        const unsigned long long nbytes = (bits + 7) / 8;
        uint8_t *packed = pool.get<uint8_t>((size_t)nbytes + 16);
        FB2_CUDA(cudaMemsetAsync(packed, 0, (size_t)nbytes + 16, st));
        k_lz_pack<<<1, 32, 0, st>>>(r.sym, (unsigned long long)r.count, (uint32_t)lo, r.job.lens, r.job.codes, packed);
        FB2_CHECK_LAUNCH();
        as.val<int32_t>((int32_t)(((uint32_t)table << 31) | (uint32_t)lo));
        const uint8_t be[4] = {(uint8_t)(ns >> 24), (uint8_t)(ns >> 16), (uint8_t)(ns >> 8), (uint8_t)ns};
        as.bytes(be, 4);
        as.dev(r.job.lens, (size_t)ns);
        as.val<uint64_t>(nbytes);
        as.dev(packed, (size_t)nbytes);
    };
    size_t k = 0;
    if (composed) {
        as.val<uint64_t>((uint64_t)nblocks);
        if (nblocks) record(k++);
    }
    as.val<uint8_t>(0b10);  // LinearQuantizer::save
    as.val<double>(eb);
    as.val<int32_t>(radius);
    as.val<int32_t>((int32_t)h_nu[0]);
    as.dev(unpred, (size_t)h_nu[0] * sizeof(T));
    as.val<uint64_t>((uint64_t)n);
    record(k);
    if (as.framed_size() > pcap) throw std::length_error("The buffer for compressed data is not large enough.");
    const size_t out = as.run_framed(pool, d_pay, st);
    tr.mark("payload assembled");
    return out;
}

template size_t lorenzo_compress<float>(const falcons_config &, const float *, uint8_t *, size_t, cudaStream_t);
template size_t lorenzo_compress<double>(const falcons_config &, const double *, uint8_t *, size_t, cudaStream_t);

template void lorenzo_decompress<float>(const falcons_config &, const ByteView &, const uint8_t *, float *,
                                        cudaStream_t);
template void lorenzo_decompress<double>(const falcons_config &, const ByteView &, const uint8_t *, double *,
                                         cudaStream_t);

}  // namespace fb2
