// Decode of the 1-D blockwise Lorenzo + Huffman path (ALGO_LORENZO_REG streams that the
// reference's interpolation tuner writes for 1-D fields; lorenzo.cuh has the format and the
// reference lines).  The payload is on the device (d_flat, logical bytes); the host reads its
// small headers, then one single-thread CTA per Huffman record decodes the selection and the
// codes, and one single-thread CTA walks the reconstruction (each a sequential chain, see
// lorenzo.cuh).
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

template void lorenzo_decompress<float>(const falcons_config &, const ByteView &, const uint8_t *, float *,
                                        cudaStream_t);
template void lorenzo_decompress<double>(const falcons_config &, const ByteView &, const uint8_t *, double *,
                                         cudaStream_t);

}  // namespace fb2
