// Test build of the device code of the 1-D Lorenzo path for the host: the same __host__ __device__
// functions (falcons_b200/csrc/lorenzo.cuh) that the decode kernels (k_lz_huff_decode,
// k_lz_reconstruct) run, and the encoder's (quantize_blocks, huff_lengths, huff_codes, huff_pack),
// called here on the CPU so that tests/test_lorenzo_host.py checks their logic against the
// reference without a GPU.  Test infrastructure; the product never loads it.
#include <cstring>
#include <stdexcept>
#include <vector>

#include "../../falcons_b200/csrc/lorenzo.cuh"

namespace {
struct FlatReader {
    const uint8_t *base;
    size_t len;
    template <class U>
    U rd(size_t &off) const {
        if (off + sizeof(U) > len || off + sizeof(U) < off) throw std::invalid_argument("truncated");
        U v;
        memcpy(&v, base + off, sizeof(U));
        off += sizeof(U);
        return v;
    }
};

template <class T>
int decode(const uint8_t *p, size_t len, size_t n, int block, int lorenzo, int lorenzo2, T *out) {
    using namespace fb2::lz;
    try {
        const FlatReader v{p, len};
        const size_t nblocks = (n + (size_t)block - 1) / (size_t)block;
        const bool composed = lorenzo && lorenzo2;
        const Layout l = parse_payload(v, n, nblocks, composed, sizeof(T));
        std::vector<int32_t> sel(nblocks + 1), codes(n + 1);
        auto run = [&](const Record &r, size_t count, int32_t *dst) {
            std::vector<uint32_t> order(r.nstates);
            HuffTables h;
            int e = huff_tables(p + r.lens_off, r.nstates, r.offset, order.data(), h);
            if (!e) e = huff_decode(p + r.bits_off, r.nbytes, h, order.data(), count, dst);
            return e;
        };
        int e = 0;
        if (composed && nblocks) e = run(l.sel, nblocks, sel.data());
        if (!e) e = run(l.codes, n, codes.data());
        if (e) return e;
        std::vector<T> unpred(l.n_unpred + 1);
        memcpy(unpred.data(), p + l.unpred_off, l.n_unpred * sizeof(T));
        e = reconstruct<T>(codes.data(), n, composed ? sel.data() : nullptr, lorenzo2 && !lorenzo ? 1 : 0, block,
                           unpred.data(), l.n_unpred, l.eb, l.radius, out);
        return e ? 16 + e : 0;
    } catch (std::exception &) {
        return -1;
    }
}
struct Out {
    std::vector<uint8_t> b;
    void put(const void *v, size_t n) {
        const uint8_t *p = static_cast<const uint8_t *>(v);
        b.insert(b.end(), p, p + n);
    }
};

// A Huffman record of sym[0, n) with the encoder functions of lorenzo.cuh: its header
// (HuffmanEncoder::save) into `head`, its bits (HuffmanEncoder::encode) into `bits`.
int record_parts(Out &head, Out &bitsout, const int32_t *sym, size_t n);

// One Huffman record of sym[0, n) (save, then encode).
int record(Out &o, const int32_t *sym, size_t n) {
    Out h, b;
    const int e = record_parts(h, b, sym, n);
    o.put(h.b.data(), h.b.size());
    o.put(b.b.data(), b.b.size());
    return e;
}

int record_parts(Out &o, Out &ob, const int32_t *sym, size_t n) {
    using namespace fb2::lz;
    std::vector<unsigned long long> hist(65536, 0);
    for (size_t i = 0; i < n; i++) {
        if (sym[i] < 0 || sym[i] > 65535) return 30;
        hist[sym[i]]++;
    }
    uint32_t lo = 0, hi = 65535;
    while (!hist[lo]) lo++;
    while (!hist[hi]) hi--;
    const uint32_t ns = hi - lo + 2;
    std::vector<unsigned long long> freq(ns, 0);
    for (uint32_t s = 0; s + 1 < ns; s++) freq[s] = hist[lo + s];
    std::vector<HuffNode> nodes(2 * ns);
    std::vector<int> heap(2 * ns + 1);
    std::vector<uint8_t> lens(ns);
    std::vector<uint32_t> codes(ns);
    if (huff_lengths(freq.data(), ns, nodes.data(), heap.data(), lens.data()) < 0) return 31;
    const int table = huff_codes(lens.data(), freq.data(), ns, n, codes.data());
    const int32_t word = (int32_t)(((uint32_t)table << 31) | lo);
    o.put(&word, 4);
    const uint8_t be[4] = {(uint8_t)(ns >> 24), (uint8_t)(ns >> 16), (uint8_t)(ns >> 8), (uint8_t)ns};
    o.put(be, 4);
    o.put(lens.data(), ns);
    unsigned long long bits = 0;
    for (size_t i = 0; i < n; i++) bits += lens[sym[i] - lo];
    const unsigned long long nbytes = (bits + 7) / 8;
    ob.put(&nbytes, 8);
    std::vector<uint8_t> packed(nbytes + 1, 0);
    huff_pack(sym, 0, n, lo, lens.data(), codes.data(), 0, packed.data());
    ob.put(packed.data(), nbytes);
    return 0;
}

// The tuner's trial buffer over B blocks of V points in the layout lorenzo.cu's
// lorenzo_trial_ratio writes: [u64 selections][selection record][quantizer header + the
// unpredictable values of all blocks][codes record header][u64 codes][codes record bits].
template <class T>
long long trial(const T *blocks, size_t B, size_t V, double eb, int radius, uint8_t *out, size_t cap) {
    using namespace fb2::lz;
    const size_t nblk = (V + 4) / 5;
    std::vector<int32_t> codes(B * V + 1), sel(B * nblk + 1);
    std::vector<T> unpred(B * V + 1);
    std::vector<uint32_t> nu(B, 0);
    for (size_t b = 0; b < B; b++) {
        const int e = quantize_blocks<T>(blocks + b * V, V, eb, radius, 5, 1, 0, codes.data() + b * V,
                                         sel.data() + b * nblk, unpred.data() + b * V, (uint32_t)V, &nu[b]);
        if (e) return -e;
    }
    Out o, ch, cb;
    const uint64_t ns = B * nblk;
    o.put(&ns, 8);
    if (record(o, sel.data(), B * nblk)) return -30;
    const uint8_t uid = 2;
    const int32_t r = radius;
    int32_t u = 0;
    for (uint32_t v : nu) u += (int32_t)v;
    o.put(&uid, 1);
    o.put(&eb, 8);
    o.put(&r, 4);
    o.put(&u, 4);
    for (size_t b = 0; b < B; b++) o.put(unpred.data() + b * V, nu[b] * sizeof(T));
    if (record_parts(ch, cb, codes.data(), B * V)) return -31;
    o.put(ch.b.data(), ch.b.size());
    const uint64_t nc = B * V;
    o.put(&nc, 8);
    o.put(cb.b.data(), cb.b.size());
    if (o.b.size() > cap) return -1;
    memcpy(out, o.b.data(), o.b.size());
    return (long long)o.b.size();
}

template <class T>
long long encode(const T *x, size_t n, double eb, int radius, int block, int l1, int l2, uint8_t *out, size_t cap) {
    using namespace fb2::lz;
    const size_t nblocks = (n + (size_t)block - 1) / (size_t)block;
    const bool composed = l1 && l2;
    std::vector<int32_t> codes(n + 1), sel(nblocks + 1);
    std::vector<T> unpred(n + 1);
    uint32_t nu = 0;
    int e = quantize_blocks<T>(x, n, eb, radius, block, composed, l2 && !l1 ? 1 : 0, codes.data(), sel.data(),
                               unpred.data(), (uint32_t)n, &nu);
    if (e) return -e;
    Out o;
    if (composed) {
        const uint64_t ns = nblocks;
        o.put(&ns, 8);
        if (nblocks && (e = record(o, sel.data(), nblocks))) return -e;
    }
    const uint8_t uid = 2;
    const int32_t r = radius, u = (int32_t)nu;
    o.put(&uid, 1);
    o.put(&eb, 8);
    o.put(&r, 4);
    o.put(&u, 4);
    o.put(unpred.data(), nu * sizeof(T));
    const uint64_t nc = n;
    o.put(&nc, 8);
    if ((e = record(o, codes.data(), n))) return -e;
    if (o.b.size() > cap) return -1;
    memcpy(out, o.b.data(), o.b.size());
    return (long long)o.b.size();
}
}  // namespace

extern "C" {
long long lzh_trial_f32(const float *b, size_t B, size_t V, double eb, int radius, uint8_t *out, size_t cap) {
    return trial<float>(b, B, V, eb, radius, out, cap);
}
long long lzh_trial_f64(const double *b, size_t B, size_t V, double eb, int radius, uint8_t *out, size_t cap) {
    return trial<double>(b, B, V, eb, radius, out, cap);
}
long long lzh_encode_f32(const float *x, size_t n, double eb, int radius, int block, int l1, int l2, uint8_t *out,
                         size_t cap) {
    return encode<float>(x, n, eb, radius, block, l1, l2, out, cap);
}
long long lzh_encode_f64(const double *x, size_t n, double eb, int radius, int block, int l1, int l2, uint8_t *out,
                         size_t cap) {
    return encode<double>(x, n, eb, radius, block, l1, l2, out, cap);
}
int lzh_decode_f32(const uint8_t *p, size_t len, size_t n, int block, int l1, int l2, float *out) {
    return decode<float>(p, len, n, block, l1, l2, out);
}
int lzh_decode_f64(const uint8_t *p, size_t len, size_t n, int block, int l1, int l2, double *out) {
    return decode<double>(p, len, n, block, l1, l2, out);
}
}
