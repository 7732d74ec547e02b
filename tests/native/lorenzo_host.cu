// Test build of the device code of the 1-D Lorenzo decoder for the host: the same
// __host__ __device__ functions (falcons_b200/csrc/lorenzo.cuh) that k_lz_huff_decode and
// k_lz_reconstruct run, called here on the CPU so that tests/test_lorenzo_host.py checks their
// logic against the reference without a GPU.  Test infrastructure; the product never loads it.
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
}  // namespace

extern "C" {
int lzh_decode_f32(const uint8_t *p, size_t len, size_t n, int block, int l1, int l2, float *out) {
    return decode<float>(p, len, n, block, l1, l2, out);
}
int lzh_decode_f64(const uint8_t *p, size_t len, size_t n, int block, int l1, int l2, double *out) {
    return decode<double>(p, len, n, block, l1, l2, out);
}
}
