// 1-D blockwise Lorenzo + Huffman path (ALGO_LORENZO_REG as the interpolation tuner configures it
// for 1-D fields: Lorenzo orders 1 and 2 composed per block, block size 5, no regression), decode
// side.  Reference: decomposition/BlockwiseDecomposition.hpp:46-72 (blocks, +radius bias),
// predictor/ComposedPredictor.hpp:52-78 (selection record), predictor/LorenzoPredictor.hpp:67-83
// (predictions), quantizer/LinearQuantizer.hpp:112-128,154-178 (recover, load),
// encoder/HuffmanEncoder.hpp:570-650 (load: code lengths -> canonical codes), 429-478 (decode:
// first bit first, one symbol per complete code).
//
// Every code depends on the reconstruction of the point before it (the predictions read the
// reconstructed values), a chain of floating-point roundings that no scan or speculative split
// reproduces bit for bit, so the reconstruction of one field is one sequential walk; so is the
// Huffman decode of a record without decode checkpoints (the reference writes none).  The
// functions here are __host__ __device__ so that the same source runs in the device kernels and,
// for the tests, on the host.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <stdexcept>

namespace fb2 {
namespace lz {

constexpr int kMaxCodeLen = 32;

// Canonical decode tables of one Huffman record (code lengths of the states s = symbol - offset).
struct HuffTables {
    uint32_t offset = 0, nstates = 0;
    int maxl = 0;
    int single = 0;        // one symbol only: no code bits (HuffmanEncoder.hpp:615-645)
    uint32_t single_state = 0;
    uint32_t count[kMaxCodeLen + 1];
    uint32_t first[kMaxCodeLen + 1];  // first canonical code of each length (MSB-first)
    uint32_t base[kMaxCodeLen + 1];   // index of that length's first state in `order`
};

// Error codes written by the decode steps (0 = success).
enum : int { kOk = 0, kBadLengths = 1, kBadBits = 2, kShort = 3, kBadUnpred = 4, kBadSelection = 5 };

// Tables from the code lengths (lens[nstates]); order[] receives the states sorted by (length,
// state), at most nstates entries.
__host__ __device__ inline int huff_tables(const uint8_t *lens, uint32_t nstates, uint32_t offset, uint32_t *order,
                                           HuffTables &h) {
    h.offset = offset;
    h.nstates = nstates;
    h.maxl = 0;
    h.single = 0;
    h.single_state = 0;
    for (int l = 0; l <= kMaxCodeLen; l++) h.count[l] = h.first[l] = h.base[l] = 0;
    uint32_t nonzero = 0, last = 0;
    for (uint32_t s = 0; s < nstates; s++) {
        const int l = lens[s];
        if (l > kMaxCodeLen) return kBadLengths;
        if (l) {
            h.count[l]++;
            nonzero++;
            last = s;
            if (l > h.maxl) h.maxl = l;
        }
    }
    if (nstates == 2) {
        h.single = 1;
        h.single_state = nonzero == 1 ? last : 0;
        return kOk;
    }
    if (h.maxl == 0) return kBadLengths;
    uint32_t c = 0, k = 0;
    for (int l = 1; l <= h.maxl; l++) {
        c = (c + (l > 1 ? h.count[l - 1] : 0)) << 1;
        h.first[l] = c;
        h.base[l] = k;
        k += h.count[l];
    }
    // the codes must fit their lengths (a complete or incomplete prefix code)
    for (int l = 1; l <= h.maxl; l++)
        if (h.count[l] && (unsigned long long)h.first[l] + h.count[l] > (1ULL << l)) return kBadLengths;
    uint32_t next[kMaxCodeLen + 1];
    for (int l = 0; l <= kMaxCodeLen; l++) next[l] = h.base[l];
    for (uint32_t s = 0; s < nstates; s++)
        if (lens[s]) order[next[lens[s]]++] = s;
    return kOk;
}

// Decodes n symbols from bits[0, nbytes) (first bit of a code in bit 0 of its byte).
__host__ __device__ inline int huff_decode(const uint8_t *bits, unsigned long long nbytes, const HuffTables &h,
                                           const uint32_t *order, size_t n, int32_t *out) {
    if (h.single) {
        for (size_t i = 0; i < n; i++) out[i] = (int32_t)(h.offset + h.single_state);
        return kOk;
    }
    size_t i = 0;
    uint32_t code = 0;
    int l = 0;
    for (unsigned long long b = 0; b < nbytes && i < n; b++) {
        uint32_t byte = bits[b];
        for (int k = 0; k < 8 && i < n; k++, byte >>= 1) {
            code = (code << 1) | (byte & 1u);
            if (++l > h.maxl) return kBadBits;
            if (h.count[l] && code - h.first[l] < h.count[l]) {
                out[i++] = (int32_t)(h.offset + order[h.base[l] + code - h.first[l]]);
                code = 0;
                l = 0;
            }
        }
    }
    return i == n ? kOk : kShort;
}

// The reconstruction: blocks of `block` points, block k predicted by Lorenzo order 1 (sel 0) or
// order 2 (sel 1) from the reconstructed values before each point (two zeros before the field);
// code c - radius is the quantization index, 0 - radius the next unpredictable value.  Without a
// selection array (a single predictor) every block uses sel_all.
template <class T>
__host__ __device__ inline int reconstruct(const int32_t *codes, size_t n, const int32_t *sel, int sel_all,
                                           int block, const T *unpred, uint32_t n_unpred, double eb, int radius,
                                           T *out) {
    if (block < 1) return kBadSelection;
    const double ebx2 = 2 * eb;
    T m1 = 0, m2 = 0;  // the values one and two points before
    uint32_t u = 0;
    size_t i = 0;
    for (size_t k = 0; i < n; k++) {
        const int s = sel ? sel[k] : sel_all;
        if (s != 0 && s != 1) return kBadSelection;
        const size_t end = (n - i < (size_t)block) ? n : i + (size_t)block;
        for (; i < end; i++) {
            const T pred = s ? (T)2 * m1 - m2 : m1;
            const int q = codes[i] - radius;
            T v;
            if (q != -radius) {
                v = (T)fma((double)q, ebx2, (double)pred);
            } else {
                if (u >= n_unpred) return kBadUnpred;
                v = unpred[u++];
            }
            out[i] = v;
            m2 = m1;
            m1 = v;
        }
    }
    return kOk;
}

// ---- the payload layout (host): FalconsGenericCompressor.hpp:64-81 after the zstd stage is undone
// [selection: u64 count, Huffman record (composed predictors only)] [quantizer: u8 uid 2, f64 eb,
// i32 radius, i32 unpredictable count, T values] [u64 code count] [codes: Huffman record];
// a Huffman record is [i32 table flag << 31 | offset] [u32 big-endian state count] [a length byte
// per state] [u64 bit bytes] [bits] (HuffmanEncoder.hpp:165-181, 200-228).
struct Record {
    size_t lens_off = 0, bits_off = 0;
    unsigned long long nbytes = 0;
    uint32_t offset = 0, nstates = 0;
};
struct Layout {
    bool composed = false;
    Record sel, codes;
    double eb = 0;
    int radius = 0;
    uint32_t n_unpred = 0;
    size_t unpred_off = 0, end = 0;
};

// Reader: v.len (logical bytes) and v.template rd<U>(off) (reads sizeof(U) bytes at off, advances
// off, throws past the end).
template <class Reader>
Record parse_record(const Reader &v, size_t &off) {
    Record r;
    const uint32_t word = v.template rd<uint32_t>(off);
    r.offset = word & 0x7FFFFFFFu;
    uint32_t ns = 0;
    for (int k = 0; k < 4; k++) ns = (ns << 8) | v.template rd<uint8_t>(off);
    if (ns < 2 || ns > 65538 || r.offset > 65535) throw std::invalid_argument("Huffman load: bad state count");
    r.nstates = ns;
    r.lens_off = off;
    if (off + ns > v.len) throw std::invalid_argument("Huffman load: insufficient data for code lengths");
    off += ns;
    r.nbytes = v.template rd<uint64_t>(off);
    if (r.nbytes > v.len - off) throw std::invalid_argument("Invalid or truncated Falcons payload");
    r.bits_off = off;
    off += (size_t)r.nbytes;
    return r;
}

template <class Reader>
Layout parse_payload(const Reader &v, size_t n, size_t nblocks, bool composed, size_t elem) {
    Layout l;
    l.composed = composed;
    size_t off = 0;
    if (composed) {
        const uint64_t nsel = v.template rd<uint64_t>(off);
        if (nsel != nblocks) throw std::invalid_argument("block selection count does not match the field");
        if (nsel) l.sel = parse_record(v, off);
    }
    if (v.template rd<uint8_t>(off) != 0b10) throw std::invalid_argument("LinearQuantizer uid mismatch");
    l.eb = v.template rd<double>(off);
    l.radius = v.template rd<int32_t>(off);
    const int32_t nu = v.template rd<int32_t>(off);
    if (l.radius < 1 || l.radius > 32768 || nu < 0 || (size_t)nu > n || (size_t)nu * elem > v.len - off)
        throw std::invalid_argument("Truncated Falcons payload");
    l.n_unpred = (uint32_t)nu;
    l.unpred_off = off;
    off += (size_t)nu * elem;
    if (v.template rd<uint64_t>(off) != n) throw std::invalid_argument("code count does not match the field");
    l.codes = parse_record(v, off);
    l.end = off;
    return l;
}

}  // namespace lz
}  // namespace fb2
