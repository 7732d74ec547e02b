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

// ---- encode side

// The blockwise quantization (BlockwiseDecomposition.hpp:37-57 with ComposedPredictor.hpp:25-50):
// block by block, the predictor is chosen by the sum (in double) of its error estimates
// |x - pred| + noise at the block's first and last point (BlockwiseIterator.hpp:153-158; the
// values inside the block are still the originals there, those before it reconstructed), the
// first smallest sum winning; then every point is quantized against the reconstruction
// (LinearQuantizer.hpp:49-80) and its code biased by +radius.  With a single predictor
// (composed == 0) every block uses sel_all and no choice is made.  The input is not modified.
// Returns kOk, or kBadUnpred when more than unpred_cap values are unpredictable.
template <class T>
__host__ __device__ inline int quantize_blocks(const T *x, size_t n, double eb, int radius, int block, int composed,
                                               int sel_all, int32_t *codes, int32_t *sel, T *unpred,
                                               uint32_t unpred_cap, uint32_t *n_unpred) {
    if (block < 1) return kBadSelection;
    const double ebx2 = 2 * eb, ebx2_r = 1.0 / ebx2;
    const T noise1 = (T)(0.5 * eb), noise2 = (T)(1.08 * eb);  // LorenzoPredictor.hpp:17-38, N = 1
    T m1 = 0, m2 = 0;  // reconstructed values one and two points before the current one
    uint32_t u = 0;
    size_t i = 0;
    for (size_t k = 0; i < n; k++) {
        const size_t b0 = i, end = (n - i < (size_t)block) ? n : i + (size_t)block;
        int s = sel_all;
        if (composed) {
            // value j for the estimates: originals inside the block, reconstructions before it
            auto at = [&](size_t j, size_t back) -> T { return j >= b0 + back ? x[j - back] : (back - (j - b0) == 1 ? m1 : m2); };
            double e1 = 0, e2 = 0;
            const size_t pts[2] = {b0, end - 1};
            // each estimate is a T value (LorenzoPredictor::estimate_error returns T)
            auto est = [](T d, T noise) -> T { return (d < 0 ? -d : d) + noise; };
            for (int q = 0; q < 2; q++) {
                const size_t j = pts[q];
                e1 += (double)est(x[j] - at(j, 1), noise1);
            }
            for (int q = 0; q < 2; q++) {
                const size_t j = pts[q];
                e2 += (double)est(x[j] - ((T)2 * at(j, 1) - at(j, 2)), noise2);
            }
            s = e2 < e1 ? 1 : 0;
            sel[k] = s;
        }
        for (; i < end; i++) {
            const T pred = s ? (T)2 * m1 - m2 : m1;
            const T xv = x[i];
            const T diff = xv - pred;
            const double v = nearbyint((double)diff * ebx2_r);
            T r = xv;
            int q = -radius;
            if (v > -radius && v < radius) {
                const int qi = (int)v;
                const T dq = (T)fma((double)qi, ebx2, (double)pred);
                const T err = dq - xv;
                if ((double)err >= -eb && (double)err <= eb) {
                    q = qi;
                    r = dq;
                }
            }
            if (q == -radius) {
                if (u >= unpred_cap) return kBadUnpred;
                unpred[u++] = xv;
            }
            codes[i] = q + radius;
            m2 = m1;
            m1 = r;
        }
    }
    *n_unpred = u;
    return kOk;
}

// Huffman code lengths (HuffmanEncoder.hpp:1001-1083): leaves for the states s = symbol - lo with
// a nonzero count, in state order, into the reference's binary min-heap (a new node climbs while
// its parent's count is larger; the removal sifts down to the smaller child, the right one only
// when strictly smaller), the two smallest merged until one node is left; a leaf's length is its
// depth (a lone leaf: 0).  nodes: 2 * nstates entries, heap: 2 * nstates + 1 entries of scratch.
struct HuffNode {
    unsigned long long freq;
    int kid0, kid1;  // children; -1 for a leaf
    uint32_t state;
};

__host__ __device__ inline void heap_up(int *heap, int &end, const HuffNode *nodes, int x) {
    int at = end++;
    while (at > 1 && nodes[heap[at >> 1]].freq > nodes[x].freq) {
        heap[at] = heap[at >> 1];
        at >>= 1;
    }
    heap[at] = x;
}

__host__ __device__ inline int heap_take(int *heap, int &end, const HuffNode *nodes) {
    const int top = heap[1];
    heap[1] = heap[--end];
    int at = 1;
    while (2 * at < end) {
        int c = 2 * at;
        if (c + 1 < end && nodes[heap[c + 1]].freq < nodes[heap[c]].freq) c++;
        if (nodes[heap[at]].freq <= nodes[heap[c]].freq) break;
        const int t = heap[at];
        heap[at] = heap[c];
        heap[c] = t;
        at = c;
    }
    return top;
}

// freq[s] for s < nstates (= max - lo + 2, the last state always empty); lens[nstates] out.
// Returns the longest length, or -1 when a length would exceed kMaxCodeLen.
__host__ __device__ inline int huff_lengths(const unsigned long long *freq, uint32_t nstates, HuffNode *nodes,
                                            int *heap, uint8_t *lens) {
    int nn = 0, end = 1;
    for (uint32_t s = 0; s < nstates; s++) {
        lens[s] = 0;
        if (!freq[s]) continue;
        nodes[nn] = HuffNode{freq[s], -1, -1, s};
        heap_up(heap, end, nodes, nn++);
    }
    if (end < 2) return 0;
    while (end > 2) {
        const int a = heap_take(heap, end, nodes), b = heap_take(heap, end, nodes);
        nodes[nn] = HuffNode{nodes[a].freq + nodes[b].freq, a, b, 0};
        heap_up(heap, end, nodes, nn++);
    }
    // depths by an explicit stack (reusing heap[] from index 1: at most nn entries of node, depth)
    int maxl = 0, sp = 0;
    int *stack = heap;  // the heap holds one entry now; 2 * nstates + 1 ints of room
    const int root = heap[1];
    stack[sp++] = root;
    stack[sp++] = 0;
    while (sp) {
        const int d = stack[--sp], x = stack[--sp];
        if (nodes[x].kid0 < 0) {
            if (d > kMaxCodeLen) return -1;
            lens[nodes[x].state] = (uint8_t)d;
            if (d > maxl) maxl = d;
        } else {
            stack[sp++] = nodes[x].kid1;
            stack[sp++] = d + 1;
            stack[sp++] = nodes[x].kid0;
            stack[sp++] = d + 1;
        }
    }
    return maxl;
}

// Canonical codes of the lengths (HuffmanEncoder.hpp:897-990): codes assigned in (length, state)
// order, stored first bit in bit 0; and the reference decoder's table flag, from how many symbols
// (freq) have length 1 and lengths 2..10.  Returns the table flag.
__host__ __device__ inline int huff_codes(const uint8_t *lens, const unsigned long long *freq, uint32_t nstates,
                                          unsigned long long total, uint32_t *codes) {
    uint32_t count[kMaxCodeLen + 1] = {0}, next[kMaxCodeLen + 1] = {0}, lfreq[kMaxCodeLen + 1] = {0};
    int maxl = 0;
    for (uint32_t s = 0; s < nstates; s++) {
        codes[s] = 0;
        if (lens[s]) {
            count[lens[s]]++;
            lfreq[lens[s]] += (uint32_t)freq[s];  // 32-bit sums, as the reference keeps them
            if (lens[s] > maxl) maxl = lens[s];
        }
    }
    if (maxl == 0) return 0;
    uint32_t c = 0;
    for (int l = 1; l <= maxl; l++) {
        c = (c + (l > 1 ? count[l - 1] : 0)) << 1;
        next[l] = c;
    }
    for (uint32_t s = 0; s < nstates; s++) {
        const int l = lens[s];
        if (!l) continue;
        const uint32_t msb = next[l]++;
        uint32_t r = 0;
        for (int b = 0; b < l; b++) r |= ((msb >> b) & 1u) << (l - 1 - b);
        codes[s] = r;
    }
    unsigned long long table = 0;
    for (int l = 2; l <= maxl && l <= 10; l++) table += lfreq[l];
    const unsigned long long rest = total - table - lfreq[1];
    const bool no_table = (double)rest >= (double)table * 0.88 || (double)lfreq[1] / (double)total >= 0.98;
    return no_table ? 0 : 1;
}

// Packs the codes of sym[i0, i1) starting at bit `bit` of out (first bit of a code first, bytes
// filled from bit 0); bytes the range shares with a neighbour are OR-ed (the caller zeroes out).
__host__ __device__ inline void huff_pack(const int32_t *sym, size_t i0, size_t i1, uint32_t offset,
                                          const uint8_t *lens, const uint32_t *codes, unsigned long long bit,
                                          uint8_t *out) {
    for (size_t i = i0; i < i1; i++) {
        const uint32_t s = (uint32_t)sym[i] - offset;
        const uint32_t c = codes[s];
        for (int b = 0, l = lens[s]; b < l; b++, bit++)
            if ((c >> b) & 1u) out[bit >> 3] |= (uint8_t)(1u << (bit & 7));
    }
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
