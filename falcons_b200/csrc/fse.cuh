// Finite State Entropy (tANS) primitives, host + device, for the FSE block format the reference
// links (zstd's standalone FSE v0.9, vendored as include/Falcons/encoder/zfse; the format is the
// one RFC 8878 section 4.1 documents for zstd):
//   - normalized-count header ("NCount"), RFC 8878 4.1.1: written and read here from the RFC's
//     description, with a plain bit packer;
//   - count normalization: this file's own rule (nearest shares, then single-cell moves by
//     marginal coded size); any normalization is valid, since the counts travel in the header;
//   - table spread and the encode/decode tables: the decoder must rebuild the encoder's cells, so
//     they follow the format's spread step (zfse fse_compress.c FSE_buildCTable_wksp,
//     fse_decompress.c FSE_buildDTable);
//   - 2-state block coding and the little-endian forward / backward bit streams (zfse
//     fse_compress.c FSE_compress_usingCTable_generic, bitstream.h): the stream layout.
// Every routine is a plain sequential function so that one GPU thread (or the host) can run it.
#pragma once
#include <math.h>
#include <stdint.h>

namespace fb2 {
namespace fse {

constexpr int kMinTableLog = 5;
constexpr int kMaxTableLog = 13;        // FSE_MAX_MEMORY_USAGE 15 in the reference's build
constexpr int kDefaultTableLog = 11;    // FSE_DEFAULT_MEMORY_USAGE 13
constexpr int kAbsMaxTableLog = 15;

__host__ __device__ __forceinline__ unsigned highbit32(uint32_t v) {
#ifdef __CUDA_ARCH__
    return 31 - __clz(v);
#else
    return 31 - __builtin_clz(v);
#endif
}

__host__ __device__ __forceinline__ uint32_t table_step(uint32_t tableSize) {
    return (tableSize >> 1) + (tableSize >> 3) + 3;
}

// ---------------------------------------------------------------- table size
// About one table cell per four symbols of the block (cells beyond that cost header bits and
// decoder memory that a short block does not earn back), but at least four cells per distinct
// symbol present (so that rounding a share to whole cells stays a small part of it), within
// [kMinTableLog, maxTableLog].
__host__ __device__ inline unsigned choose_table_log(unsigned maxTableLog, size_t srcSize, unsigned nPresent) {
    unsigned tl = 0;
    for (size_t q = srcSize >> 2; q > 1; q >>= 1) tl++;  // floor(log2(srcSize / 4))
    unsigned need = 2;
    while ((1u << need) < 4u * nPresent) need++;         // 2^need >= 4 * nPresent
    if (tl < need) tl = need;
    if (tl < (unsigned)kMinTableLog) tl = kMinTableLog;
    if (tl > maxTableLog) tl = maxTableLog;
    return tl;
}

// ---------------------------------------------------------------- count normalization
// Shares the 2^tableLog table cells among the present symbols so as to minimise the coded size,
// sum over s of count_s * log2(2^tableLog / cells_s), with at least one cell per present symbol.
// The saving of a symbol's n-th cell, count * log2(n / (n - 1)), is compared through
// count / (n - 1/2) (the midpoint value of count / x on [n - 1, n]) in integer arithmetic, so that
// host and device make the same choice.  Under that measure the best table gives every symbol
// max(1, round(count * mu)) cells for the scale mu that fills the table, so:
//   1. mu starts at cells / total and is refined a few times to (cells - symbols held at one
//      cell) / (count of the others), which absorbs the one-cell floor of rare symbols;
//   2. the few cells still missing or in excess then move one at a time: a missing cell goes to
//      the symbol whose next cell saves most, an excess cell leaves the symbol (above one cell)
//      whose last cell saves least.
// The low-probability mark (-1) is never used.  Returns tableLog on success, 1 when one symbol
// holds the whole count (the caller writes a single-symbol block instead), 0 when the table has
// fewer cells than present symbols.
__host__ __device__ inline unsigned normalize_count(int16_t *norm, unsigned tableLog, const uint32_t *count,
                                                    uint64_t total, unsigned maxSymbolValue) {
    if (tableLog < (unsigned)kMinTableLog || tableLog > (unsigned)kMaxTableLog || total == 0) return 0;
    const uint64_t cells = 1ull << tableLog;
    unsigned present = 0;
    for (unsigned s = 0; s <= maxSymbolValue; s++) {
        if (count[s] == total) return 1;
        present += count[s] != 0;
    }
    if (present > cells) return 0;
    double mu = (double)cells / (double)total;
    int64_t left = 0;
    for (int round = 0; round < 4; round++) {
        uint64_t ones = 0, ones_count = 0;
        left = (int64_t)cells;
        for (unsigned s = 0; s <= maxSymbolValue; s++) {
            if (count[s] == 0) {
                norm[s] = 0;
                continue;
            }
            const double share = floor((double)count[s] * mu + 0.5);  // nearest whole cell (built without FMA contraction)
            uint64_t n = share < (double)cells ? (uint64_t)share : cells;
            if (n <= 1) {
                n = 1;
                ones++;
                ones_count += count[s];
            }
            norm[s] = (int16_t)n;
            left -= (int64_t)norm[s];
        }
        if (left == 0 || ones_count == total) break;
        mu = (double)(cells - ones) / (double)(total - ones_count);
    }
    for (; left > 0; left--) {  // hand out the missing cells
        unsigned best = 0;
        uint64_t bc = 0, bd = 1;  // best saving so far as the fraction bc / bd
        for (unsigned s = 0; s <= maxSymbolValue; s++) {
            if (!count[s]) continue;
            const uint64_t c2 = 2 * (uint64_t)count[s], d = 2 * (uint64_t)norm[s] + 1;  // n + 1 - 1/2
            if (c2 * bd > bc * d) {
                best = s;
                bc = c2;
                bd = d;
            }
        }
        norm[best]++;
    }
    for (; left < 0; left++) {  // take back the cells in excess
        int best = -1;
        uint64_t bc = 0, bd = 1;
        for (unsigned s = 0; s <= maxSymbolValue; s++) {
            if (norm[s] < 2) continue;
            const uint64_t c2 = 2 * (uint64_t)count[s], d = 2 * (uint64_t)norm[s] - 1;  // n - 1/2
            if (best < 0 || c2 * bd < bc * d) {
                best = (int)s;
                bc = c2;
                bd = d;
            }
        }
        if (best < 0) return 0;
        norm[best]--;
    }
    return tableLog;
}

// ---------------------------------------------------------------- NCount header (RFC 8878 4.1.1)
// The bit layout, least significant bit first within little-endian bytes:
//   * 4 bits: tableLog - 5;
//   * for symbols 0, 1, ... until all 2^tableLog cells are given out: v = normalized count + 1
//     (0 stands for the low-probability mark -1).  With R = cells still to give out + 1, v lies in
//     [0, R]; let B be the bit length of R and H = 2^(B-1).  The values below 2^B - 1 - R take B - 1
//     bits; the others take B bits, the values from H upward stored plus (2^B - 1 - R);
//   * after a zero count: the number of further zero counts, as 2-bit fields (3 = three more
//     zeros and another field follows);
//   * padding to a whole byte.

// Upper bound of the header size: 4 bits, then per symbol at most tableLog + 1 bits for its
// value and 2 bits of zero-run fields.
__host__ __device__ inline size_t ncount_bound(unsigned maxSymbolValue, unsigned tableLog) {
    return (4 + (size_t)(maxSymbolValue + 1) * (tableLog + 3) + 7) / 8 + 1;
}

struct NcPacker {
    uint8_t *out;
    size_t bytes;
    uint32_t acc;
    unsigned nb;
    __host__ __device__ void put(uint32_t v, unsigned n) {
        acc |= v << nb;
        nb += n;
        while (nb >= 8) {
            out[bytes++] = (uint8_t)acc;
            acc >>= 8;
            nb -= 8;
        }
    }
    __host__ __device__ size_t finish() {
        if (nb) out[bytes++] = (uint8_t)acc;
        return bytes;
    }
};

struct NcUnpacker {
    const uint8_t *in;
    size_t size;
    size_t bit;  // bits consumed
    __host__ __device__ uint32_t get(unsigned n) {
        uint32_t v = 0;
        for (unsigned i = 0; i < n; i++, bit++) {
            const size_t byte = bit >> 3;
            if (byte < size) v |= (uint32_t)((in[byte] >> (bit & 7)) & 1u) << i;
        }
        return v;
    }
    __host__ __device__ bool overrun() const { return bit > 8 * size; }
};

// Writes the header for `norm` (its counts must fill the 2^tableLog cells); returns its size in
// bytes, 0 when the counts do not fill the table exactly.
__host__ __device__ inline size_t write_ncount(uint8_t *out, const int16_t *norm, unsigned maxSymbolValue,
                                               unsigned tableLog) {
    NcPacker pk{out, 0, 0, 0};
    pk.put(tableLog - kMinTableLog, 4);
    int R = (1 << tableLog) + 1;
    unsigned s = 0;
    while (R > 1) {
        if (s > maxSymbolValue) return 0;
        const int n = norm[s++];
        if (n < -1) return 0;
        const unsigned v = (unsigned)(n + 1);
        const unsigned B = highbit32((uint32_t)R) + 1, H = 1u << (B - 1), shortv = 2 * H - 1 - (unsigned)R;
        if (v < shortv) pk.put(v, B - 1);
        else pk.put(v >= H ? v + shortv : v, B);
        R -= n < 0 ? -n : n;
        if (R < 1) return 0;
        if (n == 0) {
            unsigned z = 0;
            while (s + z <= maxSymbolValue && norm[s + z] == 0) z++;
            if (s + z > maxSymbolValue) return 0;  // cells left but no symbol to take them
            s += z;
            for (; z >= 3; z -= 3) pk.put(3, 2);
            pk.put(z, 2);
        }
    }
    return pk.finish();
}

// Reads a header.  `*maxSV` is the largest symbol the caller accepts on input and the last coded
// symbol on output.  Returns the header size in bytes, 0 when the header is malformed or runs past
// `size` bytes.
__host__ __device__ inline size_t read_ncount(int16_t *norm, unsigned *maxSV, unsigned *tableLogOut, const uint8_t *in,
                                              size_t size) {
    if (size < 1) return 0;
    NcUnpacker up{in, size, 0};
    const unsigned tl = up.get(4) + kMinTableLog;
    if (tl > (unsigned)kAbsMaxTableLog) return 0;
    const unsigned lim = *maxSV;
    for (unsigned s = 0; s <= lim; s++) norm[s] = 0;
    int R = (1 << tl) + 1;
    unsigned s = 0;
    while (R > 1) {
        if (s > lim || up.overrun()) return 0;
        const unsigned B = highbit32((uint32_t)R) + 1, H = 1u << (B - 1), shortv = 2 * H - 1 - (unsigned)R;
        unsigned v = up.get(B - 1);
        if (v >= shortv) {
            v |= up.get(1) << (B - 1);
            if (v >= H) v -= shortv;
        }
        const int n = (int)v - 1;
        norm[s++] = (int16_t)n;
        R -= n < 0 ? -n : n;
        if (n == 0) {
            unsigned f;
            do {
                f = up.get(2);
                s += f;
            } while (f == 3 && !up.overrun());
        }
    }
    if (up.overrun() || s == 0 || s - 1 > lim) return 0;
    *maxSV = s - 1;
    *tableLogOut = tl;
    return (up.bit + 7) / 8;
}

// Chooses how a block of n symbols with histogram `count` is coded: 0 raw, 1 a single repeated
// symbol, 2 FSE with table log *tl and counts `norm` (largest coded symbol *maxSV).
__host__ __device__ inline int plan_block(const uint32_t *count, size_t n, unsigned maxTableLog, int16_t *norm,
                                          unsigned *maxSV, unsigned *tl) {
    if (n <= 2) return 0;
    unsigned m = 255, present = 0;
    while (m > 0 && count[m] == 0) m--;
    for (unsigned s = 0; s <= m; s++) {
        present += count[s] != 0;
        if (count[s] == n) return 1;
    }
    *maxSV = m;
    *tl = choose_table_log(maxTableLog, n, present);
    return normalize_count(norm, *tl, count, n, m) == *tl ? 2 : 0;
}
// ---------------------------------------------------------------- table spread (shared by both sides)
// Fills sym[0..2^tableLog) with the spread symbol of every cell.  Returns false on an invalid table.
__host__ __device__ inline bool spread(uint8_t *sym, const int16_t *norm, unsigned maxSymbolValue, unsigned tableLog) {
    const uint32_t tableSize = 1u << tableLog, mask = tableSize - 1, step = table_step(tableSize);
    uint32_t high = tableSize - 1;
    for (unsigned s = 0; s <= maxSymbolValue; s++)
        if (norm[s] == -1) sym[high--] = (uint8_t)s;
    uint32_t pos = 0;
    for (unsigned s = 0; s <= maxSymbolValue; s++) {
        for (int i = 0; i < norm[s]; i++) {
            sym[pos] = (uint8_t)s;
            pos = (pos + step) & mask;
            while (pos > high) pos = (pos + step) & mask;
        }
    }
    return pos == 0;
}

// Encoding table.  state_table has 2^tableLog entries; sym_tt has maxSymbolValue+1.
struct SymTT {
    int32_t deltaFindState;
    uint32_t deltaNbBits;
};

__host__ __device__ inline bool build_ctable(uint16_t *state_table, SymTT *sym_tt, uint8_t *scratch_sym,
                                             const int16_t *norm, unsigned maxSymbolValue, unsigned tableLog) {
    const uint32_t tableSize = 1u << tableLog;
    if (!spread(scratch_sym, norm, maxSymbolValue, tableLog)) return false;
    uint32_t cumul[257];
    cumul[0] = 0;
    for (unsigned u = 1; u <= maxSymbolValue + 1; u++)
        cumul[u] = cumul[u - 1] + (norm[u - 1] == -1 ? 1 : (uint32_t)norm[u - 1]);
    for (uint32_t u = 0; u < tableSize; u++) state_table[cumul[scratch_sym[u]]++] = (uint16_t)(tableSize + u);
    uint32_t total = 0;
    for (unsigned s = 0; s <= maxSymbolValue; s++) {
        const int n = norm[s];
        if (n == 0) {
            sym_tt[s].deltaNbBits = ((tableLog + 1) << 16) - (1u << tableLog);
            sym_tt[s].deltaFindState = 0;
        } else if (n == -1 || n == 1) {
            sym_tt[s].deltaNbBits = (tableLog << 16) - (1u << tableLog);
            sym_tt[s].deltaFindState = (int32_t)total - 1;
            total++;
        } else {
            const uint32_t maxBitsOut = tableLog - highbit32((uint32_t)(n - 1));
            const uint32_t minStatePlus = (uint32_t)n << maxBitsOut;
            sym_tt[s].deltaNbBits = (maxBitsOut << 16) - minStatePlus;
            sym_tt[s].deltaFindState = (int32_t)total - n;
            total += (uint32_t)n;
        }
    }
    return true;
}

// Decoding table entry (fse_decompress.c FSE_decode_t layout: newState, symbol, nbBits).
struct DEntry {
    uint16_t newState;
    uint8_t symbol;
    uint8_t nbBits;
};

__host__ __device__ inline bool build_dtable(DEntry *dt, const int16_t *norm, unsigned maxSymbolValue,
                                             unsigned tableLog, uint8_t *scratch_sym) {
    const uint32_t tableSize = 1u << tableLog;
    if (!spread(scratch_sym, norm, maxSymbolValue, tableLog)) return false;
    uint16_t next[256];
    for (unsigned s = 0; s <= maxSymbolValue; s++) next[s] = norm[s] == -1 ? 1 : (uint16_t)norm[s];
    for (uint32_t u = 0; u < tableSize; u++) {
        const uint8_t s = scratch_sym[u];
        const uint32_t ns = next[s]++;
        const uint8_t nb = (uint8_t)(tableLog - highbit32(ns));
        dt[u].symbol = s;
        dt[u].nbBits = nb;
        dt[u].newState = (uint16_t)((ns << nb) - tableSize);
    }
    return true;
}

// ---------------------------------------------------------------- bit I/O
// Forward little-endian bit writer (BIT_CStream semantics: LSB-first, bytes little-endian).
struct BitWriter {
    uint8_t *base;
    size_t pos;      // bytes flushed
    size_t cap;
    uint64_t acc;
    unsigned nb;     // bits in acc
    bool overflow;
    __host__ __device__ void init(uint8_t *b, size_t c) {
        base = b;
        cap = c;
        pos = 0;
        acc = 0;
        nb = 0;
        overflow = false;
    }
    __host__ __device__ __forceinline__ void add(uint64_t value, unsigned n) {
        acc |= (value & ((n == 64) ? ~0ULL : ((1ULL << n) - 1))) << nb;
        nb += n;
    }
    __host__ __device__ __forceinline__ void flush() {
        while (nb >= 8) {
            if (pos < cap) base[pos] = (uint8_t)acc;
            else overflow = true;
            pos++;
            acc >>= 8;
            nb -= 8;
        }
    }
    // Appends the end mark and returns the byte size (BIT_closeCStream).
    __host__ __device__ size_t close() {
        add(1, 1);
        flush();
        if (nb > 0) {
            if (pos < cap) base[pos] = (uint8_t)acc;
            else overflow = true;
            pos++;
        }
        return pos;
    }
};

// Backward bit reader over a closed stream (BIT_DStream semantics).
struct BitReader {
    const uint8_t *base;
    int64_t bitpos;   // number of unread bits below the read position
    __host__ __device__ bool init(const uint8_t *b, size_t size) {
        base = b;
        if (size < 1) return false;
        const uint8_t last = b[size - 1];
        if (last == 0) return false;
        bitpos = (int64_t)(size - 1) * 8 + highbit32(last);  // below the end mark
        return true;
    }
    __host__ __device__ __forceinline__ uint32_t read(unsigned n) {
        if (n == 0) return 0;
        bitpos -= n;
        int64_t p = bitpos;
        uint64_t v = 0;
        // gather the bytes covering [p, p+n)
        const int64_t byte0 = p >> 3;
        const int shift = (int)(p & 7);
        const int nbytes = (shift + (int)n + 7) >> 3;
        for (int i = 0; i < nbytes; i++) {
            const int64_t bi = byte0 + i;
            const uint64_t b = bi >= 0 ? base[bi] : 0;
            v |= b << (8 * i);
        }
        return (uint32_t)((v >> shift) & ((1ULL << n) - 1));
    }
};

// Backward bit reader with a 64-bit register window, refilled by aligned 32-bit word loads
// (fast path for device streams; same semantics as BitReader).
struct FastReader {
    const uint8_t *base;
    int64_t size;      // bytes
    int64_t pos;       // bits below the read position
    int64_t lo;        // bit offset of win's bit 0 (multiple of 8)
    uint64_t win;
    __host__ __device__ __forceinline__ uint64_t load8(int64_t byte) const {
#ifdef __CUDA_ARCH__
        if (byte >= 0 && byte + 8 <= size) {
            const uintptr_t a = reinterpret_cast<uintptr_t>(base + byte);
            const uint32_t *w = reinterpret_cast<const uint32_t *>(a & ~uintptr_t(3));
            const int sh = (int)(a & 3) * 8;
            const uint32_t w0 = __ldg(w), w1 = __ldg(w + 1);
            const uint32_t w2 = sh ? __ldg(w + 2) : 0u;
            const uint32_t l = __funnelshift_r(w0, w1, sh), h = __funnelshift_r(w1, w2, sh);
            return (uint64_t)l | ((uint64_t)h << 32);
        }
#endif
        uint64_t v = 0;
        for (int i = 0; i < 8; i++) {
            const int64_t b = byte + i;
            if (b >= 0 && b < size) v |= (uint64_t)base[b] << (8 * i);
        }
        return v;
    }
    // Loads the 64-bit window that ends at the byte boundary at or above bit p + n.
    __host__ __device__ __forceinline__ void refill(int64_t p, unsigned n) {
        const int64_t top = (p + (int64_t)n + 7) >> 3;
        lo = (top - 8) * 8;
        win = load8(top - 8);
    }
    __host__ __device__ bool init(const uint8_t *b, size_t sz) {
        base = b;
        size = (int64_t)sz;
        lo = INT64_MAX;
        win = 0;
        if (sz < 1) return false;
        const uint8_t last = b[sz - 1];
        if (last == 0) return false;
        pos = (int64_t)(sz - 1) * 8 + highbit32(last);
        return true;
    }
    __host__ __device__ __forceinline__ uint32_t read(unsigned n) {
        pos -= n;
        if (pos < lo) refill(pos, n);
        return (uint32_t)((win >> (pos - lo)) & ((1ull << n) - 1));
    }
};

// Backward bit reader over one stream with 32-bit positions (streams shorter than 256 MiB).
struct Reader32 {
    const uint8_t *base;
    int32_t size;
    int32_t pos;
    int32_t lo;
    uint64_t win;
    __device__ __forceinline__ uint64_t load8(int32_t byte) const {
        if (byte >= 0 && byte + 8 <= size) {
            const uintptr_t a = reinterpret_cast<uintptr_t>(base + byte);
            const uint32_t *w = reinterpret_cast<const uint32_t *>(a & ~uintptr_t(3));
            const int sh = (int)(a & 3) * 8;
            const uint32_t w0 = __ldg(w), w1 = __ldg(w + 1);
            const uint32_t w2 = sh ? __ldg(w + 2) : 0u;
            return (uint64_t)__funnelshift_r(w0, w1, sh) | ((uint64_t)__funnelshift_r(w1, w2, sh) << 32);
        }
        uint64_t v = 0;
        for (int i = 0; i < 8; i++) {
            const int32_t b = byte + i;
            if (b >= 0 && b < size) v |= (uint64_t)base[b] << (8 * i);
        }
        return v;
    }
    __device__ bool init(const uint8_t *b, uint32_t sz) {
        base = b;
        size = (int32_t)sz;
        lo = 0x7fffffff;
        win = 0;
        if (sz < 1) return false;
        const uint8_t last = b[sz - 1];
        if (last == 0) return false;
        pos = (int32_t)(sz - 1) * 8 + (int32_t)highbit32(last);
        return true;
    }
    __device__ __forceinline__ uint32_t read(unsigned n) {
        pos -= (int32_t)n;
        if (pos < lo) {
            const int32_t top = (pos + (int32_t)n + 7) >> 3;
            lo = (top - 8) * 8;
            win = load8(top - 8);
        }
        return (uint32_t)(win >> (pos - lo)) & ((1u << n) - 1u);
    }
};

// Backward bit reader for long-running chains: the stream is read as aligned 32-bit words
// (words sharing bytes with neighbouring data are harmless: those bits are never returned for a
// valid stream) and the next two words are prefetched, so a refill never waits on memory.
struct ReaderPF {
    const uint32_t *w;   // aligned word base
    int32_t pos;         // bit position (relative to w) below which bits are unread
    int32_t lo;          // bit offset of win's bit 0 (multiple of 32)
    uint64_t win;
    uint32_t p1, p2;     // words lo/32 - 1 and lo/32 - 2
    __device__ __forceinline__ uint32_t word(int32_t i) const { return i >= 0 ? __ldg(w + i) : 0u; }
    __device__ bool init(const uint8_t *b, uint32_t sz) {
        if (sz < 1) return false;
        const uint8_t last = b[sz - 1];
        if (last == 0) return false;
        const uintptr_t a = reinterpret_cast<uintptr_t>(b);
        w = reinterpret_cast<const uint32_t *>(a & ~uintptr_t(3));
        pos = (int32_t)(a & 3) * 8 + (int32_t)(sz - 1) * 8 + (int32_t)highbit32(last);
        const int32_t top = pos >> 5;
        lo = (top - 1) * 32;
        win = ((uint64_t)word(top) << 32) | word(top - 1);
        p1 = word(top - 2);
        p2 = word(top - 3);
        return true;
    }
    // Starts reading below stream bit `bit` (0 <= bit <= 8 * size), e.g. at a decode checkpoint.
    __device__ void init_at(const uint8_t *b, int32_t bit) {
        const uintptr_t a = reinterpret_cast<uintptr_t>(b);
        w = reinterpret_cast<const uint32_t *>(a & ~uintptr_t(3));
        pos = (int32_t)(a & 3) * 8 + bit;
        const int32_t top = pos >> 5;
        lo = (top - 1) * 32;
        win = ((uint64_t)word(top) << 32) | word(top - 1);
        p1 = word(top - 2);
        p2 = word(top - 3);
    }
    __device__ __forceinline__ uint32_t read(unsigned n) {
        pos -= (int32_t)n;
        if (pos < lo) {
            win = (win << 32) | p1;
            lo -= 32;
            p1 = p2;
            p2 = word((lo >> 5) - 2);
        }
        return (uint32_t)(win >> (pos - lo)) & ((1u << n) - 1u);
    }
    // bits consumed beyond the stream start (0 for a fully consumed valid stream)
    __device__ __forceinline__ int32_t start_bit(const uint8_t *b) const {
        return (int32_t)(reinterpret_cast<uintptr_t>(b) & 3) * 8;
    }
};

// Forward bit writer that stores whole little-endian 32-bit words to a 4-byte aligned buffer.
struct Writer32 {
    uint32_t *out;
    uint32_t cap_words;
    uint32_t nw;        // words stored
    uint64_t acc;
    uint32_t nb;
    bool overflow;
    __device__ void init(uint8_t *b, size_t cap) {
        out = reinterpret_cast<uint32_t *>(b);
        cap_words = (uint32_t)(cap / 4);
        nw = 0;
        acc = 0;
        nb = 0;
        overflow = false;
    }
    __device__ __forceinline__ void add(uint32_t v, unsigned n) {
        acc |= (uint64_t)(v & ((n >= 32) ? 0xffffffffu : ((1u << n) - 1u))) << nb;
        nb += n;
        if (nb >= 32) {
            if (nw < cap_words) out[nw] = (uint32_t)acc;
            else overflow = true;
            nw++;
            acc >>= 32;
            nb -= 32;
        }
    }
    // Appends the end mark; returns the byte length (BIT_closeCStream).
    __device__ size_t close() {
        add(1, 1);
        size_t bytes = (size_t)nw * 4;
        uint8_t *ob = reinterpret_cast<uint8_t *>(out);
        while (nb > 0) {
            if (bytes < (size_t)cap_words * 4) ob[bytes] = (uint8_t)acc;
            else overflow = true;
            bytes++;
            acc >>= 8;
            nb = nb > 8 ? nb - 8 : 0;
        }
        return bytes;
    }
};

}  // namespace fse
}  // namespace fb2

namespace fb2 {
namespace fse {

// One FSE block in the format FSE_decompress reads (zfse/fse_decompress.c): NCount header, then the
// two-state backward bit stream.  Returns 0 when the block is better stored raw, 1 when it is a
// single repeated symbol, otherwise the number of bytes written to dst.
// Scratch: state_table (1<<kMaxTableLog u16), sym_tt (256), spread scratch (1<<kMaxTableLog bytes).
struct BlockScratch {
    uint16_t state_table[1 << kMaxTableLog];
    SymTT sym_tt[256];
    uint8_t sym[1 << kMaxTableLog];
    uint32_t count[256];
    int16_t norm[256];
};

// Same, with w.count already holding the histogram of src.
__host__ __device__ inline size_t compress_block_counted(uint8_t *dst, size_t cap, const uint8_t *src, size_t n,
                                                         BlockScratch &w) {
    unsigned maxSV = 0, tableLog = 0;
    const int mode = plan_block(w.count, n, kDefaultTableLog, w.norm, &maxSV, &tableLog);
    if (mode != 2) return (size_t)mode;
    if (cap < ncount_bound(maxSV, tableLog) + 16) return 0;
    const size_t hdr = write_ncount(dst, w.norm, maxSV, tableLog);
    if (hdr == 0) return 0;
    if (!build_ctable(w.state_table, w.sym_tt, w.sym, w.norm, maxSV, tableLog)) return 0;
    BitWriter bw;
    bw.init(dst + hdr, cap - hdr);
    // S1 carries the even indices, S2 the odd ones; both start from the last symbol of their parity.
    uint32_t st[2];
    for (int k = 0; k < 2; k++) {
        const size_t i = ((n - 1) % 2 == (size_t)k) ? n - 1 : n - 2;
        const SymTT t = w.sym_tt[src[i]];
        const uint32_t nb = (t.deltaNbBits + (1u << 15)) >> 16;
        const uint32_t v = (nb << 16) - t.deltaNbBits;
        st[k] = w.state_table[(int32_t)(v >> nb) + t.deltaFindState];
    }
    for (size_t ii = n - 2; ii-- > 0;) {
        const int k = (int)(ii & 1);
        const SymTT t = w.sym_tt[src[ii]];
        const uint32_t nb = (st[k] + t.deltaNbBits) >> 16;
        bw.add(st[k], nb);
        st[k] = w.state_table[(int32_t)(st[k] >> nb) + t.deltaFindState];
        bw.flush();
    }
    bw.add(st[1], tableLog);
    bw.add(st[0], tableLog);
    bw.flush();
    const size_t body = bw.close();
    // BIT_closeCStream reports overflow when the stream reaches the last 8 bytes of the buffer.
    if (bw.overflow || body + 8 > cap - hdr) return 0;
    const size_t total = hdr + body;
    if (total >= n - 1) return 0;  // no gain over the raw block and its smaller block header
    return total;
}

__host__ __device__ inline size_t compress_block(uint8_t *dst, size_t cap, const uint8_t *src, size_t n,
                                                 BlockScratch &w) {
    if (n <= 1) return 0;
    for (int s = 0; s < 256; s++) w.count[s] = 0;
    for (size_t i = 0; i < n; i++) w.count[src[i]]++;
    return compress_block_counted(dst, cap, src, n, w);
}

// Decodes one FSE block of exactly n symbols (n >= 3) produced by compress_block / FSE_compress.
// Returns false on a malformed header.  dt must hold 1 << kMaxTableLog entries.
__host__ __device__ inline bool decompress_block(uint8_t *out, size_t n, const uint8_t *src, size_t size, DEntry *dt,
                                                 uint8_t *scratch_sym) {
    int16_t norm[256];
    unsigned maxSV = 255, tableLog = 0;
    const size_t hdr = read_ncount(norm, &maxSV, &tableLog, src, size);
    if (hdr == 0 || hdr >= size || tableLog > (unsigned)kMaxTableLog) return false;
    if (!build_dtable(dt, norm, maxSV, tableLog, scratch_sym)) return false;
    BitReader br;
    if (!br.init(src + hdr, size - hdr)) return false;
    uint32_t st[2];
    st[0] = br.read(tableLog);
    st[1] = br.read(tableLog);
    for (size_t i = 0; i < n; i++) {
        const int k = (int)(i & 1);
        const DEntry e = dt[st[k]];
        out[i] = e.symbol;
        if (i + 2 < n) st[k] = e.newState + br.read(e.nbBits);
    }
    return true;
}

}  // namespace fse
}  // namespace fb2
