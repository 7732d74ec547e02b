// Finite State Entropy (tANS) primitives, host+device, compatible with the FSE stream format that
// the reference links (zstd's standalone FSE v0.9, vendored as include/Falcons/encoder/zfse, and
// documented for zstd in RFC 8878 section 4.1):
//   - normalized-count header ("NCount"):        zfse/fse_compress.c FSE_writeNCount, entropy_common.c FSE_readNCount
//   - count normalization:                        zfse/fse_compress.c FSE_normalizeCount / FSE_normalizeM2
//   - table spread, encode/decode tables:         zfse/fse_compress.c FSE_buildCTable_wksp, fse_decompress.c FSE_buildDTable
//   - 2-state block coding:                       zfse/fse_compress.c FSE_compress_usingCTable_generic
//   - little-endian forward bit writer, backward bit reader: zfse/bitstream.h
// Implemented here from the published algorithm; every routine is a plain sequential function so
// that one GPU thread (or the host) can run it.
#pragma once
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

// ---------------------------------------------------------------- table log choice
__host__ __device__ inline unsigned min_table_log(size_t srcSize, unsigned maxSymbolValue) {
    unsigned a = highbit32((uint32_t)srcSize) + 1;
    unsigned b = highbit32(maxSymbolValue) + 2;
    return a < b ? a : b;
}

__host__ __device__ inline unsigned optimal_table_log(unsigned maxTableLog, size_t srcSize, unsigned maxSymbolValue) {
    unsigned maxBitsSrc = highbit32((uint32_t)(srcSize - 1)) - 2;
    unsigned tableLog = maxTableLog ? maxTableLog : kDefaultTableLog;
    unsigned minBits = min_table_log(srcSize, maxSymbolValue);
    if (maxBitsSrc < tableLog) tableLog = maxBitsSrc;
    if (minBits > tableLog) tableLog = minBits;
    if (tableLog < (unsigned)kMinTableLog) tableLog = kMinTableLog;
    if (tableLog > (unsigned)kMaxTableLog) tableLog = kMaxTableLog;
    return tableLog;
}

// ---------------------------------------------------------------- normalization
// Secondary method for skewed distributions.  Returns false on failure.
__host__ __device__ inline bool normalize_m2(int16_t *norm, uint32_t tableLog, const uint32_t *count, uint64_t total,
                                             uint32_t maxSymbolValue) {
    const int16_t NOT_YET = -2;
    uint32_t distributed = 0;
    const uint32_t lowThreshold = (uint32_t)(total >> tableLog);
    uint32_t lowOne = (uint32_t)((total * 3) >> (tableLog + 1));
    for (uint32_t s = 0; s <= maxSymbolValue; s++) {
        if (count[s] == 0) { norm[s] = 0; continue; }
        if (count[s] <= lowThreshold) { norm[s] = -1; distributed++; total -= count[s]; continue; }
        if (count[s] <= lowOne) { norm[s] = 1; distributed++; total -= count[s]; continue; }
        norm[s] = NOT_YET;
    }
    uint32_t toDistribute = (1u << tableLog) - distributed;
    if (toDistribute == 0) return true;
    if ((total / toDistribute) > lowOne) {
        lowOne = (uint32_t)((total * 3) / (toDistribute * 2));
        for (uint32_t s = 0; s <= maxSymbolValue; s++) {
            if (norm[s] == NOT_YET && count[s] <= lowOne) {
                norm[s] = 1;
                distributed++;
                total -= count[s];
            }
        }
        toDistribute = (1u << tableLog) - distributed;
    }
    if (distributed == maxSymbolValue + 1) {
        uint32_t maxV = 0, maxC = 0;
        for (uint32_t s = 0; s <= maxSymbolValue; s++)
            if (count[s] > maxC) { maxV = s; maxC = count[s]; }
        norm[maxV] = (int16_t)(norm[maxV] + (int16_t)toDistribute);
        return true;
    }
    if (total == 0) {
        for (uint32_t s = 0; toDistribute > 0; s = (s + 1) % (maxSymbolValue + 1))
            if (norm[s] > 0) { toDistribute--; norm[s]++; }
        return true;
    }
    const uint64_t vStepLog = 62 - tableLog;
    const uint64_t mid = (1ULL << (vStepLog - 1)) - 1;
    const uint64_t rStep = (((1ULL << vStepLog) * toDistribute) + mid) / total;
    uint64_t tmpTotal = mid;
    for (uint32_t s = 0; s <= maxSymbolValue; s++) {
        if (norm[s] == NOT_YET) {
            const uint64_t end = tmpTotal + (count[s] * rStep);
            const uint32_t sStart = (uint32_t)(tmpTotal >> vStepLog);
            const uint32_t sEnd = (uint32_t)(end >> vStepLog);
            const uint32_t weight = sEnd - sStart;
            if (weight < 1) return false;
            norm[s] = (int16_t)weight;
            tmpTotal = end;
        }
    }
    return true;
}

// Normalizes `count` (sum `total`) to 2^tableLog; -1 marks a low-probability symbol.
// Returns 0 on failure, 1 for the single-symbol case (not normalized), tableLog otherwise.
__host__ __device__ inline unsigned normalize_count(int16_t *norm, unsigned tableLog, const uint32_t *count,
                                                    uint64_t total, unsigned maxSymbolValue) {
    if (tableLog == 0) tableLog = kDefaultTableLog;
    if (tableLog < (unsigned)kMinTableLog || tableLog > (unsigned)kMaxTableLog) return 0;
    if (tableLog < min_table_log((size_t)total, maxSymbolValue)) return 0;
    const uint32_t rtb[8] = {0, 473195, 504333, 520860, 550000, 700000, 750000, 830000};
    const uint64_t scale = 62 - tableLog;
    const uint64_t step = (1ULL << 62) / total;
    const uint64_t vStep = 1ULL << (scale - 20);
    int still = 1 << tableLog;
    unsigned largest = 0;
    int16_t largestP = 0;
    const uint32_t lowThreshold = (uint32_t)(total >> tableLog);
    for (unsigned s = 0; s <= maxSymbolValue; s++) {
        if (count[s] == total) return 1;
        if (count[s] == 0) { norm[s] = 0; continue; }
        if (count[s] <= lowThreshold) {
            norm[s] = -1;
            still--;
        } else {
            int16_t proba = (int16_t)((count[s] * step) >> scale);
            if (proba < 8) {
                const uint64_t restToBeat = vStep * rtb[proba];
                proba += (count[s] * step) - ((uint64_t)proba << scale) > restToBeat;
            }
            if (proba > largestP) { largestP = proba; largest = s; }
            norm[s] = proba;
            still -= proba;
        }
    }
    if (-still >= (norm[largest] >> 1)) {
        if (!normalize_m2(norm, tableLog, count, total, maxSymbolValue)) return 0;
    } else {
        norm[largest] = (int16_t)(norm[largest] + still);
    }
    return tableLog;
}

// ---------------------------------------------------------------- NCount header
__host__ __device__ inline size_t ncount_bound(unsigned maxSymbolValue, unsigned tableLog) {
    return (((maxSymbolValue + 1) * tableLog) >> 3) + 3;
}

// Writes the normalized-count header; returns its size (0 on an invalid distribution).
__host__ __device__ inline size_t write_ncount(uint8_t *out0, const int16_t *norm, unsigned maxSymbolValue,
                                               unsigned tableLog) {
    uint8_t *out = out0;
    const int tableSize = 1 << tableLog;
    int remaining = tableSize + 1;
    int threshold = tableSize;
    int nbBits = (int)tableLog + 1;
    uint32_t bitStream = (tableLog - kMinTableLog);
    int bitCount = 4;
    unsigned symbol = 0;
    const unsigned alphabetSize = maxSymbolValue + 1;
    bool previousIs0 = false;
    while (symbol < alphabetSize && remaining > 1) {
        if (previousIs0) {
            unsigned start = symbol;
            while (symbol < alphabetSize && !norm[symbol]) symbol++;
            if (symbol == alphabetSize) break;
            while (symbol >= start + 24) {
                start += 24;
                bitStream += 0xFFFFu << bitCount;
                out[0] = (uint8_t)bitStream;
                out[1] = (uint8_t)(bitStream >> 8);
                out += 2;
                bitStream >>= 16;
            }
            while (symbol >= start + 3) {
                start += 3;
                bitStream += 3u << bitCount;
                bitCount += 2;
            }
            bitStream += (symbol - start) << bitCount;
            bitCount += 2;
            if (bitCount > 16) {
                out[0] = (uint8_t)bitStream;
                out[1] = (uint8_t)(bitStream >> 8);
                out += 2;
                bitStream >>= 16;
                bitCount -= 16;
            }
        }
        {
            int count = norm[symbol++];
            const int max = (2 * threshold - 1) - remaining;
            remaining -= count < 0 ? -count : count;
            count++;
            if (count >= threshold) count += max;
            bitStream += (uint32_t)count << bitCount;
            bitCount += nbBits;
            bitCount -= (count < max);
            previousIs0 = (count == 1);
            if (remaining < 1) return 0;
            while (remaining < threshold) { nbBits--; threshold >>= 1; }
        }
        if (bitCount > 16) {
            out[0] = (uint8_t)bitStream;
            out[1] = (uint8_t)(bitStream >> 8);
            out += 2;
            bitStream >>= 16;
            bitCount -= 16;
        }
    }
    if (remaining != 1) return 0;
    out[0] = (uint8_t)bitStream;
    out[1] = (uint8_t)(bitStream >> 8);
    out += (bitCount + 7) / 8;
    return (size_t)(out - out0);
}

__host__ __device__ __forceinline__ uint32_t read_le32_clamped(const uint8_t *p, const uint8_t *end) {
    uint32_t v = 0;
    for (int i = 0; i < 4; i++) {
        const uint8_t b = (p + i < end) ? p[i] : 0;
        v |= (uint32_t)b << (8 * i);
    }
    return v;
}

// Reads a normalized-count header.  Returns the header size, 0 on corruption.
// `*maxSV` is the alphabet bound on input and the last coded symbol on output.
__host__ __device__ inline size_t read_ncount(int16_t *norm, unsigned *maxSV, unsigned *tableLogOut, const uint8_t *in,
                                              size_t size) {
    if (size < 1) return 0;
    const uint8_t *const istart = in;
    const uint8_t *const iend = in + size;
    // The reference reader requires 4 readable bytes; emulate its zero padding for short headers.
    uint8_t pad[8];
    if (size < 4) {
        for (int i = 0; i < 8; i++) pad[i] = i < (int)size ? in[i] : 0;
        unsigned mx = *maxSV, tl = 0;
        size_t r = read_ncount(norm, &mx, &tl, pad, 4);
        if (r == 0 || r > size) return 0;
        *maxSV = mx;
        *tableLogOut = tl;
        return r;
    }
    const uint8_t *ip = istart;
    for (unsigned s = 0; s <= *maxSV; s++) norm[s] = 0;
    uint32_t bitStream = read_le32_clamped(ip, iend);
    int nbBits = (bitStream & 0xF) + kMinTableLog;
    if (nbBits > kAbsMaxTableLog) return 0;
    bitStream >>= 4;
    int bitCount = 4;
    *tableLogOut = nbBits;
    int remaining = (1 << nbBits) + 1;
    int threshold = 1 << nbBits;
    nbBits++;
    unsigned charnum = 0;
    bool previous0 = false;
    while ((remaining > 1) & (charnum <= *maxSV)) {
        if (previous0) {
            unsigned n0 = charnum;
            while ((bitStream & 0xFFFF) == 0xFFFF) {
                n0 += 24;
                if (ip < iend - 5) {
                    ip += 2;
                    bitStream = read_le32_clamped(ip, iend) >> bitCount;
                } else {
                    bitStream >>= 16;
                    bitCount += 16;
                }
            }
            while ((bitStream & 3) == 3) {
                n0 += 3;
                bitStream >>= 2;
                bitCount += 2;
            }
            n0 += bitStream & 3;
            bitCount += 2;
            if (n0 > *maxSV) return 0;
            while (charnum < n0) norm[charnum++] = 0;
            if ((ip <= iend - 7) || (ip + (bitCount >> 3) <= iend - 4)) {
                ip += bitCount >> 3;
                bitCount &= 7;
                bitStream = read_le32_clamped(ip, iend) >> bitCount;
            } else {
                bitStream >>= 2;
            }
        }
        {
            const int max = (2 * threshold - 1) - remaining;
            int count;
            if ((int)(bitStream & (threshold - 1)) < max) {
                count = bitStream & (threshold - 1);
                bitCount += nbBits - 1;
            } else {
                count = bitStream & (2 * threshold - 1);
                if (count >= threshold) count -= max;
                bitCount += nbBits;
            }
            count--;
            remaining -= count < 0 ? -count : count;
            norm[charnum++] = (int16_t)count;
            previous0 = !count;
            while (remaining < threshold) { nbBits--; threshold >>= 1; }
            if ((ip <= iend - 7) || (ip + (bitCount >> 3) <= iend - 4)) {
                ip += bitCount >> 3;
                bitCount &= 7;
            } else {
                bitCount -= (int)(8 * (iend - 4 - ip));
                ip = iend - 4;
            }
            bitStream = read_le32_clamped(ip, iend) >> (bitCount & 31);
        }
    }
    if (remaining != 1) return 0;
    if (bitCount > 32) return 0;
    *maxSV = charnum - 1;
    ip += (bitCount + 7) >> 3;
    return (size_t)(ip - istart);
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

// One FSE block in the format of FSE_compress(src, n) with maxSymbolValue 255 and tableLog 11
// (zfse/fse_compress.c FSE_compress_wksp).  Returns 0 when the block is not compressible, 1 when
// it is a single repeated symbol, otherwise the number of bytes written to dst.
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
    if (n <= 1) return 0;
    unsigned maxSV = 255;
    while (maxSV > 0 && w.count[maxSV] == 0) maxSV--;
    uint32_t maxCount = 0;
    for (unsigned s = 0; s <= maxSV; s++) maxCount = w.count[s] > maxCount ? w.count[s] : maxCount;
    if (maxCount == n) return 1;
    if (maxCount == 1) return 0;
    if (maxCount < (n >> 7)) return 0;
    const unsigned tableLog = optimal_table_log(kDefaultTableLog, n, maxSV);
    if (normalize_count(w.norm, tableLog, w.count, n, maxSV) != tableLog) return 0;
    if (cap < ncount_bound(maxSV, tableLog) + 16) return 0;
    const size_t hdr = write_ncount(dst, w.norm, maxSV, tableLog);
    if (hdr == 0) return 0;
    if (!build_ctable(w.state_table, w.sym_tt, w.sym, w.norm, maxSV, tableLog)) return 0;
    if (n <= 2) return 0;
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
    if (total >= n - 1) return 0;
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
