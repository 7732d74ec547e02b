/*
 * ORACLE — test infrastructure, not product code.
 *
 * A plain-C restatement of the reference's 1-D blockwise Lorenzo path, ALGO_LORENZO_REG as the
 * interpolation tuner configures it for 1-D fields (Lorenzo order 1 and order 2 composed per
 * block, block size 5, no regression), up to the payload that the reference hands to its
 * trailing zstd stage, and the matching decoder.  Used only by tests/ and
 * tests/golden/make_golden.py as the reference restatement of that path; nothing in falcons_b200/ links it.
 *
 * What it restates (reference = JLiu-1/Falcons, include/Falcons/...):
 *   - the blockwise decomposition    decomposition/BlockwiseDecomposition.hpp:28-72: blocks of
 *     `block` points in index order, codes biased by +radius (the escape becomes 0), two zero
 *     values before the field (block_data padding, utils/BlockwiseIterator.hpp:202-240)
 *   - the per-block predictor choice predictor/ComposedPredictor.hpp:25-50: the error estimate
 *     of each predictor summed in double over the block's first and last point
 *     (utils/BlockwiseIterator.hpp:153-158), the first smallest sum wins
 *   - 1-D Lorenzo orders 1 and 2     predictor/LorenzoPredictor.hpp:17-38 (noise 0.5 eb and
 *     1.08 eb), :56-65 (estimate = |x - pred| + noise), :67-83 (predictions)
 *   - the linear quantizer           quantizer/LinearQuantizer.hpp:49-80, 112-128, 142-152 (save)
 *   - the Huffman coder              encoder/HuffmanEncoder.hpp:1001-1083 (frequencies, leaves
 *     in symbol order), 836-870 (the binary heap and its tie order), 874-890 (code lengths),
 *     897-990 (canonical codes in (length, symbol) order stored LSB-first, the decode-table
 *     flag), 165-181 (save), 200-238 (encode), 570-650 and 429-478 (load, decode)
 *   - the payload layout             compressor/FalconsGenericCompressor.hpp:64-81,
 *     ComposedPredictor.hpp:52-62, BlockwiseDecomposition.hpp:75-79
 *
 * Its payload bytes and reconstruction are pinned against the reference build (oracle/_ref)
 * by tests/test_lorenzo_oracle.py, and by the golden vectors that tests/golden/make_golden.py
 * writes from that build.
 *
 * Entry points:
 *   long long oracle_lorenzo_payload_{f32,f64}(const T *x, size_t n, double eb, int radius,
 *                                              int block, uint8_t *out, size_t cap, T *recon)
 *       the payload bytes (or -1 when cap is too small) and the reconstruction
 *   long long oracle_lorenzo_decode_{f32,f64}(const uint8_t *p, size_t len, size_t n, int block,
 *                                             T *out)
 *       the bytes consumed (or a negative error code)
 *   long long oracle_huffman_encode(const int32_t *sym, size_t n, uint8_t *out, size_t cap)
 *   long long oracle_huffman_decode(const uint8_t *p, size_t len, size_t n, int32_t *out)
 *       one Huffman record ([offset word][state count][lengths][u64 bytes][bits]) alone
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#pragma GCC optimize("fp-contract=off")

/* ------------------------------------------------------------------ byte writer / reader */
typedef struct {
    uint8_t *p, *end;
    int overflow;
} wr_t;

static void put(wr_t *w, const void *v, size_t n) {
    if ((size_t)(w->end - w->p) < n) {
        w->overflow = 1;
        w->p = w->end;
        return;
    }
    memcpy(w->p, v, n);
    w->p += n;
}

typedef struct {
    const uint8_t *p, *end;
    int bad;
} rd_t;

static void get(rd_t *r, void *v, size_t n) {
    if ((size_t)(r->end - r->p) < n) {
        r->bad = 1;
        memset(v, 0, n);
        r->p = r->end;
        return;
    }
    memcpy(v, r->p, n);
    r->p += n;
}

/* ------------------------------------------------------------------ Huffman coder */
/* A code book over the states s = symbol - offset, 0 <= s < nstates = max - offset + 2. */
typedef struct {
    uint32_t offset, nstates;
    uint8_t *len;   /* code length of every state, 0 when unused */
    uint32_t *code; /* its code, first bit in bit 0 */
    int table;      /* the reference decoder's table flag (bit 31 of the saved offset word) */
} book_t;

static void book_free(book_t *b) {
    free(b->len);
    free(b->code);
    b->len = NULL;
    b->code = NULL;
}

typedef struct {
    uint64_t freq;
    int kid[2]; /* children, -1 for a leaf */
    uint32_t state;
} hnode_t;

/* The reference's binary min-heap over node frequencies (1-based, `end` one past the last). */
static void heap_push(int *heap, int *end, const hnode_t *nodes, int x) {
    int at = (*end)++;
    while (at > 1) {
        const int up = at >> 1;
        if (nodes[heap[up]].freq <= nodes[x].freq) break;
        heap[at] = heap[up];
        at = up;
    }
    heap[at] = x;
}

static int heap_pop(int *heap, int *end, const hnode_t *nodes) {
    if (*end < 2) return -1;
    const int top = heap[1];
    (*end)--;
    heap[1] = heap[*end];
    int at = 1;
    for (;;) {
        int c = at * 2;
        if (c >= *end) break;
        if (c + 1 < *end && nodes[heap[c + 1]].freq < nodes[heap[c]].freq) c++;
        if (!(nodes[heap[at]].freq > nodes[heap[c]].freq)) break;
        const int t = heap[at];
        heap[at] = heap[c];
        heap[c] = t;
        at = c;
    }
    return top;
}

static uint32_t reverse_bits(uint32_t v, int n) {
    uint32_t r = 0;
    for (int i = 0; i < n; i++) r |= ((v >> i) & 1u) << (n - 1 - i);
    return r;
}

/* Code lengths of the Huffman tree of the frequencies, canonical codes, the table flag. */
static int book_build(book_t *b, const int32_t *sym, size_t n) {
    memset(b, 0, sizeof(*b));
    if (n == 0) return -1;
    uint64_t *freq = calloc(65536, sizeof(uint64_t));
    if (!freq) return -2;
    for (size_t i = 0; i < n; i++) {
        if (sym[i] < 0 || sym[i] >= 65536) {
            free(freq);
            return -3;
        }
        freq[sym[i]]++;
    }
    uint32_t lo = 0, hi = 65535;
    while (!freq[lo]) lo++;
    while (!freq[hi]) hi--;
    b->offset = lo;
    b->nstates = hi - lo + 2;
    b->len = calloc(b->nstates, 1);
    b->code = calloc(b->nstates, sizeof(uint32_t));
    const size_t cap_nodes = 2 * (size_t)b->nstates + 2;
    hnode_t *nodes = calloc(cap_nodes, sizeof(hnode_t));
    int *heap = calloc(cap_nodes + 1, sizeof(int));
    if (!b->len || !b->code || !nodes || !heap) {
        free(freq);
        free(nodes);
        free(heap);
        book_free(b);
        return -2;
    }
    int nn = 0, end = 1;
    for (uint32_t s = lo; s <= hi; s++) {
        if (!freq[s]) continue;
        nodes[nn] = (hnode_t){freq[s], {-1, -1}, s - lo};
        heap_push(heap, &end, nodes, nn++);
    }
    while (end > 2) {
        const int a = heap_pop(heap, &end, nodes), c = heap_pop(heap, &end, nodes);
        nodes[nn] = (hnode_t){nodes[a].freq + nodes[c].freq, {a, c}, 0};
        heap_push(heap, &end, nodes, nn++);
    }
    /* depths of the leaves (a lone leaf is the root: length 0) */
    {
        int *stack = malloc(sizeof(int) * (size_t)(nn + 1) * 2);
        int sp = 0;
        stack[sp++] = heap[1];
        stack[sp++] = 0;
        int maxd = 0;
        while (sp) {
            const int d = stack[--sp], x = stack[--sp];
            if (nodes[x].kid[0] < 0) {
                b->len[nodes[x].state] = (uint8_t)d;
                if (d > maxd) maxd = d;
            } else {
                stack[sp++] = nodes[x].kid[1];
                stack[sp++] = d + 1;
                stack[sp++] = nodes[x].kid[0];
                stack[sp++] = d + 1;
            }
        }
        free(stack);
        if (maxd > 32) {
            free(freq);
            free(nodes);
            free(heap);
            book_free(b);
            return -4;
        }
        /* canonical codes: by length, then by state; counts and first codes per length */
        if (maxd > 0) {
            uint32_t count[34] = {0}, first[34] = {0}, len_freq[34] = {0};
            for (uint32_t s = 0; s < b->nstates; s++)
                if (b->len[s]) {
                    count[b->len[s]]++;
                    len_freq[b->len[s]] += (uint32_t)freq[s + lo];
                }
            uint32_t c = 0;
            for (int l = 1; l <= maxd; l++) {
                c = (c + (l > 1 ? count[l - 1] : 0)) << 1;
                first[l] = c;
            }
            for (int l = 1; l <= maxd; l++)
                for (uint32_t s = 0; s < b->nstates; s++)
                    if (b->len[s] == l) b->code[s] = reverse_bits(first[l]++, l);
            uint64_t table_freq = 0;
            for (int l = 2; l <= maxd && l <= 10; l++) table_freq += len_freq[l];
            const uint64_t rest = (uint64_t)n - table_freq - len_freq[1];
            b->table = !((double)rest >= (double)table_freq * 0.88 || (double)len_freq[1] / (double)n >= 0.98);
        }
    }
    free(freq);
    free(nodes);
    free(heap);
    return 0;
}

static void book_save(wr_t *w, const book_t *b) {
    const int32_t word = (int32_t)(((uint32_t)(b->table & 1) << 31) | b->offset);
    put(w, &word, 4);
    const uint8_t be[4] = {(uint8_t)(b->nstates >> 24), (uint8_t)(b->nstates >> 16), (uint8_t)(b->nstates >> 8),
                           (uint8_t)b->nstates};
    put(w, be, 4);
    put(w, b->len, b->nstates);
}

static void book_encode(wr_t *w, const book_t *b, const int32_t *sym, size_t n) {
    uint8_t *size_at = w->p;
    const uint64_t zero = 0;
    put(w, &zero, 8);
    if (w->overflow) return;
    uint8_t *start = w->p;
    uint64_t acc = 0;
    unsigned nb = 0;
    for (size_t i = 0; i < n; i++) {
        const uint32_t s = (uint32_t)sym[i] - b->offset;
        acc |= (uint64_t)b->code[s] << nb;
        nb += b->len[s];
        while (nb >= 8) {
            const uint8_t byte = (uint8_t)acc;
            put(w, &byte, 1);
            acc >>= 8;
            nb -= 8;
        }
    }
    if (nb) {
        const uint8_t byte = (uint8_t)acc;
        put(w, &byte, 1);
    }
    if (w->overflow) return;
    const uint64_t bytes = (uint64_t)(w->p - start);
    memcpy(size_at, &bytes, 8);
}

static int book_load(rd_t *r, book_t *b) {
    memset(b, 0, sizeof(*b));
    int32_t word;
    get(r, &word, 4);
    uint8_t be[4];
    get(r, be, 4);
    if (r->bad) return -1;
    b->table = (int)(((uint32_t)word >> 31) & 1u);
    b->offset = (uint32_t)word & 0x7FFFFFFFu;
    b->nstates = ((uint32_t)be[0] << 24) | ((uint32_t)be[1] << 16) | ((uint32_t)be[2] << 8) | be[3];
    if (b->nstates < 2 || b->nstates > 65538) return -2;
    b->len = malloc(b->nstates);
    b->code = calloc(b->nstates, sizeof(uint32_t));
    if (!b->len || !b->code) return -3;
    get(r, b->len, b->nstates);
    return r->bad ? -1 : 0;
}

/* Decodes n symbols of one record's bit section (canonical codes read first bit first). */
static int book_decode(rd_t *r, const book_t *b, size_t n, int32_t *out) {
    uint64_t bytes;
    get(r, &bytes, 8);
    if (r->bad || bytes > (uint64_t)(r->end - r->p)) return -1;
    const uint8_t *p = r->p, *pend = r->p + bytes;
    r->p = pend;
    int maxl = 0, nonzero = 0;
    uint32_t last = 0;
    for (uint32_t s = 0; s < b->nstates; s++)
        if (b->len[s]) {
            nonzero++;
            last = s;
            if (b->len[s] > maxl) maxl = b->len[s];
        }
    if (b->nstates == 2) {  /* one symbol: no bits */
        const uint32_t s = nonzero == 1 ? last : 0;
        for (size_t i = 0; i < n; i++) out[i] = (int32_t)(b->offset + s);
        return 0;
    }
    if (maxl == 0 || maxl > 32) return -2;
    /* canonical decode: per length the first code, the count and the states in state order */
    uint32_t count[34] = {0}, first[34] = {0}, base[34] = {0};
    for (uint32_t s = 0; s < b->nstates; s++) count[b->len[s]]++;
    count[0] = 0;
    uint32_t c = 0, k = 0;
    for (int l = 1; l <= maxl; l++) {
        c = (c + (l > 1 ? count[l - 1] : 0)) << 1;
        first[l] = c;
        base[l] = k;
        k += count[l];
    }
    uint32_t *order = malloc(sizeof(uint32_t) * (k + 1));
    if (!order) return -3;
    {
        uint32_t at = 0;
        for (int l = 1; l <= maxl; l++)
            for (uint32_t s = 0; s < b->nstates; s++)
                if (b->len[s] == l) order[at++] = s;
    }
    size_t i = 0;
    uint32_t code = 0;
    int l = 0;
    for (; p < pend && i < n; p++) {
        uint8_t byte = *p;
        for (int bit = 0; bit < 8 && i < n; bit++, byte >>= 1) {
            code = (code << 1) | (byte & 1u);
            l++;
            if (l > maxl) {
                free(order);
                return -4;
            }
            if (count[l] && code - first[l] < count[l]) {
                out[i++] = (int32_t)(b->offset + order[base[l] + code - first[l]]);
                code = 0;
                l = 0;
            }
        }
    }
    free(order);
    return i == n ? 0 : -5;
}

long long oracle_huffman_encode(const int32_t *sym, size_t n, uint8_t *out, size_t cap) {
    book_t b;
    const int e = book_build(&b, sym, n);
    if (e) return e;
    wr_t w = {out, out + cap, 0};
    book_save(&w, &b);
    book_encode(&w, &b, sym, n);
    book_free(&b);
    return w.overflow ? -1 : (long long)(w.p - out);
}

long long oracle_huffman_decode(const uint8_t *p, size_t len, size_t n, int32_t *out) {
    rd_t r = {p, p + len, 0};
    book_t b;
    int e = book_load(&r, &b);
    if (!e) e = book_decode(&r, &b, n, out);
    book_free(&b);
    return e ? e : (long long)(r.p - p);
}

/* ------------------------------------------------------------------ the Lorenzo path */
#define T float
#define SFX f32
#define FABS fabsf
#include "lorenzo_oracle_impl.h"
#undef T
#undef SFX
#undef FABS

#define T double
#define SFX f64
#define FABS fabs
#include "lorenzo_oracle_impl.h"
#undef T
#undef SFX
#undef FABS
