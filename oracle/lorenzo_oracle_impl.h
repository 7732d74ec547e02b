/* ORACLE — test infrastructure.  The T-dependent part of lorenzo_oracle.c (included once per
 * element type with T, SFX and FABS defined).  References in lorenzo_oracle.c's header. */

#define LZ_CAT2(a, b) a##_##b
#define LZ_CAT(a, b) LZ_CAT2(a, b)
#define LZ(name) LZ_CAT(name, SFX)

/* Lorenzo predictions from the values before d (LorenzoPredictor.hpp:67-83, N = 1). */
static T LZ(pred_l1)(const T *d) { return d[-1]; }
static T LZ(pred_l2)(const T *d) { return (T)2 * d[-1] - d[-2]; }

/* LinearQuantizer::quantize_and_overwrite: the code, with *x replaced by its reconstruction, or
 * -radius with *x appended to the unpredictable values. */
static int LZ(quantize)(T *x, T pred, double eb, double ebx2, double ebx2_r, int radius, T *unpred, size_t *nu) {
    const T diff = *x - pred;
    const double v = nearbyint((double)diff * ebx2_r);
    if (v > -radius && v < radius) {
        const int q = (int)v;
        const T dq = (T)fma((double)q, ebx2, (double)pred);
        const T err = dq - *x;
        if ((double)err >= -eb && (double)err <= eb) {
            *x = dq;
            return q;
        }
    }
    unpred[(*nu)++] = *x;
    return -radius;
}

long long LZ(oracle_lorenzo_payload)(const T *x, size_t n, double eb, int radius, int block, uint8_t *out,
                                     size_t cap, T *recon) {
    if (n == 0 || block < 1 || radius < 1 || 2 * (long long)radius > 65536) return -2;
    const size_t nblocks = (n + (size_t)block - 1) / (size_t)block;
    T *buf = calloc(n + 2, sizeof(T));  /* two zero values before the field */
    T *unpred = malloc(sizeof(T) * (n + 1));
    int32_t *codes = malloc(sizeof(int32_t) * n);
    int32_t *sel = malloc(sizeof(int32_t) * nblocks);
    if (!buf || !unpred || !codes || !sel) {
        free(buf);
        free(unpred);
        free(codes);
        free(sel);
        return -3;
    }
    memcpy(buf + 2, x, sizeof(T) * n);
    T *d = buf + 2;
    const double ebx2 = 2 * eb, ebx2_r = 1.0 / ebx2;
    const T noise1 = (T)(0.5 * eb), noise2 = (T)(1.08 * eb);
    size_t nu = 0;
    for (size_t k = 0; k < nblocks; k++) {
        const size_t b0 = k * (size_t)block, m = (n - b0 < (size_t)block) ? n - b0 : (size_t)block;
        /* error estimates at the block's first and last point, in that order */
        double e1 = 0, e2 = 0;
        const size_t at[2] = {b0, b0 + m - 1};
        for (int s = 0; s < 2; s++) e1 += (double)(FABS(d[at[s]] - LZ(pred_l1)(d + at[s])) + noise1);
        for (int s = 0; s < 2; s++) e2 += (double)(FABS(d[at[s]] - LZ(pred_l2)(d + at[s])) + noise2);
        const int sid = e2 < e1 ? 1 : 0;
        sel[k] = sid;
        for (size_t i = b0; i < b0 + m; i++) {
            const T pred = sid ? LZ(pred_l2)(d + i) : LZ(pred_l1)(d + i);
            codes[i] = LZ(quantize)(d + i, pred, eb, ebx2, ebx2_r, radius, unpred, &nu) + radius;
        }
    }
    if (recon) memcpy(recon, d, sizeof(T) * n);

    wr_t w = {out, out + cap, 0};
    int e = 0;
    /* ComposedPredictor::save: the selection count, then its Huffman record */
    const uint64_t ns = nblocks;
    put(&w, &ns, 8);
    book_t b;
    if ((e = book_build(&b, sel, nblocks)) == 0) {
        book_save(&w, &b);
        book_encode(&w, &b, sel, nblocks);
        book_free(&b);
    }
    /* LinearQuantizer::save */
    const uint8_t uid = 2;
    const int32_t rad = radius, nun = (int32_t)nu;
    put(&w, &uid, 1);
    put(&w, &eb, 8);
    put(&w, &rad, 4);
    put(&w, &nun, 4);
    put(&w, unpred, sizeof(T) * nu);
    /* FalconsGenericCompressor: the code count, then the codes' Huffman record */
    const uint64_t nc = n;
    put(&w, &nc, 8);
    if (!e && (e = book_build(&b, codes, n)) == 0) {
        book_save(&w, &b);
        book_encode(&w, &b, codes, n);
        book_free(&b);
    }
    free(buf);
    free(unpred);
    free(codes);
    free(sel);
    if (e) return -10 + e;
    return w.overflow ? -1 : (long long)(w.p - out);
}

long long LZ(oracle_lorenzo_decode)(const uint8_t *p, size_t len, size_t n, int block, T *out) {
    if (block < 1) return -2;
    rd_t r = {p, p + len, 0};
    uint64_t ns;
    get(&r, &ns, 8);
    const size_t nblocks = (n + (size_t)block - 1) / (size_t)block;
    if (r.bad || ns != nblocks) return -20;
    int32_t *sel = malloc(sizeof(int32_t) * (nblocks + 1));
    int32_t *codes = malloc(sizeof(int32_t) * (n + 1));
    T *buf = calloc(n + 2, sizeof(T));
    T *unpred = NULL;
    long long rc = 0;
    book_t b = {0};
    if (!sel || !codes || !buf) {
        rc = -3;
        goto done;
    }
    if (nblocks) {
        if (book_load(&r, &b) || book_decode(&r, &b, nblocks, sel)) {
            rc = -21;
            goto done;
        }
        book_free(&b);
    }
    uint8_t uid;
    double eb;
    int32_t radius, nu;
    get(&r, &uid, 1);
    get(&r, &eb, 8);
    get(&r, &radius, 4);
    get(&r, &nu, 4);
    if (r.bad || uid != 2 || nu < 0 || radius < 1) {
        rc = -22;
        goto done;
    }
    unpred = malloc(sizeof(T) * ((size_t)nu + 1));
    if (!unpred) {
        rc = -3;
        goto done;
    }
    get(&r, unpred, sizeof(T) * (size_t)nu);
    uint64_t nc;
    get(&r, &nc, 8);
    if (r.bad || nc != n) {
        rc = -23;
        goto done;
    }
    if (book_load(&r, &b) || book_decode(&r, &b, n, codes)) {
        rc = -24;
        goto done;
    }
    {
        T *d = buf + 2;
        const double ebx2 = 2 * eb;
        size_t ui = 0;
        for (size_t k = 0; k < nblocks; k++) {
            const size_t b0 = k * (size_t)block, m = (n - b0 < (size_t)block) ? n - b0 : (size_t)block;
            for (size_t i = b0; i < b0 + m; i++) {
                const T pred = sel[k] ? LZ(pred_l2)(d + i) : LZ(pred_l1)(d + i);
                const int q = codes[i] - radius;
                if (q != -radius) {
                    d[i] = (T)fma((double)q, ebx2, (double)pred);
                } else {
                    if (ui >= (size_t)nu) {
                        rc = -25;
                        goto done;
                    }
                    d[i] = unpred[ui++];
                }
            }
        }
        memcpy(out, d, sizeof(T) * n);
        rc = (long long)(r.p - p);
    }
done:
    book_free(&b);
    free(sel);
    free(codes);
    free(buf);
    free(unpred);
    return rc;
}

#undef LZ_CAT2
#undef LZ_CAT
#undef LZ
