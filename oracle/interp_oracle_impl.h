/*
 * ORACLE — test infrastructure.  Type-generic body of oracle/interp_oracle.c, included once
 * for float (T=float) and once for double.  See interp_oracle.c for what it restates.
 */
#define CAT2(a, b) a##_##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)

typedef struct {
    int N;
    long dims[4];
    long off[4];
    int cubic;
    int decomp;     /* 0 = compress, 1 = decompress */
    T *x;           /* field, C order (dims[0] slowest) */
    int16_t *q;     /* codes, stream order */
    size_t nq;
    T *u;           /* unpredictable values (anchors first) */
    size_t nu;
    size_t ui;      /* decompress: next unpredictable value */
    double eb, ebx2, ebx2_r;
    int radius;
} FN(ctx_t);

/* utils/Interpolators.hpp:49-117, floating branches (explicit fma, no contraction). */
static T FN(apply)(int f, T a, T b, T c, T d) {
    T t;
    switch (f) {
        case F_EQUAL: return a;
        case F_LINEAR: return (a + b) / 2;
        case F_LINEAR1: return FMA(-(T)0.5, a, (T)1.5 * b);
        case F_QUAD1: t = FMA((T)6, b, -c); t = FMA((T)3, a, t); return t * (T)0.125;
        case F_QUAD2: t = FMA((T)6, b, -a); t = FMA((T)3, c, t); return t * (T)0.125;
        case F_QUAD3: return (3 * a - 10 * b + 15 * c) / 8;
        default: t = (b + c) * (T)9; t = t - a; t = t - d; return t * (T)0.0625;
    }
}

/* quantizer/LinearQuantizer.hpp:49-82 (overwrite) and :84-109 (without overwrite). */
static int FN(quantize)(FN(ctx_t) * c, T *xp, T pred, int overwrite) {
    T x = *xp;
    T diff = x - pred;
    double v = nearbyint((double)diff * c->ebx2_r);
    int qi = (v >= -2147483648.0 && v < 2147483648.0) ? (int)v : (int)0x80000000u; /* x86 cvttsd2si on overflow/NaN */
    if (qi > -c->radius && qi < c->radius) {
        T dq = (T)fma((double)qi, c->ebx2, (double)pred);
        T err = dq - x;
        if (err >= -c->eb && err <= c->eb) {
            if (overwrite) *xp = dq;
            return qi;
        }
    }
    c->u[c->nu++] = x;
    return -c->radius;
}

/* quantizer/LinearQuantizer.hpp:112-133 */
static T FN(recover)(FN(ctx_t) * c, T pred, int qi) {
    if (qi != -c->radius) return (T)fma((double)qi, c->ebx2, (double)pred);
    return c->u[c->ui++];
}

/* One target: base = element offset of the line start (pass index 0), step = element step
 * of one grid unit along the pass line, t = index along the line. */
static void FN(visit)(FN(ctx_t) * c, long base, long step, long t, rule_t r, int overwrite) {
    T *x = c->x;
    T a = x[base + r.o[0] * step];
    T b = (r.f != F_EQUAL) ? x[base + r.o[1] * step] : a;
    T cc = (r.f >= F_QUAD1) ? x[base + r.o[2] * step] : a;
    T d = (r.f == F_CUBIC) ? x[base + r.o[3] * step] : a;
    T pred = FN(apply)(r.f, a, b, cc, d);
    T *xp = x + base + t * step;
    if (!c->decomp) {
        c->q[c->nq++] = (int16_t)FN(quantize)(c, xp, pred, overwrite);
    } else {
        *xp = FN(recover)(c, pred, c->q[c->nq++]);
    }
}

static long FN(count)(long dim, long st) { return (dim - 1) / st + 1; }

/* Line pass along dimension pd for the line starting at element `base`. */
static void FN(line)(FN(ctx_t) * c, long base, long pd, long s, int skip) {
    long n = (c->dims[pd] - 1) / s + 1;
    long step = s * c->off[pd];
    if (n <= 1) return;
    for (long t = 1; t < n; t += 2) FN(visit)(c, base, step, t, line_rule(c->cubic, t, n), !skip);
}

/* ---- non-tuning passes (TUNING::DISABLED float path) ---- */

/* 3-D / 2-D row pass along pd, iterated as in interpolation_1d_simd_3d_z (pd=0, outer dim 1),
 * interpolation_1d_simd_3d_y (pd=1, outer dim 0) and interpolation_1d_simd_2d_y (pd=0, no outer). */
static void FN(rows)(FN(ctx_t) * c, long pd, long s, long so, long outer_dim, long sk, long inner_dim, int skip) {
    long n = (c->dims[pd] - 1) / s + 1;
    long step = s * c->off[pd];
    if (n <= 1) return;
    long no = outer_dim >= 0 ? FN(count)(c->dims[outer_dim], so) : 1;
    long nk = FN(count)(c->dims[inner_dim], sk);
    int late_edge = c->cubic && (n % 2 == 0) && n > 2 && c->N == 3; /* the t = n-1 plane after all rows */
    for (long o = 0; o < no; o++) {
        long obase = outer_dim >= 0 ? o * so * c->off[outer_dim] : 0;
        for (long t = 1; t < n; t += 2) {
            if (late_edge && t == n - 1) continue;
            rule_t r = row_rule(c->cubic, t, n, skip);
            for (long k = 0; k < nk; k++) FN(visit)(c, obase + k * sk * c->off[inner_dim], step, t, r, !skip);
        }
    }
    if (late_edge) {
        rule_t r = row_rule(c->cubic, n - 1, n, skip);
        for (long o = 0; o < no; o++) {
            long obase = outer_dim >= 0 ? o * so * c->off[outer_dim] : 0;
            for (long k = 0; k < nk; k++) FN(visit)(c, obase + k * sk * c->off[inner_dim], step, n - 1, r, !skip);
        }
    }
}

/* interpolation() for the non-tuning float path, InterpolationDecomposition.hpp:2294-2527. */
static void FN(level_disabled)(FN(ctx_t) * c, long s, int direction, int last_level) {
    long s2 = 2 * s;
    if (c->N == 1) {
        FN(line)(c, 0, 0, s, last_level);
    } else if (c->N == 2) {
        if (direction == 0) {
            FN(rows)(c, 0, s, 0, -1, s2, 1, 0);
            for (long i = 0; i < c->dims[0]; i += s) FN(line)(c, i * c->off[0], 1, s, last_level);
        } else {
            for (long i = 0; i < c->dims[0]; i += s2) FN(line)(c, i * c->off[0], 1, s, 0);
            FN(rows)(c, 0, s, 0, -1, s, 1, last_level);
        }
    } else {
        if (direction == 0) {
            FN(rows)(c, 0, s, s2, 1, s2, 2, 0);   /* z: rows j outer, planes, x inner */
            FN(rows)(c, 1, s, s, 0, s2, 2, 0);    /* y: planes i outer, rows, x inner */
            for (long i = 0; i < c->dims[0]; i += s)
                for (long j = 0; j < c->dims[1]; j += s) FN(line)(c, i * c->off[0] + j * c->off[1], 2, s, last_level);
        } else {
            for (long i = 0; i < c->dims[0]; i += s2)
                for (long j = 0; j < c->dims[1]; j += s2) FN(line)(c, i * c->off[0] + j * c->off[1], 2, s, 0);
            FN(rows)(c, 1, s, s2, 0, s, 2, 0);
            FN(rows)(c, 0, s, s, 1, s, 2, last_level);
        }
    }
}

/* ---- tuning / 4-D passes ---- */

/* foreach over all dims (row-major, InterpolationDecomposition BlockwiseIterator.hpp:285-324) with the
 * pass dim pd restricted to t in [t0, t1) step 2; other dims use st[d]. */
static void FN(generic_sweep)(FN(ctx_t) * c, long pd, long s, const long *st, long t0, long t1, int use_boundary, int linear_tail) {
    long n = (c->dims[pd] - 1) / s + 1;
    long step = s * c->off[pd];
    long cnt[4], idx[4] = {0, 0, 0, 0};
    long total = 1;
    for (int d = 0; d < c->N; d++) {
        if (d == pd) {
            cnt[d] = t1 > t0 ? (t1 - t0 + 1) / 2 : 0;
        } else {
            cnt[d] = FN(count)(c->dims[d], st[d]);
        }
        total *= cnt[d];
    }
    for (long it = 0; it < total; it++) {
        long rem = it;
        for (int d = c->N - 1; d >= 0; d--) {
            idx[d] = rem % cnt[d];
            rem /= cnt[d];
        }
        long base = 0, t = 0;
        for (int d = 0; d < c->N; d++) {
            if (d == pd) t = t0 + 2 * idx[d];
            else base += idx[d] * st[d] * c->off[d];
        }
        rule_t r;
        if (linear_tail) {
            r = (n < 3) ? mk(F_EQUAL, n - 2, 0, 0, 0) : mk(F_LINEAR1, n - 3, n - 2, 0, 0);
        } else if (use_boundary) {
            r = generic_cubic_boundary_rule(t, n);
        } else if (c->cubic) {
            r = mk(F_CUBIC, t - 3, t - 1, t + 1, t + 3);
        } else {
            r = mk(F_LINEAR, t - 1, t + 1, 0, 0);
        }
        FN(visit)(c, base, step, t, r, 1);
    }
}

/* interpolation_1d_fastest_dim_first, InterpolationDecomposition.hpp:436-528. */
static void FN(generic_pass)(FN(ctx_t) * c, long pd, long s, const long *st) {
    long n = (c->dims[pd] - 1) / s + 1;
    if (n <= 1) return;
    if (!c->cubic) {
        FN(generic_sweep)(c, pd, s, st, 1, n - 1, 0, 0);
        if (n % 2 == 0) FN(generic_sweep)(c, pd, s, st, n - 1, n, 0, 1);
    } else {
        FN(generic_sweep)(c, pd, s, st, 3, (n >= 3) ? n - 3 : 0, 0, 0);
        long b[4];
        int nb = 0;
        b[nb++] = 1;
        if (n % 2 == 1 && n > 3) b[nb++] = n - 2;
        if (n % 2 == 0 && n > 4) b[nb++] = n - 3;
        if (n % 2 == 0 && n > 2) b[nb++] = n - 1;
        for (int i = 0; i < nb; i++) FN(generic_sweep)(c, pd, s, st, b[i], b[i] + 1, 1, 0);
    }
}

/* Legacy 1-D line interpolation_1d, InterpolationDecomposition.hpp:371-419 (always overwrites). */
static void FN(legacy_line)(FN(ctx_t) * c, long base, long pd, long s) {
    long n = (c->dims[pd] - 1) / s + 1;
    long step = s * c->off[pd];
    if (n <= 1) return;
    if (!c->cubic || n < 5) {
        for (long t = 1; t + 1 < n; t += 2) FN(visit)(c, base, step, t, mk(F_LINEAR, t - 1, t + 1, 0, 0), 1);
        if (n % 2 == 0) {
            rule_t r = (n < 4) ? mk(F_EQUAL, n - 2, 0, 0, 0) : mk(F_LINEAR1, n - 4, n - 2, 0, 0);
            FN(visit)(c, base, step, n - 1, r, 1);
        }
    } else {
        long t;
        for (t = 3; t + 3 < n; t += 2) FN(visit)(c, base, step, t, mk(F_CUBIC, t - 3, t - 1, t + 1, t + 3), 1);
        FN(visit)(c, base, step, 1, mk(F_QUAD1, 0, 2, 4, 0), 1);
        FN(visit)(c, base, step, t, mk(F_QUAD2, t - 3, t - 1, t + 1, 0), 1);
        if (n % 2 == 0) FN(visit)(c, base, step, n - 1, mk(F_QUAD3, n - 6, n - 4, n - 2, 0), 1);
    }
}

static const int FN(perm3)[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

static void FN(perm_of)(int N, int direction, int *seq) {
    /* std::next_permutation order over {0..N-1} */
    int a[4];
    for (int i = 0; i < N; i++) a[i] = i;
    for (int it = 0; it < direction; it++) {
        int i = N - 2;
        while (i >= 0 && a[i] >= a[i + 1]) i--;
        if (i < 0) break;
        int j = N - 1;
        while (a[j] <= a[i]) j--;
        int tmp = a[i]; a[i] = a[j]; a[j] = tmp;
        for (int l = i + 1, r = N - 1; l < r; l++, r--) { tmp = a[l]; a[l] = a[r]; a[r] = tmp; }
    }
    for (int i = 0; i < N; i++) seq[i] = a[i];
}

/* interpolation() with TUNING::ENABLED (or N == 4). */
static void FN(level_tuning)(FN(ctx_t) * c, long s, int direction) {
    int seq[4];
    FN(perm_of)(c->N, direction, seq);
    long s2 = 2 * s;
    if (c->N == 1) {
        FN(legacy_line)(c, 0, 0, s);
    } else if (c->N == 2) {
        int d0 = seq[0], d1 = seq[1];
        for (long j = 0; j <= c->dims[d1] - 1; j += s2) FN(legacy_line)(c, j * c->off[d1], d0, s);
        for (long i = 0; i <= c->dims[d0] - 1; i += s) FN(legacy_line)(c, i * c->off[d0], d1, s);
    } else {
        long st[4];
        for (int i = 0; i < c->N; i++) st[i] = s2;
        FN(generic_pass)(c, seq[0], s, st);
        for (int i = 1; i < c->N; i++) {
            st[seq[i - 1]] = s;
            FN(generic_pass)(c, seq[i], s, st);
        }
    }
}

/* Anchor grid in foreach order (InterpolationDecomposition.hpp:341-359). */
static void FN(anchors)(FN(ctx_t) * c, long a) {
    long cnt[4], idx[4], total = 1;
    for (int d = 0; d < c->N; d++) { cnt[d] = FN(count)(c->dims[d], a); total *= cnt[d]; }
    for (long it = 0; it < total; it++) {
        long rem = it, off = 0;
        for (int d = c->N - 1; d >= 0; d--) { idx[d] = rem % cnt[d]; rem /= cnt[d]; }
        for (int d = 0; d < c->N; d++) off += idx[d] * a * c->off[d];
        if (!c->decomp) c->u[c->nu++] = c->x[off];
        else c->x[off] = c->u[c->ui++];
    }
}

static void FN(set_eb)(FN(ctx_t) * c, double eb) {
    c->eb = eb;
    c->ebx2 = 2 * eb;
    c->ebx2_r = 1.0 / c->ebx2;
}

/* InterpolationDecomposition::compress / decompress (hpp:48-128, 131-239). */
static int FN(run)(FN(ctx_t) * c, double eb, int direction, long anchor, double alpha, double beta, int tuning) {
    int level_count = -1, use_anchor = 0;
    for (int d = 0; d < c->N; d++) {
        int lv = (int)ceil(log2((double)c->dims[d]));
        if (level_count < lv) level_count = lv;
        if (c->dims[d] > anchor) use_anchor = 1;
    }
    if (!use_anchor) anchor = 0;
    if (anchor > 0) {
        int maxl = (int)log2((double)anchor) + 1;
        if (maxl <= level_count) level_count = maxl;
    }
    c->radius = 32768;
    /* the constructor's reciprocal (0.5/eb) applies to the anchor-free first point */
    c->eb = eb; c->ebx2 = 2 * eb; c->ebx2_r = 0.5 / eb;
    if (anchor == 0) {
        if (!c->decomp) c->q[c->nq++] = (int16_t)FN(quantize)(c, c->x, 0, 1);
        else c->x[0] = FN(recover)(c, 0, c->q[c->nq++]);
    } else {
        FN(anchors)(c, anchor);
        level_count--;
    }
    for (int level = level_count; level > 0; level--) {
        double cur = eb;
        if (alpha < 0) {
            cur = (level >= 3) ? eb * 0.5 : eb;
        } else if (alpha >= 1) {
            double ratio = pow(alpha, level - 1);
            if (ratio > beta) ratio = beta;
            cur = eb / ratio;
        }
        FN(set_eb)(c, cur);
        long s = 1L << (level - 1);
        if (tuning || c->N == 4) FN(level_tuning)(c, s, direction);
        else FN(level_disabled)(c, s, direction, level == 1);
    }
    return 0;
}

static int FN(setup)(FN(ctx_t) * c, const size_t *dims, int N, int algo) {
    if (N < 1 || N > 4) return -1;
    memset(c, 0, sizeof(*c));
    c->N = N;
    for (int d = 0; d < N; d++) c->dims[d] = (long)dims[d];
    c->off[N - 1] = 1;
    for (int d = N - 2; d >= 0; d--) c->off[d] = c->off[d + 1] * c->dims[d + 1];
    c->cubic = (algo == 1);
    return 0;
}

/* Returns 0 on success.  codes must hold num elements, unpred num + anchors elements. */
int FN(oracle_interp_compress)(const size_t *dims, int N, double eb, int algo, int direction, long anchor,
                                 double alpha, double beta, int tuning, T *data, int16_t *codes, size_t *ncodes,
                                 T *unpred, size_t *nunpred) {
    FN(ctx_t) c;
    if (FN(setup)(&c, dims, N, algo)) return -1;
    c.x = data; c.q = codes; c.u = unpred;
    FN(run)(&c, eb, direction, anchor, alpha, beta, tuning);
    *ncodes = c.nq;
    *nunpred = c.nu;
    return 0;
}

int FN(oracle_interp_decompress)(const size_t *dims, int N, double eb, int algo, int direction, long anchor,
                                   double alpha, double beta, const int16_t *codes, size_t ncodes, const T *unpred,
                                   size_t nunpred, T *out) {
    FN(ctx_t) c;
    if (FN(setup)(&c, dims, N, algo)) return -1;
    c.decomp = 1;
    c.x = out; c.q = (int16_t *)codes; c.u = (T *)unpred;
    FN(run)(&c, eb, direction, anchor, alpha, beta, 0);
    if (c.nq != ncodes || c.ui != nunpred) return -2;
    return 0;
}

#undef CAT2
#undef CAT
#undef FN
