/*
 * ORACLE — test infrastructure, not product code.
 *
 * A plain-C restatement of the reference's serial interpolation decomposition
 * (prediction + linear quantization) for float and double fields, used only by the
 * tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the reference
 * of the CUDA path.  Nothing in falcons_b200/ links or calls it.
 *
 * What it restates (reference = JLiu-1/Falcons, include/Falcons/...):
 *   - interpolation formulas           utils/Interpolators.hpp:49-117 (fp-contract off, explicit fma)
 *   - the linear quantizer             quantizer/LinearQuantizer.hpp:49-133
 *   - the level loop and anchor grid   decomposition/InterpolationDecomposition.hpp:48-128, 131-239, 286-359
 *   - the per-pass drivers used by the non-tuning float path:
 *       1-D line   (interp_*_and_quantize_1D_line)   decomposition/Interpolation_quantizer.inl:2623-2700
 *       2-D rows   (interpolation_1d_simd_2d_y)      InterpolationDecomposition.hpp:602-721
 *       2-D lines  (interpolation_1d_simd_2d_x)      InterpolationDecomposition.hpp:723-816
 *       3-D z rows (interpolation_1d_simd_3d_z)      InterpolationDecomposition.hpp:819-1135
 *       3-D y rows (interpolation_1d_simd_3d_y)      InterpolationDecomposition.hpp:1136-1375
 *       3-D x line (interpolation_1d_simd_3d_x)      InterpolationDecomposition.hpp:1378-1428
 *     and their ordering in interpolation()          InterpolationDecomposition.hpp:2294-2527
 *   - the tuning / N=4 path (interpolation_1d_fastest_dim_first, :436-528, and the
 *     legacy 1-D interpolation_1d, :371-419), used by the auto-tuner's trial runs.
 *
 * The restatement is organised differently from the reference: every pass is described
 * by (pass dimension, row-or-line kind, the strides of the other dimensions) and each
 * target's predictor is a closed-form function of its index t along the pass line and
 * the line length n ("rules" below).  Emission order is produced by explicit loops that
 * follow the reference's loop nesting.  Its codes, unpredictable list and reconstruction
 * are pinned bit-for-bit against the reference build (oracle/_ref) by tests/test_oracle.py.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#pragma GCC optimize("fp-contract=off")

enum { F_EQUAL = 0, F_LINEAR, F_LINEAR1, F_QUAD1, F_QUAD2, F_QUAD3, F_CUBIC };

/* A predictor: formula + up to four operand offsets along the pass line (grid units). */
typedef struct {
    int f;
    long o[4];
} rule_t;

static rule_t mk(int f, long a, long b, long c, long d) {
    rule_t r;
    r.f = f;
    r.o[0] = a; r.o[1] = b; r.o[2] = c; r.o[3] = d;
    return r;
}

/* 1-D line rule (Interpolation_quantizer.inl:2623-2700): operands as absolute line indices. */
static rule_t line_rule(int cubic, long t, long n) {
    long odd = n / 2, even = n - odd;
    if (!cubic) {
        if (t < 2 * odd - 1) return mk(F_LINEAR, t - 1, t + 1, 0, 0);
        if (n < 3) return mk(F_EQUAL, 2 * (even - 1), 0, 0, 0);
        return mk(F_LINEAR1, 2 * (even - 2), 2 * (even - 1), 0, 0);
    }
    if (t == 1) {
        if (even < 2) return mk(F_EQUAL, 0, 0, 0, 0);
        if (even < 3) return mk(F_LINEAR, 0, 2, 0, 0);
        return mk(F_QUAD1, 0, 2, 4, 0);
    }
    if (odd < even) { /* n odd: the only edge is t = n-2 */
        if (t == 2 * odd - 1) return mk(F_QUAD2, 2 * (even - 3), 2 * (even - 2), 2 * (even - 1), 0);
    } else {           /* n even: edges t = n-3 (if odd > 2) and t = n-1 */
        if (t == 2 * odd - 1) return mk(F_LINEAR1, 2 * (even - 2), 2 * (even - 1), 0, 0);
        if (odd > 2 && t == 2 * odd - 3) return mk(F_QUAD2, 2 * (even - 3), 2 * (even - 2), 2 * (even - 1), 0);
    }
    return mk(F_CUBIC, t - 3, t - 1, t + 1, t + 3);
}

/* Row-buffer rule (2d_y / 3d_z / 3d_y): skip = final pass of level 1 (last_linear_stride = 3s). */
static rule_t row_rule(int cubic, long t, long n, int skip) {
    if (!cubic) {
        if (t < n - 1) return mk(F_LINEAR, t - 1, t + 1, 0, 0);
        if (n < 3) return mk(F_EQUAL, n - 2, 0, 0, 0);
        return mk(F_LINEAR1, n - 1 - (skip ? 3 : 2), n - 2, 0, 0);
    }
    if (t == 1) {
        if (n >= 5) return mk(F_QUAD1, 0, 2, 4, 0);
        if (n >= 3) return mk(F_LINEAR, 0, 2, 0, 0);
        return mk(F_EQUAL, 0, 0, 0, 0);
    }
    if (n % 2 == 1) {
        if (t == n - 2) return mk(F_QUAD2, n - 5, n - 3, n - 1, 0);
    } else {
        if (t == n - 1) return mk(F_LINEAR1, n - 4, n - 2, 0, 0);
        if (t == n - 3 && n > 4) return mk(F_QUAD2, n - 6, n - 4, n - 2, 0);
    }
    return mk(F_CUBIC, t - 3, t - 1, t + 1, t + 3);
}

/* Boundary rule of interpolation_1d_fastest_dim_first (InterpolationDecomposition.hpp:497-521). */
static rule_t generic_cubic_boundary_rule(long b, long n) {
    if (b >= 3) {
        if (b + 3 < n) return mk(F_CUBIC, b - 3, b - 1, b + 1, b + 3);
        if (b + 1 < n) return mk(F_QUAD2, b - 3, b - 1, b + 1, 0);
        return mk(F_LINEAR1, b - 3, b - 1, 0, 0);
    }
    if (b + 3 < n) return mk(F_QUAD1, b - 1, b + 1, b + 3, 0);
    if (b + 1 < n) return mk(F_LINEAR, b - 1, b + 1, 0, 0);
    return mk(F_EQUAL, b - 1, 0, 0, 0);
}

/* ---------------- type-generic body, instantiated for float and double ---------------- */
#define T float
#define SFX f32
#define FMA fmaf
#include "interp_oracle_impl.h"
#undef T
#undef SFX
#undef FMA

#define T double
#define SFX f64
#define FMA fma
#include "interp_oracle_impl.h"
#undef T
#undef SFX
#undef FMA
