// Interpolation decomposition on the device: the pass plan and the launchers.
//
// The reference (InterpolationDecomposition.hpp:131-239 / :48-128) sweeps the field level by
// level (stride 2^(l-1)), one 1-D pass per dimension, and emits one int16 code per target in a
// loop order that is specific to each pass.  Here every pass is a PassLaunch: a 3-index box
// (a, b, c) whose points map in closed form to (1) the element offset of the target and of its
// predictor operands and (2) the target's position p in the code stream.  Every target of a
// launch reads only points that no other target of the same launch writes, so one launch is
// embarrassingly parallel; the few targets that read a same-pass target (the linear edge row)
// get a launch of their own that runs after the main one.
#pragma once
#include <vector>

#include "common.cuh"

namespace fb2 {

enum PassKind : int { KIND_ROW = 0, KIND_LINE = 1, KIND_GENERIC = 2, KIND_LEGACY = 3 };

struct PassLaunch {
    int kind;
    int cubic;
    int skip;           // final pass of level 1: no write-back, 3-unit linear edge
    int n;              // grid points along the pass line
    long long step;     // element step of one grid unit along the pass line
    long long A, B, C;  // loop box
    long long sa, sb, sc;
    int t0;             // ROW: t = t0 + 2b
    long long rows_in_group, b_off, p_base;
    int level;          // index into the per-level quantizer parameters
    // KIND_GENERIC / KIND_LEGACY (tuning path and 4-D): mixed-radix box over N dims
    int N, pd;
    long long cnt[4], est[4];  // counts and element strides per dim (pass dim: targets)
    int g_t0;                  // pass-dim index of the first target, step 2
    int g_mode;                // 0 body (linear/cubic), 1 cubic boundary rule, 2 linear tail, 3 legacy fixed rule
    int g_rule[5];             // mode 3: formula + operand offsets relative to t
};

struct InterpParams {
    double eb;             // absolute error bound (resolved)
    int cubic;             // interpAlgo
    int direction;         // interpDirection
    long long anchor;      // interpAnchorStride (resolved, >= 0)
    double alpha, beta;    // interpAlpha / interpBeta
    int radius;            // quantbinCnt / 2
    int tuning;            // 1: the auto-tuner's trial path (TUNING::ENABLED)
    double max_abs = -1;   // largest |value| of the field (compress); negative: not known
};

struct InterpPlan {
    int N;
    long long dims[4];
    long long off[4];
    long long num;
    long long anchor;       // 0 when the anchor grid is not used
    long long n_anchor;     // anchors stored in the unpredictable list
    long long n_codes;      // codes emitted
    int first_point;        // anchor-free field: element 0 is quantized against 0 first
    std::vector<QParams> levels;      // index 0: first point (constructor reciprocal), then one per level
    std::vector<PassLaunch> passes;   // in stream order
    std::vector<long long> level_starts;  // first code position of every level (statistics change there)
    double max_abs = -1;    // InterpParams::max_abs
};

// Builds the pass plan; throws std::invalid_argument for unsupported parameters.
InterpPlan make_plan(const long long *dims, int N, const InterpParams &p);

// Scratch needed by the compress/decompress launchers (bytes).
size_t interp_workspace_bytes(const InterpPlan &plan, int elem_size);

// Device times of the pass launches of one call, for measurement: when a LaunchTimes is given,
// a CUDA event pair is recorded on the stream around every pass launch (fused levels are one
// launch each), with the level it codes; read() waits for the events and fills ms.
struct LaunchTimes {
    struct Entry {
        int level;
        cudaEvent_t a, b;
        float ms;
    };
    std::vector<Entry> e;
    void begin(int level, cudaStream_t st);
    void end(cudaStream_t st);
    void read();
    ~LaunchTimes();
};
// Codes of plan level li (an index into plan.levels), from the level starts.
long long level_codes(const InterpPlan &plan, int li);

template <class T>
void interp_compress(const InterpPlan &plan, T *d_x, int16_t *d_codes, T *d_unpred, void *d_ws,
                     unsigned long long *d_n_esc, cudaStream_t st, LaunchTimes *lt = nullptr);

// interp_compress in two steps, so that the caller can size the unpredictable list from the
// escape count (*d_n_esc after the first step) instead of the field: the passes, the escape
// count and its scan; then the anchors and the escape values into d_unpred (n_anchor + count).
template <class T>
void interp_compress_passes(const InterpPlan &plan, T *d_x, int16_t *d_codes, void *d_ws,
                            unsigned long long *d_n_esc, cudaStream_t st, LaunchTimes *lt = nullptr);
template <class T>
void interp_compress_finish(const InterpPlan &plan, const T *d_x, const int16_t *d_codes, T *d_unpred, void *d_ws,
                            cudaStream_t st);

// d_unpred holds n_unpred values: the anchors, then one value per escape code in stream order.
// An escape beyond the list is not read; interp_decompress_check reports it.
template <class T>
void interp_decompress(const InterpPlan &plan, const int16_t *d_codes, const T *d_unpred, long long n_unpred, T *d_x,
                       void *d_ws, cudaStream_t st);

// Waits for the stream and throws std::invalid_argument when the codes of the last
// interp_decompress on d_ws name more escapes than its unpredictable list holds after the anchors
// (the reference's LinearQuantizer::recover would read past its list; the reconstruction is then
// not valid).
void interp_decompress_check(const InterpPlan &plan, int elem_size, const void *d_ws, long long n_unpred,
                             cudaStream_t st);

// Loads, on the current device, every kernel interp_decompress can launch (float and double).
// Under lazy module loading a kernel is otherwise loaded at its first launch, which can allocate
// device memory for its code; calling this once up front moves that cost out of later calls.
cudaError_t interp_decompress_preload();

// max - min over a device array, result left on the device (T) and optionally returned.
template <class T>
void device_range(const T *d_x, long long n, T *d_out_range, void *d_ws, cudaStream_t st);
size_t range_workspace_bytes();

}  // namespace fb2
