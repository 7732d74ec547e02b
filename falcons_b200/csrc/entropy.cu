// Device entropy coder in the RleFseEncoder<int16_t> stream format (see entropy.cuh).
//
// Reference (JLiu-1/Falcons include/Falcons/encoder/RleFseEncoder.hpp):
//   preprocess_encode :850-895   method / delta decision from 256 x 32 sampled windows
//   encode (method 0) :897-982   runs of zeros + values as Elias-gamma class bytes + raw mantissas
//   fse_enc / fse_dec :150-187   class bytes FSE-coded in 64 Ki-symbol blocks
//   O1Lut             :354-391   context bucket of the previous code, zigzag symbol, 255 = escape
//   o1_normalize      :410-477   per-context normalization to 2^13
//   encode_o1tans     :582-751   S segments x K reverse-encoded interleaved chunks
//   encode_o1_ovf     :483-575   escape side stream (gamma + FSE, or raw int16)
//   decode            :984-1070, decode_o1tans :753-843
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "assemble.cuh"
#include "entropy.cuh"
#include "fse.cuh"
#include "scan.cuh"

namespace fb2 {
namespace {

constexpr int FBLK = 1 << 16;
constexpr int O1_NCTX = 15;
constexpr int O1_PB = 13;
constexpr int O1_M = 1 << O1_PB;
constexpr int O1_NSYM = 256;
constexpr int kMaxK = 16;

__host__ __device__ __forceinline__ int o1_ctx(int code) {
    // magnitude buckets 1,2,3,4 | 5-7 | 8-11 | >= 12, doubled for the sign (RleFseEncoder.hpp:354-384)
    const int sgn = code < 0;
    const int a = sgn ? -code : code;
    const int m = min(a - 1, 3 + (a > 4) + (a > 7) + (a > 11));
    return a == 0 ? 0 : 1 + m * 2 + sgn;
}

__host__ __device__ __forceinline__ int o1_sym(int code) {
    const uint32_t zz = ((uint32_t)code << 1) ^ (uint32_t)(code >> 31);
    return zz < (uint32_t)(O1_NSYM - 1) ? (int)zz : O1_NSYM - 1;
}

__host__ __device__ __forceinline__ int unzz(uint32_t z) { return (int)((z >> 1) ^ (~(z & 1) + 1)); }

__host__ __device__ __forceinline__ uint32_t zigzag(int v) { return ((uint32_t)v << 1) ^ (uint32_t)(v >> 31); }

// ------------------------------------------------------------------ FSE class blocks
struct BlockJob {
    unsigned long long src;   // offset into the class array
    unsigned n;               // symbols
    unsigned flag;            // decode side: 0 raw, 1 FSE, 2 RLE
    unsigned long long in;    // decode side: offset of the payload (after flag / length)
    unsigned long long inlen; // decode side: payload length
    unsigned ck = 0xFFFFFFFFu; // decode side: first checkpoint of the block (none: all ones)
    unsigned pad = 0;
};

constexpr size_t kBlockSlot = FBLK + 64;

// FSE_compress on the device: header, tables and the 2-state reverse coding of one 64 Ki block
// (zfse/fse_compress.c FSE_compress_wksp).  The two state chains are interleaved and the symbol
// loads are issued ahead of the dependent table lookups.
// Decode checkpoint of an FSE block (two interleaved states): the decoder's bit position and both
// states just before it decodes symbol q * part (q >= 1).  Recorded by the encoder, stored in the
// stream's checkpoint frame, so that one block decodes as independent parts.
struct FseCkpt {
    uint32_t bitpos;
    uint16_t s0, s1;
};

// Decode checkpoint of a tANS chain: before the decoder decodes index lo + q * part (q >= 1), its
// bit position in the chain's stream, its state, the context (of the previous code) and the number
// of escapes the chain has consumed.  Recorded by the encoder into the stream's checkpoint frame.
struct O1Ckpt {
    uint32_t bitpos;
    uint32_t esc;
    uint16_t state;
    uint16_t ctx;
};

// Checkpoints of an n-symbol FSE block: one before every symbol q * part <= n - 3, q >= 1 (the
// last two symbols only initialise the encoder states).
__host__ __device__ __forceinline__ uint32_t fse_ckpt_count(uint32_t n, uint32_t part) {
    return n >= 3 ? (n - 3) / part : 0;
}

// FSE class block encoder (zfse/fse_compress.c FSE_compress), one group of 256 threads per 64
// Ki-symbol block (four groups per CTA, below), the largest blocks first.  The group counts the
// block; its thread 0 normalizes and writes the table header; the group builds the coding tables
// in shared memory (the state table with warp match ranks, the symbol transforms per symbol, and,
// where it fits, the next-state table); two warps then code the two state chains (symbols n-3 .. 0,
// each coded by the state of its index parity) side by side, recording for every symbol only the
// state before it (the emitted bits are its low bits, their count follows from the state and the
// symbol); the group then packs in parallel: a scan of the bit counts gives every symbol its bit
// position, each thread writes the bits of one run of symbols (words shared with a neighbour
// merged with atomicOr), and thread 0 appends the two final states and the end mark.  (The
// chains of these skewed class streams converge too slowly for a speculative split.)  Writes the
// complete fse_enc record ([1][u32 len][data] | [0][raw] | [2][sym]) to the block's slot; the
// record flag goes into bits 56-63 of `sizes`.  `recs` is scratch of kFseRecWords words per block
// (the 16-bit step records of both chains).
constexpr unsigned kFseMaxLog = 11;               // the block coder's table log never exceeds 11
// Next-state table of the chains (dynamic shared memory): for every symbol s from the smallest
// to the largest present one and every state x, twice the coded state minus L, which is the byte
// offset of that state in a table row, so that a chain step is one add and one table load.
// Blocks whose table would not fit (symbol span x L x 2 bytes) take the state-table path.
constexpr size_t kFseNxtBytes = 40 * 1024;
// Per-chain record scratch (16-bit records): a chain's records are indexed by step plus the
// chain's lead (the steps that its first 16-byte symbol word holds above the chain's start).
constexpr unsigned kFseChainRec = FBLK / 2 + 32;
constexpr unsigned kFseRecWords = kFseChainRec;  // both chains, 2 records per word
// The packer's chunk of emission positions and its word buffer (the chunk's bits, at most
// kFseMaxLog per position, plus the partial word in front and one behind), staged with its records,
// symbols and slice offsets in the next-state table's space.
constexpr unsigned kPackChunk = 8192;
constexpr unsigned kStageBatch = 16;  // loads a thread has in flight while staging a chunk
constexpr unsigned kPackWords = kPackChunk * kFseMaxLog / 32 + 2;
static_assert(kPackChunk * 3 + (kPackWords + kPackChunk / 32 + 1) * 4 <= kFseNxtBytes,
              "the packer's staging fits the next-state table's space");
static_assert(kPackChunk % 1024 == 0, "one warp scans the chunk's slices, a whole number per lane");
static_assert(kFseChainRec % 8 == 0, "records of whole symbol words are stored as 16-byte vectors");
struct FseSmem {
    uint32_t count[256];
    uint32_t cumul[257];
    uint32_t scan[256];
    fse::SymTT sym_tt[256];
    int16_t norm[256];
    uint16_t state_table[1 << kFseMaxLog];
    uint8_t sym[1 << kFseMaxLog];
};
// A CTA codes G blocks side by side, one group of kFseGroupThreads threads each, with its own
// shared memory and its own named barrier.  G = 1 when the blocks and the chain encoder's CTAs
// together fit the SMs (a block alone on an SM codes fastest); G = kFseGroups otherwise: the CTA
// fills an SM (registers), so the blocks sit on a quarter as many SMs as one CTA per block would
// spread over, and the chain encoder launched beside them keeps the other SMs.
constexpr unsigned kFseGroups = 4, kFseGroupThreads = 256;
struct FseGroupSmem {
    FseSmem w;
    int mode;
    unsigned tl, hdr, s0, s1, maxsv, i0, i1, minsv, fast, high;
    unsigned lead[2];
    uint32_t sh[32];
    unsigned long long tend[2];  // traced calls: when each chain walk ended
};

// A group's barrier.  bar.sync counts whole warps, so the warp is made convergent first (after
// code where some lanes ran on alone, such as the two chain lanes).
__device__ __forceinline__ void group_sync(unsigned bar) {
    __syncwarp();
    asm volatile("bar.sync %0, %1;" ::"r"(bar), "n"(kFseGroupThreads) : "memory");
}

// Phase times of a block (traced calls only): the global timer at the block's start and after its
// count, plan, tables, chain walk, pack and output, kFsePhases words per block.
constexpr int kFsePhases = 8;
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t)::"memory");
    return t;
}
__device__ __forceinline__ void fse_phase(unsigned long long *phase, unsigned slot, int k) {
    if (phase) phase[(size_t)slot * kFsePhases + k] = global_ns();
}

// Exclusive scan over a group's threads (tid = index in the group), total of the group in `total`.
__device__ __forceinline__ uint32_t group_excl_scan(uint32_t v, uint32_t *sh, uint32_t &total, unsigned tid,
                                                    unsigned bar) {
    constexpr unsigned nw = kFseGroupThreads / 32;
    const unsigned lane = tid & 31u, wid = tid >> 5;
    const uint32_t incl = warp_incl_scan(v);
    if (lane == 31) sh[wid] = incl;
    group_sync(bar);
    if (wid == 0) {
        uint32_t x = lane < nw ? sh[lane] : 0u;
        x = warp_incl_scan(x);
        sh[lane] = x;
    }
    group_sync(bar);
    const uint32_t before = wid ? sh[wid - 1] : 0u;
    total = sh[nw - 1];
    group_sync(bar);
    return before + incl - v;
}

template <unsigned G>
__global__ void __launch_bounds__(G * kFseGroupThreads, 4 / G)
    k_fse_encode_blocks(const uint8_t *__restrict__ cls, const BlockJob *__restrict__ jobs, unsigned njobs,
                        uint8_t *__restrict__ slots, unsigned long long *__restrict__ sizes,
                        uint8_t *__restrict__ scratch, uint32_t part, FseCkpt *__restrict__ cks,
                        uint32_t *__restrict__ recs, const uint32_t *__restrict__ order,
                        unsigned long long *__restrict__ phase) {
    __shared__ FseGroupSmem groups[G];
    extern __shared__ uint4 s_nxt_all[];  // the groups' next-state tables (kFseNxtBytes each)
    const unsigned grp = threadIdx.x / kFseGroupThreads, tid = threadIdx.x % kFseGroupThreads;
    const unsigned slot = blockIdx.x * G + grp;
    if (slot >= njobs) return;  // the other groups synchronise on barriers of their own
    const unsigned bar = 1 + grp;  // named barrier of this group (0 is the CTA's)
    FseGroupSmem &gm = groups[grp];
    FseSmem &w = gm.w;
    uint4 *s_nxt4 = s_nxt_all + (size_t)grp * (kFseNxtBytes / 16);
    int &s_mode = gm.mode;  // 0 raw, 1 RLE, 2 FSE
    unsigned &s_tl = gm.tl, &s_hdr = gm.hdr, &s_s0 = gm.s0, &s_s1 = gm.s1, &s_maxsv = gm.maxsv, &s_i0 = gm.i0,
             &s_i1 = gm.i1, &s_minsv = gm.minsv, &s_fast = gm.fast, &s_high = gm.high;
    unsigned *s_lead = gm.lead;
    uint32_t *s_sh = gm.sh;
    const unsigned b = order[slot];  // the largest blocks first
    if (tid == 0) fse_phase(phase, slot, 0);
    const BlockJob jb = jobs[b];
    const uint8_t *src = cls + jb.src;
    uint8_t *out = slots + (size_t)b * kBlockSlot;
    uint32_t *bw = reinterpret_cast<uint32_t *>(scratch + (size_t)b * kBlockSlot);
    uint32_t *rec = recs + (size_t)b * kFseRecWords;
    FseCkpt *ck = cks ? cks + (size_t)b * (FBLK / part) : nullptr;
    const unsigned n = jb.n;
    for (int s = tid; s < 256; s += kFseGroupThreads) w.count[s] = 0;
    group_sync(bar);
    // Count the symbols: every thread reads a contiguous run of aligned 16-byte words (the pool's
    // allocations are 16-byte aligned with slack behind them) and adds runs of equal symbols with
    // one atomic (the class streams are dominated by a few symbols).
    {
        const unsigned lead = (unsigned)(jb.src & 15u);
        const uint4 *g4 = reinterpret_cast<const uint4 *>(src - lead);
        const unsigned nw = (lead + n + 15) / 16, per = (nw + kFseGroupThreads - 1) / kFseGroupThreads;
        const unsigned w0 = min(nw, tid * per), cnt = min(nw, w0 + per) - w0;
        unsigned cur = 256, run = 0;
        for (unsigned j = 0; j < cnt; j++) {
            const unsigned wi = w0 + j;
            const uint4 v = g4[wi];
#pragma unroll
            for (int h = 0; h < 16; h++) {
                const unsigned bi = wi * 16 + h;
                if (bi < lead || bi >= lead + n) continue;
                const uint32_t qw = h < 4 ? v.x : h < 8 ? v.y : h < 12 ? v.z : v.w;
                const unsigned sy = (qw >> ((h & 3) * 8)) & 0xFFu;
                if (sy == cur) {
                    run++;
                } else {
                    if (run) atomicAdd(&w.count[cur], run);
                    cur = sy;
                    run = 1;
                }
            }
        }
        if (run) atomicAdd(&w.count[cur], run);
    }
    group_sync(bar);
    if (tid == 0) fse_phase(phase, slot, 1);
    if (tid == 0) {
        int mode = 0;
        unsigned tl = 0, hdr = 0, maxSV = 255;
        {
            const int plan = fse::plan_block(w.count, n, kFseMaxLog, w.norm, &maxSV, &tl);
            if (plan == 1) {
                mode = 1;
            } else if (plan == 2) {
                if (kBlockSlot - 5 >= fse::ncount_bound(maxSV, tl) + 16) {
                    hdr = (unsigned)fse::write_ncount(out + 5, w.norm, maxSV, tl);
                    // the spread (zfse FSE_buildCTable): the low-probability (-1) symbols take the
                    // top cells; the cells of the others, in symbol order, go to the kept positions
                    // (j * step) & mask <= high in order of j (spread in parallel below; the
                    // sequential walk ends at position 0 exactly when the cells fill the kept
                    // positions)
                    uint32_t c = 0, high = (1u << tl) - 1;
                    for (unsigned s2 = 0; s2 <= maxSV; s2++) {
                        w.scan[s2] = c;
                        if (w.norm[s2] > 0) c += (uint32_t)w.norm[s2];
                        else if (w.norm[s2] == -1) w.sym[high--] = (uint8_t)s2;
                    }
                    w.scan[maxSV + 1] = c;
                    s_high = high;
                    if (hdr && c == high + 1) {
                        mode = 2;
                        w.cumul[0] = 0;
                        for (unsigned u = 1; u <= maxSV + 1; u++)
                            w.cumul[u] = w.cumul[u - 1] + (w.norm[u - 1] == -1 ? 1u : (uint32_t)w.norm[u - 1]);
                    }
                }
            }
        }
        s_mode = mode;
        s_tl = tl;
        s_hdr = hdr;
        s_maxsv = maxSV;
    }
    group_sync(bar);
    if (tid == 0) fse_phase(phase, slot, 2);
    if (s_mode == 2) {
        const unsigned tl = s_tl, L = 1u << tl, maxSV = s_maxsv;
        {
            // parallel spread: thread t ranks the kept positions of j in [t * per, (t + 1) * per)
            const uint32_t step = fse::table_step(L), mask = L - 1, high = s_high;
            const unsigned per = (L + kFseGroupThreads - 1) / kFseGroupThreads;
            const unsigned j0 = min(L, tid * per), j1 = min(L, j0 + per);
            uint32_t cnt = 0;
            for (unsigned j = j0; j < j1; j++) cnt += ((j * step) & mask) <= high;
            uint32_t tot;
            uint32_t kc = group_excl_scan(cnt, s_sh, tot, tid, bar);
            unsigned sy = 0;  // the symbol of cell kc: the last one whose first cell is <= kc
            for (unsigned lo = 0, hi = maxSV + 1; hi - lo > 1;) {
                const unsigned mid = (lo + hi) >> 1;
                if (w.scan[mid] <= kc) lo = mid;
                else hi = mid;
                sy = lo;
            }
            for (unsigned j = j0; j < j1; j++) {
                const uint32_t pos = (j * step) & mask;
                if (pos > high) continue;
                while (w.scan[sy + 1] <= kc) sy++;
                w.sym[pos] = (uint8_t)sy;
                kc++;
            }
            group_sync(bar);
        }
        // state table: the cells of every symbol in increasing order (match ranks within a warp)
        if (tid < 32) {
            const unsigned lane = tid;
            for (unsigned u0 = 0; u0 < L; u0 += 32) {
                const unsigned u = u0 + lane;
                const unsigned sy = u < L ? w.sym[u] : 256u + lane;
                const unsigned peers = __match_any_sync(0xffffffffu, sy);
                const unsigned rank = __popc(peers & ((1u << lane) - 1u));
                if (u < L) w.state_table[w.cumul[sy] + rank] = (uint16_t)(L + u);
                __syncwarp();
                if (u < L && rank == (unsigned)__popc(peers) - 1u) w.cumul[sy] += rank + 1;
                __syncwarp();
            }
        }
        for (unsigned sy = tid; sy <= maxSV; sy += kFseGroupThreads) {
            const int nn = w.norm[sy];
            uint32_t total = 0;  // cells of the symbols before sy
            for (unsigned s2 = 0; s2 < sy; s2++) total += w.norm[s2] == -1 ? 1u : (uint32_t)max(0, (int)w.norm[s2]);
            if (nn == 0) {
                w.sym_tt[sy].deltaNbBits = ((tl + 1) << 16) - L;
                w.sym_tt[sy].deltaFindState = 0;
            } else if (nn == -1 || nn == 1) {
                w.sym_tt[sy].deltaNbBits = (tl << 16) - L;
                w.sym_tt[sy].deltaFindState = (int32_t)total - 1;
            } else {
                const uint32_t maxBitsOut = tl - fse::highbit32((uint32_t)(nn - 1));
                const uint32_t minStatePlus = (uint32_t)nn << maxBitsOut;
                w.sym_tt[sy].deltaNbBits = (maxBitsOut << 16) - minStatePlus;
                w.sym_tt[sy].deltaFindState = (int32_t)total - nn;
            }
        }
        group_sync(bar);
        if (tid == 0) {
            unsigned lo = 0;
            while (lo < maxSV && w.count[lo] == 0) lo++;
            s_minsv = lo;
            s_fast = (size_t)(maxSV - lo + 1) * L * 2 <= kFseNxtBytes;
        }
        group_sync(bar);
        uint16_t *nxt = reinterpret_cast<uint16_t *>(s_nxt4);
        const unsigned minSV = s_minsv;
        const bool fast = s_fast != 0;
        if (fast) {
            for (unsigned e = tid; e < (maxSV - minSV + 1) * L; e += kFseGroupThreads) {
                const unsigned sy = minSV + (e >> tl), x = L + (e & (L - 1));
                if (!w.count[sy]) continue;
                const fse::SymTT t = w.sym_tt[sy];
                const uint32_t nb = (x + t.deltaNbBits) >> 16;
                nxt[e] = (uint16_t)((w.state_table[(int32_t)(x >> nb) + t.deltaFindState] - L) << 1);
            }
            group_sync(bar);
        }
        // The chains run on the group's warps cw, cw + 1, chosen so that the CTA's eight chain warps
        // sit two on each SM sub-partition (warp w of a CTA issues from sub-partition w mod 4).
        const unsigned cw = (2u * grp) & 3u;
        if (tid == 0) fse_phase(phase, slot, 3);
        if ((tid & 31u) == 0 && (tid >> 5) - cw < 2u) {
            // The two state chains, one per warp: chain k codes the symbols i <= n - 3 of parity k
            // from the top down (step j codes symbol top - 2 j), starting from the state that
            // symbol n-1 or n-2 (of parity k) initialised.  Each step records twice the state
            // before it minus L (16 bits, table log <= 11): its low bits are the emitted ones, and
            // the record of the chain's next step holds the state after it.
            const unsigned k = (tid >> 5) - cw;
            uint32_t v;  // the state minus L
            {
                const unsigned i0 = ((n - 1) % 2 == k) ? n - 1 : n - 2;
                const fse::SymTT t = w.sym_tt[src[i0]];
                const uint32_t nb = (t.deltaNbBits + (1u << 15)) >> 16;
                const uint32_t u = (nb << 16) - t.deltaNbBits;
                v = w.state_table[(int32_t)(u >> nb) + t.deltaFindState] - L;
            }
            // the decoder's states before symbols n-3 and n-4 (for checkpoints next to them)
            if (k == 0) s_i0 = v;
            else s_i1 = v;
            const int top = (int)n - 3 - (int)(((n - 3) & 1u) != k);
            const unsigned m = top >= 0 ? (unsigned)top / 2 + 1 : 0;  // steps
            uint16_t *rk = reinterpret_cast<uint16_t *>(rec) + k * kFseChainRec;
            unsigned lead = 0;
            if (fast && m > 0) {
                // The chain's symbols are every other byte of the aligned 16-byte words from the one
                // holding symbol `top` down: eight steps per word (whole words loaded three words
                // ahead), the first word holding `lead` steps above the chain's start.  A step is
                // one add and one load from the next-state table (its entries and the row offsets
                // are byte offsets); the records of a whole word leave as one 16-byte store.
                const uintptr_t a0 = reinterpret_cast<uintptr_t>(src + top);
                const unsigned par = (unsigned)(a0 & 1u), sh = 8u * par;
                lead = (14u + par - (unsigned)(a0 & 15u)) >> 1;
                const unsigned nv = lead + m;
                const uint4 *wp = reinterpret_cast<const uint4 *>(a0 & ~(uintptr_t)15);  // word g at wp - g
                // shared memory: the row of symbol s at byte (s - minSV) << (tl + 1)
                const unsigned char *tb = reinterpret_cast<const unsigned char *>(nxt);
                const unsigned rsh = tl + 1;
                auto step = [&](uint32_t o, uint32_t v2) -> uint32_t {
                    return *reinterpret_cast<const uint16_t *>(tb + o + v2);
                };
                // the chain's bytes of a word at even offsets 14, 12, .., 0 (descending steps), as the
                // byte offsets of their rows in the next-state table
                auto offsets = [&](const uint4 &q, uint32_t *o) {
                    const uint32_t h0 = __funnelshift_r(q.x, q.y, sh), h1 = __funnelshift_r(q.y, q.z, sh);
                    const uint32_t h2 = __funnelshift_r(q.z, q.w, sh), h3 = q.w >> sh;
                    o[0] = (((h3 >> 16) & 0xFFu) - minSV) << rsh;
                    o[1] = ((h3 & 0xFFu) - minSV) << rsh;
                    o[2] = (((h2 >> 16) & 0xFFu) - minSV) << rsh;
                    o[3] = ((h2 & 0xFFu) - minSV) << rsh;
                    o[4] = (((h1 >> 16) & 0xFFu) - minSV) << rsh;
                    o[5] = ((h1 & 0xFFu) - minSV) << rsh;
                    o[6] = (((h0 >> 16) & 0xFFu) - minSV) << rsh;
                    o[7] = ((h0 & 0xFFu) - minSV) << rsh;
                };
                uint32_t v2 = v << 1;  // twice the state minus L
                // steps [t0, t1) of word g one at a time (the partial first and last words)
                auto partial = [&](unsigned g, unsigned t0, unsigned t1) {
                    uint32_t o[8];
                    offsets(wp[-(int)g], o);
#pragma unroll
                    for (unsigned t = 0; t < 8; t++) {
                        if (t < t0 || t >= t1) continue;
                        rk[8 * g + t] = (uint16_t)v2;
                        v2 = step(o[t], v2);
                    }
                };
                const unsigned gs = lead ? 1u : 0u, ge = nv >> 3;  // the whole words [gs, ge)
                if (lead) partial(0, lead, min(8u, nv));
                if (gs < ge) {
                    // Whole words; the symbol words are loaded three words ahead and their row
                    // offsets formed a word ahead, so that only the adds and lookups stay on the chain.
                    uint4 q1 = gs + 1 < ge ? wp[-(int)(gs + 1)] : make_uint4(0, 0, 0, 0);
                    uint4 q2 = gs + 2 < ge ? wp[-(int)(gs + 2)] : make_uint4(0, 0, 0, 0);
                    uint32_t o[8];
                    offsets(wp[-(int)gs], o);
                    for (unsigned g = gs; g < ge; g++) {
                        const uint4 qn = q1;
                        q1 = q2;
                        if (g + 3 < ge) q2 = wp[-(int)(g + 3)];
                        uint32_t on[8];
                        offsets(qn, on);
                        uint32_t r[8];
#pragma unroll
                        for (int t = 0; t < 8; t++) {
                            r[t] = v2;
                            v2 = step(o[t], v2);
                        }
                        *reinterpret_cast<uint4 *>(rk + 8 * g) =
                            make_uint4(r[0] | (r[1] << 16), r[2] | (r[3] << 16), r[4] | (r[5] << 16), r[6] | (r[7] << 16));
#pragma unroll
                        for (int t = 0; t < 8; t++) o[t] = on[t];
                    }
                }
                if (ge >= gs && 8 * ge < nv && (ge > 0 || !lead)) partial(ge, 0, nv - 8 * ge);
                v = v2 >> 1;
            } else if (m > 0) {
                // the state-table path: the symbol transform of the next symbol and the symbol
                // after it are loaded ahead, so that only the state table lookup stays on the chain
                uint32_t sA = v + L;
                int i = top;
                fse::SymTT ta = w.sym_tt[src[i]];
                unsigned ya = src[max(i - 2, 0)];
                for (unsigned j = 0; j < m; j++, i -= 2) {
                    const fse::SymTT na = w.sym_tt[ya];
                    ya = __ldg(src + max(i - 4, 0));
                    const uint32_t nba = (sA + ta.deltaNbBits) >> 16;
                    const uint32_t xa = w.state_table[(int32_t)(sA >> nba) + ta.deltaFindState];
                    rk[j] = (uint16_t)((sA - L) << 1);
                    sA = xa;
                    ta = na;
                }
                v = sA - L;
            }
            s_lead[k] = lead;
            if (k == 0) s_s0 = v + L;
            else s_s1 = v + L;
            // the walk's end, taken by the chain lane itself (a lane that waits at the barrier
            // below may read the timer before the barrier completes)
            if (phase) gm.tend[k] = global_ns();
        }
    }
    group_sync(bar);
    if (tid == 0 && phase) phase[(size_t)slot * kFsePhases + 4] = s_mode == 2 ? max(gm.tend[0], gm.tend[1]) : global_ns();
    int mode = s_mode;
    size_t body = 0;
    if (mode == 2) {
        const unsigned tl = s_tl;
        const unsigned ns = n - 2;  // emission position e codes symbol n - 3 - e
        // the record of emission position e: even positions belong to the chain of n-3's parity
        const unsigned ka = (n - 3) & 1u;
        const unsigned offA = ka * kFseChainRec + s_lead[ka], offB = (ka ^ 1u) * kFseChainRec + s_lead[ka ^ 1u];
        const uint16_t *rec16 = reinterpret_cast<const uint16_t *>(rec);
        // the state minus L before emission position e (symbol n - 3 - e)
        auto V = [&](unsigned e) -> uint32_t { return rec16[((e & 1u) ? offB : offA) + (e >> 1)] >> 1; };
        // the number of bits that state v + L emits for symbol sy
        const uint32_t Lb = 1u << tl;
        auto NB = [&](uint32_t v, unsigned sy) -> uint32_t { return (v + Lb + w.sym_tt[sy].deltaNbBits) >> 16; };
        // The bits leave in chunks of kPackChunk emission positions.  A chunk's records and symbols
        // are staged in shared memory (the next-state table's space, free once the chains are
        // done); lane l of a warp takes position 32 s + l of the chunk's slice s; the slices' bit
        // totals, scanned, and a warp scan within the slice give every position its bit offset; the
        // bits are merged into a shared word buffer, whose words then leave as whole-word stores
        // (the chunk's two edge words, shared with the neighbouring chunks, by atomicOr into the
        // zeroed scratch).  Words past the block's slot are dropped: such a block is stored raw.
        uint16_t *sv = reinterpret_cast<uint16_t *>(s_nxt4);
        uint8_t *ss = reinterpret_cast<uint8_t *>(sv + kPackChunk);
        uint32_t *sw = reinterpret_cast<uint32_t *>(ss + kPackChunk);
        uint32_t *slice = sw + kPackWords;  // kPackChunk / 32 slice offsets, then the chunk's total
        const unsigned lane = tid & 31u, wid = tid >> 5;
        constexpr unsigned kCap = (unsigned)(kBlockSlot / 4);
        {
            const unsigned long long most = (unsigned long long)ns * tl + 2 * tl + 1;
            const unsigned zw = (unsigned)((most + 31) / 32 + 1 < kCap ? (most + 31) / 32 + 1 : kCap);
            for (unsigned z = tid; z < zw; z += kFseGroupThreads) bw[z] = 0u;
        }
        uint32_t base = 0;  // bits of the chunks before
        for (unsigned c0 = 0; c0 < ns; c0 += kPackChunk) {
            const unsigned cn = min(kPackChunk, ns - c0), nsl = (cn + 31) / 32;
            group_sync(bar);  // the previous chunk's words are out (the first time: the scratch is zero)
            // the records come from L2: each thread issues a batch of loads before it stores any
#pragma unroll
            for (unsigned h = 0; h < kPackChunk / kFseGroupThreads; h += kStageBatch) {
                uint32_t r[kStageBatch], y[kStageBatch];
#pragma unroll
                for (unsigned u = 0; u < kStageBatch; u++) {
                    const unsigned j = tid + (h + u) * kFseGroupThreads, e = c0 + j;
                    r[u] = j < cn ? rec16[((e & 1u) ? offB : offA) + (e >> 1)] : 0u;
                    y[u] = j < cn ? src[n - 3 - e] : 0u;
                }
#pragma unroll
                for (unsigned u = 0; u < kStageBatch; u++) {
                    const unsigned j = tid + (h + u) * kFseGroupThreads;
                    if (j < cn) {
                        sv[j] = (uint16_t)r[u];
                        ss[j] = (uint8_t)y[u];
                    }
                }
            }
            for (unsigned z = tid; z < kPackWords; z += kFseGroupThreads) sw[z] = 0u;
            group_sync(bar);
            for (unsigned sl = wid; sl < nsl; sl += kFseGroupThreads / 32) {
                const unsigned j = sl * 32 + lane;
                const uint32_t nb = j < cn ? NB(sv[j] >> 1, ss[j]) : 0u;
                const uint32_t t = __reduce_add_sync(0xffffffffu, nb);
                if (lane == 0) slice[sl] = t;
            }
            group_sync(bar);
            if (wid == 0) {  // exclusive scan of the slice totals; the chunk's total after them
                constexpr unsigned kPer = kPackChunk / 32 / 32;
                uint32_t a[kPer], sum = 0;
#pragma unroll
                for (unsigned q = 0; q < kPer; q++) {
                    const unsigned sl = lane * kPer + q;
                    a[q] = sl < nsl ? slice[sl] : 0u;
                    sum += a[q];
                }
                const uint32_t incl = warp_incl_scan(sum);
                uint32_t run = incl - sum;
#pragma unroll
                for (unsigned q = 0; q < kPer; q++) {
                    const unsigned sl = lane * kPer + q;
                    if (sl < nsl) slice[sl] = run;
                    run += a[q];
                }
                if (lane == 31) slice[kPackChunk / 32] = incl;
            }
            group_sync(bar);
            const uint32_t ctot = slice[kPackChunk / 32], b0 = base & 31u;
            for (unsigned sl = wid; sl < nsl; sl += kFseGroupThreads / 32) {
                const unsigned j = sl * 32 + lane;
                uint32_t v = 0, nb = 0;
                if (j < cn) {
                    v = sv[j] >> 1;
                    nb = NB(v, ss[j]);
                }
                const uint32_t incl = warp_incl_scan(nb);
                const uint32_t p = b0 + slice[sl] + incl - nb;  // bit offset in the chunk's words
                if (nb) {
                    const uint32_t bits = v & ((1u << nb) - 1u), w0 = p >> 5, sh = p & 31u;
                    atomicOr(sw + w0, bits << sh);
                    if (sh + nb > 32) atomicOr(sw + w0 + 1, bits >> (32 - sh));
                }
                if (ck && j < cn) {
                    const unsigned e = c0 + j, i = n - 3 - e;
                    if (i > 0 && (i & (part - 1)) == 0) {
                        // decoder states before symbol i: the states after symbol i (the state
                        // before symbol i - 2 of its chain) and after symbol i + 1 (before i - 1)
                        const uint32_t odd = i + 1 <= n - 3 ? V(e + 1) : ((n - 2) & 1 ? s_i1 : s_i0);
                        ck[i / part - 1] = FseCkpt{base + slice[sl] + incl, (uint16_t)V(e + 2), (uint16_t)odd};
                    }
                }
            }
            group_sync(bar);
            const unsigned wfirst = base >> 5, nw = (b0 + ctot + 31) >> 5;
            for (unsigned z = tid; z < nw; z += kFseGroupThreads) {
                const unsigned gw = wfirst + z;
                if (gw >= kCap) continue;
                if (z == 0 || z == nw - 1) atomicOr(bw + gw, sw[z]);
                else bw[gw] = sw[z];
            }
            base += ctot;
        }
        const uint32_t sym_bits = base;  // bits of all symbols
        const uint32_t total = sym_bits + 2 * tl + 1;
        body = (total + 7) / 8;
        if (body + 8 > kBlockSlot - 5 - s_hdr || s_hdr + body >= n - 1) mode = 0;  // not worth coding: raw
        group_sync(bar);
        if (mode == 2 && tid == 0) {  // final states (odd, then even) and the end mark
            uint32_t p2 = sym_bits;
            auto put = [&](uint32_t v, uint32_t nb) {
                for (uint32_t b = 0; b < nb; b++, p2++)
                    if ((v >> b) & 1u) atomicOr(bw + (p2 >> 5), 1u << (p2 & 31u));
            };
            put(s_s1 & ((1u << tl) - 1), tl);
            put(s_s0 & ((1u << tl) - 1), tl);
            put(1u, 1u);
        }
        group_sync(bar);
    }
    if (tid == 0) fse_phase(phase, slot, 5);
    if (mode == 0) {  // raw
        if (tid == 0) out[0] = 0;
        for (unsigned i = tid; i < n; i += kFseGroupThreads) out[1 + i] = src[i];
        if (tid == 0) sizes[b] = 1 + n;  // flag 0
    } else if (mode == 1) {  // a single repeated symbol
        if (tid == 0) {
            out[0] = 2;
            out[1] = src[0];
            sizes[b] = 2 | (2ULL << 56);
        }
    } else {
        const size_t r = s_hdr + body;
        uint8_t *d = out + 5 + s_hdr;
        const uint8_t *bb = reinterpret_cast<const uint8_t *>(bw);
        for (size_t i = tid; i < body; i += kFseGroupThreads) d[i] = bb[i];
        if (tid == 0) {
            out[0] = 1;
            const uint32_t rr = (uint32_t)r;
            out[1] = (uint8_t)rr;
            out[2] = (uint8_t)(rr >> 8);
            out[3] = (uint8_t)(rr >> 16);
            out[4] = (uint8_t)(rr >> 24);
            sizes[b] = (5 + r) | (1ULL << 56);
        }
    }
    if (phase) {
        group_sync(bar);
        if (tid == 0) fse_phase(phase, slot, 6);
    }
}

// One CTA of kFseDecThreads per 64 Ki block: thread 0 reads the table header, the first warp
// builds the decode table in shared memory (zfse/fse_decompress.c FSE_buildDTable), then the block
// decodes either as one sequence (thread 0, two interleaved states,
// FSE_decompress_usingDTable_generic) or, when the stream carries checkpoints for it, as
// independent parts of `part` symbols, one per thread, each starting from its checkpoint and
// verified against the next one (a mismatch sets err[1] and the caller decodes again without
// checkpoints).
constexpr int kFseDecThreads = 64;  // parts of a block decode one per thread
constexpr unsigned kPartPad = 4;     // bytes between the parts' regions of the decoded block (>= 2:
                                     // the last part may hold two symbols past `part`)
// the decoded block in shared memory: FBLK symbols plus kPartPad per part (parts of >= 64 symbols)
constexpr int kFseDecSmem = FBLK + (FBLK / 64) * kPartPad;
__global__ void __launch_bounds__(kFseDecThreads) k_fse_decode_blocks(const uint8_t *__restrict__ in,
                                                         const BlockJob *__restrict__ jobs,
                                                         uint8_t *__restrict__ cls, int *__restrict__ err,
                                                         uint32_t part, const FseCkpt *__restrict__ cks) {
    __shared__ fse::DEntry dt[1 << fse::kMaxTableLog];
    __shared__ uint8_t sym[1 << fse::kMaxTableLog];
    __shared__ int16_t s_norm[256];
    __shared__ uint32_t s_scan[257], s_next[256];
    __shared__ unsigned tl_sh, hdr_sh, maxsv_sh, high_sh;
    extern __shared__ uint4 s_out4[];  // the block's symbols (FBLK bytes), copied out at the end
    uint8_t *s_out = reinterpret_cast<uint8_t *>(s_out4);
    const BlockJob jb = jobs[blockIdx.x];
    uint8_t *dst = cls + jb.src;
    const uint8_t *p = in + jb.in;
    if (jb.flag == 0) {
        for (unsigned i = threadIdx.x; i < jb.n; i += blockDim.x) dst[i] = p[i];
        return;
    }
    if (jb.flag == 2) {
        const uint8_t v = p[0];
        for (unsigned i = threadIdx.x; i < jb.n; i += blockDim.x) dst[i] = v;
        return;
    }
    const size_t size = (size_t)jb.inlen;
    // The decode table (zfse FSE_buildDTable), built by the warp: lane 0 reads the header and lays
    // the low-probability (-1) symbols on the top cells; the lanes spread the other cells (cell k
    // in symbol order goes to the k-th position (j * step) & mask <= high in order of j) and then
    // number every symbol's cells in cell order (warp match ranks, 32 cells at a time).
    if (threadIdx.x == 0) {
        unsigned maxSV = 255, tl = 0;
        const size_t hdr = fse::read_ncount(s_norm, &maxSV, &tl, p, size);
        bool ok = hdr != 0 && hdr < size && tl <= (unsigned)fse::kMaxTableLog;
        if (ok) {
            uint32_t c = 0, high = (1u << tl) - 1;
            for (unsigned s2 = 0; s2 <= maxSV; s2++) {
                s_scan[s2] = c;
                const int nn = s_norm[s2];
                if (nn > 0) c += (uint32_t)nn;
                else if (nn == -1) sym[high--] = (uint8_t)s2;
                s_next[s2] = nn == -1 ? 1u : (uint32_t)max(nn, 0);
            }
            s_scan[maxSV + 1] = c;
            ok = c == high + 1;  // the sequential spread ends at position 0 exactly then
            high_sh = high;
        }
        tl_sh = ok ? tl : 0xFFFFFFFFu;
        hdr_sh = (unsigned)hdr;
        maxsv_sh = maxSV;
        if (!ok) atomicExch(err, 1);
    }
    __syncthreads();
    const unsigned tl = tl_sh;
    if (tl == 0xFFFFFFFFu) return;
    if (threadIdx.x < 32) {  // the table, by the first warp
        const unsigned lane = threadIdx.x, L = 1u << tl, maxSV = maxsv_sh;
        const uint32_t step = fse::table_step(L), mask = L - 1, high = high_sh;
        const unsigned per = (L + 31) / 32, j0 = min(L, lane * per), j1 = min(L, j0 + per);
        uint32_t cnt = 0;
        for (unsigned j = j0; j < j1; j++) cnt += ((j * step) & mask) <= high;
        uint32_t kc = cnt;  // exclusive warp scan
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, kc, o);
            if (lane >= (unsigned)o) kc += t;
        }
        kc -= cnt;
        unsigned sy = 0;  // the symbol of cell kc: the last one whose first cell is <= kc
        for (unsigned lo = 0, hi = maxSV + 1; hi - lo > 1;) {
            const unsigned mid = (lo + hi) >> 1;
            if (s_scan[mid] <= kc) lo = mid;
            else hi = mid;
            sy = lo;
        }
        for (unsigned j = j0; j < j1; j++) {
            const uint32_t pos = (j * step) & mask;
            if (pos > high) continue;
            while (s_scan[sy + 1] <= kc) sy++;
            sym[pos] = (uint8_t)sy;
            kc++;
        }
        __syncwarp();
        for (unsigned u0 = 0; u0 < L; u0 += 32) {
            const unsigned u = u0 + lane;
            const unsigned sv = u < L ? sym[u] : 256u + lane;
            const unsigned peers = __match_any_sync(0xffffffffu, sv);
            const unsigned rank = __popc(peers & ((1u << lane) - 1u));
            if (u < L) {
                const uint32_t ns = s_next[sv] + rank;
                const uint32_t nb = tl - fse::highbit32(ns);
                dt[u].symbol = (uint8_t)sv;
                dt[u].nbBits = (uint8_t)nb;
                dt[u].newState = (uint16_t)((ns << nb) - L);
            }
            __syncwarp();
            if (u < L && rank == (unsigned)__popc(peers) - 1u) s_next[sv] += rank + 1;
            __syncwarp();
        }
    }
    __syncthreads();
    const uint8_t *sp = p + hdr_sh;
    const uint32_t ssz = (uint32_t)(size - hdr_sh);
    const unsigned n = jb.n;
    const unsigned nparts = jb.ck == 0xFFFFFFFFu ? 1u : 1u + fse_ckpt_count(n, part);
    for (unsigned q = threadIdx.x; q < nparts; q += blockDim.x) {
        fse::ReaderPF br;
        uint32_t s0, s1;
        const unsigned start = q * (nparts > 1 ? part : 0u);
        const unsigned end = q + 1 < nparts ? start + part : n;
        if (q == 0) {
            if (!br.init(sp, ssz)) {
                atomicExch(err, 1);
                continue;
            }
            s0 = br.read(tl);
            s1 = br.read(tl);
        } else {
            const FseCkpt c = cks[jb.ck + q - 1];
            if (c.bitpos >= ssz * 8u || (c.s0 >> tl) || (c.s1 >> tl)) {
                atomicExch(err + 1, 1);
                continue;
            }
            br.init_at(sp, (int32_t)c.bitpos);
            s0 = c.s0;
            s1 = c.s1;
        }
        // Part q's symbols go to its own region of shared memory, kPartPad bytes more than a part
        // apart, four to a word: the parts' word stores then fall on different banks.
        uint8_t *so = s_out + (size_t)q * (nparts > 1 ? part + kPartPad : 0u);
        unsigned i = start;
        uint32_t wv = 0;
        unsigned k = 0;
        for (; i + 1 < end; i += 2) {
            const fse::DEntry e0 = dt[s0];
            const fse::DEntry e1 = dt[s1];
            wv |= ((uint32_t)e0.symbol | ((uint32_t)e1.symbol << 8)) << (8 * k);
            k += 2;
            if (k == 4) {
                *reinterpret_cast<uint32_t *>(so + (i + 2 - start - 4)) = wv;
                wv = 0;
                k = 0;
            }
            s0 = e0.newState + br.read(e0.nbBits);
            s1 = e1.newState + br.read(e1.nbBits);
        }
        for (unsigned t = 0; t < k; t++) so[i - start - k + t] = (uint8_t)(wv >> (8 * t));
        if (i < end) so[i - start] = dt[s0].symbol;
        if (q + 1 < nparts) {
            const FseCkpt c = cks[jb.ck + q];
            if (c.s0 != s0 || c.s1 != s1 || br.pos != br.start_bit(sp) + (int32_t)c.bitpos) atomicExch(err + 1, 1);
        }
    }
    // the symbols leave in consecutive bytes across the CTA (each thread's part decoded into
    // shared memory, so that no warp store scatters over the parts)
    __syncthreads();
    if (nparts > 1) {
        // the last part runs to the block's end (up to two symbols past `part`, which its
        // region's padding holds)
        const unsigned lp = 31 - __clz(part);
        for (unsigned i = threadIdx.x; i < n; i += blockDim.x) {
            const unsigned r = min(i >> lp, nparts - 1);
            dst[i] = s_out[(size_t)r * (part + kPartPad) + (i - r * part)];
        }
    } else {
        for (unsigned i = threadIdx.x; i < n; i += blockDim.x) dst[i] = s_out[i];
    }
}

// Walks an fse_enc record sequence (host bytes) for n symbols starting at `off`; appends jobs.
size_t parse_blocks(const ByteView &h, size_t off, unsigned long long n, unsigned long long dst_base,
                    std::vector<BlockJob> &jobs) {
    const size_t len = h.len;
    unsigned long long done = 0;
    while (done < n) {
        const unsigned bn = (unsigned)std::min<unsigned long long>(n - done, FBLK);
        if (off >= len) throw std::invalid_argument("truncated FSE block stream");
        const uint8_t flag = h.at(off++);
        BlockJob j{dst_base + done, bn, flag, 0, 0};
        if (flag == 0) {
            if (off + bn > len) throw std::invalid_argument("truncated raw block");
            j.in = off;
            j.inlen = bn;
            off += bn;
        } else if (flag == 2) {
            if (off + 1 > len) throw std::invalid_argument("truncated RLE block");
            j.in = off;
            j.inlen = 1;
            off += 1;
        } else if (flag == 1) {
            if (off + 4 > len) throw std::invalid_argument("truncated FSE block header");
            const uint32_t rr = h.rd<uint32_t>(off);
            if (off + rr > len || bn < 3) throw std::invalid_argument("truncated FSE block");
            j.in = off;
            j.inlen = rr;
            off += rr;
        } else {
            throw std::invalid_argument("invalid FSE block flag");
        }
        jobs.push_back(j);
        done += bn;
    }
    return off;
}

// ------------------------------------------------------------------ Elias-gamma groups
// vals (u32, >= 1) of all groups concatenated; gstart has G+1 entries.
struct GammaOut {
    std::vector<std::vector<std::pair<const uint8_t *, size_t>>> cls_pieces;  // per group
    std::vector<std::vector<unsigned>> cls_n;                                  // symbols per block
    std::vector<std::vector<uint8_t>> cls_flag;                                // record flag per block
    std::vector<std::vector<const FseCkpt *>> cls_ck;                          // checkpoints per block
    std::vector<size_t> cls_bytes;                                             // per group
    std::vector<const uint8_t *> man_ptr;                                      // per group
    std::vector<size_t> man_bytes;                                             // per group
};

__global__ void k_gamma_cls(const uint32_t *__restrict__ v, long long n, uint8_t *__restrict__ cls) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        cls[i] = (uint8_t)(31 - __clz(v[i]));
}

__device__ __forceinline__ int find_group(const unsigned long long *gstart, int G, unsigned long long i) {
    int lo = 0, hi = G - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (gstart[mid] <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// MSB-first packing of k low bits of each value into word-aligned per-group regions (zeroed).
__global__ void __launch_bounds__(256) k_gamma_pack(const uint32_t *__restrict__ v, const uint8_t *__restrict__ cls,
                                                    const unsigned long long *__restrict__ boff, long long n,
                                                    const unsigned long long *__restrict__ gstart, int G,
                                                    const unsigned long long *__restrict__ gword,
                                                    uint32_t *__restrict__ words) {
    __shared__ unsigned long long s_gs[1025];  // the group starts, when there are few groups
    const bool in_smem = G + 1 <= 1025;
    if (in_smem)
        for (int g = threadIdx.x; g <= G; g += blockDim.x) s_gs[g] = gstart[g];
    __syncthreads();
    const unsigned long long *gs = in_smem ? s_gs : gstart;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int k = cls[i];
        if (k == 0) continue;
        const int g = find_group(gs, G, (unsigned long long)i);
        const unsigned long long b = boff[i] - boff[gs[g]];
        const uint32_t m = v[i] & ((1u << k) - 1u);
        const unsigned long long w = gword[g] + (b >> 5);
        const int o = (int)(b & 31);
        const unsigned long long win = (unsigned long long)m << (64 - k - o);
        const uint32_t hi = (uint32_t)(win >> 32), lo = (uint32_t)win;
        if (hi) atomicOr(&words[w], __byte_perm(hi, 0, 0x0123));
        if (lo) atomicOr(&words[w + 1], __byte_perm(lo, 0, 0x0123));
    }
}

// out[i] = src[idx[i]]
__global__ void k_pick_u64(const unsigned long long *__restrict__ src, const unsigned long long *__restrict__ idx,
                           long long n, unsigned long long *__restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = src[idx[i]];
}

// The FSE block coders' shared-memory limits, set once per device (a function attribute set while
// other threads launch the same kernel would only add driver work to every call).
void enable_fse_smem() {
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    FB2_CUDA(cudaGetDevice(&dev));
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return;
    FB2_CUDA(cudaFuncSetAttribute(k_fse_encode_blocks<kFseGroups>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(kFseGroups * kFseNxtBytes)));
    FB2_CUDA(cudaFuncSetAttribute(k_fse_encode_blocks<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kFseNxtBytes));
    FB2_CUDA(cudaFuncSetAttribute(k_fse_decode_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize, kFseDecSmem));
    done.fetch_or(bit, std::memory_order_acq_rel);
}

// The FSE class blocks of the gamma classes, launched by gamma_launch; gamma_finish packs the
// mantissas and collects the blocks.  Between the two the caller may launch other work: the class
// blocks are long sequential chains, so they go to the GPU before the order-1 chain encoder.
struct GammaBlocks {
    long long T = 0;
    std::vector<unsigned long long> gstart;
    uint8_t *cls = nullptr;
    std::vector<BlockJob> jobs;
    std::vector<int> job_group;
    uint8_t *slots = nullptr;
    unsigned long long *sizes = nullptr;
    FseCkpt *cks = nullptr;
    size_t ck_per_block = 0;
    unsigned long long *phase = nullptr;  // per-block phase times, traced calls only
};

// `beside`: CTAs of whole SMs that run next to the class blocks (the chain encoder's).
GammaBlocks gamma_launch(Pool &pool, const uint32_t *d_vals, const std::vector<unsigned long long> &gstart,
                         cudaStream_t st, uint32_t ckpt_part, cudaEvent_t queued = nullptr, size_t beside = 0) {
    GammaBlocks gb;
    gb.gstart = gstart;
    const int G = (int)gstart.size() - 1;
    const long long T = (long long)gstart.back();
    gb.T = T;
    if (T == 0) {
        if (queued) FB2_CUDA(cudaEventRecord(queued, st));
        return gb;
    }
    uint8_t *cls = pool.get<uint8_t>(T);
    gb.cls = cls;
    k_gamma_cls<<<grid_for(T, 256), 256, 0, st>>>(d_vals, T, cls);
    FB2_CHECK_LAUNCH();
    for (int g = 0; g < G; g++) {
        for (unsigned long long b = gstart[g]; b < gstart[g + 1]; b += FBLK) {
            gb.jobs.push_back(BlockJob{b, (unsigned)std::min<unsigned long long>(FBLK, gstart[g + 1] - b), 0, 0, 0});
            gb.job_group.push_back(g);
        }
    }
    const size_t nj = gb.jobs.size();
    if (std::getenv("FALCONS_TRACE"))
        std::fprintf(stderr, "[falcons trace] escapes: %lld values in %d groups, %zu class blocks\n", T, G, nj);
    BlockJob *d_jobs = h2d(pool, gb.jobs, st);
    gb.slots = pool.get<uint8_t>(nj * kBlockSlot);
    uint8_t *bits = pool.get<uint8_t>(nj * kBlockSlot);
    gb.sizes = pool.get<unsigned long long>(nj);
    gb.ck_per_block = ckpt_part ? FBLK / ckpt_part : 0;
    gb.cks = ckpt_part ? pool.get<FseCkpt>(nj * gb.ck_per_block) : nullptr;
    uint32_t *recs = pool.get<uint32_t>(nj * kFseRecWords);
    std::vector<uint32_t> order(nj);
    for (size_t j = 0; j < nj; j++) order[j] = (uint32_t)j;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return gb.jobs[a].n > gb.jobs[b].n; });
    uint32_t *d_order = h2d(pool, order, st);
    if (queued) FB2_CUDA(cudaEventRecord(queued, st));  // what the blocks wait for is on the stream
    const uint32_t part = ckpt_part ? ckpt_part : 4096u;
    if (std::getenv("FALCONS_TRACE")) {
        gb.phase = pool.get<unsigned long long>(nj * kFsePhases);
        FB2_CUDA(cudaMemsetAsync(gb.phase, 0, nj * kFsePhases * 8, st));
    }
    enable_fse_smem();
    if (nj + beside > (size_t)sm_count()) {
        constexpr unsigned G = kFseGroups;
        constexpr int smem = (int)(G * kFseNxtBytes);
        k_fse_encode_blocks<G><<<(unsigned)((nj + G - 1) / G), G * kFseGroupThreads, smem, st>>>(
            cls, d_jobs, (unsigned)nj, gb.slots, gb.sizes, bits, part, gb.cks, recs, d_order, gb.phase);
    } else {
        constexpr int smem = (int)kFseNxtBytes;
        k_fse_encode_blocks<1><<<(unsigned)nj, kFseGroupThreads, smem, st>>>(
            cls, d_jobs, (unsigned)nj, gb.slots, gb.sizes, bits, part, gb.cks, recs, d_order, gb.phase);
    }
    FB2_CHECK_LAUNCH();
    return gb;
}

GammaOut gamma_finish(Pool &pool, const GammaBlocks &gb, const uint32_t *d_vals, cudaStream_t st) {
    Trace tr("gamma");
    const std::vector<unsigned long long> &gstart = gb.gstart;
    const int G = (int)gstart.size() - 1;
    const long long T = gb.T;
    GammaOut out;
    out.cls_pieces.resize(G);
    out.cls_n.resize(G);
    out.cls_flag.resize(G);
    out.cls_ck.resize(G);
    out.cls_bytes.assign(G, 0);
    out.man_ptr.assign(G, nullptr);
    out.man_bytes.assign(G, 0);
    if (T == 0) return out;
    const uint8_t *cls = gb.cls;
    unsigned long long *boff = pool.get<unsigned long long>(T + 1);
    void *sc = pool.get<uint8_t>(scan_scratch_bytes(T, 8));
    exclusive_scan<uint8_t, unsigned long long>(cls, T, boff, sc, st);
    // per-group bit totals: the scan at every group start, gathered on the device, one copy back
    unsigned long long *d_gstart = h2d(pool, gstart, st);
    unsigned long long *d_gb = pool.get<unsigned long long>(G + 1);
    k_pick_u64<<<grid_for(G + 1, 256), 256, 0, st>>>(boff, d_gstart, G + 1, d_gb);
    FB2_CHECK_LAUNCH();
    const std::vector<unsigned long long> gbits = d2h(d_gb, (size_t)G + 1, st);
    tr.mark("group bits known");
    std::vector<unsigned long long> gword(G);
    unsigned long long words = 0;
    for (int g = 0; g < G; g++) {
        const unsigned long long bits = gbits[g + 1] - gbits[g];
        out.man_bytes[g] = (size_t)((bits + 7) / 8);
        gword[g] = words;
        words += (bits + 31) / 32 + 2;
    }
    uint32_t *wbuf = pool.get<uint32_t>(words + 4);
    FB2_CUDA(cudaMemsetAsync(wbuf, 0, (words + 4) * 4, st));
    unsigned long long *d_gword = h2d(pool, gword, st);
    k_gamma_pack<<<grid_for(T, 256, 148 * 8), 256, 0, st>>>(d_vals, cls, boff, T, d_gstart, G, d_gword, wbuf);
    FB2_CHECK_LAUNCH();
    for (int g = 0; g < G; g++) out.man_ptr[g] = reinterpret_cast<const uint8_t *>(wbuf + gword[g]);
    std::vector<unsigned long long> hs = d2h(gb.sizes, gb.jobs.size(), st);
    tr.mark("class blocks coded");
    if (gb.phase && tr.on) {
        const size_t nj = gb.jobs.size();
        const std::vector<unsigned long long> ph = d2h(gb.phase, nj * kFsePhases, st);
        unsigned long long t0 = ~0ULL, t1 = 0;
        double sum[6] = {0};
        for (size_t j = 0; j < nj; j++) {
            const unsigned long long *p = ph.data() + j * kFsePhases;
            t0 = std::min(t0, p[0]);
            t1 = std::max(t1, p[6]);
            for (int k = 0; k < 6; k++)
                if (p[k] && p[k + 1]) sum[k] += (double)(p[k + 1] - p[k]);
        }
        std::fprintf(stderr,
                     "[falcons trace] gamma class blocks: %zu, span %.3f ms; per block (us): count %.1f plan %.1f "
                     "tables %.1f chain walk %.1f pack %.1f output %.1f\n",
                     nj, (double)(t1 - t0) / 1e6, sum[0] / nj / 1e3, sum[1] / nj / 1e3, sum[2] / nj / 1e3,
                     sum[3] / nj / 1e3, sum[4] / nj / 1e3, sum[5] / nj / 1e3);
    }
    for (size_t j = 0; j < gb.jobs.size(); j++) {
        const int g = gb.job_group[j];
        const size_t sz = (size_t)(hs[j] & ((1ULL << 56) - 1));
        out.cls_pieces[g].push_back({gb.slots + j * kBlockSlot, sz});
        out.cls_n[g].push_back(gb.jobs[j].n);
        out.cls_flag[g].push_back((uint8_t)(hs[j] >> 56));
        out.cls_ck[g].push_back(gb.cks ? gb.cks + j * gb.ck_per_block : nullptr);
        out.cls_bytes[g] += sz;
    }
    return out;
}

GammaOut gamma_encode(Pool &pool, const uint32_t *d_vals, const std::vector<unsigned long long> &gstart,
                      cudaStream_t st, uint32_t ckpt_part) {
    const GammaBlocks gb = gamma_launch(pool, d_vals, gstart, st, ckpt_part);
    return gamma_finish(pool, gb, d_vals, st);
}

// Adds the fse_enc records of group g, recording each record's header bytes for the index.
// Gathers the decode checkpoints of the streams in stream order and writes the FB2C frame.
struct CkptCollector {
    uint32_t o1_part = 0, fse_part = 0;
    const O1Ckpt *o1 = nullptr;
    unsigned long long n_o1 = 0;
    std::vector<std::pair<const FseCkpt *, uint32_t>> fse;
    unsigned long long n_fse = 0;
    void add_block(const FseCkpt *p, uint32_t count) {
        if (p && count) {
            fse.push_back({p, count});
            n_fse += count;
        }
    }
    void emit(Assembler &as) const {
        if (n_o1 + n_fse == 0 || !as.with_index) return;
        const unsigned long long content = kCkptHeader + n_o1 * sizeof(O1Ckpt) + n_fse * sizeof(FseCkpt);
        if (content >= 0xFFFFFFFFULL) return;
        uint8_t h[8 + kCkptHeader];
        static_assert(kCkptHeader == 32, "content header: tag, version, o1_part, fse_part, n_o1, n_fse");
        const uint32_t w[6] = {kSkippableMagic, (uint32_t)content, kCkptTag, kCkptVersion, o1_part, fse_part};
        memcpy(h, w, sizeof(w));
        memcpy(h + 24, &n_o1, 8);
        memcpy(h + 32, &n_fse, 8);
        as.tail_bytes(h, sizeof(h));
        as.tail_dev(o1, n_o1 * sizeof(O1Ckpt));
        for (auto &f : fse) as.tail_dev(f.first, (size_t)f.second * sizeof(FseCkpt));
    }
};
static_assert(sizeof(O1Ckpt) == 12 && sizeof(FseCkpt) == 8, "checkpoint record sizes are part of the frame format");

void add_class_pieces(Assembler &as, const GammaOut &go, int g, CkptCollector *cc = nullptr) {
    for (size_t b = 0; b < go.cls_pieces[g].size(); b++) {
        const auto &p = go.cls_pieces[g][b];
        if (cc && go.cls_flag[g][b] == 1) cc->add_block(go.cls_ck[g][b], fse_ckpt_count(go.cls_n[g][b], cc->fse_part));
        uint8_t h[5];
        size_t hl;
        const uint8_t flag = go.cls_flag[g][b];
        if (flag != 1) { h[0] = flag; hl = 1; }
        else {
            h[0] = 1;
            const uint32_t r = (uint32_t)(p.second - 5);
            memcpy(h + 1, &r, 4);
            hl = 5;
        }
        as.shadow(h, hl);
        as.dev(p.first, p.second);
    }
}

// Gamma decode of n values in index order: value i = (1 << k) | k mantissa bits (MSB first, at
// the group's running bit offset boff), k = cls[i].  The group starts (and, when there are few
// groups, the group tables) sit in shared memory; the mantissa bits come from at most two
// aligned words.
// Gamma unpacking in units of kUnit values: the values of group g, [gstart[g], gstart[g + 1]),
// are cut into units from the group's start; unit u of the whole list belongs to the last group g
// with ustart[g] <= u.  A warp sums a unit's classes (its mantissa bits); an exclusive scan of the
// unit sums gives every unit its first bit; a thread then reads its unit's mantissas in order
// (MSB-first bits of the group's byte region, one aligned word at a time).
constexpr unsigned kUnit = 1024;

__device__ __forceinline__ int unit_group(const unsigned long long *__restrict__ ustart, int G, unsigned long long u) {
    int lo = 0, hi = G - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (ustart[mid] <= u) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(256) k_unit_bits(const uint8_t *__restrict__ cls,
                                                   const unsigned long long *__restrict__ gstart,
                                                   const unsigned long long *__restrict__ ustart, int G,
                                                   unsigned long long nunits, unsigned long long *__restrict__ usum) {
    const unsigned long long u = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31u;
    if (u >= nunits) return;
    const int g = unit_group(ustart, G, u);
    const unsigned long long first = gstart[g] + (u - ustart[g]) * kUnit;
    const unsigned long long end = min(first + kUnit, gstart[g + 1]);
    uint32_t s = 0;
    for (unsigned long long i = first + lane; i < end; i += 32) s += cls[i];
    s = __reduce_add_sync(0xffffffffu, s);
    if (lane == 0) usum[u] = s;
}

// Escape values (zigzag + 1, gamma-coded) of every unit, a warp per unit: v[i] = (1 << k) |
// mantissa, or, with `ovf`, the escape code unzz(v - 1) at its place gdst[g] + (i - gstart[g]).
// uoff is the exclusive scan of the unit bit sums; the warp takes its unit's values 32 at a time,
// a warp scan of their classes giving each lane its mantissa's bit offset.  A class above 31 sets
// err 2, a mantissa past its group's region err 3.
__global__ void __launch_bounds__(256) k_gamma_unpack_units(
    const uint8_t *__restrict__ cls, const unsigned long long *__restrict__ gstart,
    const unsigned long long *__restrict__ ustart, int G, unsigned long long nunits,
    const unsigned long long *__restrict__ uoff, const unsigned long long *__restrict__ gman,
    const uint8_t *__restrict__ base, const unsigned long long *__restrict__ gman_len, uint32_t *__restrict__ v,
    int *__restrict__ err, const unsigned long long *__restrict__ gdst, int16_t *__restrict__ ovf) {
    const unsigned long long u = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31u;
    if (u >= nunits) return;
    const int g = unit_group(ustart, G, u);
    const unsigned long long g0 = gstart[g];
    const unsigned long long first = g0 + (u - ustart[g]) * kUnit;
    const unsigned long long end = min(first + kUnit, gstart[g + 1]);
    const unsigned long long len = gman_len[g];
    const uint8_t *rb = base + gman[g];
    unsigned long long run = uoff[u] - uoff[ustart[g]];  // bit offset of the values below
    bool bad2 = false, bad3 = false;
    for (unsigned long long i0 = first; i0 < end; i0 += 32) {
        const unsigned long long i = i0 + lane;
        const bool act = i < end;
        const unsigned k = act ? cls[i] : 0u;
        uint32_t incl = k;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (unsigned)o) incl += t;
        }
        const unsigned long long bb = run + incl - k;
        run += __shfl_sync(0xffffffffu, incl, 31);
        if (!act) continue;
        uint32_t m = 0;
        if (k > 31) {
            bad2 = true;
        } else if (k > 0) {
            if (((bb + k + 7) >> 3) > len) {
                bad3 = true;
            } else {
                const uintptr_t a = reinterpret_cast<uintptr_t>(rb + (bb >> 3));
                const uint32_t *w = reinterpret_cast<const uint32_t *>(a & ~uintptr_t(3));
                const unsigned lead = (unsigned)(a & 3);
                const unsigned need = lead + (unsigned)((((bb & 7) + k) + 7) >> 3);  // bytes from w[0]
                const uint32_t w0 = __byte_perm(w[0], 0, 0x0123);
                const uint32_t w1 = need > 4 ? __byte_perm(w[1], 0, 0x0123) : 0u;
                const unsigned long long be = ((unsigned long long)w0 << 32) | w1;  // big-endian bytes
                m = (uint32_t)((be << (lead * 8 + (unsigned)(bb & 7))) >> (64 - k));
            }
        }
        const uint32_t val = k <= 31 ? ((1u << k) | m) : 0u;
        if (ovf) ovf[gdst[g] + (i - g0)] = (int16_t)unzz(val - 1u);
        else v[i] = val;
    }
    if (bad2) atomicExch(err, 2);
    if (bad3) atomicExch(err, 3);
}

// ------------------------------------------------------------------ delta
__global__ void k_delta(const int16_t *__restrict__ in, long long n, int16_t *__restrict__ out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = i ? (int16_t)(uint16_t)((uint16_t)in[i] - (uint16_t)in[i - 1]) : in[0];
}

// Inclusive prefix sum modulo 2^16 (un-delta), tile based.
__global__ void __launch_bounds__(kScanThreads) k_tile_sum16(const int16_t *__restrict__ in, long long n,
                                                            uint32_t *__restrict__ tile_sum) {
    const long long base = (long long)blockIdx.x * kScanTile;
    uint32_t s = 0;
    for (int j = 0; j < kScanItems; j++) {
        const long long i = base + (long long)j * kScanThreads + threadIdx.x;
        if (i < n) s += (uint16_t)in[i];
    }
    __shared__ uint32_t sh[32];
    uint32_t tot;
    block_excl_scan<uint32_t>(s, sh, tot);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = tot & 0xFFFF;
}

__global__ void __launch_bounds__(kScanThreads) k_tile_undelta(int16_t *__restrict__ io, long long n,
                                                              const uint32_t *__restrict__ tile_off) {
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const long long i = base + j;
        v[j] = i < n ? (uint16_t)io[i] : 0u;
        s += v[j];
    }
    __shared__ uint32_t sh[32];
    uint32_t tot;
    uint32_t run = block_excl_scan<uint32_t>(s, sh, tot) + tile_off[blockIdx.x];
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const long long i = base + j;
        run += v[j];
        if (i < n) io[i] = (int16_t)(uint16_t)run;
    }
}

void undelta(Pool &pool, int16_t *d, long long n, cudaStream_t st) {
    if (n <= 1) return;
    const long long tiles = (n + kScanTile - 1) / kScanTile;
    uint32_t *ts = pool.get<uint32_t>(tiles + 2);
    k_tile_sum16<<<(unsigned)tiles, kScanThreads, 0, st>>>(d, n, ts);
    FB2_CHECK_LAUNCH();
    k_scan_small<uint32_t><<<1, 1024, 0, st>>>(ts, tiles);
    FB2_CHECK_LAUNCH();
    k_tile_undelta<<<(unsigned)tiles, kScanThreads, 0, st>>>(d, n, ts);
    FB2_CHECK_LAUNCH();
}

// ------------------------------------------------------------------ method 0
__global__ void __launch_bounds__(kScanThreads) k_m0_tiles(const int16_t *__restrict__ q, long long n,
                                                          uint32_t *__restrict__ cnt, long long *__restrict__ last) {
    const long long base = (long long)blockIdx.x * kScanTile;
    uint32_t c = 0;
    long long l = -1;
    for (int j = 0; j < kScanItems; j++) {
        const long long i = base + (long long)j * kScanThreads + threadIdx.x;
        if (i < n && q[i] != 0) {
            c++;
            l = i > l ? i : l;
        }
    }
    __shared__ uint32_t sh[32];
    uint32_t tot;
    block_excl_scan<uint32_t>(c, sh, tot);
    __shared__ long long lm;
    if (threadIdx.x == 0) lm = -1;
    __syncthreads();
    if (l >= 0) atomicMax(&lm, l);
    __syncthreads();
    if (threadIdx.x == 0) {
        cnt[blockIdx.x] = tot;
        last[blockIdx.x] = lm;
    }
}

// Exclusive running max of tile "last nonzero" positions (one block, chunked); last[tiles] = overall max.
__global__ void __launch_bounds__(1024) k_prefix_last(long long *__restrict__ last, long long tiles) {
    __shared__ long long sh[1024];
    __shared__ long long carry;
    if (threadIdx.x == 0) carry = -1;
    __syncthreads();
    for (long long base = 0; base < tiles; base += blockDim.x) {
        const long long i = base + threadIdx.x;
        const long long v = i < tiles ? last[i] : -1;
        sh[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < (int)blockDim.x; o <<= 1) {
            const long long y = threadIdx.x >= (unsigned)o ? sh[threadIdx.x - o] : -1;
            __syncthreads();
            if (y > sh[threadIdx.x]) sh[threadIdx.x] = y;
            __syncthreads();
        }
        const long long before = threadIdx.x ? sh[threadIdx.x - 1] : -1;
        const long long c = carry;
        if (i < tiles) last[i] = before > c ? before : c;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = sh[threadIdx.x] > c ? sh[threadIdx.x] : c;
        __syncthreads();
    }
    if (threadIdx.x == 0) last[tiles] = carry;
}

__global__ void __launch_bounds__(kScanThreads) k_m0_extract(const int16_t *__restrict__ q, long long n,
                                                            const uint32_t *__restrict__ tile_off,
                                                            const long long *__restrict__ tile_prev,
                                                            uint32_t *__restrict__ runs, uint32_t *__restrict__ vals) {
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int16_t v[kScanItems];
    uint32_t c = 0;
    long long l = -1;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const long long i = base + j;
        v[j] = i < n ? q[i] : (int16_t)0;
        if (v[j] != 0) {
            c++;
            l = i;
        }
    }
    __shared__ uint32_t sh[32];
    uint32_t tot;
    uint32_t rank = block_excl_scan<uint32_t>(c, sh, tot) + tile_off[blockIdx.x];
    // previous nonzero before this thread's items: max over lower threads of their last, else tile carry
    __shared__ long long lastv[kScanThreads];
    lastv[threadIdx.x] = l;
    __syncthreads();
    // inclusive max-scan over threads (Hillis-Steele in shared memory)
    for (int o = 1; o < kScanThreads; o <<= 1) {
        long long y = threadIdx.x >= (unsigned)o ? lastv[threadIdx.x - o] : -1;
        __syncthreads();
        if (y > lastv[threadIdx.x]) lastv[threadIdx.x] = y;
        __syncthreads();
    }
    long long prev = threadIdx.x ? lastv[threadIdx.x - 1] : -1;
    if (prev < 0) prev = tile_prev[blockIdx.x];
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        if (v[j] != 0) {
            const long long i = base + j;
            runs[rank] = (uint32_t)(i - prev);  // L + 1
            vals[rank] = zigzag((int)v[j]) + 1u;
            prev = i;
            rank++;
        }
    }
}

// ------------------------------------------------------------------ method 1
struct SegInfo {
    unsigned long long lo, n, cs;   // segment start, length, chunk size
    int K;
    int pad;
};

// Per segment: the count of every (context, symbol) key of its chains (a chain's first code has
// context 0) and every chain's escape count; writes every code's key (context << 8 | symbol) for
// the chain encoder.  CTA (g, u) takes the u-th of gridDim.y slices of every chain of segment g
// (slice edges on multiples of 8 codes) and adds its counts to the segment's totals, which start
// at zero.  Codes are read 8 at a time as 16-byte vectors when q is 16-byte aligned (the
// code before a vector comes from the lane below); runs of equal keys within a vector are counted
// with one atomic, and the lanes of a warp spread their atomics over kHistCopies histograms.
constexpr int kHistCopies = 4;
constexpr size_t kHistSmem = (size_t)kHistCopies * O1_NCTX * O1_NSYM * 4;
__global__ void __launch_bounds__(1024, 2) k_o1_hist(const int16_t *__restrict__ q, const SegInfo *__restrict__ segs,
                                                    uint32_t *__restrict__ hist, uint32_t *__restrict__ nvk,
                                                    uint16_t *__restrict__ keys, int vec) {
    extern __shared__ uint32_t hs[];  // kHistCopies histograms of O1_NCTX * O1_NSYM keys
    __shared__ uint32_t esc[kMaxK];
    constexpr int HN = O1_NCTX * O1_NSYM;
    const SegInfo sg = segs[blockIdx.x];
    const unsigned long long U = gridDim.y, u = blockIdx.y;
    for (int i = threadIdx.x; i < kHistCopies * HN; i += blockDim.x) hs[i] = 0;
    if (threadIdx.x < kMaxK) esc[threadIdx.x] = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31u;
    uint32_t *h = hs + (lane % kHistCopies) * HN;
    for (int k = 0; k < sg.K; k++) {
        const long long b = (long long)(sg.lo + (unsigned long long)k * sg.cs);
        const long long e = (long long)(sg.lo + min((unsigned long long)k * sg.cs + sg.cs, sg.n));
        if (e <= b) continue;
        // this CTA's slice [sb, se) of the chain [b, e)
        const unsigned long long len = (unsigned long long)(e - b);
        auto edge = [&](unsigned long long v) -> long long {
            if (v == 0) return b;
            if (v >= U) return e;
            const long long x = (b + (long long)(len * v / U) + 7) & ~7LL;
            return x < e ? x : e;
        };
        const long long sb = edge(u), se = edge(u + 1);
        if (se <= sb) continue;
        // codes [sb, hb) and [tb, se) one per thread, whole vectors [hb, tb) one per thread
        long long hb = se, tb = se;
        if (vec) {
            hb = min(se, (sb + 7) & ~7LL);
            tb = max(hb, se & ~7LL);
        }
        uint32_t ne = 0;
        const long long nh = hb - sb, nt = se - tb;
        for (long long j = threadIdx.x; j < nh + nt; j += blockDim.x) {
            const long long i = j < nh ? sb + j : tb + (j - nh);
            const int prev = i == b ? 0 : (int)q[i - 1];
            const int sy = o1_sym((int)q[i]);
            const uint32_t key = (uint32_t)(o1_ctx(prev) << 8) | (uint32_t)sy;
            atomicAdd(&h[key], 1u);
            keys[i] = (uint16_t)key;
            ne += sy == O1_NSYM - 1;
        }
        const long long v0 = hb >> 3, v1 = tb >> 3;
        const uint4 *q4 = reinterpret_cast<const uint4 *>(q);
        uint4 *k4 = reinterpret_cast<uint4 *>(keys);
        for (long long vb = v0 + (threadIdx.x & ~31u); vb < v1; vb += blockDim.x) {  // warp-uniform
            const long long vi = vb + lane;
            const bool act = vi < v1;
            const uint4 w = act ? __ldg(q4 + vi) : make_uint4(0, 0, 0, 0);
            const uint32_t below = __shfl_up_sync(0xffffffffu, w.w >> 16, 1);
            if (!act) continue;
            int prev = 0;  // the code before this vector (context 0 at the chain's start)
            if (vi * 8 > b) prev = (lane && vi > v0) ? (int)(int16_t)below : (int)q[vi * 8 - 1];
            const uint32_t ww[4] = {w.x, w.y, w.z, w.w};
            uint32_t kk[8];
            uint32_t rkey = ~0u, rn = 0;
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const int code = (int)(int16_t)(ww[m >> 1] >> (16 * (m & 1)));
                const int sy = o1_sym(code);
                const uint32_t key = (uint32_t)(o1_ctx(prev) << 8) | (uint32_t)sy;
                kk[m] = key;
                ne += sy == O1_NSYM - 1;
                if (key == rkey) {
                    rn++;
                } else {
                    if (rn) atomicAdd(&h[rkey], rn);
                    rkey = key;
                    rn = 1;
                }
                prev = code;
            }
            atomicAdd(&h[rkey], rn);
            k4[vi] = make_uint4(kk[0] | (kk[1] << 16), kk[2] | (kk[3] << 16), kk[4] | (kk[5] << 16), kk[6] | (kk[7] << 16));
        }
        ne = __reduce_add_sync(0xffffffffu, ne);
        if (lane == 0 && ne) atomicAdd(&esc[k], ne);
    }
    __syncthreads();
    uint32_t *gh = hist + (size_t)blockIdx.x * HN;
    for (int i = threadIdx.x; i < HN; i += blockDim.x) {
        uint32_t v = 0;
#pragma unroll
        for (int c = 0; c < kHistCopies; c++) v += hs[c * HN + i];
        if (v) atomicAdd(gh + i, v);
    }
    if (threadIdx.x < kMaxK && esc[threadIdx.x]) atomicAdd(nvk + blockIdx.x * kMaxK + threadIdx.x, esc[threadIdx.x]);
}

// Keeps every m-th decode checkpoint of every chain (the m-th, 2m-th, ... of chain c's
// src[soff[c] ..]), compacted to dst[doff[c] ..]: checkpoints m times as far apart.
__global__ void k_ck_thin(const O1Ckpt *__restrict__ src, const unsigned long long *__restrict__ soff,
                          const unsigned long long *__restrict__ doff, int nchains, uint32_t m,
                          O1Ckpt *__restrict__ dst) {
    const int c = blockIdx.y;
    if (c >= nchains) return;
    const unsigned long long n = doff[c + 1] - doff[c];
    for (unsigned long long j = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (unsigned long long)gridDim.x * blockDim.x)
        dst[doff[c] + j] = src[soff[c] + (j + 1) * m - 1];
}

// The order-1 tables (RleFseEncoder.hpp:410-477 normalizes each context's counts to O1_M cells):
// one warp per (region, context) table, lanes holding 8 symbols each, with the rule of
// fse::normalize_count: every present symbol gets its nearest share of the cells (at least one)
// under a scale refined for the one-cell floor, then single cells move by marginal coded size
// (count / (n - 1/2) compared in integers) until the table is full.  An empty context gets all
// cells on symbol 0, a context with one symbol all cells on it.
__device__ __forceinline__ void warp_best(unsigned long long &bc, unsigned long long &bd, int &bs, bool want_max) {
    // the best fraction bc / bd over the warp (ties: the lower symbol); bs < 0 marks no candidate
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long oc = __shfl_xor_sync(0xffffffffu, bc, o);
        const unsigned long long od = __shfl_xor_sync(0xffffffffu, bd, o);
        const int os = __shfl_xor_sync(0xffffffffu, bs, o);
        bool take;
        if (os < 0) take = false;
        else if (bs < 0) take = true;
        else {
            const unsigned long long l = oc * bd, r = bc * od;
            take = want_max ? (l > r || (l == r && os < bs)) : (l < r || (l == r && os < bs));
        }
        if (take) {
            bc = oc;
            bd = od;
            bs = os;
        }
    }
}

__global__ void __launch_bounds__(256) k_o1_norm(const uint32_t *__restrict__ hist, int total_tables,
                                                 uint16_t *__restrict__ nf) {
    const int wt = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (wt >= total_tables) return;
    const uint32_t *cnt = hist + (size_t)wt * O1_NSYM;
    uint16_t *freq = nf + (size_t)wt * O1_NSYM;
    constexpr int PER = O1_NSYM / 32;
    uint32_t c[PER];
    int n[PER];
    unsigned long long total = 0;
    int present = 0;
#pragma unroll
    for (int i = 0; i < PER; i++) {
        c[i] = cnt[lane + 32 * i];
        total += c[i];
        present += c[i] != 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
    present = __reduce_add_sync(0xffffffffu, (unsigned)present);
    if (total == 0 || present == 1) {
#pragma unroll
        for (int i = 0; i < PER; i++) {
            const int sy = lane + 32 * i;
            freq[sy] = (uint16_t)(total == 0 ? (sy == 0 ? O1_M : 0) : (c[i] ? O1_M : 0));
        }
        return;
    }
    double mu = (double)O1_M / (double)total;
    int left = 0;
    for (int round = 0; round < 4; round++) {
        int ones = 0, sum = 0;
        unsigned long long ones_count = 0;
#pragma unroll
        for (int i = 0; i < PER; i++) {
            if (!c[i]) {
                n[i] = 0;
                continue;
            }
            const double share = floor((double)c[i] * mu + 0.5);
            int v = share < (double)O1_M ? (int)share : O1_M;
            if (v <= 1) {
                v = 1;
                ones++;
                ones_count += c[i];
            }
            n[i] = v;
            sum += v;
        }
        sum = (int)__reduce_add_sync(0xffffffffu, (unsigned)sum);
        ones = (int)__reduce_add_sync(0xffffffffu, (unsigned)ones);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ones_count += __shfl_xor_sync(0xffffffffu, ones_count, o);
        left = O1_M - sum;
        if (left == 0 || ones_count == total) break;
        mu = (double)(O1_M - ones) / (double)(total - ones_count);
    }
    while (left != 0) {
        const bool add = left > 0;
        unsigned long long bc = 0, bd = 1;
        int bs = -1;
#pragma unroll
        for (int i = 0; i < PER; i++) {
            if (!c[i] || (!add && n[i] < 2)) continue;
            const unsigned long long c2 = 2ull * c[i], d = add ? 2ull * n[i] + 1 : 2ull * n[i] - 1;
            if (bs < 0 || (add ? c2 * bd > bc * d : c2 * bd < bc * d)) {
                bc = c2;
                bd = d;
                bs = lane + 32 * i;
            }
        }
        warp_best(bc, bd, bs, add);
        if (bs < 0) break;  // nothing movable (cannot happen: fewer symbols than cells)
        if ((bs & 31) == lane) {
#pragma unroll
            for (int i = 0; i < PER; i++)
                if (lane + 32 * i == bs) n[i] += add ? 1 : -1;
        }
        left += add ? -1 : 1;
    }
#pragma unroll
    for (int i = 0; i < PER; i++) freq[lane + 32 * i] = (uint16_t)n[i];
}

// ---- tANS tables for 15 contexts x 256 symbols, built by a whole CTA per table (zfse
// fse_compress.c FSE_buildCTable_wksp / fse_decompress.c FSE_buildDTable, restated in parallel).
constexpr int kTabThreads = 256;
struct TabSmem {
    int16_t norm[O1_NSYM];
    uint32_t cum[O1_NSYM + 1];   // cells before every symbol (a -1 symbol holds one cell)
    uint32_t occ[O1_NSYM + 1];   // spread occurrences before every symbol (positive counts only)
    uint32_t cnt[O1_NSYM];       // running per-symbol counters of the rank pass
    uint32_t part[kTabThreads];
    uint8_t sym[O1_M];
    int bad;
};

// The spread (fse::spread): symbol s takes the occurrences occ[s] .. occ[s+1]-1 of the visit order
// j -> (j * step) & mask that skips the cells above `high` (the -1 symbols' cells).  Every thread
// maps one run of j; a block scan of the kept visits gives each its occurrence number.
__device__ void cta_spread(TabSmem &w, unsigned tl) {
    const uint32_t tsize = 1u << tl, mask = tsize - 1, step = fse::table_step(tsize);
    if (threadIdx.x == 0) {
        uint32_t c = 0, o = 0, high = tsize - 1;
        for (int s2 = 0; s2 < O1_NSYM; s2++) {
            w.cum[s2] = c;
            w.occ[s2] = o;
            const int nn = w.norm[s2];
            if (nn == -1) {
                w.sym[high--] = (uint8_t)s2;
                c += 1;
            } else if (nn > 0) {
                c += (uint32_t)nn;
                o += (uint32_t)nn;
            }
        }
        w.cum[O1_NSYM] = c;
        w.occ[O1_NSYM] = o;
        w.bad = c != tsize;
    }
    __syncthreads();
    const uint32_t high = tsize - 1 - (w.cum[O1_NSYM] - w.occ[O1_NSYM]);
    const uint32_t per = tsize / blockDim.x;  // tsize is a multiple of the block size
    const uint32_t j0 = threadIdx.x * per;
    uint32_t kept = 0;
    for (uint32_t j = j0; j < j0 + per; j++) kept += ((j * step) & mask) <= high;
    w.part[threadIdx.x] = kept;
    __syncthreads();
    uint32_t k = 0;
    for (uint32_t t2 = 0; t2 < threadIdx.x; t2++) k += w.part[t2];
    for (uint32_t j = j0; j < j0 + per; j++) {
        const uint32_t pos = (j * step) & mask;
        if (pos > high) continue;
        int lo = 0, hi = O1_NSYM;  // the symbol whose occurrences hold k: occ[lo] <= k < occ[lo+1]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (w.occ[mid] <= k) lo = mid;
            else hi = mid;
        }
        w.sym[pos] = (uint8_t)lo;
        k++;
    }
    __syncthreads();
}

// For every cell u in increasing order, f(u, s, rank) with rank = the cells of symbol s before u
// (warp 0, 32 cells at a time with match ranks).
template <class F>
__device__ void cta_ranks(TabSmem &w, uint32_t tsize, F &&f) {
    for (int s2 = threadIdx.x; s2 < O1_NSYM; s2 += blockDim.x) w.cnt[s2] = 0;
    __syncthreads();
    if (threadIdx.x < 32) {
        const unsigned lane = threadIdx.x;
        for (uint32_t u0 = 0; u0 < tsize; u0 += 32) {
            const uint32_t u = u0 + lane;
            const unsigned sy = w.sym[u];
            const unsigned peers = __match_any_sync(0xffffffffu, sy);
            const unsigned rank = __popc(peers & ((1u << lane) - 1u));
            f(u, sy, w.cnt[sy] + rank);
            __syncwarp();
            if (rank == (unsigned)__popc(peers) - 1u) w.cnt[sy] += rank + 1;
            __syncwarp();
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kTabThreads) k_o1_ctable(const uint16_t *__restrict__ nf, uint16_t *__restrict__ stab,
                                                         fse::SymTT *__restrict__ stt, uint8_t *__restrict__ scratch,
                                                         int *__restrict__ err) {
    (void)scratch;
    __shared__ TabSmem w;
    const size_t t = blockIdx.x;
    for (int s2 = threadIdx.x; s2 < O1_NSYM; s2 += blockDim.x) w.norm[s2] = (int16_t)nf[t * O1_NSYM + s2];
    __syncthreads();
    cta_spread(w, O1_PB);
    if (w.bad) {
        if (threadIdx.x == 0) atomicExch(err, 4);
        return;
    }
    uint16_t *st = stab + t * O1_M;
    cta_ranks(w, O1_M, [&](uint32_t u, unsigned sy, uint32_t r) { st[w.cum[sy] + r] = (uint16_t)(O1_M + u); });
    for (int s2 = threadIdx.x; s2 < O1_NSYM; s2 += blockDim.x) {
        const int nn = w.norm[s2];
        const uint32_t total = w.cum[s2];
        fse::SymTT tt;
        if (nn == 0) {
            tt.deltaNbBits = ((O1_PB + 1) << 16) - O1_M;
            tt.deltaFindState = 0;
        } else if (nn == -1 || nn == 1) {
            tt.deltaNbBits = (O1_PB << 16) - O1_M;
            tt.deltaFindState = (int32_t)total - 1;
        } else {
            const uint32_t maxBitsOut = O1_PB - fse::highbit32((uint32_t)(nn - 1));
            const uint32_t minStatePlus = (uint32_t)nn << maxBitsOut;
            tt.deltaNbBits = (maxBitsOut << 16) - minStatePlus;
            tt.deltaFindState = (int32_t)total - nn;
        }
        stt[t * O1_NSYM + s2] = tt;
    }
}

// Decode tables, one packed u32 per cell: bits 0-12 newState, 13-16 nbBits, 17-20 the context
// of the decoded code, 21 escape, 22-31 the code (10 bits, two's complement).
__global__ void __launch_bounds__(kTabThreads) k_o1_dtable(const uint16_t *__restrict__ nf, uint32_t *__restrict__ dt,
                                                         uint8_t *__restrict__ scratch, int *__restrict__ err) {
    (void)scratch;
    __shared__ TabSmem w;
    const size_t t = blockIdx.x;
    for (int s2 = threadIdx.x; s2 < O1_NSYM; s2 += blockDim.x) w.norm[s2] = (int16_t)nf[t * O1_NSYM + s2];
    __syncthreads();
    cta_spread(w, O1_PB);
    if (w.bad) {
        if (threadIdx.x == 0) atomicExch(err, 5);
        return;
    }
    uint32_t *d = dt + t * O1_M;
    cta_ranks(w, O1_M, [&](uint32_t u, unsigned sy, uint32_t r) {
        const int nn = w.norm[sy];
        const uint32_t ns = (nn == -1 ? 1u : (uint32_t)nn) + r;
        const uint32_t nb = O1_PB - fse::highbit32(ns);
        const uint32_t newState = (ns << nb) - O1_M;
        const bool esc = sy == O1_NSYM - 1;
        const int code = esc ? 0 : unzz(sy);
        const int ctx = esc ? 0 : o1_ctx(code);
        d[u] = newState | (nb << 13) | ((uint32_t)ctx << 17) | ((uint32_t)esc << 21) | ((uint32_t)(code & 0x3FF) << 22);
    });
}

struct DecChain {
    unsigned long long in;      // stream byte offset
    unsigned long long inlen;   // stream length (0 = empty chunk)
    unsigned long long lo, n;   // output range
    unsigned long long ovf;     // first escape value of this chunk
    int table;                  // segment index (tables at table * 15)
    uint32_t nesc;              // escapes of this chunk
    uint32_t ck;                // first decode checkpoint of this chunk
    uint32_t pad;
};

// One part of a chain decoded from a checkpoint (part 0 starts at the chain's stream end).
struct DecPart {
    uint32_t chain;
    uint32_t part;
};

// ---- shared-memory resident context tables
// A CTA encodes or decodes chains that share one table set; the tables of the contexts that carry
// most symbols are staged in shared memory (the rest are read from global memory).  `map` packs,
// per context, its shared-memory slot (4 bits, 15 = not resident); `rev` packs the context of
// every slot.
// A chain CTA holds up to 64 chains that share one table set (kept in shared memory, so one CTA
// fills an SM).  The chains are spread over all 8 warps, 8 lanes each, so that every scheduler of
// the SM has two warps of independent chain steps to interleave.
constexpr int kChainThreads = 256;
constexpr int kMaxChainsPerCta = 64;
__device__ __forceinline__ int chain_slot() {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    return lane < kMaxChainsPerCta / (kChainThreads / 32) ? lane * (kChainThreads / 32) + warp : -1;
}
constexpr int kDecSlots = 7;   // 7 x 8192 x u32 decode tables = 224 KiB
struct ChainCta {
    int table;
    int first;
    int count;
    int pad;
    unsigned long long map, rev;
};

__global__ void __launch_bounds__(kChainThreads) k_o1_decode_smem(const uint8_t *__restrict__ in,
                                                      const DecChain *__restrict__ chains,
                                                      const ChainCta *__restrict__ ctas,
                                                      const uint32_t *__restrict__ dt,
                                                      const int16_t *__restrict__ ovf, unsigned long long n_ovf,
                                                      int16_t *__restrict__ out, int *__restrict__ err) {
    extern __shared__ uint4 smem_raw[];
    uint32_t *sdt = reinterpret_cast<uint32_t *>(smem_raw);
    const ChainCta w = ctas[blockIdx.x];
    const uint32_t *__restrict__ tb = dt + (size_t)w.table * O1_NCTX * O1_M;
    for (int j = 0; j < kDecSlots; j++) {
        const int c = (int)((w.rev >> (4 * j)) & 15);
        if (c >= O1_NCTX) continue;
        const uint4 *src = reinterpret_cast<const uint4 *>(tb + (size_t)c * O1_M);
        uint4 *dst = reinterpret_cast<uint4 *>(sdt + (size_t)j * O1_M);
        for (int i = threadIdx.x; i < O1_M * 4 / 16; i += blockDim.x) dst[i] = __ldg(src + i);
    }
    __syncthreads();
    const int lc = chain_slot();
    if (lc < 0 || lc >= w.count) return;
    const DecChain ch = chains[w.first + lc];
    if (ch.n == 0) return;
    fse::ReaderPF br;
    const uint8_t *sb = in + ch.in;
    if (ch.inlen == 0 || ch.inlen >= (1ull << 28) || !br.init(sb, (uint32_t)ch.inlen)) {
        atomicExch(err, 6);
        return;
    }
    const unsigned long long map = w.map;
    uint32_t state = br.read(O1_PB);
    uint32_t ctx = 0;
    const int16_t *__restrict__ ov = ovf + ch.ovf;
    const uint32_t nov = (uint32_t)min((unsigned long long)0x7fffffff, n_ovf - ch.ovf);
    int16_t *o = out + ch.lo;
    const uint32_t n = (uint32_t)ch.n;
    uint32_t oi = 0;
    // escape values queued two deep, so each load has several steps to arrive
    int q0 = nov > 0 ? (int)__ldg(ov) : 0;
    int q1 = nov > 1 ? (int)__ldg(ov + 1) : 0;
    for (uint32_t j = 0; j < n; j++) {
        const uint32_t sl = (uint32_t)(map >> (4 * ctx)) & 15u;
        const uint32_t e = sl < (uint32_t)kDecSlots ? sdt[sl * O1_M + state] : __ldg(tb + ctx * O1_M + state);
        const bool esc = (e >> 21) & 1u;
        const int code = esc ? q0 : ((int)e >> 22);
        ctx = esc ? 13u + (uint32_t)(code < 0) : ((e >> 17) & 15u);
        if (esc) {
            oi++;
            q0 = q1;
            q1 = oi + 1 < nov ? (int)__ldg(ov + oi + 1) : 0;
        }
        o[j] = (int16_t)code;
        state = (e & 0x1FFFu) + br.read((e >> 13) & 15u);
    }
    if (oi > nov) atomicExch(err, 7);
    if (br.pos < br.start_bit(sb) - 16) atomicExch(err, 8);
}

// Context frequencies of one table set: the stationary distribution of the context chain implied
// by the normalized tables (the next context is a function of the decoded code; escapes split
// between the two large-magnitude contexts).  Returns (map, rev) for `slots` resident tables.
// ---- parallel chain encoder
// Every chain is cut into parts of `part` codes, one part per thread, all parts of a chain in one
// CTA.  A tANS encoder walks its chain backwards and only its state carries from one code to the
// next, so:
//   1. every part runs from a guessed entering state (the top part from the exact initial state),
//      writing its bits to its own staging area and keeping the state and the bit count at every
//      64th index (`sparse`, `sparse_bits`) and its exit state;
//   2. repair rounds: each part reruns from the exit state of the part above, writing the bits
//      again into a second staging area, until its state equals a kept one (from there on the two
//      runs, and their bits, are identical); a part that never meets its kept states has a new
//      exit state, so the part below repairs again in the next round.  Encoder states from
//      different starting points meet after a few hundred codes, so one round nearly always
//      suffices, and the loop ends after at most one round per part;
//   3. (the bits of a part: the repaired bits above the meeting index, then the speculative ones)
//   4. the bit counts give every part its offset in the chain's stream; every part shifts its
//      staged bits into place (words shared with a neighbour are merged with atomicOr);
//   5. every part start is a decode checkpoint: state, bit position, context and escape count.
// The stream is bit-identical to a sequential encoder's (the tANS states are fully determined).
// All 15 context state tables stay in shared memory: the two contexts that carry most codes (from
// the table set's histogram) as 16-bit states, the other 13 as 13-bit entries (state - 8192)
// packed into words; one word per key holds the symbol transform.  k_spec_image lays this out once
// per table set in global memory, and every CTA copies it in.
constexpr int kSpecThreads = 1024;
constexpr int kSpecHot = 2;
constexpr unsigned kSpecPackWords = (O1_NCTX - kSpecHot) * O1_M * O1_PB / 32 + 1;  // + 1: a read of w + 1
constexpr size_t kSpecSmem =
    ((size_t)kSpecHot * O1_M * 2 + (size_t)kSpecPackWords * 4 + (size_t)O1_NCTX * O1_NSYM * 4 + 15) & ~(size_t)15;
// Which table slot every context of a table set takes (4 bits each; slots 0 and 1 are the 16-bit
// tables).
struct SpecMeta {
    unsigned long long map;
};
constexpr int kSparseShift = 6;  // kept speculative states: every 64th index
struct SpecCta {
    int table;
    int first;  // first chain
    int count;  // chains
    int ppc;    // threads per chain (>= parts of every chain of the CTA)
    unsigned long long map, rev;
};

// Staging words of one part: 13 bits per code at most, plus the final state and end mark.
__host__ __device__ __forceinline__ size_t spec_stage_words(uint32_t part) { return ((size_t)part * 13 + 64) / 32 + 4; }

// keys[i] = context of code i (from code i-1; 0 at a chain's first code) << 8 | symbol of code i,
// written by k_o1_hist.

// Calls f(i, keys[i]) for i = top down to bottom, reading the keys through aligned 16-byte vectors
// (8 keys) fetched two vectors ahead.
template <class F>
__device__ __forceinline__ void walk_keys(const uint16_t *__restrict__ keys, long long top, long long bottom, F &&f) {
    long long i = top;
    for (; i >= bottom && (i & 7) != 7; i--) f(i, (uint32_t)__ldg(keys + i));
    if (i - 7 >= bottom) {
        const uint4 *kv = reinterpret_cast<const uint4 *>(keys);
        const uint4 z = make_uint4(0, 0, 0, 0);
        uint4 v0 = __ldg(kv + ((i - 7) >> 3));
        uint4 v1 = i - 15 >= 0 ? __ldg(kv + ((i - 15) >> 3)) : z;
        while (i - 7 >= bottom) {
            const uint4 v2 = i - 23 >= 0 ? __ldg(kv + ((i - 23) >> 3)) : z;
            f(i, v0.w >> 16);
            f(i - 1, v0.w & 0xFFFFu);
            f(i - 2, v0.z >> 16);
            f(i - 3, v0.z & 0xFFFFu);
            f(i - 4, v0.y >> 16);
            f(i - 5, v0.y & 0xFFFFu);
            f(i - 6, v0.x >> 16);
            f(i - 7, v0.x & 0xFFFFu);
            i -= 8;
            v0 = v1;
            v1 = v2;
        }
    }
    for (; i >= bottom; i--) f(i, (uint32_t)__ldg(keys + i));
}

// As walk_keys, but stops (and returns true) at the first index for which f returns true.
template <class F>
__device__ __forceinline__ bool walk_keys_until(const uint16_t *__restrict__ keys, long long top, long long bottom,
                                                F &&f) {
    long long i = top;
    for (; i >= bottom && (i & 7) != 7; i--)
        if (f(i, (uint32_t)__ldg(keys + i))) return true;
    if (i - 7 >= bottom) {
        const uint4 *kv = reinterpret_cast<const uint4 *>(keys);
        const uint4 z = make_uint4(0, 0, 0, 0);
        uint4 v0 = __ldg(kv + ((i - 7) >> 3));
        uint4 v1 = i - 15 >= 0 ? __ldg(kv + ((i - 15) >> 3)) : z;
        while (i - 7 >= bottom) {
            const uint4 v2 = i - 23 >= 0 ? __ldg(kv + ((i - 23) >> 3)) : z;
            if (f(i, v0.w >> 16) || f(i - 1, v0.w & 0xFFFFu) || f(i - 2, v0.z >> 16) || f(i - 3, v0.z & 0xFFFFu) ||
                f(i - 4, v0.y >> 16) || f(i - 5, v0.y & 0xFFFFu) || f(i - 6, v0.x >> 16) || f(i - 7, v0.x & 0xFFFFu))
                return true;
            i -= 8;
            v0 = v1;
            v1 = v2;
        }
    }
    for (; i >= bottom; i--)
        if (f(i, (uint32_t)__ldg(keys + i))) return true;
    return false;
}

// Per key (context << 8 | symbol) the encoder's symbol transform, as one word: deltaFindState +
// 8192 (bits 0-13), minStatePlus - 8192 (14-27) and maxBitsOut (28-31); the emitted bit count of
// state x is maxBitsOut - (x < minStatePlus), which is (x + deltaNbBits) >> 16 with deltaNbBits =
// (maxBitsOut << 16) - minStatePlus.
__host__ __device__ __forceinline__ uint32_t enc_word(const fse::SymTT &t) {
    const uint32_t mbo = (t.deltaNbBits + 0xFFFFu) >> 16, msp = (mbo << 16) - t.deltaNbBits;
    return (uint32_t)(t.deltaFindState + O1_M) | ((msp - O1_M) << 14) | (mbo << 28);
}

// The chain encoder's shared-memory image of table set blockIdx.y (kSpecSmem bytes at image +
// blockIdx.y * kSpecSmem / 4, laid out as k_o1_encode_spec's dynamic shared memory), filled by all
// blocks of the grid's x dimension: the 16-bit tables of the two contexts with the most codes in
// the set's histogram, the other contexts' 13-bit packed entries, and the transform word of every key.
__global__ void __launch_bounds__(256) k_spec_image(const uint16_t *__restrict__ stab,
                                                    const fse::SymTT *__restrict__ stt,
                                                    const uint32_t *__restrict__ thist, uint32_t *__restrict__ image,
                                                    SpecMeta *__restrict__ meta) {
    __shared__ uint32_t s_tot[O1_NCTX];
    __shared__ uint8_t s_rev[O1_NCTX];  // context of every slot
    const size_t tb = (size_t)blockIdx.y * O1_NCTX;
    const uint16_t *__restrict__ S = stab + tb * O1_M;
    if (threadIdx.x < O1_NCTX) s_tot[threadIdx.x] = 0;
    __syncthreads();
    {
        // codes per context: 16 threads per context, 16 symbols each
        const unsigned c = threadIdx.x / 16, s0 = (threadIdx.x % 16) * 16;
        if (c < (unsigned)O1_NCTX) {
            uint32_t v = 0;
#pragma unroll
            for (int u = 0; u < 16; u++) v += __ldg(thist + (tb + c) * O1_NSYM + s0 + u);
            atomicAdd(&s_tot[c], v);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int h0 = 0, h1 = 1;
        if (s_tot[h1] > s_tot[h0]) h0 = 1, h1 = 0;
        for (int c = 2; c < O1_NCTX; c++) {
            if (s_tot[c] > s_tot[h0]) h1 = h0, h0 = c;
            else if (s_tot[c] > s_tot[h1]) h1 = c;
        }
        unsigned long long m = 0;
        int slot = kSpecHot;
        s_rev[0] = (uint8_t)h0;
        s_rev[1] = (uint8_t)h1;
        for (int c = 0; c < O1_NCTX; c++) {
            const int sl = c == h0 ? 0 : c == h1 ? 1 : slot++;
            m |= (unsigned long long)sl << (4 * c);
            if (sl >= kSpecHot) s_rev[sl] = (uint8_t)c;
        }
        if (blockIdx.x == 0) meta[blockIdx.y].map = m;
    }
    __syncthreads();
    uint32_t *img = image + (size_t)blockIdx.y * (kSpecSmem / 4);
    uint32_t *hot2 = img;                                    // 16-bit tables, two entries per word
    uint32_t *pk = img + kSpecHot * O1_M / 2;                // packed state tables
    uint32_t *r_enc = pk + kSpecPackWords;                   // symbol transform per key
    constexpr unsigned kHotWords = kSpecHot * O1_M / 2, kKeys = O1_NCTX * O1_NSYM;
    constexpr unsigned kPacked = (O1_NCTX - kSpecHot) * O1_M;
    const unsigned total = kHotWords + kSpecPackWords + kKeys;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        if (i < kHotWords) {
            const unsigned e = 2 * i;  // entries e, e + 1 of the same context
            const uint16_t *row = S + (size_t)s_rev[e / O1_M] * O1_M + (e % O1_M);
            hot2[i] = (uint32_t)__ldg(row) | ((uint32_t)__ldg(row + 1) << 16);
        } else if (i < kHotWords + kSpecPackWords) {
            // word wd holds the bits [32 wd, 32 wd + 32) of the packed entries (entry j at bit 13 j;
            // entry j is state u = j % 8192 of the context in slot kSpecHot + j / 8192)
            const unsigned wd = i - kHotWords;
            uint32_t v = 0;
            const unsigned j0 = wd * 32 / O1_PB, j1 = min((wd * 32 + 31) / O1_PB, kPacked - 1);
            uint32_t ev[4];  // a word spans at most 4 entries
#pragma unroll
            for (unsigned u = 0; u < 4; u++) {
                const unsigned j = min(j0 + u, kPacked - 1);
                ev[u] = (uint32_t)__ldg(S + (size_t)s_rev[kSpecHot + j / O1_M] * O1_M + (j % O1_M)) - O1_M;  // 13 bits
            }
#pragma unroll
            for (unsigned u = 0; u < 4; u++) {
                const unsigned j = j0 + u;
                if (j > j1 || j >= kPacked) break;
                const int sh = (int)(j * O1_PB) - (int)(wd * 32);
                v |= sh >= 0 ? ev[u] << sh : ev[u] >> -sh;
            }
            pk[wd] = v;
        } else {
            const unsigned k = i - kHotWords - kSpecPackWords;
            r_enc[k] = enc_word(stt[tb * O1_NSYM + k]);
        }
    }
}

__global__ void __launch_bounds__(kSpecThreads) k_o1_encode_spec(
    const uint16_t *__restrict__ keys, const SegInfo *__restrict__ segs, const SpecCta *__restrict__ ctas,
    const uint32_t *__restrict__ image, const SpecMeta *__restrict__ meta,
    uint16_t *__restrict__ sparse,
    uint16_t *__restrict__ sparse_bits, uint32_t *__restrict__ stage, uint32_t *__restrict__ rstage,
    uint8_t *__restrict__ slots, const unsigned long long *__restrict__ slot_off,
    unsigned long long *__restrict__ blen, uint32_t part, O1Ckpt *__restrict__ cks,
    const unsigned long long *__restrict__ ck_off, uint32_t ck_every, int *__restrict__ err) {
    extern __shared__ uint4 smem_raw[];
    uint16_t *hot = reinterpret_cast<uint16_t *>(smem_raw);           // kSpecHot 16-bit tables
    uint32_t *pk = reinterpret_cast<uint32_t *>(hot + kSpecHot * O1_M);  // packed state tables
    uint32_t *r_enc = pk + kSpecPackWords;                              // symbol transform per key
    // after the walks, the transforms' space holds the parts' bit and escape counts
    uint16_t *s_bits = reinterpret_cast<uint16_t *>(r_enc), *s_esc = s_bits + kSpecThreads;
    __shared__ uint16_t s_exit[kSpecThreads + 1];
    __shared__ uint8_t s_chg[kSpecThreads + 1];
    const SpecCta w = ctas[blockIdx.x];
    const unsigned long long smap = meta[w.table].map;  // table slot of every context (4 bits each)
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(image + (size_t)w.table * (kSpecSmem / 4));
        for (unsigned i = threadIdx.x; i < kSpecSmem / 16; i += blockDim.x) smem_raw[i] = __ldg(src + i);
    }
    const int t = threadIdx.x;
    const int ci = t / w.ppc, p = t % w.ppc;
    const int chain = w.first + ci;
    long long lo = 0, hi = 0;
    if (ci < w.count) {
        const int g = chain / kMaxK, k = chain % kMaxK;
        const SegInfo sg = segs[g];
        if (k < sg.K) {
            lo = (long long)(sg.lo + (unsigned long long)k * sg.cs);
            hi = min(lo + (long long)sg.cs, (long long)(sg.lo + sg.n));
        }
        if (p == 0 && hi <= lo) blen[chain] = 0;
    }
    const int nparts = hi > lo ? (int)((hi - lo + part - 1) / part) : 0;
    const bool active = ci < w.count && p < nparts;
    const bool is_top = active && p == nparts - 1;
    const long long a = lo + (long long)p * part;
    const long long top = active ? min(a + (long long)part, hi) - 1 : 0;
    s_chg[t] = 0;
    s_exit[t] = 0;
    if (t == 0) {
        s_chg[kSpecThreads] = 0;
        s_exit[kSpecThreads] = 0;
    }
    __syncthreads();
    // a key's transform word and table slot
    struct EncRec {
        uint32_t e, slot;
    };
    auto rec_of = [&](uint32_t k) -> EncRec {
        return EncRec{r_enc[k], (uint32_t)(smap >> (4 * (k >> 8))) & 15u};
    };
    auto nbits = [](uint32_t x, const EncRec r) -> uint32_t {
        return (r.e >> 28) - ((x - (((r.e >> 14) & 0x3FFFu) + O1_M)) >> 31);
    };
    auto next_state = [&](uint32_t x, const EncRec r, uint32_t nb) -> uint32_t {
        const uint32_t idx = (x >> nb) + (r.e & 0x3FFFu) - O1_M;  // within the context's table
        if (r.slot < (uint32_t)kSpecHot) return hot[(r.slot << O1_PB) + idx];
        const uint32_t bit = (((r.slot - kSpecHot) << O1_PB) + idx) * O1_PB;
        const uint32_t wd = bit >> 5;
        return O1_M + (__funnelshift_r(pk[wd], pk[wd + 1], bit & 31u) & (O1_M - 1));
    };
    auto init_state = [&](uint32_t k) -> uint32_t {
        // FSE_initCState2: the state that codes symbol k with the fewest bits
        const EncRec r = rec_of(k);
        const uint32_t mbo = r.e >> 28, msp = ((r.e >> 14) & 0x3FFFu) + O1_M;
        const uint32_t dnb = (mbo << 16) - msp;
        const uint32_t nb = (dnb + (1u << 15)) >> 16;
        return next_state((nb << 16) - dnb, r, nb);
    };
    // the first code of a chain has context 0, so index lo is coded apart from the walks
    const long long istart = is_top ? hi - 2 : top;
    const long long bottom = p == 0 ? a + 1 : a;
    const uint32_t k_lo = p == 0 && active ? ((uint32_t)__ldg(keys + lo) & 0xFFu) : 0u;
    // Bit writer into a part's staging words (LSB first, as the stream).  The CTA's staging areas
    // are interleaved (word j of thread t at j * kSpecThreads + t), so that the placement step's
    // reads of the same word j by a warp share cache lines.
    struct Stager {
        uint32_t *w;
        uint64_t acc = 0;
        uint32_t accn = 0, nw = 0, bits = 0;
        __device__ void put(uint32_t v, uint32_t nb) {
            acc |= (uint64_t)(v & ((1u << nb) - 1u)) << accn;
            accn += nb;
            bits += nb;
            if (accn >= 32) {
                w[(size_t)(nw++) * kSpecThreads] = (uint32_t)acc;
                acc >>= 32;
                accn -= 32;
            }
        }
        __device__ void flush() {
            if (accn > 0) w[(size_t)nw * kSpecThreads] = (uint32_t)acc;
        }
    };
    const size_t stw = spec_stage_words(part);
    uint32_t *sw = stage + (size_t)blockIdx.x * kSpecThreads * stw + t;   // speculative bits
    uint32_t *rw = rstage + (size_t)blockIdx.x * kSpecThreads * stw + t;  // repaired bits
    // 1. speculative pass: walk and emit from the guessed state, keeping the state and the bit
    //    count after every 64th index
    uint32_t esc = 0, spec_bits = 0, spec_exit = 0;
    if (active) {
        Stager sg{sw};
        uint32_t x;
        if (is_top) {
            const uint32_t k0 = hi - 1 == lo ? k_lo : (uint32_t)__ldg(keys + hi - 1);
            x = init_state(k0);
            esc += (k0 & 0xFFu) == 0xFFu;
            if (((hi - 1) & 63) == 0) {
                sparse[(hi - 1) >> 6] = (uint16_t)x;
                sparse_bits[(hi - 1) >> 6] = 0;
            }
        } else {
            x = init_state((uint32_t)__ldg(keys + top + 1));
        }
        auto step = [&](long long i, uint32_t k) {
            const EncRec r = rec_of(k);
            const uint32_t nb = nbits(x, r);
            sg.put(x, nb);
            x = next_state(x, r, nb);
            esc += (k & 0xFFu) == 0xFFu;
            if (((uint32_t)i & 63u) == 0) {
                sparse[i >> 6] = (uint16_t)x;
                sparse_bits[i >> 6] = (uint16_t)sg.bits;
            }
        };
        walk_keys(keys, istart, bottom, step);
        if (p == 0 && istart >= lo) step(lo, k_lo);
        if (p == 0) {
            sg.put(x & (O1_M - 1), O1_PB);  // the final state, then the end mark
            sg.put(1u, 1u);
        }
        sg.flush();
        spec_bits = sg.bits;
        spec_exit = x;
        s_exit[t] = (uint16_t)x;
    }
    // every part's speculative exit state is read by the part below it, which may be in another warp
    __syncthreads();
    // 2. repair rounds (err[2] counts the re-run codes, err[3] the rounds, for diagnostics): a part
    //    whose entering state changed walks again from it, emitting into its repair staging, until
    //    its state meets a kept one at index m; its bits are then the repaired bits of the codes
    //    above m followed by the speculative bits from m on.  A part that never meets has all its
    //    bits in the repair staging and a new exit state, so the part below repairs again.
    bool need = active && !is_top;
    uint32_t repaired = 0;
    int mode = 0;                    // 0 speculative bits, 1 met, 2 repaired whole
    uint32_t rep_bits = 0, cut = 0;  // repaired bits; speculative bit where the suffix starts
    for (int round = 0;; round++) {
        if (round > nparts + 2 && need) atomicExch(err, 5);
        if (t == 0) atomicMax(err + 3, round);
        const uint32_t E = need ? s_exit[t + 1] : 0u;
        // an entering state outside the table would index outside the shared tables: refuse it
        const bool valid = E >= (uint32_t)O1_M && E < 2u * O1_M;
        if (need && !valid) atomicExch(err, 6);
        __syncthreads();
        bool changed = false;
        if (need && valid && round <= nparts + 2) {
            Stager rg{rw};
            uint32_t x = E;
            // the kept state of the next 64th index below, loaded one kept index ahead
            long long ck_i = top & ~63LL;
            uint32_t ck_x = ck_i >= a ? sparse[ck_i >> 6] : 0u;
            auto rstep = [&](long long i, uint32_t k) -> bool {
                const EncRec r = rec_of(k);
                const uint32_t nb = nbits(x, r);
                rg.put(x, nb);
                x = next_state(x, r, nb);
                repaired++;
                if (i != ck_i) return false;
                if (ck_x == x) {
                    cut = sparse_bits[i >> 6];
                    return true;
                }
                ck_i -= 64;
                ck_x = ck_i >= a ? sparse[ck_i >> 6] : 0u;
                return false;
            };
            // index lo (a chain's first code, context 0) is coded apart from the walk
            bool met = walk_keys_until(keys, top, p == 0 ? a + 1 : a, rstep);
            if (!met && p == 0) met = rstep(lo, k_lo);
            if (!met && p == 0) {
                rg.put(x & (O1_M - 1), O1_PB);
                rg.put(1u, 1u);
            }
            rg.flush();
            rep_bits = rg.bits;
            // the exit state: the speculative run's once met, else this run's
            const uint32_t ex = met ? spec_exit : x;
            mode = met ? 1 : 2;
            changed = ex != s_exit[t];
            s_exit[t] = (uint16_t)ex;
        }
        s_chg[t] = changed;
        __syncthreads();
        need = active && !is_top && s_chg[t + 1] != 0;
        if (!__syncthreads_or(need)) break;
    }
    if (repaired) atomicAdd(err + 2, (int)repaired);
    // the part's bits: [rw bits 0, rep_bits) then [sw bits cut, spec_bits)
    const uint32_t bits = mode == 0 ? spec_bits : mode == 1 ? rep_bits + (spec_bits - cut) : rep_bits;
    // 4. offsets (the top part's bits come first), escapes below each part, placement
    __syncthreads();  // the symbol transforms' space is reused for the counts
    s_bits[t] = active ? (uint16_t)bits : (uint16_t)0;
    s_esc[t] = active ? (uint16_t)esc : (uint16_t)0;
    __syncthreads();
    uint32_t off = 0, esc_below = 0;
    if (active) {
        for (int q = p + 1; q < nparts; q++) off += s_bits[t - p + q];
        for (int q = 0; q < p; q++) esc_below += s_esc[t - p + q];
    }
    uint32_t *ow = active ? reinterpret_cast<uint32_t *>(slots + slot_off[chain]) : nullptr;
    if (active) ow[off >> 5] = 0u;  // the first word may be shared with the part above: zeroed, then OR-ed
    __syncthreads();
    if (active) {
        // Output words [w0, wend).  Word w0 was zeroed by this part; the last word, when the part
        // ends inside it and a part follows, is the next part's first word (zeroed by it).  Both are
        // merged with atomicOr, every other word is this part's alone.
        const uint32_t w0 = off >> 5, wend = (off + bits + 31) >> 5;
        const uint32_t shared_last = (p > 0 && ((off + bits) & 31u)) ? wend - 1 : 0xFFFFFFFFu;
        uint32_t wi = w0;
        auto store = [&](uint32_t v) {
            if (wi == w0 || wi == shared_last) atomicOr(ow + wi, v);
            else ow[wi] = v;
            wi++;
        };
        uint64_t acc = 0;
        uint32_t accn = off & 31u;
        // appends bits [b0, b1) of staging words src, loading kBatch + 1 staging words (those
        // inside the part's staging column) before placing kBatch words
        constexpr uint32_t kBatch = 8;
        auto append = [&](const uint32_t *src, uint32_t b0, uint32_t b1) {
            const uint32_t sh = b0 & 31u;
            for (uint32_t bp = b0; bp < b1; bp += 32 * kBatch) {
                const uint32_t j0 = bp >> 5;
                uint32_t wv[kBatch + 1];
#pragma unroll
                for (uint32_t u = 0; u <= kBatch; u++)
                    wv[u] = j0 + u < (uint32_t)stw ? src[(size_t)(j0 + u) * kSpecThreads] : 0u;
#pragma unroll
                for (uint32_t u = 0; u < kBatch; u++) {
                    const uint32_t q = bp + 32 * u;
                    if (q >= b1) break;
                    const uint32_t n = min(32u, b1 - q);
                    uint32_t v = sh ? __funnelshift_r(wv[u], wv[u + 1], sh) : wv[u];
                    if (n < 32) v &= (1u << n) - 1u;
                    acc |= (uint64_t)v << accn;
                    accn += n;
                    if (accn >= 32) {
                        store((uint32_t)acc);
                        acc >>= 32;
                        accn -= 32;
                    }
                }
            }
        };
        if (mode != 0) append(rw, 0, rep_bits);
        if (mode != 2) append(sw, mode == 1 ? cut : 0u, spec_bits);
        if (accn > 0) store((uint32_t)acc);
        if (p == 0) blen[chain] = ((unsigned long long)off + bits + 7) / 8;
        // 5. decode checkpoint at every ck_every-th part start: the state the decoder holds
        // before index a
        if (p > 0 && cks && (uint32_t)p % ck_every == 0)
            cks[ck_off[chain] + (uint32_t)p / ck_every - 1] = O1Ckpt{off + bits, esc_below, (uint16_t)(s_exit[t] & (O1_M - 1)),
                                                (uint16_t)(__ldg(keys + a) >> 8)};
    }
}

// A decode table entry of a context not resident in shared memory (kept out of line so that the
// global load is only issued when taken).
__device__ __noinline__ uint32_t far_entry(const uint32_t *__restrict__ tb, uint32_t ctx, uint32_t state) {
    return __ldg(tb + ctx * O1_M + state);
}

// Decodes the parts of tANS chains, one part per thread (the chains' checkpoints give every part's
// starting bit position, state, context and escape offset).  The CTA's parts share one table set,
// staged in shared memory as for k_o1_decode_smem.  Each part that ends at a checkpoint checks that
// it arrived there (state, context, bit position, escapes); a mismatch sets err[1].
constexpr int kPartThreads = 1024;
__global__ void __launch_bounds__(kPartThreads) k_o1_decode_parts(const uint8_t *__restrict__ in,
                                                                 const DecChain *__restrict__ chains,
                                                                 const uint32_t *__restrict__ pstart,
                                                                 uint32_t nchains,
                                                                 const ChainCta *__restrict__ ctas,
                                                                 const uint32_t *__restrict__ dt,
                                                                 const int16_t *__restrict__ ovf,
                                                                 unsigned long long n_ovf,
                                                                 const O1Ckpt *__restrict__ cks, uint32_t part,
                                                                 int16_t *__restrict__ out, int *__restrict__ err) {
    extern __shared__ uint4 smem_raw[];
    uint32_t *sdt = reinterpret_cast<uint32_t *>(smem_raw);
    const ChainCta w = ctas[blockIdx.x];
    const uint32_t *__restrict__ tb = dt + (size_t)w.table * O1_NCTX * O1_M;
    for (int j = 0; j < kDecSlots; j++) {
        const int c = (int)((w.rev >> (4 * j)) & 15);
        if (c >= O1_NCTX) continue;
        const uint4 *src = reinterpret_cast<const uint4 *>(tb + (size_t)c * O1_M);
        uint4 *dst = reinterpret_cast<uint4 *>(sdt + (size_t)j * O1_M);
        for (int i = threadIdx.x; i < O1_M * 4 / 16; i += blockDim.x) dst[i] = __ldg(src + i);
    }
    __syncthreads();
    if ((int)threadIdx.x >= w.count) return;
    // this thread's part: the last chain (from the CTA's first one on) whose first part is at or
    // before the item
    DecPart pp;
    {
        const uint32_t item = (uint32_t)(w.first + (int)threadIdx.x);
        uint32_t lo = (uint32_t)w.pad, hi = nchains;  // pstart[lo] <= item < pstart[hi]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(pstart + mid) <= item) lo = mid;
            else hi = mid;
        }
        pp = DecPart{lo, item - __ldg(pstart + lo)};
    }
    const DecChain ch = chains[pp.chain];
    const unsigned long long start = (unsigned long long)pp.part * part;
    if (ch.n == 0 || start >= ch.n || ch.inlen == 0 || ch.inlen >= (1ull << 28)) {
        atomicExch(err, 6);
        return;
    }
    const uint32_t n = (uint32_t)min((unsigned long long)part, ch.n - start);
    const bool last = start + n >= ch.n;
    const uint8_t *sb = in + ch.in;
    const uint32_t sbits = (uint32_t)ch.inlen * 8u;
    fse::ReaderPF br;
    uint32_t state, ctx, oi0;
    if (pp.part == 0) {
        if (!br.init(sb, (uint32_t)ch.inlen)) {
            atomicExch(err, 6);
            return;
        }
        state = br.read(O1_PB);
        ctx = 0;
        oi0 = 0;
    } else {
        const O1Ckpt c = cks[ch.ck + pp.part - 1];
        if (c.bitpos >= sbits || c.state >= O1_M || c.ctx >= O1_NCTX || c.esc > ch.nesc) {
            atomicExch(err + 1, 1);
            return;
        }
        br.init_at(sb, (int32_t)c.bitpos);
        state = c.state;
        ctx = c.ctx;
        oi0 = c.esc;
    }
    const unsigned long long avail = n_ovf > ch.ovf + oi0 ? n_ovf - ch.ovf - oi0 : 0;
    const uint32_t nov = (uint32_t)min((unsigned long long)(ch.nesc - oi0), avail);
    int16_t *o = out + ch.lo + start;
    const unsigned long long map = w.map;
    uint32_t oi = 0;
    // Escape values come in 16-byte chunks of eight (ovf is 16-byte aligned, with slack behind
    // it); the chunk after the current one is loaded a whole chunk ahead, so that taking the next
    // value never waits on memory.
    const uint4 *ov4 = reinterpret_cast<const uint4 *>(ovf);
    const long long eb = (long long)(ch.ovf + oi0);
    long long ec = eb >> 3;
    int ek = (int)(eb & 7);
    auto echunk = [&](long long c) -> uint4 {
        return (unsigned long long)(c << 3) < n_ovf ? __ldg(ov4 + c) : make_uint4(0, 0, 0, 0);
    };
    auto ext = [](const uint4 &u, int k) -> int {
        const uint32_t wd = k < 4 ? (k < 2 ? u.x : u.y) : (k < 6 ? u.z : u.w);
        return (int)(int16_t)(k & 1 ? wd >> 16 : wd & 0xFFFFu);
    };
    uint4 ecur = nov > 0 ? echunk(ec) : make_uint4(0, 0, 0, 0);
    uint4 enxt = nov > 0 ? echunk(ec + 1) : make_uint4(0, 0, 0, 0);
    int q0 = nov > 0 ? ext(ecur, ek) : 0;
    auto step = [&]() -> int {
        const uint32_t sl = (uint32_t)(map >> (4 * ctx)) & 15u;
        uint32_t e;
        if (sl < (uint32_t)kDecSlots) e = sdt[sl * O1_M + state];
        else e = far_entry(tb, ctx, state);  // a real branch: the global load is never speculated
        const bool esc = (e >> 21) & 1u;
        const int code = esc ? q0 : ((int)e >> 22);
        ctx = esc ? 13u + (uint32_t)(code < 0) : ((e >> 17) & 15u);
        if (esc) {
            oi++;
            if (++ek == 8) {
                ecur = enxt;
                ec++;
                enxt = echunk(ec + 1);
                ek = 0;
            }
            q0 = oi < nov ? ext(ecur, ek) : 0;
        }
        state = (e & 0x1FFFu) + br.read((e >> 13) & 15u);
        return code;
    };
    // codes leave in aligned groups of eight (one 16-byte store) between a scalar head and tail
    const unsigned long long base = ch.lo + start;
    uint32_t j = 0;
    for (; j < n && ((base + j) & 7); j++) o[j] = (int16_t)step();
    for (; j + 8 <= n; j += 8) {
        uint32_t wv[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int a = step();
            const int b = step();
            wv[k] = (uint32_t)(uint16_t)a | ((uint32_t)(uint16_t)b << 16);
        }
        *reinterpret_cast<uint4 *>(o + j) = make_uint4(wv[0], wv[1], wv[2], wv[3]);
    }
    for (; j < n; j++) o[j] = (int16_t)step();
    if (oi > nov) atomicExch(err, 7);
    if (!last) {
        const O1Ckpt c = cks[ch.ck + pp.part];
        if (c.state != state || c.ctx != ctx || br.pos != br.start_bit(sb) + (int32_t)c.bitpos || c.esc != oi0 + oi)
            atomicExch(err + 1, 1);
    } else if (br.pos < br.start_bit(sb) - 16) {
        atomicExch(err, 8);
    }
}

std::pair<unsigned long long, unsigned long long> hot_contexts(const uint16_t *nf, int slots) {
    double P[O1_NCTX][O1_NCTX] = {};
    for (int c = 0; c < O1_NCTX; c++) {
        for (int s = 0; s < O1_NSYM; s++) {
            int f = (int16_t)nf[c * O1_NSYM + s];
            if (f < 0) f = 1;
            if (f == 0) continue;
            const double pr = f / (double)O1_M;
            if (s == O1_NSYM - 1) {
                P[c][13] += pr / 2;
                P[c][14] += pr / 2;
            } else {
                P[c][o1_ctx(unzz(s))] += pr;
            }
        }
    }
    double pi[O1_NCTX], nx[O1_NCTX];
    for (int c = 0; c < O1_NCTX; c++) pi[c] = 1.0 / O1_NCTX;
    for (int it = 0; it < 200; it++) {
        for (int c = 0; c < O1_NCTX; c++) nx[c] = 0;
        for (int a = 0; a < O1_NCTX; a++)
            for (int b = 0; b < O1_NCTX; b++) nx[b] += pi[a] * P[a][b];
        double sum = 0;
        for (int c = 0; c < O1_NCTX; c++) sum += nx[c];
        for (int c = 0; c < O1_NCTX; c++) pi[c] = sum > 0 ? nx[c] / sum : 1.0 / O1_NCTX;
    }
    int order[O1_NCTX];
    for (int c = 0; c < O1_NCTX; c++) order[c] = c;
    std::sort(order, order + O1_NCTX, [&](int a, int b) { return pi[a] > pi[b]; });
    unsigned long long map = ~0ULL, rev = ~0ULL;
    for (int j = 0; j < slots && j < O1_NCTX; j++) {
        const int c = order[j];
        map &= ~(15ULL << (4 * c));
        map |= (unsigned long long)j << (4 * c);
        rev &= ~(15ULL << (4 * j));
        rev |= (unsigned long long)c << (4 * j);
    }
    return {map, rev};
}

// CTAs of up to 64 consecutive chains that share a table set.
// Groups consecutive items (chains or parts) of one table into CTAs.  One CTA fills an SM (its
// tables take the shared memory), so the CTAs should be at most one per SM: every run of one table
// gets CTAs in proportion to its size (greedily, always to the run whose CTAs are largest), and
// a run's items are split evenly among its CTAs.  More items than SMs x max_per take several waves.
struct ItemRun {
    size_t first, len;
    int table;
};

// Runs of consecutive items with one table.
std::vector<ItemRun> table_runs(const std::vector<int> &chain_table) {
    std::vector<ItemRun> runs;
    const size_t n = chain_table.size();
    for (size_t i = 0; i < n;) {
        size_t j = i;
        while (j < n && chain_table[j] == chain_table[i]) j++;
        runs.push_back({i, j - i, chain_table[i]});
        i = j;
    }
    return runs;
}

std::vector<ChainCta> run_ctas(const std::vector<ItemRun> &runs, size_t n, const std::vector<unsigned long long> &maps,
                               const std::vector<unsigned long long> &revs, size_t max_per) {
    std::vector<ChainCta> out;
    const size_t sms = (size_t)sm_count();
    std::vector<size_t> ctas(runs.size(), 1);
    if (runs.size() <= sms && n <= sms * max_per) {
        auto size_of = [&](size_t r) { return (runs[r].len + ctas[r] - 1) / ctas[r]; };
        for (size_t used = runs.size(); used < sms; used++) {
            size_t best = 0;
            for (size_t r = 1; r < runs.size(); r++)
                if (size_of(r) > size_of(best)) best = r;
            if (size_of(best) <= 1) break;
            ctas[best]++;
        }
    }
    for (size_t r = 0; r < runs.size(); r++) {
        size_t c = std::max<size_t>(ctas[r], (runs[r].len + max_per - 1) / max_per);
        c = std::min(c, runs[r].len);
        const int t = runs[r].table;
        for (size_t k = 0; k < c; k++) {
            const size_t a = runs[r].first + runs[r].len * k / c;
            const size_t b = runs[r].first + runs[r].len * (k + 1) / c;
            if (b > a) out.push_back(ChainCta{t, (int)a, (int)(b - a), 0, maps[t], revs[t]});
        }
    }
    return out;
}

std::vector<ChainCta> chain_ctas(const std::vector<int> &chain_table, const std::vector<unsigned long long> &maps,
                                 const std::vector<unsigned long long> &revs, size_t max_per = kMaxChainsPerCta) {
    return run_ctas(table_runs(chain_table), chain_table.size(), maps, revs, max_per);
}

void enable_big_smem() {
    // once per device (a set of flags, one bit per device ordinal below 64)
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    FB2_CUDA(cudaGetDevice(&dev));
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return;
    FB2_CUDA(cudaFuncSetAttribute(k_o1_decode_smem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kDecSlots * O1_M * 4));
    FB2_CUDA(cudaFuncSetAttribute(k_o1_decode_parts, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kDecSlots * O1_M * 4));
    FB2_CUDA(cudaFuncSetAttribute(k_o1_encode_spec, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSpecSmem));
    FB2_CUDA(cudaFuncSetAttribute(k_o1_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHistSmem));
    done.fetch_or(bit, std::memory_order_acq_rel);
}

// Sum of the per-segment histograms of each table region (segments [rs[r], rs[r+1])).
__global__ void k_region_hist(const uint32_t *__restrict__ seg_hist, const int *__restrict__ rs,
                              uint32_t *__restrict__ reg_hist) {
    const int r = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= O1_NCTX * O1_NSYM) return;
    uint32_t s = 0;
    for (int g = rs[r]; g < rs[r + 1]; g++) s += seg_hist[(size_t)g * O1_NCTX * O1_NSYM + i];
    reg_hist[(size_t)r * O1_NCTX * O1_NSYM + i] = s;
}

// Flags segments whose 15 x 256 table equals the previous segment's (decode-side deduplication).
__global__ void k_table_same(const uint8_t *__restrict__ in, const unsigned long long *__restrict__ nf_off,
                             int nseg, int *__restrict__ same) {
    const int g = blockIdx.x;
    if (g >= nseg) return;
    __shared__ int diff;
    if (threadIdx.x == 0) diff = (g == 0);
    __syncthreads();
    if (g > 0) {
        const uint8_t *a = in + nf_off[g], *b = in + nf_off[g - 1];
        for (int i = threadIdx.x; i < O1_NCTX * O1_NSYM * 2; i += blockDim.x)
            if (a[i] != b[i]) diff = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) same[g] = !diff;
}

// Escape (|code| >= 128) extraction in index order: tile count + scan + scatter of zz+1 values.
__global__ void __launch_bounds__(kScanThreads) k_esc_tiles(const int16_t *__restrict__ q, long long n,
                                                           uint32_t *__restrict__ cnt) {
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    uint32_t c = 0;
    // 16-byte vectors when the code array is 16-byte aligned (tile starts are multiples of 16 codes)
    if (base + kScanItems <= n && (reinterpret_cast<uintptr_t>(q) & 15) == 0) {
        const int4 *p4 = reinterpret_cast<const int4 *>(q + base);
        const int4 a = __ldg(p4), b = __ldg(p4 + 1);
        const int32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
        for (int j = 0; j < kScanItems; j++)
            c += o1_sym((int16_t)(j & 1 ? w[j >> 1] >> 16 : w[j >> 1] & 0xFFFF)) == O1_NSYM - 1;
    } else {
        for (long long i = base; i < n && i < base + kScanItems; i++) c += o1_sym(q[i]) == O1_NSYM - 1;
    }
    __shared__ uint32_t sh[32];
    uint32_t tot;
    block_excl_scan<uint32_t>(c, sh, tot);
    if (threadIdx.x == 0) cnt[blockIdx.x] = tot;
}

// Escapes before each of npos code positions: the tile offset of the position's tile (exclusive
// scan of the tile counts) plus the escapes of the tile before the position, one warp per position.
__global__ void __launch_bounds__(256) k_esc_before(const int16_t *__restrict__ q,
                                                    const uint32_t *__restrict__ tile_off,
                                                    const unsigned long long *__restrict__ pos, int npos,
                                                    unsigned long long *__restrict__ out) {
    const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = (int)(threadIdx.x & 31u);
    if (w >= npos) return;
    const unsigned long long p = pos[w], t = p / kScanTile;
    uint32_t c = 0;
    for (unsigned long long i = t * kScanTile + lane; i < p; i += 32) c += o1_sym(q[i]) == O1_NSYM - 1;
    c = __reduce_add_sync(0xffffffffu, c);
    if (lane == 0) out[w] = (unsigned long long)tile_off[t] + c;
}

__global__ void __launch_bounds__(kScanThreads) k_esc_extract(const int16_t *__restrict__ q, long long n,
                                                             const uint32_t *__restrict__ tile_off,
                                                             uint32_t *__restrict__ vals, int16_t *__restrict__ raw) {
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int16_t v[kScanItems];
    uint32_t c = 0;
    static_assert(kScanItems == 16, "two 16-byte vectors per thread");
    if (base + kScanItems <= n && (reinterpret_cast<uintptr_t>(q) & 15) == 0) {
        const int4 *p4 = reinterpret_cast<const int4 *>(q + base);
        const int4 a = __ldg(p4), b = __ldg(p4 + 1);
        const int32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
        for (int j = 0; j < kScanItems; j++) v[j] = (int16_t)(j & 1 ? w[j >> 1] >> 16 : w[j >> 1] & 0xFFFF);
    } else {
#pragma unroll
        for (int j = 0; j < kScanItems; j++) v[j] = base + j < n ? q[base + j] : (int16_t)0;
    }
#pragma unroll
    for (int j = 0; j < kScanItems; j++) c += (base + j < n && o1_sym(v[j]) == O1_NSYM - 1);
    __shared__ uint32_t sh[32];
    // the tile's escapes are staged in shared memory in order, then leave as contiguous runs
    __shared__ int16_t sv[kScanTile];
    uint32_t tot;
    uint32_t r = block_excl_scan<uint32_t>(c, sh, tot);
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        if (base + j < n && o1_sym(v[j]) == O1_NSYM - 1) sv[r++] = v[j];
    }
    __syncthreads();
    const uint32_t t0 = tile_off[blockIdx.x];
    for (uint32_t k = threadIdx.x; k < tot; k += blockDim.x) {
        const int16_t e = sv[k];
        vals[t0 + k] = zigzag((int)e) + 1u;
        raw[t0 + k] = e;
    }
}



__global__ void k_m0_scatter(const uint32_t *__restrict__ runs, const uint32_t *__restrict__ vals,
                             const unsigned long long *__restrict__ start, long long nv, long long n,
                             int16_t *__restrict__ out) {
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < nv; j += (long long)gridDim.x * blockDim.x) {
        const unsigned long long pos = start[j] + runs[j] - 1;
        if ((long long)pos < n) out[pos] = (int16_t)unzz(vals[j] - 1u);
    }
}

__global__ void k_sample_windows(const int16_t *__restrict__ q, const unsigned long long *__restrict__ off, int nw,
                                 int wl, int16_t *__restrict__ outp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nw * wl) outp[i] = q[off[i / wl] + (i % wl)];
}

// Decodes gamma groups whose class streams are fse_enc records in host-visible bytes `h`
// (also present on the device at `d`).  vals must hold the group totals.
void gamma_decode(Pool &pool, const uint8_t *d, const ByteView &h,
                  const std::vector<size_t> &cls_off, const std::vector<size_t> &man_off,
                  const std::vector<size_t> &man_len, const std::vector<unsigned long long> &gstart,
                  uint32_t *d_vals, int *d_err, cudaStream_t st, const FseCkpt *d_fck = nullptr,
                  uint32_t fpart = 0, unsigned long long n_fck = 0, const unsigned long long *d_gdst = nullptr,
                  int16_t *d_ovf = nullptr) {
    const int G = (int)gstart.size() - 1;
    const long long T = (long long)gstart.back();
    if (T == 0) return;
    std::vector<BlockJob> jobs;
    for (int g = 0; g < G; g++) parse_blocks(h, cls_off[g], gstart[g + 1] - gstart[g], gstart[g], jobs);
    if (d_fck && fpart) {
        // the checkpoints belong to the FSE-coded blocks in stream order
        unsigned long long used = 0;
        for (auto &j : jobs)
            if (j.flag == 1) {
                const uint32_t c = fse_ckpt_count(j.n, fpart);
                j.ck = c ? (uint32_t)used : 0xFFFFFFFFu;
                used += c;
            }
        if (used != n_fck)
            for (auto &j : jobs) j.ck = 0xFFFFFFFFu;
    }
    uint8_t *cls = pool.get<uint8_t>(T);
    BlockJob *dj = h2d(pool, jobs, st);
    enable_fse_smem();
    k_fse_decode_blocks<<<(unsigned)jobs.size(), kFseDecThreads, kFseDecSmem, st>>>(d, dj, cls, d_err, fpart ? fpart : FBLK, d_fck);
    FB2_CHECK_LAUNCH();
    std::vector<unsigned long long> gman(G), glen(G), ust(G + 1, 0);
    for (int g = 0; g < G; g++) {
        gman[g] = man_off[g];
        glen[g] = man_len[g];
        ust[g + 1] = ust[g] + (gstart[g + 1] - gstart[g] + kUnit - 1) / kUnit;
    }
    const unsigned long long NU = ust[G];
    unsigned long long *d_gstart = h2d(pool, gstart, st);
    unsigned long long *d_gman = h2d(pool, gman, st);
    unsigned long long *d_glen = h2d(pool, glen, st);
    unsigned long long *d_ust = h2d(pool, ust, st);
    unsigned long long *usum = pool.get<unsigned long long>(NU + 1);
    unsigned long long *uoff = pool.get<unsigned long long>(NU + 1);
    void *sc = pool.get<uint8_t>(scan_scratch_bytes((long long)NU, 8));
    k_unit_bits<<<grid_for((long long)NU * 32, 256), 256, 0, st>>>(cls, d_gstart, d_ust, G, NU, usum);
    FB2_CHECK_LAUNCH();
    exclusive_scan<unsigned long long, unsigned long long>(usum, (long long)NU, uoff, sc, st);
    k_gamma_unpack_units<<<grid_for((long long)NU * 32, 256), 256, 0, st>>>(cls, d_gstart, d_ust, G, NU, uoff, d_gman,
                                                                           d, d_glen, d_vals, d_err, d_gdst, d_ovf);
    FB2_CHECK_LAUNCH();
}



}  // namespace

// ================================================================== public
EntropyChoice choose_entropy(Context &ctx, const int16_t *d_codes, size_t n, cudaStream_t st) {
    (void)ctx;
    // RleFseEncoder::preprocess_encode: 256 windows x 32 codes
    size_t NW = 256, WL = 32;
    if (n < NW * WL) {
        WL = n / NW;
        if (!WL) WL = 1;
    }
    size_t step = (n > NW * WL) ? (n - WL) / NW : WL;
    if (!step) step = 1;
    std::vector<unsigned long long> offs;
    for (size_t w = 0; w < NW; w++) {
        const size_t off = w * step;
        if (off + WL > n) break;
        offs.push_back(off);
    }
    EntropyChoice ch{0, false};
    size_t z = 0, zd = 0, cnt = 0, cntd = 0;
    if (!offs.empty()) {
        Pool pool(st);
        unsigned long long *d_off = h2d(pool, offs, st);
        int16_t *d_s = pool.get<int16_t>(offs.size() * WL);
        const int tot = (int)(offs.size() * WL);
        k_sample_windows<<<(tot + 255) / 256, 256, 0, st>>>(d_codes, d_off, (int)offs.size(), (int)WL, d_s);
        FB2_CHECK_LAUNCH();
        std::vector<int16_t> s = d2h(d_s, (size_t)tot, st);
        for (size_t w = 0; w < offs.size(); w++) {
            int16_t prev = s[w * WL];
            for (size_t t = 0; t < WL; t++) {
                const int16_t x = s[w * WL + t];
                if (x == 0) z++;
                if (t > 0 && x == prev) zd++;
                prev = x;
            }
            cnt += WL;
            cntd += WL - 1;
        }
    }
    const double p0 = cnt ? 1.0 * z / cnt : 1.0;
    const double dzeros = (cnt && cntd) ? (1.0 * zd / cntd - p0) : 0.0;
    ch.delta = dzeros > 0.005;
    ch.method = (p0 >= 0.80) ? 0 : 1;
    if (n < (size_t)20 * O1_NCTX * O1_NSYM) ch.method = 0;
    return ch;
}

void entropy_encode_into(Pool &pool, Assembler &as, const int16_t *d_codes_in, size_t n, const EntropyChoice &ch,
                         cudaStream_t st, const EntropyTuning &tune) {
    Trace tr("encode");
    const long long N = (long long)n;
    const int16_t *q = d_codes_in;
    if (ch.delta && N > 0) {
        int16_t *dq = pool.get<int16_t>(N);
        k_delta<<<grid_for(N, 256), 256, 0, st>>>(d_codes_in, N, dq);
        FB2_CHECK_LAUNCH();
        q = dq;
    }
    const uint8_t mb = (uint8_t)(ch.method | (ch.delta ? 0x80 : 0));
    CkptCollector cc;
    {
        const uint32_t part = tune.ckpt_part;
        const bool pow2 = part >= 64 && part <= (uint32_t)FBLK && (part & (part - 1)) == 0;
        cc.o1_part = cc.fse_part = pow2 ? part : 0;
    }
    as.val<uint8_t>(mb);
    as.val<uint16_t>(0);  // lo_
    as.val<uint16_t>(0);  // mode_
    if (ch.method == 0) {
        const long long tiles = std::max<long long>(1, (N + kScanTile - 1) / kScanTile);
        uint32_t *tcnt = pool.get<uint32_t>(tiles + 2);
        long long *tlast = pool.get<long long>(tiles + 2);
        FB2_CUDA(cudaMemsetAsync(tcnt, 0, (tiles + 2) * 4, st));
        if (N > 0) {
            k_m0_tiles<<<(unsigned)tiles, kScanThreads, 0, st>>>(q, N, tcnt, tlast);
            FB2_CHECK_LAUNCH();
        } else {
            FB2_CUDA(cudaMemsetAsync(tlast, 0xff, 8, st));
        }
        k_scan_small<uint32_t><<<1, 1024, 0, st>>>(tcnt, tiles);
        FB2_CHECK_LAUNCH();
        k_prefix_last<<<1, 1024, 0, st>>>(tlast, tiles);
        FB2_CHECK_LAUNCH();
        const uint32_t nv32 = d2h(tcnt + tiles, 1, st)[0];
        const long long lastnz = d2h(tlast + tiles, 1, st)[0];
        const unsigned long long nv = nv32;
        const bool trailing = N > 0 && lastnz < N - 1;
        const unsigned long long nr = nv + (trailing ? 1 : 0);
        uint32_t *buf = pool.get<uint32_t>(nr + nv + 2);  // runs [0, nr), values [nr, nr + nv)
        if (N > 0 && nv > 0) {
            k_m0_extract<<<(unsigned)tiles, kScanThreads, 0, st>>>(q, N, tcnt, tlast, buf, buf + nr);
            FB2_CHECK_LAUNCH();
        }
        if (trailing) {
            const uint32_t tr = (uint32_t)(N - 1 - lastnz + 1);  // L + 1
            FB2_CUDA(cudaMemcpyAsync(buf + nv, &tr, 4, cudaMemcpyHostToDevice, st));
            FB2_CUDA(cudaStreamSynchronize(st));
        }
        GammaOut go = gamma_encode(pool, buf, {0ULL, nr, nr + nv}, st, cc.fse_part);
        as.val<uint64_t>(nr);
        as.val<uint64_t>(nv);
        as.val<uint64_t>(go.cls_bytes[0]);
        as.val<uint64_t>(go.cls_bytes[1]);
        as.val<uint64_t>(go.man_bytes[0]);
        as.val<uint64_t>(go.man_bytes[1]);
        add_class_pieces(as, go, 0, &cc);
        add_class_pieces(as, go, 1, &cc);
        as.dev(go.man_ptr[0], go.man_bytes[0]);
        as.dev(go.man_ptr[1], go.man_bytes[1]);
    } else {
        // ---- segmentation: K chains per segment, S segments (decoder reads S and K from the stream)
        const int K = std::max(1, std::min(kMaxK, tune.o1_streams));
        // S segments as the reference sizes them, N / 8 Mi within [1, 16] (RleFseEncoder.hpp:582-587):
        // every segment carries its own 7.5 KiB table set, so few segments keep the payload as small
        // as the reference's; parallelism comes from the chains and their parts instead.
        long long S = tune.o1_segment > 0 ? std::max<long long>(1, (N + tune.o1_segment - 1) / tune.o1_segment)
                                          : std::min<long long>(16, std::max<long long>(1, N / (8LL << 20)));
        if (S > N) S = std::max<long long>(1, N);
        // every segment must be non-empty: an empty one ends after its N and K words
        while (S > 1 && (S - 1) * ((N + S - 1) / S) >= N) S--;
        const long long seg = (N + S - 1) / S;
        std::vector<SegInfo> segs(S);
        for (long long g = 0; g < S; g++) {
            const long long lo = g * seg;
            const long long hi = std::min<long long>(lo + seg, N);
            const long long ng = std::max<long long>(0, hi - lo);
            segs[g] = SegInfo{(unsigned long long)lo, (unsigned long long)ng,
                              (unsigned long long)((ng + K - 1) / K), K, 0};
        }
        SegInfo *d_segs = h2d(pool, segs, st);
        // encoder part size (also the decode checkpoint spacing): a chain's parts fit one CTA
        unsigned long long max_cs = 1;
        for (const auto &sg : segs) max_cs = std::max<unsigned long long>(max_cs, sg.cs);
        uint32_t enc_part = std::min<uint32_t>(cc.o1_part ? cc.o1_part : 1024u, 1024u);
        while ((max_cs + enc_part - 1) / enc_part > (unsigned long long)kSpecThreads) enc_part *= 2;
        if (cc.o1_part && cc.o1_part < enc_part) cc.o1_part = enc_part;
        const uint32_t ck_every = cc.o1_part ? cc.o1_part / enc_part : 1u;
        const int ppc = (int)((max_cs + enc_part - 1) / enc_part);
        // decode checkpoints of every chain: one before each index lo + q * part, q >= 1
        const long long nchains_all = S * kMaxK;
        std::vector<unsigned long long> ck_off(nchains_all + 1, 0);
        for (long long g = 0; g < S; g++)
            for (int k = 0; k < kMaxK; k++) {
                unsigned long long cnt = 0;
                if (k < K && cc.o1_part) {
                    const unsigned long long clo = segs[g].lo + (unsigned long long)k * segs[g].cs;
                    const unsigned long long chi = std::min(clo + segs[g].cs, segs[g].lo + segs[g].n);
                    if (chi > clo) cnt = (chi - clo - 1) / cc.o1_part;
                }
                ck_off[g * kMaxK + k + 1] = ck_off[g * kMaxK + k] + cnt;
            }
        cc.n_o1 = ck_off.back();
        O1Ckpt *o1ck = cc.n_o1 ? pool.get<O1Ckpt>(cc.n_o1) : nullptr;
        cc.o1 = o1ck;
        unsigned long long *d_ck_off = o1ck ? h2d(pool, ck_off, st) : nullptr;
        uint32_t *hist = pool.get<uint32_t>((size_t)S * O1_NCTX * O1_NSYM);
        uint32_t *nvk = pool.get<uint32_t>((size_t)S * kMaxK);
        uint16_t *keys = pool.get<uint16_t>((size_t)N + 8);
        FB2_CUDA(cudaMemsetAsync(hist, 0, (size_t)S * O1_NCTX * O1_NSYM * 4, st));
        FB2_CUDA(cudaMemsetAsync(nvk, 0, (size_t)S * kMaxK * 4, st));
        // The escape side stream (escape values in index order, their gamma classes, the FSE class
        // blocks) needs only the codes, so it forks before the histogram pass and runs next to it,
        // the table builds and the chain encoder.
        const long long tiles = std::max<long long>(1, (N + kScanTile - 1) / kScanTile);
        uint32_t *tcnt = pool.get<uint32_t>(tiles + 2);
        FB2_CUDA(cudaMemsetAsync(tcnt, 0, (tiles + 2) * 4, st));
        const bool fork = tune.side != nullptr && tune.fork_ev != nullptr && tune.join_ev != nullptr;
        cudaStream_t es = fork ? tune.side : st;
        if (fork) {
            FB2_CUDA(cudaEventRecord(tune.fork_ev, st));
            FB2_CUDA(cudaStreamWaitEvent(es, tune.fork_ev, 0));
        }
        struct Join {  // the calling stream waits for the second one before anything is freed
            bool on;
            cudaStream_t st, es;
            cudaEvent_t ev;
            void operator()() {
                if (on) {
                    cudaEventRecord(ev, es);
                    cudaStreamWaitEvent(st, ev, 0);
                    on = false;
                }
            }
            ~Join() { (*this)(); }
        } join{fork, st, es, tune.join_ev};
        Pool spool(es);  // scratch of the escape side stream, handed to `pool` once joined
        if (N > 0) {
            k_esc_tiles<<<(unsigned)tiles, kScanThreads, 0, es>>>(q, N, tcnt);
            FB2_CHECK_LAUNCH();
        }
        k_scan_small<uint32_t><<<1, 1024, 0, es>>>(tcnt, tiles);
        FB2_CHECK_LAUNCH();
        // escapes before every segment start (the groups of the escape stream)
        unsigned long long *d_gstart = spool.get<unsigned long long>(S + 1);
        {
            std::vector<unsigned long long> pos(S + 1);
            for (long long g = 0; g < S; g++) pos[g] = segs[g].lo;
            pos[S] = (unsigned long long)N;
            unsigned long long *d_pos = h2d(spool, pos, es);
            k_esc_before<<<(unsigned)((S + 1 + 7) / 8), 256, 0, es>>>(q, tcnt, d_pos, (int)(S + 1), d_gstart);
            FB2_CHECK_LAUNCH();
        }
        tr.gpu("escape counts done", es);
        enable_big_smem();
        tr.gpu("histogram start", st);
        {
            // about four CTAs per SM over all segments, a slice at least 64 Ki codes long
            const long long want = (4LL * 148 + S - 1) / S;
            const long long U = std::max<long long>(1, std::min<long long>(want, (seg + 65535) / 65536));
            k_o1_hist<<<dim3((unsigned)S, (unsigned)U), 1024, kHistSmem, st>>>(
                q, d_segs, hist, nvk, keys, (reinterpret_cast<uintptr_t>(q) & 15) == 0);
        }
        FB2_CHECK_LAUNCH();
        tr.gpu("histogram done", st);
        // table regions: segments whose statistics come from the same part of the code stream
        // share one table set (tune.regions holds the code positions where statistics change)
        std::vector<int> seg_region(S, 0), rs{0};
        if (tune.per_segment_tables) {
            for (long long g = 0; g < S; g++) seg_region[g] = (int)g;
            for (long long g = 1; g <= S; g++) rs.push_back((int)g);
        } else {
            int prev_rr = -1;
            for (long long g = 0; g < S; g++) {
                int rr = 0;
                for (long long b : tune.regions)
                    if (b > 0 && (unsigned long long)b <= segs[g].lo) rr++;
                if (g > 0 && rr != prev_rr) rs.push_back((int)g);
                seg_region[g] = (int)rs.size() - 1;
                prev_rr = rr;
            }
            rs.push_back((int)S);
        }
        const int R = (int)rs.size() - 1;
        uint32_t *rhist = hist;
        if (!tune.per_segment_tables) {
            rhist = pool.get<uint32_t>((size_t)R * O1_NCTX * O1_NSYM);
            int *d_rs = h2d(pool, rs, st);
            k_region_hist<<<dim3((O1_NCTX * O1_NSYM + 255) / 256, R), 256, 0, st>>>(hist, d_rs, rhist);
            FB2_CHECK_LAUNCH();
        }
        int *d_tab = h2d(pool, seg_region, st);
        const int ntab = R * O1_NCTX;
        uint16_t *nf = pool.get<uint16_t>((size_t)ntab * O1_NSYM);
        k_o1_norm<<<(ntab + 7) / 8, 256, 0, st>>>(rhist, ntab, nf);
        FB2_CHECK_LAUNCH();
        uint16_t *stab = pool.get<uint16_t>((size_t)ntab * O1_M);
        fse::SymTT *stt = pool.get<fse::SymTT>((size_t)ntab * O1_NSYM);
        uint8_t *spread = pool.get<uint8_t>((size_t)ntab * O1_M);
        int *d_err = pool.get<int>(8);
        FB2_CUDA(cudaMemsetAsync(d_err, 0, 32, st));
        k_o1_ctable<<<ntab, kTabThreads, 0, st>>>(nf, stab, stt, spread, d_err);
        FB2_CHECK_LAUNCH();
        // the chain encoder's shared-memory image of every table set
        uint32_t *image = pool.get<uint32_t>((size_t)R * (kSpecSmem / 4));
        SpecMeta *meta = pool.get<SpecMeta>((size_t)R);
        {
            const unsigned items = kSpecHot * O1_M / 2 + kSpecPackWords + O1_NCTX * O1_NSYM;
            k_spec_image<<<dim3((items + 255) / 256, (unsigned)R), 256, 0, st>>>(stab, stt, rhist, image, meta);
            FB2_CHECK_LAUNCH();
        }
        // escapes in index order, on the second stream (the host waits here for their count; the
        // histogram pass and the table builds, launched above, run meanwhile)
        const std::vector<unsigned long long> gstart = d2h(d_gstart, (size_t)S + 1, es);
        const unsigned long long E = gstart[S];
        uint32_t *evals = spool.get<uint32_t>(E + 1);
        int16_t *eraw = spool.get<int16_t>(E + 1);
        if (E > 0) {
            k_esc_extract<<<(unsigned)tiles, kScanThreads, 0, es>>>(q, N, tcnt, evals, eraw);
            FB2_CHECK_LAUNCH();
        }
        tr.gpu("escapes extracted", es);
        // the class blocks (long sequential chains) reach the GPU before the chain encoder, so that
        // they take a few SMs of their own instead of waiting for the chain encoder's last wave
        const bool queue_first = fork && tune.queued_ev != nullptr;
        const GammaBlocks gblocks = gamma_launch(spool, evals, gstart, es, cc.fse_part,
                                                 queue_first ? tune.queued_ev : nullptr, (size_t)(S * K));
        tr.gpu("class blocks done", es);
        if (queue_first) FB2_CUDA(cudaStreamWaitEvent(st, tune.queued_ev, 0));
        tr.mark("class blocks launched");
        // chain output slots
        const long long nchains = S * kMaxK;
        std::vector<unsigned long long> soff(nchains + 1, 0);
        for (long long g = 0; g < S; g++)
            for (int k = 0; k < kMaxK; k++) {
                const unsigned long long c = (k < K) ? segs[g].cs * 2 + 64 : 0;
                soff[g * kMaxK + k + 1] = soff[g * kMaxK + k] + ((c + 15) & ~15ULL);
            }
        unsigned long long *d_soff = h2d(pool, soff, st);
        uint8_t *slots = pool.get<uint8_t>(soff.back() + 16);
        unsigned long long *blen = pool.get<unsigned long long>(nchains);
        {
            tr.mark("tables launched");
            const std::vector<unsigned long long> maps(R, 0), revs(R, 0);  // every table is resident
            std::vector<int> chain_table((size_t)nchains);
            for (long long ch = 0; ch < nchains; ch++) chain_table[ch] = seg_region[ch / kMaxK];
            const std::vector<ChainCta> groups = chain_ctas(chain_table, maps, revs, (size_t)(kSpecThreads / ppc));
            std::vector<SpecCta> ctas;
            for (const ChainCta &c : groups) ctas.push_back(SpecCta{c.table, c.first, c.count, ppc, c.map, c.rev});
            SpecCta *d_ctas = h2d(pool, ctas, st);
            uint16_t *sparse = pool.get<uint16_t>(((size_t)N >> kSparseShift) + 2);
            uint16_t *sparse_bits = pool.get<uint16_t>(((size_t)N >> kSparseShift) + 2);
            uint32_t *stage = pool.get<uint32_t>(ctas.size() * kSpecThreads * spec_stage_words(enc_part));
            uint32_t *rstage = pool.get<uint32_t>(ctas.size() * kSpecThreads * spec_stage_words(enc_part));
            enable_big_smem();
            tr.gpu("chain encoder start", st);
            k_o1_encode_spec<<<(unsigned)ctas.size(), kSpecThreads, kSpecSmem, st>>>(
                keys, d_segs, d_ctas, image, meta, sparse, sparse_bits, stage, rstage, slots, d_soff, blen, enc_part, o1ck,
                d_ck_off, ck_every, d_err);
            FB2_CHECK_LAUNCH();
            tr.gpu("chain encoder done", st);
            tr.mark("chains launched");
        }
        GammaOut go = gamma_finish(spool, gblocks, evals, es);
        tr.gpu("escape mantissas packed", es);
        // the chains' escape counts (stream header) from the histogram pass; their sums per segment
        // are the escape groups counted above
        const std::vector<uint32_t> h_nvk = d2h(nvk, (size_t)S * kMaxK, st);
        for (long long g = 0; g < S; g++) {
            unsigned long long e = 0;
            for (int k = 0; k < K; k++) e += h_nvk[g * kMaxK + k];
            if (e != gstart[g + 1] - gstart[g]) throw std::runtime_error("escape counts of the two passes differ");
        }
        tr.mark("escapes coded");
        std::vector<unsigned long long> h_blen = d2h(blen, (size_t)nchains, st);
        std::vector<int> h_err = d2h(d_err, 5, st);
        tr.gpu_dump();
        if (h_err[0]) throw std::runtime_error("tANS encoding failed (table construction or chain repair)");
        // Decode checkpoints cost 12 bytes each: keep them within 1.5 % of the chains' bytes by
        // keeping every m-th one (m a power of two; the decoder's parts become m times longer, so
        // streams whose codes take a few bits each, where the checkpoints weigh most, decode with
        // fewer, longer parts).
        if (cc.n_o1) {
            unsigned long long chain_bytes = 0;
            for (auto b : h_blen) chain_bytes += b;
            uint32_t m = 1;
            while (m < (1u << 16) && 12ull * (cc.n_o1 / m) * 1000 > 15 * chain_bytes) m *= 2;
            if (m > 1) {
                std::vector<unsigned long long> noff(nchains_all + 1, 0);
                const unsigned long long part2 = (unsigned long long)cc.o1_part * m;
                for (long long g = 0; g < S; g++)
                    for (int k = 0; k < kMaxK; k++) {
                        unsigned long long cnt = 0;
                        if (k < K) {
                            const unsigned long long clo = segs[g].lo + (unsigned long long)k * segs[g].cs;
                            const unsigned long long chi = std::min(clo + segs[g].cs, segs[g].lo + segs[g].n);
                            if (chi > clo) cnt = (chi - clo - 1) / part2;
                        }
                        noff[g * kMaxK + k + 1] = noff[g * kMaxK + k] + cnt;
                    }
                O1Ckpt *thin = noff.back() ? pool.get<O1Ckpt>(noff.back()) : nullptr;
                if (thin) {
                    unsigned long long *d_noff = h2d(pool, noff, st);
                    k_ck_thin<<<dim3(4, (unsigned)nchains_all), 256, 0, st>>>(o1ck, d_ck_off, d_noff,
                                                                            (int)nchains_all, m, thin);
                    FB2_CHECK_LAUNCH();
                }
                cc.o1 = thin;
                cc.n_o1 = noff.back();
                cc.o1_part = (uint32_t)part2;
            }
        }
        if (tr.on)
            std::fprintf(stderr, "[falcons trace] encode chain repair: %d codes re-run, %d rounds, %d far lookups; "
                         "%lld segments, %d chains each\n", h_err[2], h_err[3], h_err[4], S, K);
        tr.mark("chains done");
        join();
        pool.ptrs.insert(pool.ptrs.end(), spool.ptrs.begin(), spool.ptrs.end());
        spool.ptrs.clear();
        for (auto b : h_blen)
            if (b == ~0ULL) throw std::runtime_error("tANS chain overflow");
        as.val<uint64_t>((uint64_t)S);
        as.host.reserve(as.host.size() + (size_t)S * (16 + 16 * K + 32));
        as.pieces.reserve(as.pieces.size() + (size_t)S * (K + 8) + 64);
        for (long long g = 0; g < S; g++) {
            // the segment's header words (N, K, chain lengths, escape counts) in one piece
            uint64_t hw[2 + 2 * kMaxK];
            hw[0] = segs[g].n;
            hw[1] = (uint64_t)K;
            for (int k = 0; k < K; k++) hw[2 + k] = h_blen[g * kMaxK + k];
            for (int k = 0; k < K; k++) hw[2 + K + k] = h_nvk[g * kMaxK + k];
            as.bytes(hw, (size_t)(2 + 2 * K) * 8);
            as.dev(nf + (size_t)seg_region[g] * O1_NCTX * O1_NSYM, O1_NCTX * O1_NSYM * 2);
            for (int k = 0; k < K; k++) as.dev(slots + soff[g * kMaxK + k], h_blen[g * kMaxK + k]);
            const unsigned long long ne = gstart[g + 1] - gstart[g];
            if (ne == 0) {
                as.val<uint8_t>(0);
            } else {
                const size_t raw = ne * 2;
                const size_t cm = go.cls_bytes[g] + go.man_bytes[g] + 16;
                if (cm >= raw) {
                    as.val<uint8_t>(0);
                    as.dev(eraw + gstart[g], raw);
                } else {
                    as.val<uint8_t>(1);
                    as.val<uint64_t>(go.cls_bytes[g]);
                    as.val<uint64_t>(go.man_bytes[g]);
                    add_class_pieces(as, go, (int)g, &cc);
                    as.dev(go.man_ptr[g], go.man_bytes[g]);
                }
            }
        }
    }
    cc.emit(as);
}

size_t entropy_encode(Context &ctx, const int16_t *d_codes, size_t n, const EntropyChoice &ch, uint8_t *d_out,
                      size_t cap, cudaStream_t st, const EntropyTuning &tune) {
    (void)ctx;
    Pool pool(st);
    Assembler as;
    entropy_encode_into(pool, as, d_codes, n, ch, st, tune);
    if (as.pos > cap) throw std::length_error("The buffer for compressed data is not large enough.");
    as.run(pool, d_out, st);
    return (size_t)as.pos;
}

bool parse_ckpt_header(const uint8_t *h, const uint8_t *d_content, size_t avail, DecodeCheckpoints &out) {
    if (avail < kCkptHeader) return false;
    uint32_t w[4];
    uint64_t n1, n2;
    memcpy(w, h, 16);
    memcpy(&n1, h + 16, 8);
    memcpy(&n2, h + 24, 8);
    if (w[0] != kCkptTag || w[1] != kCkptVersion) return false;
    if (n1 > avail / sizeof(O1Ckpt) || n2 > avail / sizeof(FseCkpt)) return false;
    if (kCkptHeader + n1 * sizeof(O1Ckpt) + n2 * sizeof(FseCkpt) != avail) return false;
    out.d_o1 = d_content + kCkptHeader;
    out.n_o1 = n1;
    out.o1_part = w[2];
    out.d_fse = out.d_o1 + n1 * sizeof(O1Ckpt);
    out.n_fse = n2;
    out.fse_part = w[3];
    return true;
}

size_t entropy_decode(Context &ctx, const uint8_t *d_in, const ByteView &h, size_t n, int16_t *d_codes,
                      cudaStream_t st, const DecodeCheckpoints *ck) {
    Trace tr("decode");
    Pool pool(st);
    tr.gpu("decode begin", st);
    // checkpoint arrays, copied to aligned scratch (their place in the stream has any alignment)
    auto pow2 = [](uint32_t v) { return v >= 64 && v <= (uint32_t)FBLK && (v & (v - 1)) == 0; };
    const O1Ckpt *o1ck = nullptr;
    const FseCkpt *fck = nullptr;
    uint32_t o1_part = 0, f_part = 0;
    unsigned long long n_o1ck = 0, n_fck = 0;
    if (ck && ck->n_o1 && ck->d_o1 && pow2(ck->o1_part) && ck->n_o1 < (1ULL << 32)) {
        O1Ckpt *d = pool.get<O1Ckpt>(ck->n_o1);
        launch_gather(pool, {Piece{ck->d_o1, 0, ck->n_o1 * sizeof(O1Ckpt)}}, reinterpret_cast<uint8_t *>(d), st);
        o1ck = d;
        o1_part = ck->o1_part;
        n_o1ck = ck->n_o1;
    }
    if (ck && ck->n_fse && ck->d_fse && pow2(ck->fse_part) && ck->n_fse < (1ULL << 32)) {
        FseCkpt *d = pool.get<FseCkpt>(ck->n_fse);
        launch_gather(pool, {Piece{ck->d_fse, 0, ck->n_fse * sizeof(FseCkpt)}}, reinterpret_cast<uint8_t *>(d), st);
        fck = d;
        f_part = ck->fse_part;
        n_fck = ck->n_fse;
    }
    const size_t len = h.len;
    size_t off = 0;
    const uint8_t mb = h.rd<uint8_t>(off);
    h.rd<uint16_t>(off);
    h.rd<uint16_t>(off);
    const bool delta = (mb & 0x80) != 0;
    const int method = mb & 0x7F;
    const long long N = (long long)n;
    int *d_err = pool.get<int>(4);
    FB2_CUDA(cudaMemsetAsync(d_err, 0, 16, st));
    if (method == 0) {
        const unsigned long long nr = h.rd<uint64_t>(off), nv = h.rd<uint64_t>(off);
        const unsigned long long s_rcl = h.rd<uint64_t>(off), s_vcl = h.rd<uint64_t>(off);
        const unsigned long long rbp = h.rd<uint64_t>(off), vbp = h.rd<uint64_t>(off);
        const size_t o_rcl = off, o_vcl = o_rcl + s_rcl, o_rman = o_vcl + s_vcl, o_vman = o_rman + rbp;
        const size_t end = o_vman + vbp;
        if (end > len || nv > (unsigned long long)N || nr > (unsigned long long)N + 1)
            throw std::invalid_argument("Invalid or truncated Falcons entropy payload");
        uint32_t *buf = pool.get<uint32_t>(nr + nv + 2);
        gamma_decode(pool, d_in, h, {o_rcl, o_vcl}, {o_rman, o_vman}, {(size_t)rbp, (size_t)vbp},
                     {0ULL, nr, nr + nv}, buf, d_err, st, fck, f_part, n_fck);
        FB2_CUDA(cudaMemsetAsync(d_codes, 0, (size_t)N * 2, st));
        if (nv > 0) {
            unsigned long long *start = pool.get<unsigned long long>(nr + 1);
            void *sc = pool.get<uint8_t>(scan_scratch_bytes((long long)nr, 8));
            exclusive_scan<uint32_t, unsigned long long>(buf, (long long)nr, start, sc, st);
            k_m0_scatter<<<grid_for((long long)nv, 256), 256, 0, st>>>(buf, buf + nr, start, (long long)nv, N,
                                                                      d_codes);
            FB2_CHECK_LAUNCH();
        }
        off = end;
    } else if (method == 1) {
        unsigned long long S = h.rd<uint64_t>(off);
        if (S == 0) S = 1;
        if (S > (unsigned long long)std::max<long long>(N, 1)) throw std::invalid_argument("invalid segment count");
        const unsigned long long seg = ((unsigned long long)N + S - 1) / S;
        std::vector<DecChain> chains;
        std::vector<size_t> nf_off(S);
        std::vector<size_t> cls_off, man_off, man_len;
        std::vector<unsigned long long> gstart{0};
        std::vector<int> gseg;
        struct RawOvf {
            size_t off;
            unsigned long long n, dst;
        };
        std::vector<RawOvf> raws;
        unsigned long long ovf_total = 0;
        for (unsigned long long g = 0; g < S; g++) {
            const unsigned long long lo = g * seg;
            unsigned long long hi = lo + seg;
            if (hi > (unsigned long long)N) hi = N;
            const unsigned long long ng = hi > lo ? hi - lo : 0;
            h.rd<uint64_t>(off);  // stored N (the decoder uses the computed length)
            const unsigned long long K = h.rd<uint64_t>(off);
            if (ng == 0) continue;
            if (K < 1 || K > (unsigned long long)kMaxK) throw std::invalid_argument("invalid tANS stream count");
            const unsigned long long cs = (ng + K - 1) / K;
            unsigned long long bl[kMaxK], nk[kMaxK];
            for (unsigned long long k = 0; k < K; k++) bl[k] = h.rd<uint64_t>(off);
            for (unsigned long long k = 0; k < K; k++) nk[k] = h.rd<uint64_t>(off);
            nf_off[g] = off;
            off += O1_NCTX * O1_NSYM * 2;
            unsigned long long sp = off, tot_ov = 0;
            for (unsigned long long k = 0; k < K; k++) {
                const unsigned long long clo = lo + k * cs;
                unsigned long long chi = clo + cs;
                if (chi > hi) chi = hi;
                DecChain c{sp, bl[k], clo, chi > clo ? chi - clo : 0, ovf_total + tot_ov, (int)g,
                           (uint32_t)std::min<unsigned long long>(nk[k], 0xFFFFFFFFULL), 0, 0};
                chains.push_back(c);
                sp += bl[k];
                tot_ov += nk[k];
            }
            off = sp;
            if (off > len) throw std::invalid_argument("Invalid or truncated Falcons entropy payload");
            // escape block (decode_o1_ovf)
            const uint8_t mode = h.rd<uint8_t>(off);
            if (tot_ov > 0) {
                if (mode == 0) {
                    if (off + tot_ov * 2 > len) throw std::invalid_argument("truncated escape block");
                    raws.push_back(RawOvf{off, tot_ov, ovf_total});
                    off += tot_ov * 2;
                } else {
                    const unsigned long long s_vcl = h.rd<uint64_t>(off);
                    const unsigned long long vbp = h.rd<uint64_t>(off);
                    cls_off.push_back(off);
                    man_off.push_back(off + s_vcl);
                    man_len.push_back(vbp);
                    gstart.push_back(gstart.back() + tot_ov);
                    gseg.push_back((int)g);
                    // decoded values land at the group's position in a separate array, moved below
                    raws.push_back(RawOvf{~size_t(0), tot_ov, ovf_total});
                    off += s_vcl + vbp;
                    if (off > len) throw std::invalid_argument("truncated escape block");
                }
            }
            ovf_total += tot_ov;
        }
        for (unsigned long long g = 0; g < S; g++)
            if (nf_off[g] + O1_NCTX * O1_NSYM * 2 > len) throw std::invalid_argument("truncated tANS tables");
        tr.mark("segments parsed");
        // escape values, decoded on the side stream while this stream builds the decode tables
        // (raw blocks are copied; gamma groups are unpacked straight into their place)
        int16_t *ovf = pool.get<int16_t>(ovf_total + 1);
        SideFork fork(ctx, st);
        Pool spool(fork.side);
        {
            std::vector<Piece> pcs;
            std::vector<unsigned long long> conv_dst;
            for (auto &r : raws) {
                if (r.off != ~size_t(0)) pcs.push_back(Piece{d_in + r.off, r.dst * 2, r.n * 2});
                else conv_dst.push_back(r.dst);
            }
            if (!conv_dst.empty()) {
                unsigned long long *d_cd = h2d(spool, conv_dst, fork.side);
                gamma_decode(spool, d_in, h, cls_off, man_off, man_len, gstart, nullptr, d_err, fork.side, fck, f_part,
                             n_fck, d_cd, ovf);
            }
            launch_gather(spool, pcs, reinterpret_cast<uint8_t *>(ovf), fork.side);
        }
        tr.gpu("escapes decoded", fork.side);
        tr.mark("escapes launched");
        // decode tables: consecutive segments with identical tables share one decode table set
        std::vector<int> uid(S, 0);
        std::vector<unsigned long long> lead;
        {
            std::vector<unsigned long long> nfo(nf_off.begin(), nf_off.end());
            unsigned long long *d_nfo = h2d(pool, nfo, st);
            int *d_same = pool.get<int>(S);
            k_table_same<<<(unsigned)S, 256, 0, st>>>(d_in, d_nfo, (int)S, d_same);
            FB2_CHECK_LAUNCH();
            std::vector<int> same = d2h(d_same, (size_t)S, st);
            for (unsigned long long g = 0; g < S; g++) {
                if (g == 0 || !same[g]) lead.push_back(nf_off[g]);
                uid[g] = (int)lead.size() - 1;
            }
        }
        tr.mark("shared tables found");
        const int U = (int)lead.size();
        const int ntab = U * O1_NCTX;
        uint16_t *nf = pool.get<uint16_t>((size_t)ntab * O1_NSYM);
        {
            std::vector<Piece> pcs;
            for (int u = 0; u < U; u++)
                pcs.push_back(Piece{d_in + lead[u], (unsigned long long)u * O1_NCTX * O1_NSYM * 2, O1_NCTX * O1_NSYM * 2});
            launch_gather(pool, pcs, reinterpret_cast<uint8_t *>(nf), st);
        }
        // the host ranks the tables' contexts while the device builds the decode tables
        const std::vector<uint16_t> hnf = d2h(nf, (size_t)ntab * O1_NSYM, st);
        tr.mark("tables read");
        uint32_t *dt = pool.get<uint32_t>((size_t)ntab * O1_M);
        uint8_t *spread = pool.get<uint8_t>(16);
        k_o1_dtable<<<ntab, kTabThreads, 0, st>>>(nf, dt, spread, d_err);
        FB2_CHECK_LAUNCH();
        tr.gpu("decode tables built", st);
        for (auto &c : chains) c.table = uid[c.table];
        // checkpoint base of every chain; the checkpoints are used only if their count matches
        bool parts_ok = false;
        if (o1ck) {
            unsigned long long tot = 0;
            for (auto &c : chains) {
                c.ck = (uint32_t)tot;
                if (c.n) tot += (c.n - 1) / o1_part;
            }
            parts_ok = tot == n_o1ck;
        }
        DecChain *dch = h2d(pool, chains, st);
        {
            tr.mark("decode tables launched");
            std::vector<unsigned long long> maps(U), revs(U);
            for (int u = 0; u < U; u++) {
                auto mr = hot_contexts(hnf.data() + (size_t)u * O1_NCTX * O1_NSYM, kDecSlots);
                maps[u] = mr.first;
                revs[u] = mr.second;
            }
            tr.mark("hot contexts ranked");
            enable_big_smem();
            fork.join();  // the chains consume the escape values
            if (parts_ok) {
                // parts of every chain (their first indices in pstart), CTAs over runs of one table
                std::vector<uint32_t> pstart(chains.size() + 1, 0);
                std::vector<int> chain_table(chains.size());
                for (size_t i = 0; i < chains.size(); i++) {
                    const unsigned long long np = chains[i].n ? 1 + (chains[i].n - 1) / o1_part : 0;
                    pstart[i + 1] = pstart[i] + (uint32_t)np;
                    chain_table[i] = chains[i].table;
                }
                std::vector<ItemRun> runs = table_runs(chain_table);
                for (auto &r : runs) {
                    const size_t a = pstart[r.first], b = pstart[r.first + r.len];
                    r.first = a;
                    r.len = b - a;
                }
                std::vector<ChainCta> ctas = run_ctas(runs, pstart.back(), maps, revs, kPartThreads);
                for (auto &c : ctas)  // the chain of the CTA's first part
                    c.pad = (int)(std::upper_bound(pstart.begin(), pstart.end(), (uint32_t)c.first) - pstart.begin()) - 1;
                tr.mark("parts listed");
                ChainCta *d_ctas = h2d(pool, ctas, st);
                uint32_t *d_pstart = h2d(pool, pstart, st);
                k_o1_decode_parts<<<(unsigned)ctas.size(), kPartThreads, kDecSlots * O1_M * 4, st>>>(
                    d_in, dch, d_pstart, (uint32_t)chains.size(), d_ctas, dt, ovf, ovf_total, o1ck, o1_part, d_codes,
                    d_err);
                FB2_CHECK_LAUNCH();
            } else {
                std::vector<int> chain_table(chains.size());
                for (size_t i = 0; i < chains.size(); i++) chain_table[i] = chains[i].table;
                std::vector<ChainCta> ctas = chain_ctas(chain_table, maps, revs);
                ChainCta *d_ctas = h2d(pool, ctas, st);
                k_o1_decode_smem<<<(unsigned)ctas.size(), kChainThreads, kDecSlots * O1_M * 4, st>>>(
                    d_in, dch, d_ctas, dt, ovf, ovf_total, d_codes, d_err);
                FB2_CHECK_LAUNCH();
            }
        }
    } else {
        throw std::invalid_argument("unsupported entropy method");
    }
    tr.mark("chains launched");
    tr.gpu("chains decoded", st);
    if (delta) undelta(pool, d_codes, N, st);
    std::vector<int> he = d2h(d_err, 2, st);
    tr.gpu_dump();
    tr.mark("chains done");
    if (he[1] && ck) {
        // a checkpoint did not match the stream: decode again, sequentially
        if (tr.on) std::fprintf(stderr, "[falcons trace] decode checkpoint mismatch: decoding sequentially\n");
        return entropy_decode(ctx, d_in, h, n, d_codes, st, nullptr);
    }
    if (he[0]) throw std::invalid_argument("Invalid or corrupted Falcons entropy payload");
    return off;
}


}  // namespace fb2
