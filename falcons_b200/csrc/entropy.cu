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
};

constexpr size_t kBlockSlot = FBLK + 64;

// FSE_compress on the device: header, tables and the 2-state reverse coding of one 64 Ki block
// (zfse/fse_compress.c FSE_compress_wksp).  The two state chains are interleaved and the symbol
// loads are issued ahead of the dependent table lookups.
__device__ size_t fse_block_encode(uint8_t *dst, size_t cap, const uint8_t *__restrict__ src, size_t n,
                                   fse::BlockScratch &w, uint8_t *__restrict__ bits, size_t &hdr_out,
                                   size_t &body_out) {
    if (n <= 2) return 0;
    unsigned maxSV = 255;
    while (maxSV > 0 && w.count[maxSV] == 0) maxSV--;
    uint32_t maxCount = 0;
    for (unsigned s2 = 0; s2 <= maxSV; s2++) maxCount = w.count[s2] > maxCount ? w.count[s2] : maxCount;
    if (maxCount == n) return 1;
    if (maxCount == 1) return 0;
    if (maxCount < (n >> 7)) return 0;
    const unsigned tl = fse::optimal_table_log(fse::kDefaultTableLog, n, maxSV);
    if (fse::normalize_count(w.norm, tl, w.count, n, maxSV) != tl) return 0;
    if (cap < fse::ncount_bound(maxSV, tl) + 16) return 0;
    const size_t hdr = fse::write_ncount(dst, w.norm, maxSV, tl);
    if (hdr == 0) return 0;
    if (!fse::build_ctable(w.state_table, w.sym_tt, w.sym, w.norm, maxSV, tl)) return 0;
    fse::Writer32 bw;
    bw.init(bits, cap - hdr);
    uint32_t st[2];
    for (int k = 0; k < 2; k++) {
        const size_t i = ((n - 1) % 2 == (size_t)k) ? n - 1 : n - 2;
        const fse::SymTT t = w.sym_tt[src[i]];
        const uint32_t nb = (t.deltaNbBits + (1u << 15)) >> 16;
        const uint32_t v = (nb << 16) - t.deltaNbBits;
        st[k] = w.state_table[(int32_t)(v >> nb) + t.deltaFindState];
    }
    // symbols n-3 .. 0 in that order; index parity selects the state
    long long ii = (long long)n - 3;
    uint8_t sa = ii >= 1 ? src[ii] : 0, sb = ii >= 1 ? src[ii - 1] : 0;
    while (ii >= 1) {
        const uint8_t na = ii >= 3 ? src[ii - 2] : 0, nbs = ii >= 3 ? src[ii - 3] : 0;  // next pair, early
        const fse::SymTT ta = w.sym_tt[sa], tb = w.sym_tt[sb];
        const int ka = (int)(ii & 1), kb = ka ^ 1;
        const uint32_t nba = (st[ka] + ta.deltaNbBits) >> 16;
        const uint32_t nbb = (st[kb] + tb.deltaNbBits) >> 16;
        bw.add(st[ka], nba);
        bw.add(st[kb], nbb);
        st[ka] = w.state_table[(int32_t)(st[ka] >> nba) + ta.deltaFindState];
        st[kb] = w.state_table[(int32_t)(st[kb] >> nbb) + tb.deltaFindState];
        sa = na;
        sb = nbs;
        ii -= 2;
    }
    if (ii == 0) {
        const fse::SymTT t = w.sym_tt[src[0]];
        const uint32_t nb = (st[0] + t.deltaNbBits) >> 16;
        bw.add(st[0], nb);
        st[0] = w.state_table[(int32_t)(st[0] >> nb) + t.deltaFindState];
    }
    bw.add(st[1], tl);
    bw.add(st[0], tl);
    const size_t body = bw.close();
    if (bw.overflow || body + 8 > cap - hdr) return 0;
    const size_t total = hdr + body;
    if (total >= n - 1) return 0;
    hdr_out = hdr;
    body_out = body;
    return total;
}

// One CTA per 64 Ki block: parallel histogram, then the sequential FSE coder in thread 0 writing
// the bitstream to an aligned scratch area, then a cooperative move into the record.
// Writes the complete fse_enc record ([flag][u32 len][data] | [0][raw] | [2][sym]) to its slot.
__global__ void __launch_bounds__(256) k_fse_encode_blocks(const uint8_t *__restrict__ cls,
                                                          const BlockJob *__restrict__ jobs,
                                                          uint8_t *__restrict__ slots,
                                                          unsigned long long *__restrict__ sizes,
                                                          uint8_t *__restrict__ scratch) {
    __shared__ fse::BlockScratch w;
    const BlockJob jb = jobs[blockIdx.x];
    const uint8_t *src = cls + jb.src;
    uint8_t *out = slots + (size_t)blockIdx.x * kBlockSlot;
    uint8_t *bits = scratch + (size_t)blockIdx.x * kBlockSlot;
    for (int s = threadIdx.x; s < 256; s += blockDim.x) w.count[s] = 0;
    __syncthreads();
    for (unsigned i = threadIdx.x; i < jb.n; i += blockDim.x) atomicAdd(&w.count[src[i]], 1u);
    __syncthreads();
    __shared__ unsigned long long r_sh, hdr_sh, body_sh;
    if (threadIdx.x == 0) {
        size_t h = 0, b = 0;
        r_sh = fse_block_encode(out + 5, kBlockSlot - 5, src, jb.n, w, bits, h, b);
        hdr_sh = h;
        body_sh = b;
    }
    __syncthreads();
    const unsigned long long r = r_sh;
    if (r == 0 || r >= jb.n) {  // raw
        if (threadIdx.x == 0) out[0] = 0;
        for (unsigned i = threadIdx.x; i < jb.n; i += blockDim.x) out[1 + i] = src[i];
        if (threadIdx.x == 0) sizes[blockIdx.x] = 1 + jb.n;
    } else if (r == 1) {  // a single repeated symbol
        if (threadIdx.x == 0) {
            out[0] = 2;
            out[1] = src[0];
            sizes[blockIdx.x] = 2;
        }
    } else {
        uint8_t *d = out + 5 + hdr_sh;
        for (unsigned long long i = threadIdx.x; i < body_sh; i += blockDim.x) d[i] = bits[i];
        if (threadIdx.x == 0) {
            out[0] = 1;
            const uint32_t rr = (uint32_t)r;
            out[1] = (uint8_t)rr;
            out[2] = (uint8_t)(rr >> 8);
            out[3] = (uint8_t)(rr >> 16);
            out[4] = (uint8_t)(rr >> 24);
            sizes[blockIdx.x] = 5 + r;
        }
    }
}

// One warp per 64 Ki block: the decode table lives in shared memory and lane 0 runs the two
// interleaved state chains (zfse/fse_decompress.c FSE_decompress_usingDTable_generic).
__global__ void __launch_bounds__(32) k_fse_decode_blocks(const uint8_t *__restrict__ in,
                                                         const BlockJob *__restrict__ jobs,
                                                         uint8_t *__restrict__ cls, int *__restrict__ err) {
    __shared__ fse::DEntry dt[1 << fse::kMaxTableLog];
    __shared__ uint8_t sym[1 << fse::kMaxTableLog];
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
    if (threadIdx.x != 0) return;
    int16_t norm[256];
    unsigned maxSV = 255, tl = 0;
    const size_t size = (size_t)jb.inlen;
    const size_t hdr = fse::read_ncount(norm, &maxSV, &tl, p, size);
    if (hdr == 0 || hdr >= size || tl > (unsigned)fse::kMaxTableLog || !fse::build_dtable(dt, norm, maxSV, tl, sym)) {
        atomicExch(err, 1);
        return;
    }
    fse::Reader32 br;
    if (!br.init(p + hdr, (uint32_t)(size - hdr))) {
        atomicExch(err, 1);
        return;
    }
    uint32_t s0 = br.read(tl), s1 = br.read(tl);
    const unsigned n = jb.n;
    unsigned i = 0;
    for (; i + 1 < n; i += 2) {
        const fse::DEntry e0 = dt[s0];
        const fse::DEntry e1 = dt[s1];
        dst[i] = e0.symbol;
        dst[i + 1] = e1.symbol;
        s0 = e0.newState + br.read(e0.nbBits);
        s1 = e1.newState + br.read(e1.nbBits);
    }
    if (i < n) dst[i] = dt[s0].symbol;
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
__global__ void k_gamma_pack(const uint32_t *__restrict__ v, const uint8_t *__restrict__ cls,
                             const unsigned long long *__restrict__ boff, long long n,
                             const unsigned long long *__restrict__ gstart, int G,
                             const unsigned long long *__restrict__ gword, uint32_t *__restrict__ words) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int k = cls[i];
        if (k == 0) continue;
        const int g = find_group(gstart, G, (unsigned long long)i);
        const unsigned long long b = boff[i] - boff[gstart[g]];
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

GammaOut gamma_encode(Pool &pool, const uint32_t *d_vals, const std::vector<unsigned long long> &gstart,
                      cudaStream_t st) {
    const int G = (int)gstart.size() - 1;
    const long long T = (long long)gstart.back();
    GammaOut out;
    out.cls_pieces.resize(G);
    out.cls_n.resize(G);
    out.cls_bytes.assign(G, 0);
    out.man_ptr.assign(G, nullptr);
    out.man_bytes.assign(G, 0);
    if (T == 0) return out;
    uint8_t *cls = pool.get<uint8_t>(T);
    k_gamma_cls<<<grid_for(T, 256), 256, 0, st>>>(d_vals, T, cls);
    FB2_CHECK_LAUNCH();
    unsigned long long *boff = pool.get<unsigned long long>(T + 1);
    void *sc = pool.get<uint8_t>(scan_scratch_bytes(T, 8));
    exclusive_scan<uint8_t, unsigned long long>(cls, T, boff, sc, st);
    // per-group bit totals: the scan at every group start, gathered on the device, one copy back
    unsigned long long *d_gstart = h2d(pool, gstart, st);
    unsigned long long *d_gb = pool.get<unsigned long long>(G + 1);
    k_pick_u64<<<grid_for(G + 1, 256), 256, 0, st>>>(boff, d_gstart, G + 1, d_gb);
    FB2_CHECK_LAUNCH();
    const std::vector<unsigned long long> gb = d2h(d_gb, (size_t)G + 1, st);
    std::vector<unsigned long long> gword(G);
    unsigned long long words = 0;
    for (int g = 0; g < G; g++) {
        const unsigned long long bits = gb[g + 1] - gb[g];
        out.man_bytes[g] = (size_t)((bits + 7) / 8);
        gword[g] = words;
        words += (bits + 31) / 32 + 2;
    }
    uint32_t *wbuf = pool.get<uint32_t>(words + 4);
    FB2_CUDA(cudaMemsetAsync(wbuf, 0, (words + 4) * 4, st));
    unsigned long long *d_gword = h2d(pool, gword, st);
    k_gamma_pack<<<grid_for(T, 256), 256, 0, st>>>(d_vals, cls, boff, T, d_gstart, G, d_gword, wbuf);
    FB2_CHECK_LAUNCH();
    for (int g = 0; g < G; g++) out.man_ptr[g] = reinterpret_cast<const uint8_t *>(wbuf + gword[g]);
    // FSE class blocks
    std::vector<BlockJob> jobs;
    std::vector<int> job_group;
    for (int g = 0; g < G; g++) {
        for (unsigned long long b = gstart[g]; b < gstart[g + 1]; b += FBLK) {
            jobs.push_back(BlockJob{b, (unsigned)std::min<unsigned long long>(FBLK, gstart[g + 1] - b), 0, 0, 0});
            job_group.push_back(g);
        }
    }
    BlockJob *d_jobs = h2d(pool, jobs, st);
    uint8_t *slots = pool.get<uint8_t>(jobs.size() * kBlockSlot);
    uint8_t *bits = pool.get<uint8_t>(jobs.size() * kBlockSlot);
    unsigned long long *sizes = pool.get<unsigned long long>(jobs.size());
    k_fse_encode_blocks<<<(unsigned)jobs.size(), 256, 0, st>>>(cls, d_jobs, slots, sizes, bits);
    FB2_CHECK_LAUNCH();
    std::vector<unsigned long long> hs = d2h(sizes, jobs.size(), st);
    for (size_t j = 0; j < jobs.size(); j++) {
        const int g = job_group[j];
        out.cls_pieces[g].push_back({slots + j * kBlockSlot, (size_t)hs[j]});
        out.cls_n[g].push_back(jobs[j].n);
        out.cls_bytes[g] += (size_t)hs[j];
    }
    return out;
}

// Adds the fse_enc records of group g, recording each record's header bytes for the index.
void add_class_pieces(Assembler &as, const GammaOut &go, int g) {
    for (size_t b = 0; b < go.cls_pieces[g].size(); b++) {
        const auto &p = go.cls_pieces[g][b];
        const unsigned n = go.cls_n[g][b];
        uint8_t h[5];
        size_t hl;
        if (p.second == 1 + (size_t)n) { h[0] = 0; hl = 1; }
        else if (p.second == 2) { h[0] = 2; hl = 1; }
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

__global__ void k_gamma_unpack(const uint8_t *__restrict__ cls, const unsigned long long *__restrict__ boff,
                               long long n, const unsigned long long *__restrict__ gstart, int G,
                               const unsigned long long *__restrict__ gman, const uint8_t *__restrict__ base,
                               const unsigned long long *__restrict__ gman_len, uint32_t *__restrict__ v,
                               int *__restrict__ err) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int k = cls[i];
        uint32_t m = 0;
        if (k > 31) {
            atomicExch(err, 2);
        } else if (k > 0) {
            const int g = find_group(gstart, G, (unsigned long long)i);
            const unsigned long long b = boff[i] - boff[gstart[g]];
            const uint8_t *p = base + gman[g];
            const unsigned long long lenb = gman_len[g];
            const unsigned long long byte0 = b >> 3;
            if (((b + k + 7) >> 3) > lenb) {
                atomicExch(err, 3);
            } else {
                unsigned long long acc = 0;
                const int nbytes = (int)((((b & 7) + k) + 7) >> 3);
                for (int j = 0; j < nbytes; j++) acc = (acc << 8) | p[byte0 + j];
                const int drop = nbytes * 8 - (int)(b & 7) - k;
                m = (uint32_t)((acc >> drop) & ((1ull << k) - 1));
            }
        }
        v[i] = (k <= 31) ? ((1u << k) | m) : 0u;
    }
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

__global__ void __launch_bounds__(1024) k_o1_hist(const int16_t *__restrict__ q, const SegInfo *__restrict__ segs,
                                                 uint32_t *__restrict__ hist, uint32_t *__restrict__ nvk) {
    __shared__ uint32_t h[O1_NCTX * O1_NSYM];
    __shared__ uint32_t esc[kMaxK];
    const SegInfo sg = segs[blockIdx.x];
    for (int i = threadIdx.x; i < O1_NCTX * O1_NSYM; i += blockDim.x) h[i] = 0;
    if (threadIdx.x < kMaxK) esc[threadIdx.x] = 0;
    __syncthreads();
    for (unsigned long long r = threadIdx.x; r < sg.n; r += blockDim.x) {
        const unsigned long long i = sg.lo + r;
        const int k = (int)(r / sg.cs);
        const bool first = (r % sg.cs) == 0;
        const int code = q[i];
        const int prev = first ? 0 : (int)q[i - 1];
        const int s = o1_sym(code);
        atomicAdd(&h[o1_ctx(prev) * O1_NSYM + s], 1u);
        if (s == O1_NSYM - 1) atomicAdd(&esc[k], 1u);
    }
    __syncthreads();
    uint32_t *gh = hist + (size_t)blockIdx.x * O1_NCTX * O1_NSYM;
    for (int i = threadIdx.x; i < O1_NCTX * O1_NSYM; i += blockDim.x) gh[i] = h[i];
    if (threadIdx.x < kMaxK) nvk[blockIdx.x * kMaxK + threadIdx.x] = esc[threadIdx.x];
}

// o1_normalize (RleFseEncoder.hpp:410-477) for one (segment, context) per thread.
__global__ void k_o1_norm(const uint32_t *__restrict__ hist, int total_tables, uint16_t *__restrict__ nf) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total_tables) return;
    const uint32_t *cnt = hist + (size_t)t * O1_NSYM;
    uint16_t *freq = nf + (size_t)t * O1_NSYM;
    unsigned long long total = 0;
    int nonzero = 0;
    for (int s = 0; s < O1_NSYM; s++) {
        total += cnt[s];
        nonzero += cnt[s] != 0;
    }
    if (total == 0) {
        for (int s = 0; s < O1_NSYM; s++) freq[s] = 0;
        freq[0] = O1_M;
        return;
    }
    if (nonzero > 1) {
        int16_t norm[O1_NSYM];
        if (fse::normalize_count(norm, O1_PB, cnt, total, O1_NSYM - 1) == (unsigned)O1_PB) {
            for (int s = 0; s < O1_NSYM; s++) freq[s] = (uint16_t)norm[s];
            return;
        }
    }
    int sum = 0, maxf = 0, argmax = 0;
    int f[O1_NSYM];
    for (int s = 0; s < O1_NSYM; s++) {
        if (cnt[s]) {
            int v = (int)((unsigned long long)cnt[s] * O1_M / total);
            if (v == 0) v = 1;
            f[s] = v;
            sum += v;
            if (v > maxf) { maxf = v; argmax = s; }
        } else {
            f[s] = 0;
        }
    }
    int e = O1_M - sum;
    if (e > 0) {
        f[argmax] += e;
    } else if (e < 0) {
        e = -e;
        int take = (maxf - 1 < e) ? (maxf - 1) : e;
        f[argmax] -= take;
        e -= take;
        while (e > 0) {
            int mi = -1;
            int mv = 1;
            for (int s = 0; s < O1_NSYM; s++)
                if (f[s] > mv) { mv = f[s]; mi = s; }
            if (mi < 0) break;
            take = f[mi] - 1;
            if (take > e) take = e;
            f[mi] -= take;
            e -= take;
        }
    }
    for (int s = 0; s < O1_NSYM; s++) freq[s] = (uint16_t)f[s];
}

__global__ void __launch_bounds__(32) k_o1_ctable(const uint16_t *__restrict__ nf, uint16_t *__restrict__ stab,
                                                 fse::SymTT *__restrict__ stt, uint8_t *__restrict__ scratch,
                                                 int *__restrict__ err) {
    (void)scratch;
    __shared__ uint8_t sym[O1_M];
    if (threadIdx.x != 0) return;
    const size_t t = blockIdx.x;
    int16_t norm[O1_NSYM];
    for (int s = 0; s < O1_NSYM; s++) norm[s] = (int16_t)nf[t * O1_NSYM + s];
    if (!fse::build_ctable(stab + t * O1_M, stt + t * O1_NSYM, sym, norm, O1_NSYM - 1, O1_PB)) atomicExch(err, 4);
}

// Decode table of one context with everything a decode step needs in one 32-bit word:
//   bits 0-12 next state base, 13-16 bits to read, 17-20 context of the decoded code,
//   bit 21 escape (value from the side stream), bits 22-31 the decoded code (signed).
__global__ void __launch_bounds__(128) k_o1_dtable(const uint16_t *__restrict__ nf, uint32_t *__restrict__ dt,
                                                 uint8_t *__restrict__ scratch, int *__restrict__ err) {
    (void)scratch;
    __shared__ uint8_t sym[O1_M];
    __shared__ fse::DEntry e[O1_M];
    const size_t t = blockIdx.x;
    if (threadIdx.x == 0) {
        int16_t norm[O1_NSYM];
        for (int s = 0; s < O1_NSYM; s++) norm[s] = (int16_t)nf[t * O1_NSYM + s];
        if (!fse::build_dtable(e, norm, O1_NSYM - 1, O1_PB, sym)) atomicExch(err, 5);
    }
    __syncthreads();
    for (int u = threadIdx.x; u < O1_M; u += blockDim.x) {
        const fse::DEntry d = e[u];
        const bool esc = d.symbol == O1_NSYM - 1;
        const int code = esc ? 0 : unzz(d.symbol);
        const int ctx = esc ? 0 : o1_ctx(code);
        dt[t * O1_M + u] = (uint32_t)d.newState | ((uint32_t)d.nbBits << 13) | ((uint32_t)ctx << 17) |
                           ((uint32_t)esc << 21) | ((uint32_t)(code & 0x3FF) << 22);
    }
}

// One thread per (segment, chunk) chain: reverse tANS encode with per-symbol context tables
// (RleFseEncoder.hpp:671-707).  tab[g] selects the table set of segment g.
__global__ void __launch_bounds__(32) k_o1_encode(const int16_t *__restrict__ q, const SegInfo *__restrict__ segs,
                                                  int nseg, const int *__restrict__ tab,
                                                  const uint16_t *__restrict__ stab,
                                                  const fse::SymTT *__restrict__ stt, uint8_t *__restrict__ slots,
                                                  const unsigned long long *__restrict__ slot_off,
                                                  unsigned long long *__restrict__ blen) {
    const int chain = blockIdx.x * blockDim.x + threadIdx.x;
    const int g = chain / kMaxK, k = chain % kMaxK;
    if (g >= nseg) return;
    const SegInfo sg = segs[g];
    if (k >= sg.K) return;
    const unsigned long long lo = sg.lo + (unsigned long long)k * sg.cs;
    unsigned long long hi = lo + sg.cs;
    if (hi > sg.lo + sg.n) hi = sg.lo + sg.n;
    if (lo >= hi) {
        blen[chain] = 0;
        return;
    }
    const size_t tb = (size_t)tab[g] * O1_NCTX;
    const uint16_t *__restrict__ S = stab + tb * O1_M;
    const fse::SymTT *__restrict__ T = stt + tb * O1_NSYM;
    fse::Writer32 bw;
    const unsigned long long cap = slot_off[chain + 1] - slot_off[chain];
    bw.init(slots + slot_off[chain], (size_t)cap);
    unsigned long long idx = hi - 1;
    int cur = q[idx];
    int prev = idx > lo ? (int)__ldg(q + idx - 1) : 0;
    fse::SymTT t = T[o1_ctx(prev) * O1_NSYM + o1_sym(cur)];
    uint32_t nb = (t.deltaNbBits + (1u << 15)) >> 16;
    uint32_t v = (nb << 16) - t.deltaNbBits;
    uint32_t state = S[o1_ctx(prev) * O1_M + (int32_t)(v >> nb) + t.deltaFindState];
    // walk down: the symbol at idx-1 becomes current, its predecessor is loaded one step ahead
    int nxt = (idx >= lo + 2) ? (int)__ldg(q + idx - 2) : 0;
    while (idx > lo) {
        idx--;
        cur = prev;
        prev = idx > lo ? nxt : 0;
        if (idx >= lo + 2) nxt = (int)__ldg(q + idx - 2);
        const int c = o1_ctx(prev);
        t = T[c * O1_NSYM + o1_sym(cur)];
        nb = (state + t.deltaNbBits) >> 16;
        bw.add(state, nb);
        state = S[c * O1_M + (int32_t)(state >> nb) + t.deltaFindState];
    }
    bw.add(state, O1_PB);
    const size_t len = bw.close();
    blen[chain] = bw.overflow ? ~0ULL : len;
}

struct DecChain {
    unsigned long long in;      // stream byte offset
    unsigned long long inlen;   // stream length (0 = empty chunk)
    unsigned long long lo, n;   // output range
    unsigned long long ovf;     // first escape value of this chunk
    int table;                  // segment index (tables at table * 15)
    int pad;
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
constexpr int kEncSlots = 13;  // 13 x 8192 x u16 encode state tables = 208 KiB
constexpr int kDecSlots = 7;   // 7 x 8192 x u32 decode tables = 224 KiB
struct ChainCta {
    int table;
    int first;
    int count;
    int pad;
    unsigned long long map, rev;
};

__global__ void __launch_bounds__(kChainThreads) k_o1_encode_smem(const int16_t *__restrict__ q, const SegInfo *__restrict__ segs,
                                                      const ChainCta *__restrict__ ctas,
                                                      const uint16_t *__restrict__ stab,
                                                      const fse::SymTT *__restrict__ stt, uint8_t *__restrict__ slots,
                                                      const unsigned long long *__restrict__ slot_off,
                                                      unsigned long long *__restrict__ blen) {
    extern __shared__ uint4 smem_raw[];
    uint16_t *sst = reinterpret_cast<uint16_t *>(smem_raw);
    const ChainCta w = ctas[blockIdx.x];
    const size_t tb = (size_t)w.table * O1_NCTX;
    const uint16_t *__restrict__ S = stab + tb * O1_M;
    const fse::SymTT *__restrict__ T = stt + tb * O1_NSYM;
    for (int j = 0; j < kEncSlots; j++) {
        const int c = (int)((w.rev >> (4 * j)) & 15);
        if (c >= O1_NCTX) continue;
        const uint4 *src = reinterpret_cast<const uint4 *>(S + (size_t)c * O1_M);
        uint4 *dst = reinterpret_cast<uint4 *>(sst + (size_t)j * O1_M);
        for (int i = threadIdx.x; i < O1_M * 2 / 16; i += blockDim.x) dst[i] = __ldg(src + i);
    }
    __syncthreads();
    const int lc = chain_slot();
    if (lc < 0 || lc >= w.count) return;
    const int chain = w.first + lc;
    const int g = chain / kMaxK, k = chain % kMaxK;
    const SegInfo sg = segs[g];
    if (k >= sg.K) return;
    const unsigned long long lo = sg.lo + (unsigned long long)k * sg.cs;
    unsigned long long hi = lo + sg.cs;
    if (hi > sg.lo + sg.n) hi = sg.lo + sg.n;
    if (lo >= hi) {
        blen[chain] = 0;
        return;
    }
    const unsigned long long map = w.map;
    fse::Writer32 bw;
    const unsigned long long cap = slot_off[chain + 1] - slot_off[chain];
    bw.init(slots + slot_off[chain], (size_t)cap);
    auto stlookup = [&](int c, int idx) -> uint32_t {
        const int sl = (int)((map >> (4 * c)) & 15);
        return sl < kEncSlots ? sst[sl * O1_M + idx] : __ldg(S + (size_t)c * O1_M + idx);
    };
    // codes are read through a 6-deep register queue (Q[i] = q[idx - i]) and the symbol transform
    // of the next step is loaded during the current one, so no step waits on global memory
    const long long L0 = (long long)lo;
    long long idx = (long long)hi - 1;
    auto ld = [&](long long i) -> int { return i >= L0 ? (int)__ldg(q + i) : 0; };
    int Q0 = ld(idx), Q1 = ld(idx - 1), Q2 = ld(idx - 2), Q3 = ld(idx - 3), Q4 = ld(idx - 4), Q5 = ld(idx - 5);
    int c = o1_ctx(idx > L0 ? Q1 : 0);
    fse::SymTT t = T[c * O1_NSYM + o1_sym(Q0)];
    uint32_t nb = (t.deltaNbBits + (1u << 15)) >> 16;
    uint32_t v = (nb << 16) - t.deltaNbBits;
    uint32_t state = stlookup(c, (int32_t)(v >> nb) + t.deltaFindState);
    // advance to idx - 1
    Q0 = Q1; Q1 = Q2; Q2 = Q3; Q3 = Q4; Q4 = Q5; Q5 = ld(idx - 6);
    idx--;
    int cn = o1_ctx(idx > L0 ? Q1 : 0);
    fse::SymTT tn = idx >= L0 ? T[cn * O1_NSYM + o1_sym(Q0)] : t;
    while (idx >= L0) {
        c = cn;
        t = tn;
        // prefetch for idx - 1
        const int n0 = Q1, n1 = Q2;
        cn = o1_ctx(idx - 1 > L0 ? n1 : 0);
        if (idx - 1 >= L0) tn = T[cn * O1_NSYM + o1_sym(n0)];
        nb = (state + t.deltaNbBits) >> 16;
        bw.add(state, nb);
        state = stlookup(c, (int32_t)(state >> nb) + t.deltaFindState);
        Q0 = Q1; Q1 = Q2; Q2 = Q3; Q3 = Q4; Q4 = Q5; Q5 = ld(idx - 6);
        idx--;
    }
    bw.add(state, O1_PB);
    const size_t len = bw.close();
    blen[chain] = bw.overflow ? ~0ULL : len;
}

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
// Groups consecutive chains of one table into CTAs of at most `per` chains; `per` is chosen so
// that the CTAs cover the SMs once (one chain CTA fills an SM).
std::vector<ChainCta> chain_ctas(const std::vector<int> &chain_table, const std::vector<unsigned long long> &maps,
                                 const std::vector<unsigned long long> &revs) {
    std::vector<ChainCta> out;
    const size_t sms = (size_t)sm_count();
    const size_t per = std::max<size_t>(8, std::min<size_t>(kMaxChainsPerCta, (chain_table.size() + sms - 1) / sms));
    size_t i = 0;
    while (i < chain_table.size()) {
        const int t = chain_table[i];
        size_t j = i;
        while (j < chain_table.size() && chain_table[j] == t && j - i < per) j++;
        out.push_back(ChainCta{t, (int)i, (int)(j - i), 0, maps[t], revs[t]});
        i = j;
    }
    return out;
}

void enable_big_smem() {
    static bool done = false;
    if (done) return;
    FB2_CUDA(cudaFuncSetAttribute(k_o1_encode_smem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kEncSlots * O1_M * 2));
    FB2_CUDA(cudaFuncSetAttribute(k_o1_decode_smem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kDecSlots * O1_M * 4));
    done = true;
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
    const long long base = (long long)blockIdx.x * kScanTile;
    uint32_t c = 0;
    for (int j = 0; j < kScanItems; j++) {
        const long long i = base + (long long)j * kScanThreads + threadIdx.x;
        if (i < n && o1_sym(q[i]) == O1_NSYM - 1) c++;
    }
    __shared__ uint32_t sh[32];
    uint32_t tot;
    block_excl_scan<uint32_t>(c, sh, tot);
    if (threadIdx.x == 0) cnt[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanThreads) k_esc_extract(const int16_t *__restrict__ q, long long n,
                                                             const uint32_t *__restrict__ tile_off,
                                                             uint32_t *__restrict__ vals, int16_t *__restrict__ raw) {
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int16_t v[kScanItems];
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const long long i = base + j;
        v[j] = i < n ? q[i] : (int16_t)0;
        c += (i < n && o1_sym(v[j]) == O1_NSYM - 1);
    }
    __shared__ uint32_t sh[32];
    uint32_t tot;
    uint32_t r = block_excl_scan<uint32_t>(c, sh, tot) + tile_off[blockIdx.x];
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const long long i = base + j;
        if (i < n && o1_sym(v[j]) == O1_NSYM - 1) {
            vals[r] = zigzag((int)v[j]) + 1u;
            raw[r] = v[j];
            r++;
        }
    }
}



__global__ void __launch_bounds__(32) k_o1_decode(const uint8_t *__restrict__ in, const DecChain *__restrict__ chains,
                                                 int nchains, const uint32_t *__restrict__ dt,
                                                 const int16_t *__restrict__ ovf, unsigned long long n_ovf,
                                                 int16_t *__restrict__ out, int *__restrict__ err) {
    const int ci = blockIdx.x * blockDim.x + threadIdx.x;
    if (ci >= nchains) return;
    const DecChain ch = chains[ci];
    if (ch.n == 0) return;
    fse::Reader32 br;
    if (ch.inlen == 0 || ch.inlen >= (1ull << 28) || !br.init(in + ch.in, (uint32_t)ch.inlen)) {
        atomicExch(err, 6);
        return;
    }
    const uint32_t *__restrict__ tb = dt + (size_t)ch.table * O1_NCTX * O1_M;
    uint32_t state = br.read(O1_PB);
    uint32_t ctx = 0;
    const int16_t *__restrict__ ov = ovf + ch.ovf;
    const uint32_t nov = (uint32_t)min((unsigned long long)0x7fffffff, n_ovf - ch.ovf);
    int16_t *o = out + ch.lo;
    const uint32_t n = (uint32_t)ch.n;
    uint32_t oi = 0;
    int next_ov = nov ? (int)__ldg(ov) : 0;  // escape value prefetched one step ahead
    for (uint32_t j = 0; j < n; j++) {
        const uint32_t e = __ldg(tb + ctx * O1_M + state);
        const bool esc = (e >> 21) & 1u;
        const int code = esc ? next_ov : ((int)e >> 22);
        ctx = esc ? 13u + (uint32_t)(code < 0) : ((e >> 17) & 15u);
        oi += esc;
        if (esc) next_ov = oi < nov ? (int)__ldg(ov + oi) : 0;
        o[j] = (int16_t)code;
        state = (e & 0x1FFFu) + br.read((e >> 13) & 15u);
    }
    if (oi > nov) atomicExch(err, 7);
    // the step after the last symbol reads at most 13 bits below the stream start
    if (br.pos < -16) atomicExch(err, 8);
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
                  uint32_t *d_vals, int *d_err, cudaStream_t st) {
    const int G = (int)gstart.size() - 1;
    const long long T = (long long)gstart.back();
    if (T == 0) return;
    std::vector<BlockJob> jobs;
    for (int g = 0; g < G; g++) parse_blocks(h, cls_off[g], gstart[g + 1] - gstart[g], gstart[g], jobs);
    uint8_t *cls = pool.get<uint8_t>(T);
    BlockJob *dj = h2d(pool, jobs, st);
    k_fse_decode_blocks<<<(unsigned)jobs.size(), 32, 0, st>>>(d, dj, cls, d_err);
    FB2_CHECK_LAUNCH();
    unsigned long long *boff = pool.get<unsigned long long>(T + 1);
    void *sc = pool.get<uint8_t>(scan_scratch_bytes(T, 8));
    exclusive_scan<uint8_t, unsigned long long>(cls, T, boff, sc, st);
    std::vector<unsigned long long> gman(G), glen(G);
    for (int g = 0; g < G; g++) {
        gman[g] = man_off[g];
        glen[g] = man_len[g];
    }
    unsigned long long *d_gstart = h2d(pool, gstart, st);
    unsigned long long *d_gman = h2d(pool, gman, st);
    unsigned long long *d_glen = h2d(pool, glen, st);
    k_gamma_unpack<<<grid_for(T, 256), 256, 0, st>>>(cls, boff, T, d_gstart, G, d_gman, d, d_glen, d_vals, d_err);
    FB2_CHECK_LAUNCH();
}

__global__ void k_ovf_convert(const uint32_t *gv, const unsigned long long *src, const unsigned long long *dst,
                              const unsigned long long *cnt, int ng, int16_t *out) {
    for (int g = blockIdx.x; g < ng; g += gridDim.x)
        for (unsigned long long i = threadIdx.x; i < cnt[g]; i += blockDim.x)
            out[dst[g] + i] = (int16_t)unzz(gv[src[g] + i] - 1u);
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
        uint32_t nv32 = 0;
        long long lastnz = -1;
        FB2_CUDA(cudaMemcpyAsync(&nv32, tcnt + tiles, 4, cudaMemcpyDeviceToHost, st));
        FB2_CUDA(cudaMemcpyAsync(&lastnz, tlast + tiles, 8, cudaMemcpyDeviceToHost, st));
        FB2_CUDA(cudaStreamSynchronize(st));
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
        GammaOut go = gamma_encode(pool, buf, {0ULL, nr, nr + nv}, st);
        as.val<uint64_t>(nr);
        as.val<uint64_t>(nv);
        as.val<uint64_t>(go.cls_bytes[0]);
        as.val<uint64_t>(go.cls_bytes[1]);
        as.val<uint64_t>(go.man_bytes[0]);
        as.val<uint64_t>(go.man_bytes[1]);
        add_class_pieces(as, go, 0);
        add_class_pieces(as, go, 1);
        as.dev(go.man_ptr[0], go.man_bytes[0]);
        as.dev(go.man_ptr[1], go.man_bytes[1]);
    } else {
        // ---- segmentation: K chains per segment, S segments (decoder reads S and K from the stream)
        const int K = std::max(1, std::min(kMaxK, tune.o1_streams));
        long long seg_target = tune.o1_segment;
        if (seg_target <= 0) {
            const char *env = getenv("FALCONS_O1_SEGMENT");
            seg_target = env ? atoll(env) : (1LL << 18);  // 256 Ki symbols -> 16 Ki per chain
            if (seg_target < 1024) seg_target = 1024;
        }
        long long S = std::max<long long>(1, (N + seg_target - 1) / seg_target);
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
        uint32_t *hist = pool.get<uint32_t>((size_t)S * O1_NCTX * O1_NSYM);
        uint32_t *nvk = pool.get<uint32_t>((size_t)S * kMaxK);
        k_o1_hist<<<(unsigned)S, 1024, 0, st>>>(q, d_segs, hist, nvk);
        FB2_CHECK_LAUNCH();
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
        k_o1_norm<<<(ntab + 63) / 64, 64, 0, st>>>(rhist, ntab, nf);
        FB2_CHECK_LAUNCH();
        uint16_t *stab = pool.get<uint16_t>((size_t)ntab * O1_M);
        fse::SymTT *stt = pool.get<fse::SymTT>((size_t)ntab * O1_NSYM);
        uint8_t *spread = pool.get<uint8_t>((size_t)ntab * O1_M);
        int *d_err = pool.get<int>(4);
        FB2_CUDA(cudaMemsetAsync(d_err, 0, 16, st));
        k_o1_ctable<<<ntab, 32, 0, st>>>(nf, stab, stt, spread, d_err);
        FB2_CHECK_LAUNCH();
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
            std::vector<uint16_t> hnf = d2h(nf, (size_t)ntab * O1_NSYM, st);
            tr.mark("tables normalized");
            std::vector<unsigned long long> maps(R), revs(R);
            for (int r = 0; r < R; r++) {
                auto mr = hot_contexts(hnf.data() + (size_t)r * O1_NCTX * O1_NSYM, kEncSlots);
                maps[r] = mr.first;
                revs[r] = mr.second;
            }
            std::vector<int> chain_table((size_t)nchains);
            for (long long ch = 0; ch < nchains; ch++) chain_table[ch] = seg_region[ch / kMaxK];
            std::vector<ChainCta> ctas = chain_ctas(chain_table, maps, revs);
            ChainCta *d_ctas = h2d(pool, ctas, st);
            enable_big_smem();
            k_o1_encode_smem<<<(unsigned)ctas.size(), kChainThreads, kEncSlots * O1_M * 2, st>>>(q, d_segs, d_ctas, stab, stt, slots,
                                                                                   d_soff, blen);
            FB2_CHECK_LAUNCH();
            tr.mark("chains launched");
        }
        // escapes in index order
        const long long tiles = std::max<long long>(1, (N + kScanTile - 1) / kScanTile);
        uint32_t *tcnt = pool.get<uint32_t>(tiles + 2);
        FB2_CUDA(cudaMemsetAsync(tcnt, 0, (tiles + 2) * 4, st));
        if (N > 0) {
            k_esc_tiles<<<(unsigned)tiles, kScanThreads, 0, st>>>(q, N, tcnt);
            FB2_CHECK_LAUNCH();
        }
        k_scan_small<uint32_t><<<1, 1024, 0, st>>>(tcnt, tiles);
        FB2_CHECK_LAUNCH();
        std::vector<uint32_t> h_nvk = d2h(nvk, (size_t)S * kMaxK, st);
        std::vector<unsigned long long> h_blen = d2h(blen, (size_t)nchains, st);
        std::vector<int> h_err = d2h(d_err, 1, st);
        if (h_err[0]) throw std::runtime_error("tANS table construction failed");
        tr.mark("chains done");
        unsigned long long E = 0;
        std::vector<unsigned long long> gstart(S + 1, 0);
        for (long long g = 0; g < S; g++) {
            unsigned long long e = 0;
            for (int k = 0; k < K; k++) e += h_nvk[g * kMaxK + k];
            gstart[g + 1] = gstart[g] + e;
        }
        E = gstart[S];
        uint32_t *evals = pool.get<uint32_t>(E + 1);
        int16_t *eraw = pool.get<int16_t>(E + 1);
        if (E > 0) {
            k_esc_extract<<<(unsigned)tiles, kScanThreads, 0, st>>>(q, N, tcnt, evals, eraw);
            FB2_CHECK_LAUNCH();
        }
        GammaOut go = gamma_encode(pool, evals, gstart, st);
        tr.mark("escapes coded");
        for (auto b : h_blen)
            if (b == ~0ULL) throw std::runtime_error("tANS chain overflow");
        as.val<uint64_t>((uint64_t)S);
        for (long long g = 0; g < S; g++) {
            as.val<uint64_t>(segs[g].n);
            as.val<uint64_t>((uint64_t)K);
            for (int k = 0; k < K; k++) as.val<uint64_t>(h_blen[g * kMaxK + k]);
            for (int k = 0; k < K; k++) as.val<uint64_t>(h_nvk[g * kMaxK + k]);
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
                    add_class_pieces(as, go, (int)g);
                    as.dev(go.man_ptr[g], go.man_bytes[g]);
                }
            }
        }
    }
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

size_t entropy_decode(Context &ctx, const uint8_t *d_in, const ByteView &h, size_t n, int16_t *d_codes,
                      cudaStream_t st) {
    (void)ctx;
    Trace tr("decode");
    Pool pool(st);
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
                     {0ULL, nr, nr + nv}, buf, d_err, st);
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
                DecChain c{sp, bl[k], clo, chi > clo ? chi - clo : 0, ovf_total + tot_ov, (int)g, 0};
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
        // escape values
        int16_t *ovf = pool.get<int16_t>(ovf_total + 1);
        {
            uint32_t *gv = pool.get<uint32_t>(gstart.back() + 1);
            gamma_decode(pool, d_in, h, cls_off, man_off, man_len, gstart, gv, d_err, st);
            // place: raw blocks are copied, gamma groups converted
            std::vector<Piece> pcs;
            size_t gi = 0;
            std::vector<unsigned long long> conv_src, conv_dst, conv_n;
            for (auto &r : raws) {
                if (r.off != ~size_t(0)) {
                    pcs.push_back(Piece{d_in + r.off, r.dst * 2, r.n * 2});
                } else {
                    conv_src.push_back(gstart[gi]);
                    conv_dst.push_back(r.dst);
                    conv_n.push_back(r.n);
                    gi++;
                }
            }
            launch_gather(pool, pcs, reinterpret_cast<uint8_t *>(ovf), st);
            if (!conv_src.empty()) {
                unsigned long long *d_cs = h2d(pool, conv_src, st), *d_cd = h2d(pool, conv_dst, st),
                                   *d_cn = h2d(pool, conv_n, st);
                const int ng = (int)conv_src.size();
                k_ovf_convert<<<std::min(ng, 65535), 256, 0, st>>>(gv, d_cs, d_cd, d_cn, ng, ovf);
                FB2_CHECK_LAUNCH();
            }
        }
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
        const int U = (int)lead.size();
        const int ntab = U * O1_NCTX;
        uint16_t *nf = pool.get<uint16_t>((size_t)ntab * O1_NSYM);
        {
            std::vector<Piece> pcs;
            for (int u = 0; u < U; u++)
                pcs.push_back(Piece{d_in + lead[u], (unsigned long long)u * O1_NCTX * O1_NSYM * 2, O1_NCTX * O1_NSYM * 2});
            launch_gather(pool, pcs, reinterpret_cast<uint8_t *>(nf), st);
        }
        uint32_t *dt = pool.get<uint32_t>((size_t)ntab * O1_M);
        uint8_t *spread = pool.get<uint8_t>(16);
        k_o1_dtable<<<ntab, 128, 0, st>>>(nf, dt, spread, d_err);
        FB2_CHECK_LAUNCH();
        for (auto &c : chains) c.table = uid[c.table];
        DecChain *dch = h2d(pool, chains, st);
        {
            std::vector<uint16_t> hnf = d2h(nf, (size_t)ntab * O1_NSYM, st);
            tr.mark("decode tables built");
            std::vector<unsigned long long> maps(U), revs(U);
            for (int u = 0; u < U; u++) {
                auto mr = hot_contexts(hnf.data() + (size_t)u * O1_NCTX * O1_NSYM, kDecSlots);
                maps[u] = mr.first;
                revs[u] = mr.second;
            }
            std::vector<int> chain_table(chains.size());
            for (size_t i = 0; i < chains.size(); i++) chain_table[i] = chains[i].table;
            std::vector<ChainCta> ctas = chain_ctas(chain_table, maps, revs);
            ChainCta *d_ctas = h2d(pool, ctas, st);
            enable_big_smem();
            k_o1_decode_smem<<<(unsigned)ctas.size(), kChainThreads, kDecSlots * O1_M * 4, st>>>(d_in, dch, d_ctas, dt, ovf,
                                                                                   ovf_total, d_codes, d_err);
            FB2_CHECK_LAUNCH();
        }
    } else {
        throw std::invalid_argument("unsupported entropy method");
    }
    tr.mark("chains launched");
    if (delta) undelta(pool, d_codes, N, st);
    std::vector<int> he = d2h(d_err, 1, st);
    tr.mark("chains done");
    if (he[0]) throw std::invalid_argument("Invalid or corrupted Falcons entropy payload");
    return off;
}


}  // namespace fb2
