#include "assemble.cuh"

namespace fb2 {

Pool::Pool(cudaStream_t s) : st(s) {
    // once per device (one bit per device ordinal below 64): keep freed blocks of the default
    // memory pool for reuse by the next call
    static std::atomic<unsigned long long> configured{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(configured.load(std::memory_order_acquire) & bit)) {
        cudaMemPool_t mp;
        if (cudaDeviceGetDefaultMemPool(&mp, dev) == cudaSuccess) {
            uint64_t thr = ~0ULL;
            cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        configured.fetch_or(bit, std::memory_order_acq_rel);
    }
}

Pool::~Pool() {
    for (void *p : ptrs) cudaFreeAsync(p, st);
}

namespace {
std::mutex g_stage_mu;
std::vector<void *> g_stage_free;  // page-locked buffers of kStageBytes not in use (kept for the process)
}  // namespace

void *stage_acquire() {
    {
        std::lock_guard<std::mutex> lk(g_stage_mu);
        if (!g_stage_free.empty()) {
            void *p = g_stage_free.back();
            g_stage_free.pop_back();
            return p;
        }
    }
    void *p = nullptr;
    if (cudaHostAlloc(&p, kStageBytes, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();  // the caller falls back to a pageable copy
        return nullptr;
    }
    return p;
}

void stage_release(void *p) {
    std::lock_guard<std::mutex> lk(g_stage_mu);
    g_stage_free.push_back(p);
}

void stage_reserve(int n) {
    for (int i = 0; i < n; i++) {
        void *p = nullptr;
        if (cudaHostAlloc(&p, kStageBytes, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        stage_release(p);
    }
}

namespace {
// Pieces are cut into chunks of kGatherChunk bytes (at multiples of 16 bytes, which keeps the
// alignment of source and destination), a CTA per chunk: chunk c belongs to the last piece whose
// first chunk (cstart, an exclusive scan of the pieces' chunk counts) is at or before c.
constexpr unsigned long long kGatherChunk = 32 * 1024;

__global__ void k_gather(const Piece *__restrict__ pieces, const unsigned *__restrict__ cstart, int np,
                         unsigned nchunks, uint8_t *__restrict__ out) {
    for (unsigned c = blockIdx.x; c < nchunks; c += gridDim.x) {
        int lo = 0, hi = np - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (cstart[mid] <= c) lo = mid;
            else hi = mid - 1;
        }
        const Piece whole = pieces[lo];
        const unsigned long long o = (unsigned long long)(c - cstart[lo]) * kGatherChunk;
        const Piece pc{whole.src + o, whole.dst + o, min(kGatherChunk, whole.len - o)};
        const uint8_t *s = pc.src;
        uint8_t *d = out + pc.dst;
        // bytes up to the first 16-byte destination boundary, whole 16-byte destination words, and
        // the remaining bytes
        unsigned long long head = (16 - ((uintptr_t)d & 15)) & 15;
        if (head > pc.len) head = pc.len;
        for (unsigned long long i = threadIdx.x; i < head; i += blockDim.x) d[i] = s[i];
        const uint8_t *s2 = s + head;
        uint4 *dv = reinterpret_cast<uint4 *>(d + head);
        const unsigned long long nv = (pc.len - head) / 16;
        const unsigned so = (unsigned)((uintptr_t)s2 & 15);
        if (so == 0) {
            const uint4 *sv = reinterpret_cast<const uint4 *>(s2);
            for (unsigned long long i = threadIdx.x; i < nv; i += blockDim.x) dv[i] = sv[i];
        } else {
            // a destination word from the two aligned source words that hold its 16 bytes (both
            // hold bytes of the piece, so they are readable)
            const uint4 *sa = reinterpret_cast<const uint4 *>(s2 - so);
            const unsigned q = so >> 2, r = 8 * (so & 3);
            for (unsigned long long i = threadIdx.x; i < nv; i += blockDim.x) {
                const uint4 A = sa[i], B = sa[i + 1];
                uint32_t w0, w1, w2, w3, w4;
                if (q == 0) { w0 = A.x; w1 = A.y; w2 = A.z; w3 = A.w; w4 = B.x; }
                else if (q == 1) { w0 = A.y; w1 = A.z; w2 = A.w; w3 = B.x; w4 = B.y; }
                else if (q == 2) { w0 = A.z; w1 = A.w; w2 = B.x; w3 = B.y; w4 = B.z; }
                else { w0 = A.w; w1 = B.x; w2 = B.y; w3 = B.z; w4 = B.w; }
                dv[i] = make_uint4(__funnelshift_r(w0, w1, r), __funnelshift_r(w1, w2, r), __funnelshift_r(w2, w3, r),
                                   __funnelshift_r(w3, w4, r));
            }
        }
        for (unsigned long long i = head + nv * 16 + threadIdx.x; i < pc.len; i += blockDim.x) d[i] = s[i];
    }
}
}  // namespace

void launch_gather(Pool &pool, const std::vector<Piece> &pieces, uint8_t *d_out, cudaStream_t st) {
    if (pieces.empty()) return;
    // the pieces and their first chunks go to the device in one copy
    const size_t np = pieces.size();
    std::vector<unsigned char> blob(np * sizeof(Piece) + (np + 1) * sizeof(unsigned));
    Piece *hp = reinterpret_cast<Piece *>(blob.data());
    unsigned *hc = reinterpret_cast<unsigned *>(blob.data() + np * sizeof(Piece));
    unsigned long long chunks = 0;
    for (size_t i = 0; i < np; i++) {
        hp[i] = pieces[i];
        hc[i] = (unsigned)chunks;
        chunks += pieces[i].len ? (pieces[i].len + kGatherChunk - 1) / kGatherChunk : 1;
    }
    hc[np] = (unsigned)chunks;
    if (chunks >= (1ull << 32)) throw std::length_error("gather too large");
    uint8_t *d = h2d(pool, blob, st);
    const Piece *dp = reinterpret_cast<const Piece *>(d);
    const unsigned *dc = reinterpret_cast<const unsigned *>(d + np * sizeof(Piece));
    k_gather<<<(unsigned)std::min<unsigned long long>(chunks, 65535), 256, 0, st>>>(dp, dc, (int)np, (unsigned)chunks,
                                                                                    d_out);
    FB2_CHECK_LAUNCH();
}

size_t zstd_raw_frame_header(uint8_t *out, size_t content) {
    // Frame_Header_Descriptor: Single_Segment_flag (bit 5) with the smallest Frame_Content_Size field.
    int fcs_flag, fcs_bytes;
    if (content < 256) { fcs_flag = 0; fcs_bytes = 1; }
    else if (content < 65536 + 256) { fcs_flag = 1; fcs_bytes = 2; }
    else if (content <= 0xFFFFFFFFull) { fcs_flag = 2; fcs_bytes = 4; }
    else { fcs_flag = 3; fcs_bytes = 8; }
    size_t p = 0;
    const uint32_t magic = kZstdMagic;
    memcpy(out + p, &magic, 4);
    p += 4;
    out[p++] = (uint8_t)((fcs_flag << 6) | (1 << 5));
    uint64_t v = (fcs_flag == 1) ? (uint64_t)content - 256 : (uint64_t)content;
    for (int i = 0; i < fcs_bytes; i++) out[p++] = (uint8_t)(v >> (8 * i));
    return p;
}

size_t zstd_raw_frame_size(size_t content) {
    uint8_t tmp[16];
    const size_t hdr = zstd_raw_frame_header(tmp, content);
    const size_t blocks = content == 0 ? 1 : (content + kZstdBlock - 1) / kZstdBlock;
    return hdr + blocks * 3 + content;
}

void Assembler::run(Pool &pool, uint8_t *d_out, cudaStream_t st) {
    if (pieces.empty()) return;
    uint8_t *dh = h2d(pool, host, st);
    std::vector<Piece> p = pieces;
    for (auto &r : host_refs) p[r.first].src = dh + r.second;
    launch_gather(pool, p, d_out, st);
    FB2_CUDA(cudaStreamSynchronize(st));  // the host vectors must outlive the async copies
}

bool SparseIndex::read(void *dst, unsigned long long o, size_t n) const {
    // reads are mostly in increasing order: try the entry of the previous read and the next one
    for (size_t e = last; e < off.size() && e < last + 2; e++) {
        if (off[e] <= o && o + n <= off[e] + len[e]) {
            memcpy(dst, bytes.data() + pos[e] + (o - off[e]), n);
            last = e;
            return true;
        }
    }
    // last entry with off <= o
    size_t lo = 0, hi = off.size();
    while (lo < hi) {
        const size_t mid = (lo + hi) / 2;
        if (off[mid] <= o) lo = mid + 1;
        else hi = mid;
    }
    if (lo == 0) return false;
    const size_t e = lo - 1;
    if (o + n > off[e] + len[e]) return false;
    memcpy(dst, bytes.data() + pos[e] + (o - off[e]), n);
    last = e;
    return true;
}

bool SparseIndex::parse(const uint8_t *c, size_t size, SparseIndex &out) {
    if (size < 12) return false;
    uint32_t tag, count;
    memcpy(&tag, c, 4);
    memcpy(&count, c + 4, 4);
    if (tag != kIndexTag) return false;
    size_t p = 8;
    for (uint32_t i = 0; i < count; i++) {
        if (p + 12 > size) return false;
        unsigned long long o;
        uint32_t l;
        memcpy(&o, c + p, 8);
        memcpy(&l, c + p + 8, 4);
        p += 12;
        if (p + l > size) return false;
        out.off.push_back(o);
        out.len.push_back(l);
        out.pos.push_back(out.bytes.size());
        out.bytes.insert(out.bytes.end(), c + p, c + p + l);
        p += l;
    }
    for (size_t i = 1; i < out.off.size(); i++)
        if (out.off[i] < out.off[i - 1]) return false;
    return true;
}

size_t Assembler::index_frame_size() const {
    size_t n = 16;
    for (auto &r : host_refs) n += 12 + (size_t)pieces[r.first].len;
    for (auto &sh : shadows) n += 12 + sh.second.size();
    return n;
}

std::vector<uint8_t> Assembler::index_frame() const {
    // host pieces and shadows are each recorded in offset order: merge them
    using Entry = std::pair<unsigned long long, std::pair<const uint8_t *, size_t>>;
    std::vector<Entry> e1, e2, e;
    e1.reserve(host_refs.size());
    e2.reserve(shadows.size());
    for (auto &r : host_refs) e1.push_back({pieces[r.first].dst, {host.data() + r.second, (size_t)pieces[r.first].len}});
    for (auto &sh : shadows) e2.push_back({sh.first, {sh.second.data(), sh.second.size()}});
    e.resize(e1.size() + e2.size());
    auto less = [](const Entry &a, const Entry &b) { return a.first < b.first; };
    if (std::is_sorted(e1.begin(), e1.end(), less) && std::is_sorted(e2.begin(), e2.end(), less)) {
        std::merge(e1.begin(), e1.end(), e2.begin(), e2.end(), e.begin(), less);
    } else {
        std::copy(e1.begin(), e1.end(), e.begin());
        std::copy(e2.begin(), e2.end(), e.begin() + (long)e1.size());
        std::stable_sort(e.begin(), e.end(), less);
    }
    size_t total = 16;
    for (auto &x : e) total += 12 + x.second.second;
    std::vector<uint8_t> c;
    c.reserve(total);
    c.resize(16);
    const uint32_t magic = kSkippableMagic, tag = kIndexTag, count = (uint32_t)e.size();
    memcpy(c.data() + 8, &tag, 4);
    memcpy(c.data() + 12, &count, 4);
    for (auto &x : e) {
        const unsigned long long o = x.first;
        const uint32_t l = (uint32_t)x.second.second;
        const size_t at = c.size();
        c.resize(at + 12 + l);
        memcpy(c.data() + at, &o, 8);
        memcpy(c.data() + at + 8, &l, 4);
        memcpy(c.data() + at + 12, x.second.first, l);
    }
    const uint32_t fsz = (uint32_t)(c.size() - 8);
    memcpy(c.data(), &magic, 4);
    memcpy(c.data() + 4, &fsz, 4);
    return c;
}

size_t Assembler::run_framed(Pool &pool, uint8_t *d_out, cudaStream_t st) {
    Trace tr("assemble");
    const size_t L = pos;
    std::vector<uint8_t> hb;  // the host bytes, then the length word, frame header, block headers
    hb.reserve(host.size() + 64 + 3 * (pos / kZstdBlock + 2) + (with_index ? index_frame_size() + tail_host.size() : 0));
    hb.insert(hb.end(), host.begin(), host.end());
    std::vector<Piece> out;
    out.reserve(pieces.size() + pieces.size() / 4 + pos / kZstdBlock + tail.size() + 16);
    auto add_host = [&](const uint8_t *b, size_t n, unsigned long long dst) {
        const size_t off = hb.size();
        hb.insert(hb.end(), b, b + n);
        out.push_back(Piece{reinterpret_cast<const uint8_t *>(off), dst, n});  // patched below
    };
    std::vector<size_t> host_pieces;  // indices into `out` whose src is a host offset
    uint8_t tmp[16];
    const uint64_t L64 = L;
    host_pieces.push_back(out.size());
    add_host(reinterpret_cast<const uint8_t *>(&L64), 8, 0);
    const size_t fh = zstd_raw_frame_header(tmp, L);
    host_pieces.push_back(out.size());
    add_host(tmp, fh, 8);
    const size_t base = 8 + fh;
    const size_t nblocks = L == 0 ? 1 : (L + kZstdBlock - 1) / kZstdBlock;
    for (size_t b = 0; b < nblocks; b++) {
        const size_t bs = std::min(kZstdBlock, L - b * kZstdBlock);
        const uint32_t h = (uint32_t)((b + 1 == nblocks) ? 1 : 0) | (0u << 1) | ((uint32_t)bs << 3);
        uint8_t hh[3] = {(uint8_t)h, (uint8_t)(h >> 8), (uint8_t)(h >> 16)};
        host_pieces.push_back(out.size());
        add_host(hh, 3, base + b * (kZstdBlock + 3));
    }
    // logical pieces split at block boundaries
    std::vector<bool> is_host(pieces.size(), false);
    std::vector<size_t> host_off(pieces.size(), 0);
    for (auto &r : host_refs) {
        is_host[r.first] = true;
        host_off[r.first] = r.second;
    }
    for (size_t i = 0; i < pieces.size(); i++) {
        const Piece &pc = pieces[i];
        unsigned long long x = pc.dst, rem = pc.len, so = 0;
        while (rem) {
            const unsigned long long in_blk = kZstdBlock - x % kZstdBlock;
            const unsigned long long c = std::min(rem, in_blk);
            const unsigned long long phys = base + (x / kZstdBlock) * (kZstdBlock + 3) + 3 + (x % kZstdBlock);
            if (is_host[i]) {
                host_pieces.push_back(out.size());
                out.push_back(Piece{reinterpret_cast<const uint8_t *>(host_off[i] + so), phys, c});
            } else {
                out.push_back(Piece{pc.src + so, phys, c});
            }
            x += c;
            so += c;
            rem -= c;
        }
    }
    tr.mark("pieces split");
    size_t total = 8 + zstd_raw_frame_size(L);
    if (with_index) {
        const std::vector<uint8_t> idx = index_frame();
        host_pieces.push_back(out.size());
        add_host(idx.data(), idx.size(), total);
        total += idx.size();
        for (size_t i = 0; i < tail.size(); i++) {
            if (tail[i].src == nullptr) {
                host_pieces.push_back(out.size());
                add_host(tail_host.data() + tail_off[i], tail[i].len, total + tail[i].dst);
            } else {
                out.push_back(Piece{tail[i].src, total + tail[i].dst, tail[i].len});
            }
        }
        total += tail_len;
    }
    tr.mark("index frame built");
    uint8_t *dh = h2d(pool, hb, st);
    tr.mark("host bytes copied");
    if (tr.on)
        std::fprintf(stderr, "[falcons trace] assemble: %zu host bytes, %zu pieces\n", hb.size(), out.size());
    for (size_t i : host_pieces) out[i].src = dh + reinterpret_cast<uintptr_t>(out[i].src);
    launch_gather(pool, out, d_out, st);
    tr.mark("gather launched");
    FB2_CUDA(cudaStreamSynchronize(st));
    tr.mark("gathered");
    return total;
}

void logical_pieces(const uint8_t *d_base, bool framed, size_t off, size_t n, unsigned long long dst,
                    std::vector<Piece> &out) {
    if (!framed) {
        if (n) out.push_back(Piece{d_base + off, dst, n});
        return;
    }
    while (n) {
        const size_t c = std::min(n, kZstdBlock - off % kZstdBlock);
        const size_t phys = (off / kZstdBlock) * (kZstdBlock + 3) + 3 + (off % kZstdBlock);
        out.push_back(Piece{d_base + phys, dst, c});
        off += c;
        dst += c;
        n -= c;
    }
}

}  // namespace fb2
