// Stream assembly helpers shared by the entropy stage and the pipeline:
//   Pool       stream-ordered device scratch (cudaMallocAsync on the default pool, retained)
//   Assembler  a list of byte pieces (device or host-built) laid out back to back and copied into
//              place by one gather kernel; optionally framed as a Zstandard frame of raw blocks
//              (RFC 8878 section 3.1: magic, frame header with content size, 3-byte block headers)
//   ByteView   logical read access to a byte range that may sit inside such a raw-block frame
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <vector>

#include "common.cuh"

namespace fb2 {

constexpr size_t kZstdBlock = 128 * 1024;   // Block_Maximum_Size
constexpr uint32_t kZstdMagic = 0xFD2FB528u;

struct Pool {
    cudaStream_t st;
    std::vector<void *> ptrs;
    explicit Pool(cudaStream_t s);
    template <class T>
    T *get(size_t count) {
        void *p = nullptr;
        FB2_CUDA(cudaMallocAsync(&p, std::max<size_t>(count * sizeof(T), 16) + 64, st));
        ptrs.push_back(p);
        return static_cast<T *>(p);
    }
    ~Pool();
};

// Pinned host staging for small device-to-host reads: a process-wide free list of page-locked
// buffers of kStageBytes, one taken per read and given back after it (the list grows only while
// more reads are in flight at once than ever before).  A copy into pageable memory goes through
// the driver's own staging, which concurrent callers share.
constexpr size_t kStageBytes = 1 << 20;
void *stage_acquire();
void stage_release(void *p);
// Adds n buffers to the free list (page-locking host memory synchronizes the device, so a context
// reserves its share when it is created rather than on a call that other streams are running beside).
void stage_reserve(int n);

template <class T>
std::vector<T> d2h(const T *d, size_t n, cudaStream_t st) {
    std::vector<T> h(n);
    if (n) {
        const size_t bytes = n * sizeof(T);
        void *stage = bytes <= kStageBytes ? stage_acquire() : nullptr;
        if (stage) {
            cudaError_t e = cudaMemcpyAsync(stage, d, bytes, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e == cudaSuccess) std::memcpy(h.data(), stage, bytes);
            stage_release(stage);
            FB2_CUDA(e);
        } else {
            FB2_CUDA(cudaMemcpyAsync(h.data(), d, bytes, cudaMemcpyDeviceToHost, st));
            FB2_CUDA(cudaStreamSynchronize(st));
        }
    }
    return h;
}

template <class T>
T *h2d(Pool &pool, const std::vector<T> &h, cudaStream_t st) {
    T *d = pool.get<T>(h.size());
    if (!h.empty()) FB2_CUDA(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    return d;
}

inline unsigned grid_for(long long n, int threads, long long cap = 1 << 20) {
    return (unsigned)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, cap));
}

// Number of SMs of the current device (cached per device).
inline int sm_count() {
    static std::atomic<int> cache[64];
    int dev = 0;
    FB2_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return 148;
    int v = cache[dev].load(std::memory_order_relaxed);
    if (v == 0) {
        FB2_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
        if (v <= 0) v = 148;
        cache[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

struct Piece {
    const uint8_t *src;
    unsigned long long dst;
    unsigned long long len;
};

// Copies every piece to out + dst (one CTA per 32 KiB chunk of a piece, 16-byte destination words).
void launch_gather(Pool &pool, const std::vector<Piece> &pieces, uint8_t *d_out, cudaStream_t st);

// Size of a raw-block zstd frame holding `content` bytes.
size_t zstd_raw_frame_size(size_t content);
// Frame header bytes (magic + descriptor + content size); returns its length.
size_t zstd_raw_frame_header(uint8_t *out, size_t content);

// Header index carried in a zstd skippable frame after the payload frame (RFC 8878 section 3.1.2;
// decoders, the reference's included, skip it).  It holds every header byte of the payload
// (logical offset + bytes), so a decoder whose stream sits in device memory can parse the block
// structure without copying the stream to the host.
constexpr uint32_t kSkippableMagic = 0x184D2A5Bu;
constexpr uint32_t kIndexTag = 0x49324246u;  // "FB2I"

struct SparseIndex {
    std::vector<unsigned long long> off;   // sorted logical offsets
    std::vector<uint32_t> len;
    std::vector<size_t> pos;               // into bytes
    std::vector<uint8_t> bytes;
    mutable size_t last = 0;               // entry of the previous read
    // Returns false when [o, o+n) is not fully covered by one entry.
    bool read(void *dst, unsigned long long o, size_t n) const;
    static bool parse(const uint8_t *content, size_t size, SparseIndex &out);
};

struct Assembler {
    std::vector<Piece> pieces;                         // logical layout
    std::vector<uint8_t> host;                         // host-built bytes
    std::vector<std::pair<size_t, size_t>> host_refs;  // (piece index, host offset)
    std::vector<std::pair<unsigned long long, std::vector<uint8_t>>> shadows;  // header bytes of device pieces
    unsigned long long pos = 0;
    bool with_index = true;
    // Records that the next device piece starts with these (host-known) header bytes.
    void shadow(const void *b, size_t n) {
        shadows.push_back({pos, std::vector<uint8_t>(static_cast<const uint8_t *>(b), static_cast<const uint8_t *>(b) + n)});
    }
    std::vector<uint8_t> index_frame() const;
    size_t index_frame_size() const;
    void dev(const void *src, size_t len) {
        if (!len) return;
        pieces.push_back(Piece{static_cast<const uint8_t *>(src), pos, len});
        pos += len;
    }
    void bytes(const void *p, size_t len) {
        if (!len) return;
        const size_t off = host.size();
        host.insert(host.end(), static_cast<const uint8_t *>(p), static_cast<const uint8_t *>(p) + len);
        if (!host_refs.empty() && host_refs.back().first + 1 == pieces.size() &&
            host_refs.back().second + pieces.back().len == off) {
            pieces.back().len += len;  // extends the previous host piece (one gather piece, one index entry)
        } else {
            host_refs.push_back({pieces.size(), off});
            pieces.push_back(Piece{nullptr, pos, len});
        }
        pos += len;
    }
    template <class T>
    void val(T v) {
        bytes(&v, sizeof(T));
    }
    // Bytes written after the index frame (further skippable frames): host bytes or device pieces.
    std::vector<Piece> tail;                 // src == nullptr: host bytes at tail_host + tail_off
    std::vector<uint8_t> tail_host;
    std::vector<size_t> tail_off;
    unsigned long long tail_len = 0;
    void tail_bytes(const void *p, size_t n) {
        if (!n) return;
        tail_off.push_back(tail_host.size());
        tail_host.insert(tail_host.end(), static_cast<const uint8_t *>(p), static_cast<const uint8_t *>(p) + n);
        tail.push_back(Piece{nullptr, tail_len, n});
        tail_len += n;
    }
    void tail_dev(const void *src, size_t n) {
        if (!n) return;
        tail_off.push_back(0);
        tail.push_back(Piece{static_cast<const uint8_t *>(src), tail_len, n});
        tail_len += n;
    }
    // Copies the logical layout to d_out[0, pos).  Synchronizes the stream.
    void run(Pool &pool, uint8_t *d_out, cudaStream_t st);
    // Writes [u64 pos][zstd raw-block frame of the layout] to d_out; returns the bytes written.
    size_t run_framed(Pool &pool, uint8_t *d_out, cudaStream_t st);
    size_t framed_size() const {
        return 8 + zstd_raw_frame_size(pos) + (with_index ? index_frame_size() + tail_len : 0);
    }
};

// Logical bytes [0, len) stored either flat or as the content of a raw-block zstd frame.
struct ByteView {
    const SparseIndex *sparse = nullptr;  // when set, reads are served from the header index
    const uint8_t *base = nullptr;   // host pointer (flat bytes or the frame's first block header)
    size_t len = 0;                  // logical length (from origin)
    bool framed = false;
    size_t origin = 0;               // logical offset of index 0
    size_t phys(size_t i) const {
        i += origin;
        return framed ? (i / kZstdBlock) * (kZstdBlock + 3) + 3 + (i % kZstdBlock) : i;
    }
    ByteView sub(size_t off) const {
        if (off > len) throw std::invalid_argument("Invalid or truncated Falcons payload");
        ByteView v = *this;
        v.origin += off;
        v.len -= off;
        return v;
    }
    uint8_t at(size_t i) const {
        if (i >= len) throw std::invalid_argument("Invalid or truncated Falcons payload");
        if (sparse) {
            uint8_t b;
            read(&b, i, 1);
            return b;
        }
        return base[phys(i)];
    }
    void read(void *dst, size_t off, size_t n) const {
        if (off + n > len || off + n < off) throw std::invalid_argument("Invalid or truncated Falcons payload");
        uint8_t *d = static_cast<uint8_t *>(dst);
        if (sparse) {
            if (!sparse->read(d, origin + off, n)) throw std::out_of_range("header index does not cover the read");
            return;
        }
        if (!framed) {
            memcpy(d, base + origin + off, n);
            return;
        }
        while (n) {
            const size_t in_blk = kZstdBlock - (origin + off) % kZstdBlock;
            const size_t c = std::min(n, in_blk);
            memcpy(d, base + phys(off), c);
            d += c;
            off += c;
            n -= c;
        }
    }
    template <class T>
    T rd(size_t &off) const {
        T v;
        read(&v, off, sizeof(T));
        off += sizeof(T);
        return v;
    }
};

// Device counterpart: pieces that move logical [off, off+n) of a (possibly framed) device buffer
// to dst (flat).  Returns the pieces (the caller launches the gather).
void logical_pieces(const uint8_t *d_base, bool framed, size_t off, size_t n, unsigned long long dst,
                    std::vector<Piece> &out);

}  // namespace fb2
