// Host <-> device transfers through a context-owned pinned ring (fm_staging.cu).
//
// Pageable cudaMemcpyAsync serialises the host with the stream and copies through the
// driver's own bounce buffer; the ring instead lets the host fill (or drain) one 8 MiB
// chunk while the copy engine moves another, and the host-side copies of a chunk are
// split over a few worker threads.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <functional>
#include <vector>

struct fm_ctx;

namespace fm {

constexpr int kStageChunks = 4;
constexpr size_t kStageChunk = size_t(8) << 20;

class CopyPool;

// The ring and the copy pool live in the context; created on first use.
cudaError_t staging_ensure(fm_ctx* ctx);
void staging_release(fm_ctx* ctx);

// Runs fn(0 .. tasks-1) on the context's copy threads and the caller (serially without
// them); returns when all are done.  fn must not throw.
void host_parallel(fm_ctx* ctx, int tasks, const std::function<void(int)>& fn);

// One host-side copy of a batch (see copy_segments).
struct Segment {
    void* dst;
    const void* src;
    size_t bytes;
};

// Copies every segment, the bytes split evenly over the context's copy threads.
void copy_segments(fm_ctx* ctx, const std::vector<Segment>& segs);

// Host -> device through the ring, on one stream.  Host bytes are gathered into the ring
// when a chunk is closed (one parallel copy for all the pieces in it), and bytes bound for
// consecutive device addresses go as one cudaMemcpyAsync.
struct Stager {
    fm_ctx* ctx;
    cudaStream_t s;
    int chunk = -1;
    size_t used = kStageChunk;
    std::vector<Segment> host;      // pending host -> ring copies
    std::vector<Segment> device;    // pending ring -> device copies (dst = device)
    cudaError_t err = cudaSuccess;

    Stager(fm_ctx* c, cudaStream_t stream) : ctx(c), s(stream) {}
    // Queues a copy of `bytes` from host memory to `dst_dev` (stream-ordered on `s`); the
    // host memory must stay valid until the next flush() or close().  `pad_before` device
    // bytes just below dst_dev are free padding of the same allocation: when the previous
    // copy ends within them, the ring is padded alike and the two copies become one (the
    // padding receives unspecified bytes).
    void put(void* dst_dev, const void* src_host, size_t bytes, size_t pad_before = 0);
    // Performs the queued host copies and issues the device copies.
    void flush();
    // flush(), then marks the current chunk busy until its copies finish.
    void close();

private:
    void next_chunk();
};

// Device -> host copies through the ring, on `s`, after the work already on `s`; returns
// when every byte is in host memory.
struct OutCopy {
    void* dst_host;
    const void* src_dev;
    size_t bytes;
};
cudaError_t copy_out(fm_ctx* ctx, cudaStream_t s, const std::vector<OutCopy>& copies);

}  // namespace fm
