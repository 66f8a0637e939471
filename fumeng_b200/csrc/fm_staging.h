// Host <-> device transfers through a context-owned pinned ring (fm_staging.cu).
//
// Pageable cudaMemcpyAsync serialises the host with the stream and copies through the
// driver's own bounce buffer; the ring instead lets the host fill (or drain) one 8 MiB
// chunk while the copy engine moves another, and host-side copies of large chunks are
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

// memcpy split over the context's copy threads (plain memcpy below 1 MiB).
void host_copy(fm_ctx* ctx, void* dst, const void* src, size_t bytes);

// Runs fn(0 .. tasks-1) on the context's copy threads and the caller (serially without
// them); returns when all are done.  fn must not throw.
void host_parallel(fm_ctx* ctx, int tasks, const std::function<void(int)>& fn);

// Host -> device: bytes bound for consecutive device addresses go as one copy.
struct Stager {
    fm_ctx* ctx;
    cudaStream_t s;
    int chunk = -1;
    size_t used = kStageChunk;
    char* run_dst = nullptr;
    const char* run_src = nullptr;
    size_t run_len = 0;
    cudaError_t err = cudaSuccess;

    Stager(fm_ctx* c, cudaStream_t stream) : ctx(c), s(stream) {}
    // Copies `bytes` from host memory to `dst_dev` (stream-ordered on `s`); the host
    // buffer may be reused as soon as this returns.
    void put(void* dst_dev, const void* src_host, size_t bytes);
    // Issues the pending copy.
    void flush();
    // Issues what is pending and marks the current chunk busy until its copies finish.
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
