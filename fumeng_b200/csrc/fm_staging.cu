// Pinned staging ring and host copy threads (interface in fm_staging.h).
#include "fm_staging.h"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <new>
#include <thread>

#include "fm_internal.h"

namespace fm {

// A few threads that split large host copies with the calling thread.
class CopyPool {
public:
    explicit CopyPool(int workers)
    {
        for (int i = 0; i < workers; ++i) threads_.emplace_back([this] { loop(); });
    }
    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : threads_) t.join();
    }
    int size() const { return (int)threads_.size() + 1; }

    // Runs fn(0 .. tasks-1) on the workers and the caller; returns when every task is done
    // and no worker is still inside this call's task loop.
    void run(int tasks, const std::function<void(int)>& fn)
    {
        {
            std::lock_guard<std::mutex> lk(m_);
            fn_ = &fn;
            tasks_ = tasks;
            next_.store(0);
            done_ = 0;
            ++gen_;
        }
        cv_.notify_all();
        const int mine = work();
        std::unique_lock<std::mutex> lk(m_);
        done_ += mine;
        done_cv_.wait(lk, [&] { return done_ == tasks_ && active_ == 0; });
        fn_ = nullptr;
    }

private:
    // Takes tasks of the current round until none is left; returns how many it ran.
    int work()
    {
        int finished = 0;
        for (;;) {
            const int i = next_.fetch_add(1);
            if (i >= tasks_) break;
            (*fn_)(i);
            ++finished;
        }
        return finished;
    }
    void loop()
    {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return stop_ || (gen_ != seen && fn_); });
                if (stop_) return;
                seen = gen_;
                ++active_;   // the round cannot end (nor the next begin) while this is set
            }
            const int finished = work();
            std::lock_guard<std::mutex> lk(m_);
            done_ += finished;
            --active_;
            if (done_ == tasks_ && active_ == 0) done_cv_.notify_all();
        }
    }
    std::vector<std::thread> threads_;
    std::mutex m_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)>* fn_ = nullptr;
    std::atomic<int> next_{0};
    int tasks_ = 0, done_ = 0, active_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

cudaError_t staging_ensure(fm_ctx* ctx)
{
    if (ctx->stage) return cudaSuccess;
    std::vector<cudaEvent_t> evs;
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < kStageChunks && e == cudaSuccess; ++k) {
        cudaEvent_t ev = nullptr;
        e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) evs.push_back(ev);
    }
    void* p = nullptr;
    if (e == cudaSuccess) e = cudaHostAlloc(&p, kStageChunk * kStageChunks, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        for (cudaEvent_t ev : evs) cudaEventDestroy(ev);
        return e;
    }
    ctx->stage = static_cast<char*>(p);
    ctx->stage_events = evs;
    if (!ctx->copy_pool) {
        const unsigned hw = std::thread::hardware_concurrency();
        const int workers = (int)std::min<unsigned>(hw > 1 ? hw - 1 : 0, 7);
        ctx->copy_pool = new (std::nothrow) CopyPool(workers);
    }
    return cudaSuccess;
}

void staging_release(fm_ctx* ctx)
{
    for (cudaEvent_t e : ctx->stage_events) {
        cudaEventSynchronize(e);
        cudaEventDestroy(e);
    }
    ctx->stage_events.clear();
    if (ctx->stage) cudaFreeHost(ctx->stage);
    ctx->stage = nullptr;
    delete ctx->copy_pool;
    ctx->copy_pool = nullptr;
}

void host_parallel(fm_ctx* ctx, int tasks, const std::function<void(int)>& fn)
{
    if (tasks <= 0) return;
    if (!ctx->copy_pool || ctx->copy_pool->size() == 1 || tasks == 1) {
        for (int i = 0; i < tasks; ++i) fn(i);
        return;
    }
    ctx->copy_pool->run(tasks, fn);
}

void copy_segments(fm_ctx* ctx, const std::vector<Segment>& segs)
{
    size_t total = 0;
    for (const Segment& g : segs) total += g.bytes;
    constexpr size_t kSlice = size_t(256) << 10;
    CopyPool* pool = ctx->copy_pool;
    const int tasks = pool ? (int)std::min<size_t>((total + kSlice - 1) / kSlice, (size_t)pool->size()) : 1;
    if (tasks <= 1) {
        for (const Segment& g : segs) std::memcpy(g.dst, g.src, g.bytes);
        return;
    }
    const size_t per = (total + tasks - 1) / tasks;
    pool->run(tasks, [&](int i) {
        // bytes [a, b) of the concatenated segments
        const size_t a = per * (size_t)i, b = std::min(total, a + per);
        size_t pos = 0;
        for (const Segment& g : segs) {
            const size_t lo = std::max(a, pos), hi = std::min(b, pos + g.bytes);
            if (lo < hi)
                std::memcpy(static_cast<char*>(g.dst) + (lo - pos), static_cast<const char*>(g.src) + (lo - pos), hi - lo);
            pos += g.bytes;
            if (pos >= b) break;
        }
    });
}

void Stager::flush()
{
    if (!host.empty()) {
        copy_segments(ctx, host);
        host.clear();
    }
    for (const Segment& g : device)
        if (err == cudaSuccess) err = cudaMemcpyAsync(g.dst, g.src, g.bytes, cudaMemcpyHostToDevice, s);
    device.clear();
}

// Closes the current chunk (its copies are issued) and waits until the next chunk's
// previous copies have finished with it.
void Stager::next_chunk()
{
    flush();
    if (chunk >= 0 && err == cudaSuccess) err = cudaEventRecord(ctx->stage_events[chunk], s);
    chunk = (chunk + 1) % kStageChunks;
    if (err == cudaSuccess) err = cudaEventSynchronize(ctx->stage_events[chunk]);
    used = 0;
}

void Stager::put(void* dst_dev, const void* src_host, size_t bytes, size_t pad_before)
{
    char* dst = static_cast<char*>(dst_dev);
    const char* src = static_cast<const char*>(src_host);
    if (pad_before && !device.empty() && used < kStageChunk) {
        Segment& last = device.back();
        char* end = static_cast<char*>(last.dst) + last.bytes;
        const size_t gap = (size_t)(dst - end);
        if (dst >= end && gap <= pad_before && static_cast<const char*>(last.src) + last.bytes ==
                                                   ctx->stage + (size_t)chunk * kStageChunk + used &&
            used + gap < kStageChunk) {
            used += gap;
            last.bytes += gap;
        }
    }
    while (bytes > 0 && err == cudaSuccess) {
        if (used == kStageChunk) next_chunk();
        if (err != cudaSuccess) return;
        const size_t k = std::min(bytes, kStageChunk - used);
        char* h = ctx->stage + (size_t)chunk * kStageChunk + used;
        host.push_back(Segment{h, src, k});
        Segment* last = device.empty() ? nullptr : &device.back();
        if (last && static_cast<char*>(last->dst) + last->bytes == dst &&
            static_cast<const char*>(last->src) + last->bytes == h)
            last->bytes += k;
        else
            device.push_back(Segment{dst, h, k});
        used += k;
        dst += k;
        src += k;
        bytes -= k;
    }
}

void Stager::close()
{
    flush();
    if (chunk >= 0 && err == cudaSuccess) err = cudaEventRecord(ctx->stage_events[chunk], s);
    used = kStageChunk;
}

cudaError_t copy_out(fm_ctx* ctx, cudaStream_t s, const std::vector<OutCopy>& copies)
{
    cudaError_t e = staging_ensure(ctx);
    if (e != cudaSuccess) return e;
    // chunks of the ring, each a list of (host destination, offset in chunk, bytes)
    struct Part {
        char* dst;
        size_t off, bytes;
    };
    std::vector<std::vector<Part>> pending(kStageChunks);
    int slot = 0;
    size_t used = 0;
    auto drain = [&](int k) -> cudaError_t {
        cudaError_t r = cudaEventSynchronize(ctx->stage_events[k]);
        if (r != cudaSuccess) return r;
        const char* base = ctx->stage + (size_t)k * kStageChunk;
        std::vector<Segment> segs;
        for (const Part& p : pending[k]) segs.push_back(Segment{p.dst, base + p.off, p.bytes});
        copy_segments(ctx, segs);
        pending[k].clear();
        return cudaSuccess;
    };
    // closes the filling chunk and moves to the next, draining it first if it holds data
    auto advance = [&]() -> cudaError_t {
        cudaError_t r = cudaEventRecord(ctx->stage_events[slot], s);
        if (r != cudaSuccess) return r;
        slot = (slot + 1) % kStageChunks;
        used = 0;
        if (!pending[slot].empty()) return drain(slot);
        return cudaEventSynchronize(ctx->stage_events[slot]);   // an earlier host -> device use
    };
    if (e == cudaSuccess) e = cudaEventSynchronize(ctx->stage_events[0]);
    for (const OutCopy& c : copies) {
        char* dst = static_cast<char*>(c.dst_host);
        const char* src = static_cast<const char*>(c.src_dev);
        size_t bytes = c.bytes;
        while (bytes > 0 && e == cudaSuccess) {
            if (used == kStageChunk) {
                e = advance();
                if (e != cudaSuccess) break;
            }
            const size_t k = std::min(bytes, kStageChunk - used);
            e = cudaMemcpyAsync(ctx->stage + (size_t)slot * kStageChunk + used, src, k, cudaMemcpyDeviceToHost, s);
            pending[slot].push_back(Part{dst, used, k});
            used += k;
            dst += k;
            src += k;
            bytes -= k;
        }
    }
    if (e == cudaSuccess && used > 0) e = advance();
    for (int k = 0; k < kStageChunks && e == cudaSuccess; ++k) {
        const int j = (slot + k) % kStageChunks;
        if (!pending[j].empty()) e = drain(j);
    }
    return e;
}

}  // namespace fm
