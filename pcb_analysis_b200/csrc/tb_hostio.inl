// Large host <-> device copies through pinned staging (included in
// tb_system.cu).
//
// A copy from or to pageable host memory moves its host side with a single
// thread's memcpy through the driver's own pinned buffer, and a fresh NumPy
// result array takes its page faults inside that memcpy.  A board's arrays
// are hundreds of megabytes each (c3: 571 MB per node field, 1.6 GB of
// element flux), so the host side, not the link, set the pace of the public
// call.  Here the host side of a large copy is split across worker threads,
// into and out of two pinned chunks of this process per device, used
// alternately: one chunk's DMA runs while the other is filled or drained.
// Copies below kIoDirect bytes stay plain cudaMemcpyAsync calls.  (Uses
// <algorithm>, <cstring>, <mutex>, <thread> and <vector>, included by the
// including file at global scope; it sits in that file's unnamed namespace.)

constexpr size_t kIoChunk = size_t(64) << 20;   // bytes per pinned chunk
constexpr size_t kIoDirect = size_t(16) << 20;  // smaller copies go straight through the driver
constexpr int kIoMaxDevices = 64;

struct PinnedRing {
    std::mutex mu;
    void* buf[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
};

PinnedRing& pinned_ring(int device) {
    static PinnedRing rings[kIoMaxDevices];
    return rings[device];
}

// The ring of `device`, made on first use (the caller holds its lock and has
// made `device` current).  It lives as long as the process.
int ring_ready(PinnedRing& r) {
    if (r.buf[0] != nullptr) return TB_OK;
    for (int b = 0; b < 2; ++b) {
        TB_CUDA(cudaHostAlloc(&r.buf[b], kIoChunk, cudaHostAllocPortable));
        TB_CUDA(cudaEventCreateWithFlags(&r.done[b], cudaEventDisableTiming));
    }
    return TB_OK;
}

int io_threads() {
    static const int n = [] {
        const unsigned hw = std::thread::hardware_concurrency();
        return (int)std::min(16u, std::max(1u, hw / 2));
    }();
    return n;
}

// memcpy of `bytes` split into page-aligned slices, one per worker thread.
void parallel_memcpy(void* dst, const void* src, size_t bytes) {
    const int threads = bytes < (size_t(4) << 20) ? 1 : io_threads();
    const size_t slice = ((bytes + threads - 1) / threads + 4095) / 4096 * 4096;
    std::vector<std::thread> workers;
    for (int t = 1; t < threads; ++t) {
        const size_t off = (size_t)t * slice;
        if (off >= bytes) break;
        const size_t n = std::min(slice, bytes - off);
        workers.emplace_back([=] { std::memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, n); });
    }
    std::memcpy(dst, src, std::min(slice, bytes));
    for (auto& w : workers) w.join();
}

// Host -> device on the system's stream.  Returns once the host array has
// been read (as a pageable cudaMemcpyAsync does); the last chunks' DMA may
// still be in flight, ordered before the stream's later work.
int host_to_device(tb_system* s, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return TB_OK;
    if (bytes < kIoDirect || s->device >= kIoMaxDevices) {
        TB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s->stream));
        return TB_OK;
    }
    PinnedRing& r = pinned_ring(s->device);
    std::lock_guard<std::mutex> lock(r.mu);
    TB_CHECK(ring_ready(r));
    size_t k = 0;
    for (size_t off = 0; off < bytes; off += kIoChunk, ++k) {
        const int b = (int)(k & 1);
        const size_t n = std::min(kIoChunk, bytes - off);
        TB_CUDA(cudaEventSynchronize(r.done[b]));  // this chunk's previous DMA has read it
        parallel_memcpy(r.buf[b], static_cast<const char*>(src) + off, n);
        TB_CUDA(cudaMemcpyAsync(static_cast<char*>(dst) + off, r.buf[b], n, cudaMemcpyHostToDevice, s->stream));
        TB_CUDA(cudaEventRecord(r.done[b], s->stream));
    }
    return TB_OK;
}

// Device -> host on the system's stream, after the stream's earlier work.
// Returns once the host array holds the data.
int device_to_host(tb_system* s, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return TB_OK;
    if (bytes < kIoDirect || s->device >= kIoMaxDevices) {
        TB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s->stream));
        TB_CUDA(cudaStreamSynchronize(s->stream));
        return TB_OK;
    }
    PinnedRing& r = pinned_ring(s->device);
    std::lock_guard<std::mutex> lock(r.mu);
    TB_CHECK(ring_ready(r));
    const size_t chunks = (bytes + kIoChunk - 1) / kIoChunk;
    auto issue = [&](size_t k) -> int {
        const int b = (int)(k & 1);
        const size_t off = k * kIoChunk;
        const size_t n = std::min(kIoChunk, bytes - off);
        TB_CUDA(cudaMemcpyAsync(r.buf[b], static_cast<const char*>(src) + off, n, cudaMemcpyDeviceToHost, s->stream));
        TB_CUDA(cudaEventRecord(r.done[b], s->stream));
        return TB_OK;
    };
    TB_CHECK(issue(0));
    if (chunks > 1) TB_CHECK(issue(1));
    for (size_t k = 0; k < chunks; ++k) {
        const int b = (int)(k & 1);
        const size_t off = k * kIoChunk;
        const size_t n = std::min(kIoChunk, bytes - off);
        TB_CUDA(cudaEventSynchronize(r.done[b]));
        parallel_memcpy(static_cast<char*>(dst) + off, r.buf[b], n);
        if (k + 2 < chunks) TB_CHECK(issue(k + 2));
    }
    return TB_OK;
}
