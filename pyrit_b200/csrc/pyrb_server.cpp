// Served chunk builds behind the C ABI (pyrb_server_*): continuous batching of
// chunk-build requests on one GPU.
//
// The reference streams a world on a worker thread that builds batches of chunks
// (World.gpuWorkImpl, src/world.zig:937-1025), admits work by its free device memory
// (World.vramFree, :814-821) and evicts unused chunks from its pools
// (src/world_plan.zig:273-292). This server does the same for a stream of independent
// requests against a device-resident pool of chunk voxel lists:
//
// * pyrb_server_submit queues a request (a pool chunk plus up to max_edits overlay
//   edits) from any thread;
// * a worker thread keeps up to max_inflight batches enqueued on the server's stream:
//   whenever one completes, every request that arrived meanwhile (up to the batch
//   caps) forms the next batch -- one pyrb_build_batch_async launch sequence --
//   so requests that arrive while others build join the next batch;
// * all scratch and all results are sub-allocated from one device arena of
//   budget_bytes (first fit with coalescing, the idea of src/range_alloc.zig:25-58).
//   A batch is admitted when its exact need (the build's own bounds,
//   pyrb_build_memory) fits into the largest free range, after evicting the least
//   recently completed results (released ones first);
// * pyrb_server_poll hands out finished results (device buffers of the batch and the
//   chunk's root, first voxel and prim); latency = submit -> the worker saw the batch
//   complete (host clock).
//
// Everything runs on the server's one stream, so a range freed after a launch (the
// build releases its scratch right after enqueueing) can be handed to the next
// launch at once: stream order keeps the GPU from reusing it early.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "pyrit_b200.h"

namespace pyrb {
pyrb_result set_error(pyrb_result r, const char* msg);  // pyrb_build.cu
}

namespace {

using Clock = std::chrono::steady_clock;

// Errors go to the calling thread's message (pyrb_error_message).
pyrb_result srv_fail(pyrb_result r, const char* fmt, ...) {
    char msg[256];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(msg, sizeof(msg), fmt, ap);
    va_end(ap);
    return pyrb::set_error(r, msg);
}

// First-fit range allocator with coalescing over one device buffer.
class Arena {
public:
    static constexpr uint64_t kAlign = 256;
    bool init(uint64_t bytes) {
        size_ = bytes / kAlign * kAlign;
        if (cudaMalloc(reinterpret_cast<void**>(&base_), size_) != cudaSuccess) {
            cudaGetLastError();
            base_ = 0;
            return false;
        }
        free_[0] = size_;
        return true;
    }
    ~Arena() {
        if (base_) cudaFree(reinterpret_cast<void*>(base_));
    }
    uint64_t alloc(uint64_t bytes) {
        const uint64_t n = (std::max<uint64_t>(bytes, 1) + kAlign - 1) / kAlign * kAlign;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            const uint64_t off = it->first, len = it->second;
            free_.erase(it);
            if (len > n) free_[off + n] = len - n;
            live_[base_ + off] = n;
            used_ += n;
            peak_ = std::max(peak_, used_);
            return base_ + off;
        }
        return 0;
    }
    void release(uint64_t addr) {
        auto it = live_.find(addr);
        if (it == live_.end()) return;
        uint64_t off = addr - base_, n = it->second;
        live_.erase(it);
        used_ -= n;
        auto nx = free_.lower_bound(off);
        if (nx != free_.begin()) {
            auto pv = std::prev(nx);
            if (pv->first + pv->second == off) {
                off = pv->first;
                n += pv->second;
                free_.erase(pv);
            }
        }
        nx = free_.lower_bound(off);
        if (nx != free_.end() && off + n == nx->first) {
            n += nx->second;
            free_.erase(nx);
        }
        free_[off] = n;
    }
    uint64_t largest_free() const {
        uint64_t m = 0;
        for (const auto& f : free_) m = std::max(m, f.second);
        return m;
    }
    uint64_t used() const { return used_; }
    uint64_t peak() const { return peak_; }

private:
    uint64_t base_ = 0, size_ = 0, used_ = 0, peak_ = 0;
    std::map<uint64_t, uint64_t> free_;            // offset -> length
    std::unordered_map<uint64_t, uint64_t> live_;  // address -> length
};

struct Request {
    uint64_t id;
    uint32_t chunk;
    std::vector<uint32_t> edits;  // 4 words per edit
    Clock::time_point submitted;
};

// Pinned staging and device copies of one batch's per-chunk arrays.
struct Slot {
    uint32_t *h_log2 = nullptr, *h_voff = nullptr, *h_eoff = nullptr, *h_edits = nullptr;
    uint64_t* h_starts = nullptr;
    uint32_t *h_roots = nullptr, *h_first = nullptr, *h_fprim = nullptr, *h_counts = nullptr;
    uint32_t *d_log2 = nullptr, *d_voff = nullptr, *d_eoff = nullptr, *d_edits = nullptr;
    uint64_t* d_starts = nullptr;
    std::vector<uint32_t> log2;  // host copy the build reads while it plans
    bool alloc(uint32_t K, uint32_t E) {
        const uint32_t e4 = std::max(E, 1u) * 4;
        bool ok = cudaHostAlloc(&h_log2, K * 4, 0) == cudaSuccess && cudaHostAlloc(&h_voff, (K + 1) * 4, 0) == cudaSuccess &&
                  cudaHostAlloc(&h_eoff, (K + 1) * 4, 0) == cudaSuccess && cudaHostAlloc(&h_edits, e4 * 4, 0) == cudaSuccess &&
                  cudaHostAlloc(&h_starts, K * 8, 0) == cudaSuccess && cudaHostAlloc(&h_roots, K * 4, 0) == cudaSuccess &&
                  cudaHostAlloc(&h_first, K * 4, 0) == cudaSuccess && cudaHostAlloc(&h_fprim, K * 4, 0) == cudaSuccess &&
                  cudaHostAlloc(&h_counts, PYRB_COUNTS_WORDS * 4, 0) == cudaSuccess;
        ok = ok && cudaMalloc(&d_log2, K * 4) == cudaSuccess && cudaMalloc(&d_voff, (K + 1) * 4) == cudaSuccess &&
             cudaMalloc(&d_eoff, (K + 1) * 4) == cudaSuccess && cudaMalloc(&d_edits, e4 * 4) == cudaSuccess &&
             cudaMalloc(&d_starts, K * 8) == cudaSuccess;
        log2.resize(K);
        if (!ok) cudaGetLastError();
        return ok;
    }
    void release() {
        for (void* p : {(void*)h_log2, (void*)h_voff, (void*)h_eoff, (void*)h_edits, (void*)h_starts, (void*)h_roots,
                        (void*)h_first, (void*)h_fprim, (void*)h_counts})
            if (p) cudaFreeHost(p);
        for (void* p : {(void*)d_log2, (void*)d_voff, (void*)d_eoff, (void*)d_edits, (void*)d_starts})
            if (p) cudaFree(p);
    }
};

struct Batch {
    uint64_t seq = 0;
    std::vector<Request> reqs;
    Slot* slot = nullptr;
    pyrb_built built = {};
    cudaEvent_t done = nullptr;
    uint32_t unreleased = 0;
};

}  // namespace

struct pyrb_server {
    pyrb_server_config cfg = {};
    std::vector<uint32_t> pool_log2, pool_sizes;
    std::vector<uint64_t> pool_starts;
    cudaStream_t stream = nullptr;
    int device = 0;
    Arena arena;
    std::vector<Slot> slots;
    std::vector<Slot*> free_slots;
    std::deque<Request> pending;
    std::deque<Batch*> inflight;
    std::list<Batch*> resident;                        // completed batches, least recently completed first
    std::unordered_map<uint64_t, Batch*> owner;        // request id -> its completed batch
    std::vector<pyrb_server_result> completed;         // waiting for pyrb_server_poll
    pyrb_server_stats stats = {};
    uint64_t seq = 0;
    std::mutex mu;
    std::condition_variable cv;
    std::thread worker;
    bool stop = false;
    pyrb_exec exec = {};

    static uint64_t arena_alloc(void* ctx, uint64_t bytes) { return static_cast<pyrb_server*>(ctx)->arena.alloc(bytes); }
    static void arena_free(void* ctx, uint64_t p) { static_cast<pyrb_server*>(ctx)->arena.release(p); }

    void free_batch(Batch* b) {
        pyrb_built_free(&exec, &b->built);
        if (b->done) cudaEventDestroy(b->done);
        delete b;
    }

    // Evicts the least recently completed batch, preferring batches whose results were
    // all released. Returns false when nothing is resident.
    bool evict_one() {
        if (resident.empty()) return false;
        auto it = std::find_if(resident.begin(), resident.end(), [](Batch* b) { return b->unreleased == 0; });
        if (it == resident.end()) it = resident.begin();
        Batch* b = *it;
        resident.erase(it);
        for (const Request& r : b->reqs) owner.erase(r.id);
        free_batch(b);
        ++stats.evictions;
        return true;
    }

    void retire(Batch* b) {
        pyrb_result rc = pyrb_build_finish(b->slot->h_counts, &b->built);
        const auto now = Clock::now();
        const uint32_t K = uint32_t(b->reqs.size());
        std::vector<uint32_t> roots(b->slot->h_roots, b->slot->h_roots + K), first(b->slot->h_first, b->slot->h_first + K),
            fprim(b->slot->h_fprim, b->slot->h_fprim + K);
        // voxels of chunk k: up to the next non-empty chunk's first voxel
        std::vector<uint32_t> vox(K, 0);
        uint32_t next = b->built.voxel_count;
        for (int k = int(K) - 1; k >= 0; --k) {
            if (first[k] != 0xFFFFFFFFu) {
                vox[k] = next - first[k];
                next = first[k];
            }
        }
        for (uint32_t k = 0; k < K; ++k) {
            pyrb_server_result r = {};
            r.id = b->reqs[k].id;
            r.status = rc;
            r.root = roots[k];
            r.first_voxel = first[k];
            r.first_prim = fprim[k];
            r.voxel_count = rc == PYRB_OK ? vox[k] : 0;
            r.batch = b->built;
            r.latency_ms = std::chrono::duration<double, std::milli>(now - b->reqs[k].submitted).count();
            completed.push_back(r);
        }
        stats.voxels += rc == PYRB_OK ? b->built.voxel_count : 0;
        free_slots.push_back(b->slot);
        b->slot = nullptr;
        if (rc == PYRB_OK) {
            b->unreleased = K;
            for (const Request& r : b->reqs) owner[r.id] = b;
            resident.push_back(b);
        } else {
            ++stats.failed_batches;
            free_batch(b);
        }
    }

    // Forms and launches the next batch from the pending requests; returns false when
    // nothing could be launched.
    bool launch_next() {
        if (pending.empty() || free_slots.empty()) return false;
        Slot* s = free_slots.back();
        uint32_t K = 0;
        uint64_t entries = 0;
        uint32_t ne = 0;
        while (K < pending.size() && K < cfg.max_batch_requests) {
            const Request& r = pending[K];
            const uint64_t add = uint64_t(pool_sizes[r.chunk]) + r.edits.size() / 4;
            if (K > 0 && entries + add > cfg.max_batch_entries) break;
            entries += add;
            ne += uint32_t(r.edits.size() / 4);
            ++K;
        }
        // staging: per chunk edge, voxel offsets and starts, edit offsets and edits
        s->h_voff[0] = 0;
        s->h_eoff[0] = 0;
        for (uint32_t k = 0; k < K; ++k) {
            const Request& r = pending[k];
            s->log2[k] = s->h_log2[k] = pool_log2[r.chunk];
            s->h_starts[k] = pool_starts[r.chunk];
            s->h_voff[k + 1] = s->h_voff[k] + pool_sizes[r.chunk];
            const uint32_t m = uint32_t(r.edits.size() / 4);
            if (m) std::memcpy(s->h_edits + uint64_t(s->h_eoff[k]) * 4, r.edits.data(), uint64_t(m) * 16);
            s->h_eoff[k + 1] = s->h_eoff[k] + m;
        }
        // admission: the build's exact need must fit the largest free range
        uint64_t scratch = 0, outs = 0;
        if (pyrb_build_memory(0, cfg.rt_log2, K, s->log2.data(), entries, &scratch, &outs) != PYRB_OK) return false;
        const uint64_t need = scratch + outs + 8 * Arena::kAlign;
        while (arena.largest_free() < need && evict_one()) {
        }
        if (arena.largest_free() < need) {
            if (!inflight.empty()) return false;  // wait for a batch to complete
            // nothing in flight, nothing resident: these requests can never fit
            const auto now = Clock::now();
            for (uint32_t k = 0; k < K; ++k) {
                pyrb_server_result r = {};
                r.id = pending.front().id;
                r.status = PYRB_ERROR_OUT_OF_MEMORY;
                r.root = r.first_voxel = r.first_prim = 0xFFFFFFFFu;
                r.latency_ms = std::chrono::duration<double, std::milli>(now - pending.front().submitted).count();
                completed.push_back(r);
                pending.pop_front();
            }
            ++stats.failed_batches;
            return true;
        }
        cudaMemcpyAsync(s->d_log2, s->h_log2, uint64_t(K) * 4, cudaMemcpyHostToDevice, stream);
        cudaMemcpyAsync(s->d_voff, s->h_voff, uint64_t(K + 1) * 4, cudaMemcpyHostToDevice, stream);
        cudaMemcpyAsync(s->d_starts, s->h_starts, uint64_t(K) * 8, cudaMemcpyHostToDevice, stream);
        cudaMemcpyAsync(s->d_eoff, s->h_eoff, uint64_t(K + 1) * 4, cudaMemcpyHostToDevice, stream);
        if (ne) cudaMemcpyAsync(s->d_edits, s->h_edits, uint64_t(ne) * 16, cudaMemcpyHostToDevice, stream);
        pyrb_batch bd = {};
        bd.count = K;
        bd.log2_host = s->log2.data();
        bd.log2 = reinterpret_cast<uint64_t>(s->d_log2);
        bd.voxels = cfg.pool_voxels;
        bd.voxel_offsets = reinterpret_cast<uint64_t>(s->d_voff);
        bd.edits = ne ? reinterpret_cast<uint64_t>(s->d_edits) : 0;
        bd.edit_offsets = ne ? reinterpret_cast<uint64_t>(s->d_eoff) : 0;
        bd.voxel_total = s->h_voff[K];
        bd.edit_total = ne;
        bd.voxel_starts = reinterpret_cast<uint64_t>(s->d_starts);
        Batch* b = new Batch();
        b->seq = seq++;
        const pyrb_result rc = pyrb_build_batch_async(&exec, &bd, cfg.rt_log2, s->h_roots, s->h_first, s->h_fprim,
                                                      s->h_counts, &b->built);
        if (rc != PYRB_OK) {
            delete b;
            if (rc == PYRB_ERROR_OUT_OF_MEMORY && !inflight.empty()) return false;
            const auto now = Clock::now();
            for (uint32_t k = 0; k < K; ++k) {
                pyrb_server_result r = {};
                r.id = pending.front().id;
                r.status = rc;
                r.root = r.first_voxel = r.first_prim = 0xFFFFFFFFu;
                r.latency_ms = std::chrono::duration<double, std::milli>(now - pending.front().submitted).count();
                completed.push_back(r);
                pending.pop_front();
            }
            ++stats.failed_batches;
            return true;
        }
        cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
        cudaEventRecord(b->done, stream);
        free_slots.pop_back();
        b->slot = s;
        b->reqs.assign(std::make_move_iterator(pending.begin()), std::make_move_iterator(pending.begin() + K));
        pending.erase(pending.begin(), pending.begin() + K);
        inflight.push_back(b);
        ++stats.batches;
        stats.max_batch_requests = std::max(stats.max_batch_requests, K);
        stats.peak_bytes = std::max(stats.peak_bytes, arena.peak());
        return true;
    }

    void run() {
        cudaSetDevice(device);
        std::unique_lock<std::mutex> lk(mu);
        while (!stop) {
            bool progress = false;
            while (!inflight.empty() && cudaEventQuery(inflight.front()->done) == cudaSuccess) {
                Batch* b = inflight.front();
                inflight.pop_front();
                retire(b);
                progress = true;
            }
            while (inflight.size() < cfg.max_inflight && launch_next()) progress = true;
            if (progress) continue;
            if (inflight.empty() && pending.empty()) {
                cv.wait(lk, [&] { return stop || !pending.empty(); });
            } else {
                // batches on the GPU: poll their completion often (the latency includes it)
                lk.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(5));
                lk.lock();
            }
        }
    }
};

extern "C" {

PYRB_API pyrb_result pyrb_server_create(const pyrb_server_config* cfg, pyrb_server** out) {
    if (!cfg || !out) return srv_fail(PYRB_ERROR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (!cfg->pool_count || !cfg->pool_log2 || !cfg->pool_starts || !cfg->pool_sizes || !cfg->pool_voxels)
        return srv_fail(PYRB_ERROR_INVALID_ARGUMENT, "the server needs a chunk pool");
    if (!cfg->budget_bytes || !cfg->max_inflight || !cfg->max_batch_requests || !cfg->max_batch_entries)
        return srv_fail(PYRB_ERROR_INVALID_ARGUMENT, "budget, max_inflight and the batch caps must be non-zero");
    for (uint32_t c = 0; c < cfg->pool_count; ++c)
        if (cfg->pool_log2[c] < 3 || cfg->pool_log2[c] > 10)
            return srv_fail(PYRB_ERROR_INVALID_ARGUMENT, "pool chunk %u: log2 %u outside [3, 10]", c, cfg->pool_log2[c]);
    auto* s = new pyrb_server();
    s->cfg = *cfg;
    s->pool_log2.assign(cfg->pool_log2, cfg->pool_log2 + cfg->pool_count);
    s->pool_starts.assign(cfg->pool_starts, cfg->pool_starts + cfg->pool_count);
    s->pool_sizes.assign(cfg->pool_sizes, cfg->pool_sizes + cfg->pool_count);
    s->cfg.pool_log2 = s->pool_log2.data();
    s->cfg.pool_starts = s->pool_starts.data();
    s->cfg.pool_sizes = s->pool_sizes.data();
    cudaGetDevice(&s->device);
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete s;
        return srv_fail(PYRB_ERROR_CUDA, "stream creation failed");
    }
    if (!s->arena.init(cfg->budget_bytes)) {
        cudaStreamDestroy(s->stream);
        delete s;
        return srv_fail(PYRB_ERROR_OUT_OF_MEMORY, "device arena of %llu bytes", (unsigned long long)cfg->budget_bytes);
    }
    s->slots.resize(cfg->max_inflight);
    for (Slot& sl : s->slots) {
        if (!sl.alloc(cfg->max_batch_requests, cfg->max_batch_requests * std::max(cfg->max_edits, 1u))) {
            for (Slot& x : s->slots) x.release();
            cudaStreamDestroy(s->stream);
            delete s;
            return srv_fail(PYRB_ERROR_OUT_OF_MEMORY, "staging buffers");
        }
        s->free_slots.push_back(&sl);
    }
    s->exec.ctx = s;
    s->exec.stream = s->stream;
    s->exec.alloc = &pyrb_server::arena_alloc;
    s->exec.free = &pyrb_server::arena_free;
    s->worker = std::thread([s] { s->run(); });
    *out = s;
    return PYRB_OK;
}

PYRB_API pyrb_result pyrb_server_submit(pyrb_server* s, uint64_t id, uint32_t chunk, const uint32_t* edits,
                                        uint32_t n_edits) {
    if (!s) return srv_fail(PYRB_ERROR_INVALID_ARGUMENT, "server is NULL");
    if (chunk >= s->cfg.pool_count) return srv_fail(PYRB_ERROR_INVALID_ARGUMENT, "chunk %u outside the pool", chunk);
    if (n_edits > s->cfg.max_edits) return srv_fail(PYRB_ERROR_INVALID_ARGUMENT, "%u edits (at most %u)", n_edits, s->cfg.max_edits);
    if (n_edits && !edits) return srv_fail(PYRB_ERROR_INVALID_ARGUMENT, "edits is NULL");
    Request r;
    r.id = id;
    r.chunk = chunk;
    r.edits.assign(edits, edits + uint64_t(n_edits) * 4);
    r.submitted = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->pending.push_back(std::move(r));
        ++s->stats.requests;
    }
    s->cv.notify_one();
    return PYRB_OK;
}

PYRB_API uint32_t pyrb_server_poll(pyrb_server* s, pyrb_server_result* out, uint32_t cap) {
    if (!s || !out) return 0;
    std::lock_guard<std::mutex> lk(s->mu);
    const uint32_t n = uint32_t(std::min<size_t>(cap, s->completed.size()));
    std::copy(s->completed.begin(), s->completed.begin() + n, out);
    s->completed.erase(s->completed.begin(), s->completed.begin() + n);
    return n;
}

PYRB_API pyrb_result pyrb_server_release(pyrb_server* s, uint64_t id) {
    if (!s) return srv_fail(PYRB_ERROR_INVALID_ARGUMENT, "server is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->owner.find(id);
    if (it == s->owner.end()) return PYRB_OK;  // released before, or evicted
    Batch* b = it->second;
    s->owner.erase(it);
    if (b->unreleased) --b->unreleased;
    if (b->unreleased == 0) {
        s->resident.remove(b);
        s->free_batch(b);
    }
    return PYRB_OK;
}

PYRB_API void pyrb_server_get_stats(pyrb_server* s, pyrb_server_stats* out) {
    if (!s || !out) return;
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    out->pending = uint32_t(s->pending.size());
    out->inflight = uint32_t(s->inflight.size());
    out->arena_used = s->arena.used();
}

PYRB_API pyrb_result pyrb_server_drain(pyrb_server* s, uint32_t timeout_ms) {
    if (!s) return srv_fail(PYRB_ERROR_INVALID_ARGUMENT, "server is NULL");
    const auto until = Clock::now() + std::chrono::milliseconds(timeout_ms);
    while (Clock::now() < until) {
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->pending.empty() && s->inflight.empty()) return PYRB_OK;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    return srv_fail(PYRB_ERROR_CUDA, "requests still pending after %u ms", timeout_ms);
}

PYRB_API void pyrb_server_destroy(pyrb_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaStreamSynchronize(s->stream);
    for (Batch* b : s->inflight) s->free_batch(b);
    for (Batch* b : s->resident) s->free_batch(b);
    for (Slot& sl : s->slots) sl.release();
    cudaStreamDestroy(s->stream);
    delete s;
}

}  // extern "C"
