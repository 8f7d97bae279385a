// cs_server.cu — the serving loop: compaction requests over device-resident columns,
// admitted by an output-memory budget and batched as they arrive.
//
// Threads. Clients submit from any thread (a short critical section). One scheduler
// thread per server admits queued requests into the output arena in arrival order, and,
// whenever a batch slot is free and admitted requests wait, packs them into one
// multi-column plan (cs_plan.h) and enqueues it on that slot's stream: upload of the
// plan's packed maps (one host-to-device copy from the slot's page-locked image), the
// plan's kernels, ONE device-to-host copy of the slot's header and per-request counts
// (contiguous in the slot buffer), and an event. While any batch is in flight the
// scheduler polls the slots' events between admission rounds (it spins on one host core
// for as long as the GPU holds work, and sleeps on a condition variable when it does not):
// a host callback (cudaLaunchHostFunc) costs well over 100 us per batch on this path,
// polling a few microseconds. With several slots, a batch formed from requests that
// arrived while earlier batches run is launched on another stream and its kernels share
// the GPU with them.
//
// Memory. Output space comes from one arena allocated at creation. A request reserves
// n * elem_bytes bytes (all selected, the most it can need) when admitted; the reservation
// shrinks to count * elem_bytes at completion and returns to the arena on release. The
// head of the queue blocks admission of later requests (arrival order is kept). Each
// slot owns a plan buffer sized for max_batch columns holding max_batch_elems elements:
// header | statuses | flags || maps | offsets | counts. Statuses are epoch tagged, so a
// slot's next batch needs no clearing; the maps region is rewritten per batch.
//
// Errors. A bounded device wait that ran out sets the slot header's sticky error word;
// every request of that batch then completes with CS_ERR_TIMEOUT and the word is cleared
// in stream order before the slot's next batch.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "compressstore.h"
#include "cs_internal.cuh"
#include "cs_plan.h"

using namespace cs;

namespace {

inline uint64_t now_ns()
{
    return static_cast<uint64_t>(
        std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
            .count());
}

inline size_t a256(size_t x)
{
    return (x + 255) & ~static_cast<size_t>(255);
}

inline bool aligned_to(const void* p, uintptr_t a)
{
    return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0;
}

// First-fit allocator over [0, size) with coalescing free list (offsets and sizes are
// multiples of 256).
class Arena {
  public:
    void reset(size_t size)
    {
        free_.clear();
        if (size) free_[0] = size;
        size_ = size;
        used_ = peak_ = 0;
    }
    bool alloc(size_t bytes, size_t* off)
    {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const size_t rest = it->second - bytes;
            const size_t roff = it->first + bytes;
            free_.erase(it);
            if (rest) free_[roff] = rest;
            used_ += bytes;
            peak_ = std::max(peak_, used_);
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes)
    {
        if (!bytes) return;
        used_ -= bytes;
        auto next = free_.lower_bound(off);
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                off = prev->first;
                bytes += prev->second;
                free_.erase(prev);
            }
        }
        if (next != free_.end() && off + bytes == next->first) {
            bytes += next->second;
            free_.erase(next);
        }
        free_[off] = bytes;
    }
    size_t size() const { return size_; }
    size_t used() const { return used_; }
    size_t peak() const { return peak_; }

  private:
    std::map<size_t, size_t> free_;
    size_t size_ = 0, used_ = 0, peak_ = 0;
};

enum ReqState : int { RS_QUEUED = 0, RS_ADMITTED = 1, RS_RUNNING = 2, RS_DONE = 3 };

struct Req {
    cs_request r{};
    size_t off = 0, bytes = 0; // arena reservation
    uint64_t t_submit = 0, t_launch = 0, t_done = 0;
    uint64_t count = 0;
    int32_t status = CS_PENDING;
    uint32_t batch_size = 0;
    int state = RS_QUEUED;
};

// Page-locked host side of a slot: the slot header, then (batch mode) the counts, copied
// back together.
struct SlotHost {
    ws_header hdr;
    uint64_t counts[1]; // max_batch entries follow
};

} // namespace

struct cs_server;

namespace {
struct Slot {
    cs_server* srv = nullptr;
    cudaStream_t stream = nullptr;
    uint8_t* dbuf = nullptr;    // plan buffer (batch mode) or workspace + count word (per-call)
    uint8_t* himg = nullptr;    // page-locked maps image (batch mode)
    SlotHost* hres = nullptr;   // page-locked results
    cudaEvent_t done = nullptr; // recorded after the results copy
    std::vector<uint64_t> tickets;
    bool busy = false;          // holds a batch (from formation to completion)
    bool launched = false;      // its work and event are enqueued
    bool clear_err = false;
};
} // namespace

struct cs_server {
    int device = 0;
    int sms = 0;
    cs_server_config cfg{};
    uint8_t* arena_base = nullptr;
    Arena arena;
    PlanCounts caps;
    PlanLayout layout;
    size_t ws_bytes = 0; // per-call workspace bytes (count word follows)
    int bps[4] = {1, 1, 1, 1};
    std::vector<Slot> slots;

    std::mutex mu;
    std::condition_variable cv_sched, cv_done;
    std::unordered_map<uint64_t, Req> reqs;
    std::deque<uint64_t> queued, admitted, done;
    uint64_t next_ticket = 1;
    bool stopping = false;
    std::thread sched;

    uint64_t submitted = 0, completed = 0, rejected = 0, batches = 0, batched = 0, launches = 0;
};

namespace {

int to_status(cudaError_t e)
{
    if (e == cudaSuccess) return CS_SUCCESS;
    if (e == cudaErrorMemoryAllocation) return CS_ERR_OUT_OF_MEMORY;
    return CS_ERR_CUDA;
}

size_t reservation(uint64_t n, uint32_t w)
{
    return a256(std::max<uint64_t>(n * w, 16));
}

// Complete a request (lock held).
void finish_locked(cs_server* s, uint64_t ticket, Req& r, int32_t status, uint64_t count, uint64_t t)
{
    r.status = status;
    r.count = status == CS_SUCCESS ? count : 0;
    r.t_done = t;
    r.state = RS_DONE;
    const size_t keep = status == CS_SUCCESS && r.count ? reservation(r.count, r.r.elem_bytes) : 0;
    if (r.bytes > keep) {
        s->arena.release(r.off + keep, r.bytes - keep);
        r.bytes = keep;
    }
    s->done.push_back(ticket);
    ++s->completed;
}

// Complete the requests of a slot whose event fired (lock held).
void complete_slot_locked(cs_server* s, Slot& sl, cudaError_t e)
{
    const uint64_t t = now_ns();
    const uint32_t err = e == cudaSuccess ? sl.hres->hdr.err : 0u;
    for (size_t i = 0; i < sl.tickets.size(); ++i) {
        auto it = s->reqs.find(sl.tickets[i]);
        if (it == s->reqs.end()) continue;
        Req& r = it->second;
        const uint64_t c = s->cfg.mode == CS_SERVE_BATCH ? sl.hres->counts[i] : sl.hres->hdr.count_word;
        int32_t st = CS_SUCCESS;
        if (e != cudaSuccess) st = CS_ERR_CUDA;
        else if (err) st = err == DEVERR_RANGE ? CS_ERR_INVALID_VALUE : CS_ERR_TIMEOUT;
        else if (c == CS_COUNT_ERROR) st = CS_ERR_TIMEOUT;
        else if (c > r.r.n) st = CS_ERR_CUDA; // cannot happen for a clean run
        finish_locked(s, sl.tickets[i], r, st, c, t);
    }
    if (err) sl.clear_err = true;
    sl.tickets.clear();
    sl.busy = false;
    sl.launched = false;
}

// Poll the events of launched slots; complete those that finished (lock held). Returns
// whether any slot still holds GPU work.
bool reap_locked(cs_server* s)
{
    bool pending = false, completed = false;
    for (Slot& sl : s->slots) {
        if (!sl.busy || !sl.launched) {
            pending |= sl.busy;
            continue;
        }
        const cudaError_t e = cudaEventQuery(sl.done);
        if (e == cudaErrorNotReady) {
            pending = true;
            continue;
        }
        if (e != cudaSuccess) cudaGetLastError();
        complete_slot_locked(s, sl, e);
        completed = true;
    }
    if (completed) s->cv_done.notify_all();
    return pending;
}

inline void spin_pause(uint64_t ns)
{
    const uint64_t until = now_ns() + ns;
    while (now_ns() < until) {
#if defined(__x86_64__) || defined(__i386__)
        __builtin_ia32_pause();
#endif
    }
}

void admit_locked(cs_server* s)
{
    while (!s->queued.empty()) {
        const uint64_t t = s->queued.front();
        auto it = s->reqs.find(t);
        if (it == s->reqs.end()) {
            s->queued.pop_front();
            continue;
        }
        Req& r = it->second;
        size_t off = 0;
        if (!s->arena.alloc(r.bytes, &off)) break; // arrival order: the head waits for space
        r.off = off;
        r.state = RS_ADMITTED;
        s->queued.pop_front();
        s->admitted.push_back(t);
    }
}

// Enqueue one batch on a slot (no lock held; the requests are RUNNING and stay put).
int launch_slot(cs_server* s, Slot& sl, const std::vector<Req*>& rs)
{
    cudaStream_t st = sl.stream;
    cudaError_t e = cudaSuccess;
    ws_header* hdr = reinterpret_cast<ws_header*>(sl.dbuf);
    if (sl.clear_err) {
        e = cudaMemsetAsync(&hdr->err, 0, sizeof(uint32_t), st);
        if (e != cudaSuccess) return to_status(e);
        sl.clear_err = false;
    }
    uint64_t* d_counts = nullptr;
    uint32_t kernels = 0;
    size_t result_bytes = sizeof(ws_header);
    if (s->cfg.mode == CS_SERVE_BATCH) {
        std::vector<cs_column> cols(rs.size());
        PlanDevice d0 = plan_device(sl.dbuf, s->layout, PlanMaps{});
        d_counts = d0.counts;
        for (size_t i = 0; i < rs.size(); ++i) {
            const Req& r = *rs[i];
            cols[i].d_in = r.r.d_in;
            cols[i].d_mask = r.r.d_mask;
            cols[i].d_out = s->arena_base + r.off;
            cols[i].n = r.r.n;
            cols[i].elem_bytes = r.r.elem_bytes;
            cols[i].reserved = 0;
            cols[i].d_count = d_counts + i;
        }
        std::vector<ColumnDesc> desc;
        std::vector<uint64_t> chunk_base;
        PlanCounts c;
        int rc = plan_columns(cols.data(), static_cast<uint32_t>(cols.size()), desc, chunk_base, c, nullptr);
        if (rc != CS_SUCCESS) return rc;
        const PlanMaps m = plan_maps(c);
        const PlanDevice d = plan_device(sl.dbuf, s->layout, m);
        plan_write_image(sl.himg, m, d, desc, chunk_base);
        e = cudaMemcpyAsync(d.maps, sl.himg, m.bytes, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return to_status(e);
        uint32_t grid[4];
        for (int wi = 0; wi < 4; ++wi) {
            const uint64_t g = static_cast<uint64_t>(s->bps[wi]) * s->sms;
            grid[wi] = static_cast<uint32_t>(std::min<uint64_t>(g, c.units[wi]));
        }
        rc = plan_launch(d, c, grid, s->sms, s->cfg.timeout_ns, st);
        if (rc != CS_SUCCESS) return rc;
        kernels = plan_kernels(c);
        result_bytes = s->layout.off_counts + 8 * rs.size(); // header and counts are contiguous
    } else {
        d_counts = &hdr->count_word; // one request per launch; its count travels with the header
        cs_config cc{};
        cc.timeout_ns = s->cfg.timeout_ns;
        for (size_t i = 0; i < rs.size(); ++i) {
            const Req& r = *rs[i];
            const uint64_t before = cs_launch_count();
            const int rc = compressstore_ex(r.r.d_in, r.r.d_mask, s->arena_base + r.off, r.r.n, r.r.elem_bytes,
                                            d_counts + i, sl.dbuf, s->ws_bytes, &cc,
                                            reinterpret_cast<cs_stream_t>(st));
            if (rc != CS_SUCCESS) return rc;
            kernels += static_cast<uint32_t>(cs_launch_count() - before);
        }
    }
    e = cudaMemcpyAsync(sl.hres, hdr, result_bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(sl.done, st);
    if (e != cudaSuccess) return to_status(e);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->launches += kernels;
    }
    return CS_SUCCESS;
}

void scheduler_main(cs_server* s)
{
    cudaSetDevice(s->device);
    const uint32_t per_batch = s->cfg.mode == CS_SERVE_BATCH ? s->cfg.max_batch : 1u;
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        if (s->stopping) break;
        const bool in_flight = reap_locked(s);
        admit_locked(s);
        Slot* free_slot = nullptr;
        for (Slot& sl : s->slots)
            if (!sl.busy) {
                free_slot = &sl;
                break;
            }
        if (!free_slot || s->admitted.empty()) {
            if (in_flight) { // GPU work outstanding: poll again shortly
                lk.unlock();
                spin_pause(1000);
                lk.lock();
            } else {
                s->cv_sched.wait(lk);
            }
            continue;
        }
        // one batch: every admitted request in order, up to the slot's capacity
        std::vector<Req*> rs;
        std::vector<uint64_t> tickets;
        uint64_t elems = 0;
        const uint64_t t = now_ns();
        while (!s->admitted.empty() && rs.size() < per_batch) {
            auto it = s->reqs.find(s->admitted.front());
            if (it == s->reqs.end()) {
                s->admitted.pop_front();
                continue;
            }
            Req& r = it->second;
            if (!rs.empty() && elems + r.r.n > s->cfg.max_batch_elems) break;
            elems += r.r.n;
            r.state = RS_RUNNING;
            r.t_launch = t;
            rs.push_back(&r);
            tickets.push_back(it->first);
            s->admitted.pop_front();
        }
        if (rs.empty()) continue;
        for (Req* r : rs) r->batch_size = static_cast<uint32_t>(rs.size());
        free_slot->busy = true;
        free_slot->tickets = tickets;
        ++s->batches;
        s->batched += rs.size();
        lk.unlock();
        const int rc = launch_slot(s, *free_slot, rs);
        if (rc != CS_SUCCESS) cudaStreamSynchronize(free_slot->stream); // let enqueued work drain
        lk.lock();
        if (rc == CS_SUCCESS) {
            free_slot->launched = true;
        } else {
            // nothing of this batch will complete on the device: fail its requests here
            const uint64_t tf = now_ns();
            for (size_t i = 0; i < tickets.size(); ++i) {
                auto it = s->reqs.find(tickets[i]);
                if (it != s->reqs.end()) finish_locked(s, tickets[i], it->second, rc, 0, tf);
            }
            free_slot->tickets.clear();
            free_slot->busy = false;
            s->cv_done.notify_all();
        }
    }
}

void fill_result(const cs_server* s, const Req& r, cs_result* res)
{
    if (!res) return;
    res->d_out = r.bytes ? s->arena_base + r.off : nullptr;
    res->count = r.count;
    res->latency_ns = r.t_done - r.t_submit;
    res->queue_ns = r.t_launch ? r.t_launch - r.t_submit : 0;
    res->status = r.status;
    res->batch_size = r.batch_size;
}

void free_server(cs_server* s)
{
    for (Slot& sl : s->slots) {
        if (sl.stream) {
            cudaStreamSynchronize(sl.stream);
            cudaStreamDestroy(sl.stream);
        }
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.dbuf) cudaFree(sl.dbuf);
        if (sl.himg) cudaFreeHost(sl.himg);
        if (sl.hres) cudaFreeHost(sl.hres);
    }
    if (s->arena_base) cudaFree(s->arena_base);
    delete s;
}

} // namespace

extern "C" {

int cs_server_create(cs_server** out, const cs_server_config* cfg)
{
    if (!out) return CS_ERR_INVALID_VALUE;
    *out = nullptr;
    auto s = new cs_server();
    if (cfg) s->cfg = *cfg;
    cs_server_config& c = s->cfg;
    if (c.mode != CS_SERVE_BATCH && c.mode != CS_SERVE_PER_CALL) {
        delete s;
        return CS_ERR_INVALID_VALUE;
    }
    if (!c.max_batch_elems) c.max_batch_elems = 1ull << 28;
    if (!c.max_batch) c.max_batch = 64;
    if (!c.slots) c.slots = 3;
    if (!c.timeout_ns) c.timeout_ns = 2000000000ull;
    if (c.max_batch > 4096 || c.slots > 16 || c.max_batch_elems > (1ull << 34)) {
        delete s;
        return CS_ERR_NOT_SUPPORTED;
    }
    int major = 0;
    if (cudaGetDevice(&s->device) != cudaSuccess ||
        cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, s->device) != cudaSuccess ||
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, s->device) != cudaSuccess || major != 10) {
        delete s;
        return CS_ERR_NO_DEVICE;
    }
    if (!c.out_budget_bytes) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            delete s;
            return CS_ERR_CUDA;
        }
        c.out_budget_bytes = std::min<uint64_t>(4ull << 30, fr / 4);
    }
    c.out_budget_bytes &= ~0xffull;
    if (c.out_budget_bytes < 256) {
        delete s;
        return CS_ERR_INVALID_VALUE;
    }
    const uint32_t per_batch = c.mode == CS_SERVE_BATCH ? c.max_batch : 1u;
    size_t slot_bytes = 0, img_bytes = 0;
    if (c.mode == CS_SERVE_BATCH) {
        s->caps = plan_capacity(c.max_batch_elems, c.max_batch);
        s->layout = plan_layout(s->caps, true);
        slot_bytes = s->layout.total;
        img_bytes = s->layout.maps_bytes;
    } else {
        cs_config cc{};
        for (uint32_t w = 1; w <= 8; w <<= 1)
            s->ws_bytes = std::max(s->ws_bytes, compressstore_workspace_size(c.max_batch_elems, w, &cc));
        s->ws_bytes = a256(s->ws_bytes);
        slot_bytes = s->ws_bytes;
    }
    for (int wi = 0; wi < 4; ++wi) s->bps[wi] = std::max(1, compact_tma_blocks_per_sm(1u << wi, 1));

    cudaError_t e = cudaMalloc(&s->arena_base, c.out_budget_bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        s->arena_base = nullptr;
        free_server(s);
        return CS_ERR_OUT_OF_MEMORY;
    }
    s->arena.reset(c.out_budget_bytes);
    s->slots.resize(c.slots);
    for (Slot& sl : s->slots) {
        sl.srv = s;
        e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMalloc(&sl.dbuf, slot_bytes);
        if (e == cudaSuccess && img_bytes) e = cudaMallocHost(&sl.himg, img_bytes);
        if (e == cudaSuccess) e = cudaMallocHost(&sl.hres, sizeof(SlotHost) + 8ull * per_batch);
        if (e == cudaSuccess) {
            if (c.mode == CS_SERVE_BATCH) {
                e = launch_ws_init(reinterpret_cast<ws_header*>(sl.dbuf), slot_bytes, sl.stream);
            } else {
                const int rc = cs_workspace_init(sl.dbuf, s->ws_bytes, reinterpret_cast<cs_stream_t>(sl.stream));
                if (rc != CS_SUCCESS) e = cudaErrorUnknown;
            }
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(sl.stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            free_server(s);
            return e == cudaErrorMemoryAllocation ? CS_ERR_OUT_OF_MEMORY : CS_ERR_CUDA;
        }
    }
    s->sched = std::thread(scheduler_main, s);
    *out = s;
    return CS_SUCCESS;
}

int cs_server_submit(cs_server* s, const cs_request* req, uint64_t* ticket)
{
    if (!s || !req || !ticket) return CS_ERR_INVALID_VALUE;
    const cs_request& r = *req;
    const uint32_t w = r.elem_bytes;
    int rc = CS_SUCCESS;
    if (w != 1 && w != 2 && w != 4 && w != 8) rc = CS_ERR_INVALID_VALUE;
    else if (r.n > s->cfg.max_batch_elems) rc = CS_ERR_NOT_SUPPORTED;
    else if (r.n && (!r.d_in || !r.d_mask)) rc = CS_ERR_INVALID_VALUE;
    else if (r.n && (!aligned_to(r.d_in, 16) || !aligned_to(r.d_mask, 16))) rc = CS_ERR_MISALIGNED;
    else if (reservation(r.n, w) > s->arena.size()) rc = CS_ERR_ADMISSION;
    const uint64_t t = now_ns();
    std::unique_lock<std::mutex> lk(s->mu);
    if (rc != CS_SUCCESS) {
        ++s->rejected;
        return rc;
    }
    if (s->stopping) return CS_ERR_INVALID_VALUE;
    const uint64_t id = s->next_ticket++;
    Req& q = s->reqs[id];
    q.r = r;
    q.t_submit = t;
    ++s->submitted;
    *ticket = id;
    if (r.n == 0) {
        q.bytes = 0;
        q.t_launch = t;
        finish_locked(s, id, q, CS_SUCCESS, 0, t);
        lk.unlock();
        s->cv_done.notify_all();
        return CS_SUCCESS;
    }
    q.bytes = reservation(r.n, w);
    s->queued.push_back(id);
    lk.unlock();
    s->cv_sched.notify_one();
    return CS_SUCCESS;
}

int cs_server_poll(cs_server* s, uint64_t ticket, cs_result* res)
{
    if (!s) return CS_ERR_INVALID_VALUE;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return CS_ERR_INVALID_VALUE;
    if (it->second.state != RS_DONE) return CS_PENDING;
    fill_result(s, it->second, res);
    return CS_SUCCESS;
}

int cs_server_wait(cs_server* s, uint64_t ticket, uint64_t timeout_ns, cs_result* res)
{
    if (!s) return CS_ERR_INVALID_VALUE;
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::nanoseconds(timeout_ns);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end()) return CS_ERR_INVALID_VALUE;
        if (it->second.state == RS_DONE) {
            fill_result(s, it->second, res);
            return CS_SUCCESS;
        }
        if (timeout_ns == 0) s->cv_done.wait(lk);
        else if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout) {
            auto jt = s->reqs.find(ticket);
            if (jt != s->reqs.end() && jt->second.state == RS_DONE) {
                fill_result(s, jt->second, res);
                return CS_SUCCESS;
            }
            return CS_PENDING;
        }
    }
}

int cs_server_next(cs_server* s, uint64_t timeout_ns, uint64_t* ticket, cs_result* res)
{
    if (!s || !ticket) return CS_ERR_INVALID_VALUE;
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::nanoseconds(timeout_ns);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        while (!s->done.empty()) {
            const uint64_t t = s->done.front();
            s->done.pop_front();
            auto it = s->reqs.find(t);
            if (it == s->reqs.end()) continue; // released meanwhile
            *ticket = t;
            fill_result(s, it->second, res);
            return CS_SUCCESS;
        }
        if (timeout_ns == 0) s->cv_done.wait(lk);
        else if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && s->done.empty())
            return CS_PENDING;
    }
}

int cs_server_release(cs_server* s, uint64_t ticket)
{
    if (!s) return CS_ERR_INVALID_VALUE;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end() || it->second.state != RS_DONE) return CS_ERR_INVALID_VALUE;
        s->arena.release(it->second.off, it->second.bytes);
        s->reqs.erase(it);
        while (!s->done.empty() && !s->reqs.count(s->done.front())) s->done.pop_front();
    }
    s->cv_sched.notify_one(); // space for the head of the queue
    return CS_SUCCESS;
}

int cs_server_stats_get(cs_server* s, cs_server_stats* st)
{
    if (!s || !st) return CS_ERR_INVALID_VALUE;
    std::lock_guard<std::mutex> lk(s->mu);
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->rejected = s->rejected;
    st->batches = s->batches;
    st->batched_requests = s->batched;
    st->arena_bytes = s->arena.size();
    st->arena_used = s->arena.used();
    st->arena_peak = s->arena.peak();
    st->kernel_launches = s->launches;
    return CS_SUCCESS;
}

int cs_server_replay(cs_server* s, const cs_request* reqs, const uint64_t* arrival_ns, uint32_t count,
                     cs_result* results)
{
    if (!s || (count && (!reqs || !arrival_ns || !results))) return CS_ERR_INVALID_VALUE;
    std::mutex map_mu;
    std::unordered_map<uint64_t, uint32_t> index_of;
    std::atomic<int64_t> expected{-1};
    std::atomic<int> reaper_rc{CS_SUCCESS};
    std::thread reaper([&] {
        int64_t got = 0;
        uint64_t idle_since = now_ns();
        for (;;) {
            const int64_t exp = expected.load();
            if (exp >= 0 && got >= exp) break;
            uint64_t t = 0;
            cs_result r{};
            const int rc = cs_server_next(s, 20000000ull, &t, &r);
            if (rc == CS_PENDING) {
                if (now_ns() - idle_since > 120000000000ull) { // two minutes without a completion
                    reaper_rc.store(CS_ERR_TIMEOUT);
                    break;
                }
                continue;
            }
            if (rc != CS_SUCCESS) {
                reaper_rc.store(rc);
                break;
            }
            idle_since = now_ns();
            uint32_t idx = 0;
            for (;;) { // the submitter records the ticket right after submit returns
                {
                    std::lock_guard<std::mutex> lk(map_mu);
                    auto it = index_of.find(t);
                    if (it != index_of.end()) {
                        idx = it->second;
                        break;
                    }
                }
                std::this_thread::yield();
            }
            r.d_out = nullptr;
            results[idx] = r;
            cs_server_release(s, t);
            ++got;
        }
    });
    const uint64_t start = now_ns();
    int64_t ok = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const uint64_t due = start + arrival_ns[i];
        for (;;) {
            const uint64_t now = now_ns();
            if (now >= due) break;
            if (due - now > 200000) std::this_thread::sleep_for(std::chrono::nanoseconds(due - now - 100000));
            else std::this_thread::yield();
        }
        uint64_t t = 0;
        const int rc = cs_server_submit(s, &reqs[i], &t);
        if (rc != CS_SUCCESS) {
            results[i] = cs_result{};
            results[i].status = rc;
            continue;
        }
        {
            std::lock_guard<std::mutex> lk(map_mu);
            index_of[t] = i;
        }
        ++ok;
    }
    expected.store(ok);
    reaper.join();
    return reaper_rc.load();
}

int cs_server_destroy(cs_server* s)
{
    if (!s) return CS_SUCCESS;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    s->cv_sched.notify_all();
    if (s->sched.joinable()) s->sched.join();
    free_server(s); // synchronises every slot stream first
    return CS_SUCCESS;
}

} // extern "C"
