// server.cu -- serving loop with continuous batching over the host-buffer
// API.  A worker thread keeps up to `max_inflight` batches on the GPU; each
// time a slot frees, every request queued so far (up to the batch limits and
// the HBM admission of the context) is fused into ONE launch: its tiles are
// concatenated and each request gets its own RGB8 canvas of the batch output
// (hpvcd_output.canvases).  Requests that arrive while batches run wait in
// the queue and join the next batch; outputs are copied to the requests'
// buffers as their batch completes.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "hpvcd_gpu.h"
#include "hostcopy.h"

#define HPVCD_API extern "C" __attribute__((visibility("default")))

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// Page-locked host arena, recycled between batches (cudaMallocHost is slow).
struct Arena {
    unsigned char* p = nullptr;
    size_t cap = 0;
};

struct ReqMeta {
    uint32_t first_pic, n_pics;
    hpvcd_canvas canvas;
    void* dst;
    uint64_t dst_bytes;
    uint64_t user;
    Clock::time_point t_submit;
    uint64_t out_off;
};

// Requests accumulate in an open batch: their buffers are packed straight
// into the batch's page-locked input arena (laid out as the device input
// arena of the fused launch, so the whole batch goes up in one DMA).
struct Batch {
    Arena in, out;
    size_t in_used = 0, out_used = 0;
    std::vector<hpvcd_picture> pics;        // pointers are arena offsets until launch
    std::vector<hpvcd_tile_place> place;
    std::vector<hpvcd_canvas> canvases;
    std::vector<hpvcd_wp_table> wp;         // weighted-prediction tables by picture
    std::vector<ReqMeta> reqs;
    Clock::time_point t_first, t_launch;
    hpvcd_ticket ticket = 0;
    uint32_t packers = 0;  // submits still copying into `in`
    bool zero_copy = false;  // inputs and outputs live in the callers' page-locked memory
};

}  // namespace

struct hpvcd_server {
    hpvcd_server_cfg cfg{};
    hpvcd_gpu* gpu = nullptr;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::unique_ptr<Batch>> open;    // filling / waiting for a slot
    std::vector<std::unique_ptr<Batch>> running;
    std::vector<Arena> free_arenas;
    std::deque<hpvcd_completion> done;
    uint32_t pending = 0;
    uint32_t slots = 2;
    bool stop = false;
    std::thread worker;

    uint32_t max_pics() const { return cfg.max_batch_pictures ? cfg.max_batch_pictures : 4096; }
    // 128 MiB of inputs per batch by default: several batches in flight
    // overlap one batch's host <-> device copies with another's decode
    uint64_t max_bytes() const { return cfg.max_batch_bytes ? cfg.max_batch_bytes : (128ull << 20); }

    // Give `a` at least `need` bytes: the smallest recycled arena that fits,
    // else a new page-locked allocation.  Only called on empty arenas (open
    // batches never grow; a request that does not fit starts a new batch).
    bool grow(Arena& a, size_t need) {
        if (a.cap >= need) return true;
        if (a.p) {
            free_arenas.push_back(a);
            a = Arena{};
        }
        size_t best = SIZE_MAX;
        for (size_t i = 0; i < free_arenas.size(); ++i)
            if (free_arenas[i].cap >= need && (best == SIZE_MAX || free_arenas[i].cap < free_arenas[best].cap))
                best = i;
        if (best != SIZE_MAX) {
            a = free_arenas[best];
            free_arenas.erase(free_arenas.begin() + best);
            return true;
        }
        const size_t cap = ((need + need / 4) + ((1u << 20) - 1)) & ~(size_t)((1u << 20) - 1);
        unsigned char* p = nullptr;
        if (cudaMallocHost(&p, cap) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        a.p = p;
        a.cap = cap;
        return true;
    }

    void recycle(Batch& b) {
        if (b.in.p) free_arenas.push_back(b.in);
        if (b.out.p) free_arenas.push_back(b.out);
        b.in = Arena{};
        b.out = Arena{};
    }

    // The canvases of a decoded batch from its page-locked output arena into
    // the callers' buffers (copy pool; needs no lock: the batch is owned by
    // the worker once it left `running`).
    static void copy_out(const Batch& b) {
        if (b.zero_copy) return;
        std::vector<hpvcd_host::CopyTask> tasks;
        tasks.reserve(b.reqs.size());
        for (const ReqMeta& r : b.reqs)
            tasks.push_back(hpvcd_host::CopyTask{r.dst, b.out.p + r.out_off,
                                                 (size_t)r.canvas.width * r.canvas.height * 3});
        hpvcd_host::parallel_copy(tasks.data(), tasks.size());
    }

    // Completion records for every request of `b` (outputs already copied).
    void complete(Batch& b, hpvcd_status st) {
        const auto now = Clock::now();
        for (const ReqMeta& r : b.reqs)
            done.push_back(hpvcd_completion{r.user, (int32_t)st, (uint32_t)b.pics.size(),
                                            ms_between(r.t_submit, now), ms_between(r.t_submit, b.t_launch)});
        recycle(b);
        cv_done.notify_all();
    }

    // A batch that failed before or at launch: nothing to copy.
    void finish(Batch& b, hpvcd_status st) { complete(b, st); }

    // Launch the front open batch; false when HBM admission asks to wait.
    bool launch_front() {
        Batch& b = *open.front();
        if (!b.zero_copy && !grow(b.out, b.out_used ? b.out_used : 256)) {
            finish(b, HPVCD_ERR_ALLOC);
            open.pop_front();
            return true;
        }
        std::vector<hpvcd_picture> pics(b.pics);
        std::vector<void*> dsts;
        for (const ReqMeta& r : b.reqs) dsts.push_back(r.dst);
        for (size_t i = 0; i < pics.size() && !b.zero_copy; ++i) {  // arena offsets -> pointers
            hpvcd_picture& p = pics[i];
            auto fix = [&](const void* off) -> const void* {
                return off ? (const void*)(b.in.p + ((uintptr_t)off - 1)) : nullptr;
            };
            p.tus = (const hpvcd_tu*)fix(p.tus);
            p.ctu_tu_start = (const uint32_t*)fix(p.ctu_tu_start);
            p.coeffs = (const int16_t*)fix(p.coeffs);
            p.cells = (const hpvcd_cell*)fix(p.cells);
            p.sao = (const hpvcd_sao_ctb*)fix(p.sao);
            p.pus = (const hpvcd_pu*)fix(p.pus);
            p.scaling = (const hpvcd_scaling*)fix(p.scaling);
            p.ctb_region = (const uint16_t*)fix(p.ctb_region);
            p.slice_deblock = (const int8_t*)fix(p.slice_deblock);
            for (int c = 0; c < 3; ++c) p.pred[c] = fix(p.pred[c]);
            if (p.wp) p.wp = &b.wp[i];
        }
        hpvcd_output o{};
        o.kind = HPVCD_OUT_RGB8;
        o.place = b.place.data();
        o.host_dst = b.out.p;
        o.host_dst_bytes = b.out.cap;
        o.n_canvases = (uint32_t)b.canvases.size();
        o.canvases = b.canvases.data();
        if (b.zero_copy) o.canvas_dst = dsts.data();
        b.t_launch = Clock::now();
        hpvcd_ticket t = 0;
        const hpvcd_status st = hpvcd_gpu_submit(gpu, pics.data(), (uint32_t)pics.size(), &o, &t);
        if ((st == HPVCD_ERR_ALLOC || st == HPVCD_ERR_BUSY) && !running.empty()) return false;  // wait
        std::unique_ptr<Batch> bp = std::move(open.front());
        open.pop_front();
        if (st != HPVCD_OK) {
            finish(*bp, st);
            return true;
        }
        bp->ticket = t;
        running.push_back(std::move(bp));
        return true;
    }

    void run() {
        cudaSetDevice(cfg.device);
        std::unique_lock<std::mutex> lock(mu);
        std::vector<std::pair<std::unique_ptr<Batch>, hpvcd_status>> decoded;
        while (true) {
            bool progressed = false;
            // Decoded batches give back their ticket slot first (the output
            // is already in the page-locked arena, or the callers' memory)...
            for (size_t i = 0; i < running.size();) {
                Batch& b = *running[i];
                const hpvcd_status w = hpvcd_gpu_wait(gpu, b.ticket, 0);
                if (w == HPVCD_ERR_BUSY) {
                    ++i;
                    continue;
                }
                const hpvcd_status st = w == HPVCD_OK ? hpvcd_gpu_read(gpu, b.ticket, b.out.p, b.out.cap) : w;
                decoded.emplace_back(std::move(running[i]), st);
                running.erase(running.begin() + i);
                progressed = true;
            }
            while (!open.empty() && running.size() < slots) {
                const Batch& f = *open.front();
                if (f.packers) break;  // a submit is still copying into it
                const bool full = open.size() > 1 || f.pics.size() >= max_pics();
                const bool window_open = cfg.batching && cfg.batch_window_us && !full &&
                                         std::chrono::duration<double, std::micro>(Clock::now() - f.t_first)
                                                 .count() < (double)cfg.batch_window_us;
                if (window_open) break;
                if (!launch_front()) break;
                progressed = true;
            }
            // ...so the next batches are already decoding while their
            // canvases go to the callers' buffers, without the lock
            if (!decoded.empty()) {
                lock.unlock();
                for (auto& d : decoded)
                    if (d.second == HPVCD_OK) copy_out(*d.first);
                lock.lock();
                for (auto& d : decoded) complete(*d.first, d.second);
                decoded.clear();
            }
            if (stop && open.empty() && running.empty()) break;
            if (!progressed) cv_work.wait_for(lock, std::chrono::microseconds(running.empty() ? 500 : 50));
        }
    }
};

HPVCD_API hpvcd_status hpvcd_server_create(const hpvcd_server_cfg* cfg, hpvcd_server** out) {
    if (!cfg || !out) return HPVCD_ERR_INVALID_ARG;
    *out = nullptr;
    hpvcd_server* s = new (std::nothrow) hpvcd_server();
    if (!s) return HPVCD_ERR_ALLOC;
    s->cfg = *cfg;
    const uint32_t inflight = cfg->max_inflight ? std::min<uint32_t>(cfg->max_inflight, 16) : 3;
    hpvcd_gpu_cfg gc{cfg->device, inflight, cfg->hbm_budget};
    const hpvcd_status st = hpvcd_gpu_create(&gc, &s->gpu);
    if (st != HPVCD_OK) {
        delete s;
        return st;
    }
    s->slots = inflight;
    s->worker = std::thread([s]() { s->run(); });
    *out = s;
    return HPVCD_OK;
}

HPVCD_API hpvcd_status hpvcd_server_submit(hpvcd_server* s, const hpvcd_request* req) {
    if (!s || !req || !req->pics || !req->n_pics || !req->place || !req->dst) return HPVCD_ERR_INVALID_ARG;
    if (req->canvas.width == 0 || req->canvas.height == 0) return HPVCD_ERR_INVALID_ARG;
    const uint64_t ob = (uint64_t)req->canvas.width * req->canvas.height * 3;
    if (req->dst_bytes < ob) return HPVCD_ERR_INVALID_ARG;
    const bool zc = (req->flags & HPVCD_REQ_ZERO_COPY) != 0;
    if (zc) {
        // the caller keeps packed page-locked inputs and a page-locked dst
        // alive until completion: nothing is copied on the host
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->open.empty() || !s->cfg.batching || !s->open.back()->zero_copy ||
            s->open.back()->pics.size() + req->n_pics > s->max_pics() ||
            s->open.back()->out_used + ob > s->max_bytes()) {
            std::unique_ptr<Batch> nbatch(new (std::nothrow) Batch());
            if (!nbatch) return HPVCD_ERR_ALLOC;
            nbatch->zero_copy = true;
            nbatch->t_first = Clock::now();
            s->open.push_back(std::move(nbatch));
        }
        Batch& b = *s->open.back();
        const uint32_t first = (uint32_t)b.pics.size();
        const uint32_t ci = (uint32_t)b.canvases.size();
        for (uint32_t i = 0; i < req->n_pics; ++i) {
            b.pics.push_back(req->pics[i]);
            hpvcd_tile_place tp = req->place[i];
            tp.canvas = ci;
            b.place.push_back(tp);
        }
        b.canvases.push_back(req->canvas);
        b.reqs.push_back(ReqMeta{first, req->n_pics, req->canvas, req->dst, req->dst_bytes, req->user,
                                 Clock::now(), b.out_used});
        b.out_used += ob;
        s->pending++;
        s->cv_work.notify_one();
        return HPVCD_OK;
    }
    const uint64_t nb = hpvcd_gpu_packed_size(req->pics, req->n_pics);
    Batch* bp;
    size_t in_off;
    uint32_t first;
    {
        // Reserve room in the open batch (arenas are sized to the batch byte
        // limit up front, so they never move while submits copy into them).
        std::lock_guard<std::mutex> lock(s->mu);
        const uint64_t cap = std::max<uint64_t>(s->max_bytes(), nb);
        if (s->open.empty() || !s->cfg.batching || s->open.back()->zero_copy ||
            s->open.back()->pics.size() + req->n_pics > s->max_pics() ||
            s->open.back()->in_used + nb + s->open.back()->out_used + ob > cap ||
            s->open.back()->in_used + nb > s->open.back()->in.cap) {
            std::unique_ptr<Batch> nbatch(new (std::nothrow) Batch());
            // room for this request, and (batching) for the ones that follow
            const uint64_t want = s->cfg.batching ? std::max<uint64_t>(nb, std::min<uint64_t>(cap, 256ull << 20)) : nb;
            if (!nbatch || !s->grow(nbatch->in, want)) return HPVCD_ERR_ALLOC;
            nbatch->t_first = Clock::now();
            s->open.push_back(std::move(nbatch));
        }
        bp = s->open.back().get();
        in_off = bp->in_used;
        first = (uint32_t)bp->pics.size();
        bp->in_used += nb;
        bp->pics.resize(first + req->n_pics);
        bp->wp.resize(first + req->n_pics);
        bp->place.resize(first + req->n_pics);
        const uint32_t ci = (uint32_t)bp->canvases.size();
        bp->canvases.push_back(req->canvas);
        bp->reqs.push_back(ReqMeta{first, req->n_pics, req->canvas, req->dst, req->dst_bytes, req->user,
                                   Clock::now(), bp->out_used});
        bp->out_used += ob;
        for (uint32_t i = 0; i < req->n_pics; ++i) {
            hpvcd_tile_place tp = req->place[i];
            tp.canvas = ci;
            bp->place[first + i] = tp;
        }
        bp->packers++;
        s->pending++;
    }
    // Copy the request's buffers into the page-locked arena (no lock held).
    std::vector<hpvcd_picture> packed(req->n_pics);
    unsigned char* base = bp->in.p;
    hpvcd_status st = hpvcd_gpu_pack_inputs(req->pics, req->n_pics, base + in_off, nb, packed.data());
    {
        std::lock_guard<std::mutex> lock(s->mu);
        for (uint32_t i = 0; i < req->n_pics; ++i) {
            hpvcd_picture p = packed[i];
            // keep 1 + arena offset; the launch turns offsets into pointers
            auto off = [&](const void* ptr) -> const void* {
                return ptr ? (const void*)((uintptr_t)((const unsigned char*)ptr - base) + 1) : nullptr;
            };
            p.tus = (const hpvcd_tu*)off(p.tus);
            p.ctu_tu_start = (const uint32_t*)off(p.ctu_tu_start);
            p.coeffs = (const int16_t*)off(p.coeffs);
            p.cells = (const hpvcd_cell*)off(p.cells);
            p.sao = (const hpvcd_sao_ctb*)off(p.sao);
            p.pus = (const hpvcd_pu*)off(p.pus);
            p.scaling = (const hpvcd_scaling*)off(p.scaling);
            p.ctb_region = (const uint16_t*)off(p.ctb_region);
            p.slice_deblock = (const int8_t*)off(p.slice_deblock);
            for (int c = 0; c < 3; ++c) p.pred[c] = off(p.pred[c]);
            bp->wp[first + i] = req->pics[i].wp ? *req->pics[i].wp : hpvcd_wp_table{};
            p.wp = req->pics[i].wp ? (const hpvcd_wp_table*)1 : nullptr;  // resolved at launch
            bp->pics[first + i] = p;
        }
        if (st != HPVCD_OK)  // a malformed request poisons its batch: fail it loudly
            for (uint32_t i = 0; i < req->n_pics; ++i) bp->pics[first + i].width = 0;
        bp->packers--;
    }
    s->cv_work.notify_one();
    return st;
}

HPVCD_API uint32_t hpvcd_server_poll(hpvcd_server* s, hpvcd_completion* out, uint32_t max, int32_t timeout_ms) {
    if (!s || !out || !max) return 0;
    std::unique_lock<std::mutex> lock(s->mu);
    if (s->done.empty()) {
        if (timeout_ms < 0)
            s->cv_done.wait(lock, [s]() { return !s->done.empty(); });
        else
            s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), [s]() { return !s->done.empty(); });
    }
    uint32_t k = 0;
    while (k < max && !s->done.empty()) {
        out[k++] = s->done.front();
        s->done.pop_front();
        s->pending--;
    }
    return k;
}

extern "C" hpvcd_status hpvcd_gpu_set_selector(hpvcd_gpu*, hpvcd_mlp*, const hpvcd_sched*, uint32_t);
extern "C" hpvcd_status hpvcd_gpu_selector_picks(hpvcd_gpu*, uint64_t*, uint32_t);

// The batches this server launches get their schedule from the selector
// network (NULL: the default schedule).
HPVCD_API hpvcd_status hpvcd_server_set_selector(hpvcd_server* s, hpvcd_mlp* mlp, const hpvcd_sched* cands,
                                                 uint32_t n) {
    if (!s) return HPVCD_ERR_INVALID_ARG;
    return hpvcd_gpu_set_selector(s->gpu, mlp, cands, n);
}

HPVCD_API hpvcd_status hpvcd_server_selector_picks(hpvcd_server* s, uint64_t* counts, uint32_t n) {
    if (!s) return HPVCD_ERR_INVALID_ARG;
    return hpvcd_gpu_selector_picks(s->gpu, counts, n);
}

HPVCD_API uint32_t hpvcd_server_pending(hpvcd_server* s) {
    if (!s) return 0;
    std::lock_guard<std::mutex> lock(s->mu);
    return s->pending;
}

HPVCD_API hpvcd_status hpvcd_server_destroy(hpvcd_server* s) {
    if (!s) return HPVCD_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (Arena& a : s->free_arenas) cudaFreeHost(a.p);
    hpvcd_gpu_destroy(s->gpu);
    delete s;
    return HPVCD_OK;
}
