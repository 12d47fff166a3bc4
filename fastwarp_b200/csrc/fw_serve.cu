// fw_serve.cu -- the continuous-batching registration server (include/fastwarp_serve.h).
//
// N execution slots, each a thread with its own context (stream, scratch). A FIFO queue of
// requests; a slot takes the first queued request whose device-memory estimate fits in what is
// left of the HBM budget (smaller requests may pass a large one that does not fit yet), runs the
// whole SyN stage (one CUDA graph per level), releases the memory, and takes the next. Several
// slots run at once, so the latency-bound coarse levels of one registration overlap the
// bandwidth-bound fine levels of another.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <thread>
#include <list>
#include <vector>

#include "../../include/fastwarp_serve.h"
#include "../../include/fastwarp_transform_io.h"
#include "fw_internal.cuh"

using Clock = std::chrono::steady_clock;

namespace {

// Pinned host buffers kept by size for reuse (cudaHostAlloc is slow and synchronises the
// device): the staging of host inputs and the host results, so both copies run as DMA at full
// link speed without a bounce through pageable memory. Process-wide: results outlive servers.
// Requests of many grid sizes would leave a buffer of every size behind: past kMaxKept bytes the
// buffers returned longest ago are released.
struct PinnedPool {
    static constexpr size_t kMaxKept = (size_t)8 << 30;
    struct Kept {
        size_t bytes;
        void* p;
    };
    std::mutex mu;
    std::list<Kept> free;  // in the order they were returned
    size_t kept = 0;
    void* get(size_t bytes) {
        {
            std::lock_guard<std::mutex> lock(mu);
            for (auto it = free.rbegin(); it != free.rend(); ++it)
                if (it->bytes == bytes) {
                    void* p = it->p;
                    kept -= bytes;
                    free.erase(std::next(it).base());
                    return p;
                }
        }
        void* p = nullptr;
        if (cudaHostAlloc(&p, bytes, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return p;
    }
    void put(void* p, size_t bytes) {
        if (!p) return;
        std::list<Kept> drop;
        {
            std::lock_guard<std::mutex> lock(mu);
            free.push_back(Kept{bytes, p});
            kept += bytes;
            while (kept > kMaxKept && free.size() > 1) {
                kept -= free.front().bytes;
                drop.splice(drop.end(), free, free.begin());
            }
        }
        for (auto& k : drop) cudaFreeHost(k.p);
    }
};

PinnedPool& pinned() {
    static PinnedPool* pool = new PinnedPool();  // kept to process exit (results may outlive it)
    return *pool;
}

struct Job {
    uint64_t ticket = 0;
    fw_syn_request req{};
    std::vector<float*> fixed_host, moving_host;  // pinned staging of host inputs
    size_t fixed_bytes = 0, moving_bytes = 0;
    float* mask_host[2] = {nullptr, nullptr};     // pinned staging of host masks
    size_t mask_bytes[2] = {0, 0};
    std::vector<const fw_image*> fixed_dev, moving_dev;
    uint64_t bytes = 0;
    Clock::time_point submitted;
    fw_syn_result result{};
    bool done = false;
    bool taken = false;
    bool linear = false;           // a linear-stage request (lreq / lres)
    int slot = -1;                 // the slot running it (-1 while queued)
    fw_linear_request lreq{};
    fw_linear_result lres{};
    int status() const { return linear ? lres.status : result.status; }
};

// Device memory of one linear stage: the uploaded inputs, the smoothed copies with the Deriche
// temporaries, the device MI level (16-byte samples, at most one per fixed voxel) and scratch.
int estimate_linear(const fw_linear_request* q, uint64_t* out) {
    using namespace fw;
    HostGrid fg, mg;
    FW_TRY(make_grid(&q->fixed_grid, fg));
    FW_TRY(make_grid(&q->moving_grid, mg));
    const fw_linear_recipe* r = &q->recipe;
    FW_CHECK(r->levels >= 1 && r->levels <= FW_MAX_LEVELS, "serve: recipe has no levels");
    const uint64_t nf = (uint64_t)fg.count(), nm = (uint64_t)mg.count();
    uint64_t b = 0;
    if (q->fixed) b += 4 * (nf + nm);
    b += 4 * (nf + nm) + 24 * std::max(nf, nm);
    b += 16 * nf + 4 * nm;
    b += 4u << 20;
    *out = b;
    return 0;
}

int estimate(const fw_syn_request* q, uint64_t* out) {
    using namespace fw;
    HostGrid fg, mg;
    FW_TRY(make_grid(&q->fixed_grid, fg));
    FW_TRY(make_grid(&q->moving_grid, mg));
    const fw_syn_recipe* r = &q->recipe;
    FW_CHECK(r->levels >= 1 && r->levels <= FW_MAX_LEVELS, "serve: recipe has no levels");
    FW_CHECK(r->channels >= 1 && r->channels <= FW_MAX_CHANNELS, "serve: 1..=4 channels");
    fw_grid last;
    FW_TRY(fw_syn_level_grid(r, &q->fixed_grid, r->levels - 1, &last));
    int64_t n = 1, nprev = 0;
    for (int a = 0; a < 3; ++a) n *= last.size[a];
    if (r->levels > 1) {
        fw_grid prev;
        FW_TRY(fw_syn_level_grid(r, &q->fixed_grid, r->levels - 2, &prev));
        nprev = prev.size[0] * prev.size[1] * prev.size[2];
    }
    const uint64_t C = (uint64_t)r->channels;
    const uint64_t nf = (uint64_t)fg.count(), nm = (uint64_t)mg.count();
    const uint64_t ps = (uint64_t)plane_stride(n), psp = (uint64_t)plane_stride(nprev);
    bool smooth = false;
    for (int l = 0; l < r->levels; ++l) smooth = smooth || r->smoothing_sigmas[l] > 0.0;
    uint64_t b = 0;
    if (q->fixed == nullptr) b += 0;
    else b += 4 * C * (nf + nm);                       // uploaded inputs
    if (smooth) b += 4 * C * (nf + nm) + 24 * std::max(nf, nm);  // smoothed copies + Deriche temp
    int fields = 4 + 2 + 1 /* inversion residual */ + (r->update_field_variance > 0 ? 2 : 0) +
                 (C > 1 ? 2 : 0) + (r->total_field_variance > 0 ? 1 : 0) + 2 /* outputs */;
    b += 12 * ps * (uint64_t)fields;
    b += 4 * (uint64_t)n * 2 * C;                      // warped images
    b += 12 * psp * 4;                                 // state of the previous level at a transition
    const fw_grid* mg_[2] = {&q->fixed_mask_grid, &q->moving_mask_grid};
    const bool mask_[2] = {q->fixed_mask || q->fixed_mask_dev, q->moving_mask || q->moving_mask_dev};
    for (int k = 0; k < 2; ++k) {
        if (!mask_[k]) continue;
        b += 4 * (uint64_t)n * 2;                      // resolved on the level grid (+ product)
        if (k == 0 ? q->fixed_mask != nullptr : q->moving_mask != nullptr)
            b += 4 * (uint64_t)(mg_[k]->size[0] * mg_[k]->size[1] * mg_[k]->size[2]);  // upload
    }
    b += 2u << 20;                                     // records and scalars
    *out = b;
    return 0;
}

}  // namespace

struct fw_server {
    int device = 0;
    uint64_t budget = 0;
    int slots = 0;
    std::vector<fw_ctx*> ctxs;
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Job*> queue;
    std::map<uint64_t, Job*> jobs;
    uint64_t next_ticket = 1;
    uint64_t reserved = 0, peak = 0;
    uint64_t submitted = 0, completed = 0, failed = 0, active = 0;
    bool stopping = false;
    cudaEvent_t epoch = nullptr;
    bool epoch_set = false;
};

namespace {

void run_job(fw_server* s, fw_ctx* ctx, Job* j) {
    using namespace fw;
    fw_syn_result& res = j->result;
    res.tag = j->req.tag;
    res.device_bytes = j->bytes;
    const fw_syn_request& q = j->req;
    const int C = q.recipe.channels;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, ctx->stream);
    std::vector<fw_image*> up;
    std::vector<const fw_image*> fi(C), mi(C);
    int rc = 0;
    if (!j->fixed_dev.empty()) {
        for (int c = 0; c < C; ++c) {
            fi[c] = j->fixed_dev[c];
            mi[c] = j->moving_dev[c];
        }
    } else {
        HostGrid fg, mg;
        rc = make_grid(&q.fixed_grid, fg);
        if (!rc) rc = make_grid(&q.moving_grid, mg);
        for (int c = 0; c < C && !rc; ++c) {
            fw_image *a = nullptr, *b = nullptr;
            rc = enqueue_image_upload_f32(ctx, fg, j->fixed_host[c], &a);
            if (!rc) up.push_back(a);
            if (!rc) rc = enqueue_image_upload_f32(ctx, mg, j->moving_host[c], &b);
            if (!rc) up.push_back(b);
            fi[c] = a;
            mi[c] = b;
        }
    }
    // the recipe's masks: device images as given, host data uploaded from the pinned staging
    const fw_image* masks[2] = {q.fixed_mask_dev, q.moving_mask_dev};
    const fw_grid* mgrids[2] = {&q.fixed_mask_grid, &q.moving_mask_grid};
    for (int k = 0; k < 2 && !rc; ++k) {
        if (!j->mask_host[k]) continue;
        HostGrid mgk;
        rc = make_grid(mgrids[k], mgk);
        fw_image* im = nullptr;
        if (!rc) rc = enqueue_image_upload_f32(ctx, mgk, j->mask_host[k], &im);
        if (!rc) {
            up.push_back(im);
            masks[k] = im;
        }
    }
    int64_t cap = 0;
    for (int l = 0; l < q.recipe.levels; ++l) cap += q.recipe.iterations[l];
    std::vector<fw_syn_iteration> recs((size_t)std::max<int64_t>(cap, 1));
    int64_t count = 0;
    fw_field *w = nullptr, *iw = nullptr;
    if (!rc)
        rc = syn_run_device(ctx, &q.recipe, fi.data(), mi.data(), masks[0], masks[1],
                            q.has_initial ? &q.initial : nullptr, nullptr, nullptr,
                            &w, &iw, recs.data(), (int64_t)recs.size(), &count);
    for (auto* im : up) fw_image_free(im);
    if (!rc) {
        res.iterations = count;
        res.final_energy = count > 0 ? recs[(size_t)std::min<int64_t>(count, cap) - 1].energy : 0.0;
        res.grid = to_c(w->grid);
        if (q.keep_on_device) {
            res.warp_dev = w;
            res.inverse_dev = iw;
            w = iw = nullptr;
        } else {
            // AoS float32 made on the device and copied straight into pinned result buffers
            size_t bytes = 3 * sizeof(float) * (size_t)w->grid.count();
            res.warp = static_cast<float*>(pinned().get(bytes));
            res.inverse_warp = static_cast<float*>(pinned().get(bytes));
            if (!res.warp || !res.inverse_warp) rc = fail(FW_ERR_MEMORY, "serve: host allocation failed");
            if (!rc) rc = enqueue_field_download_f32(ctx, w, res.warp);
            if (!rc) rc = enqueue_field_download_f32(ctx, iw, res.inverse_warp);
        }
    }
    fw_field_free(w);
    fw_field_free(iw);
    cudaEventRecord(e1, ctx->stream);
    if (sync(ctx) && !rc) rc = FW_ERR_CUDA;
    // the uploads have completed: the staging goes back to the pool
    for (auto* p : j->fixed_host) pinned().put(p, j->fixed_bytes);
    for (auto* p : j->moving_host) pinned().put(p, j->moving_bytes);
    j->fixed_host.clear();
    j->moving_host.clear();
    for (int k = 0; k < 2; ++k) {
        pinned().put(j->mask_host[k], j->mask_bytes[k]);
        j->mask_host[k] = nullptr;
    }
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->epoch_set) {
            float a = 0.0f, b = 0.0f;
            cudaEventElapsedTime(&a, s->epoch, e0);
            cudaEventElapsedTime(&b, s->epoch, e1);
            res.device_start_ms = a;
            res.device_end_ms = b;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    res.status = rc;
    if (rc) {
        std::strncpy(res.error, fw_last_error(), sizeof(res.error) - 1);
        fw_server_result_free(&res);
        fw_field_free(res.warp_dev);
        fw_field_free(res.inverse_dev);
        res.warp_dev = res.inverse_dev = nullptr;
    }
}

void run_linear_job(fw_ctx* ctx, Job* j) {
    using namespace fw;
    fw_linear_result& res = j->lres;
    const fw_linear_request& q = j->lreq;
    res.tag = q.tag;
    res.device_bytes = j->bytes;
    res.nlevels = q.recipe.levels;
    res.transform = q.start;
    std::vector<fw_image*> up;
    const fw_image *fi = nullptr, *mi = nullptr;
    int rc = 0;
    if (!j->fixed_dev.empty()) {
        fi = j->fixed_dev[0];
        mi = j->moving_dev[0];
    } else {
        HostGrid fg, mg;
        rc = make_grid(&q.fixed_grid, fg);
        if (!rc) rc = make_grid(&q.moving_grid, mg);
        fw_image *a = nullptr, *b = nullptr;
        if (!rc) rc = enqueue_image_upload_f32(ctx, fg, j->fixed_host[0], &a);
        if (!rc) up.push_back(a);
        if (!rc) rc = enqueue_image_upload_f32(ctx, mg, j->moving_host[0], &b);
        if (!rc) up.push_back(b);
        fi = a;
        mi = b;
    }
    if (!rc) rc = fw_linear_stage_run(ctx, &q.recipe, fi, mi, &res.transform, res.levels);
    for (auto* im : up) fw_image_free(im);
    if (sync(ctx) && !rc) rc = FW_ERR_CUDA;
    for (auto* p : j->fixed_host) pinned().put(p, j->fixed_bytes);
    for (auto* p : j->moving_host) pinned().put(p, j->moving_bytes);
    j->fixed_host.clear();
    j->moving_host.clear();
    res.status = rc;
    if (rc) std::strncpy(res.error, fw_last_error(), sizeof(res.error) - 1);
}

void worker(fw_server* s, int slot) {
    cudaSetDevice(s->device);
    fw_ctx* ctx = s->ctxs[slot];
    for (;;) {
        Job* j = nullptr;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            for (;;) {
                for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
                    if (s->reserved + (*it)->bytes <= s->budget) {
                        j = *it;
                        s->queue.erase(it);
                        break;
                    }
                }
                if (j || (s->stopping && s->queue.empty())) break;
                s->cv_work.wait(lock);
            }
            if (!j) return;
            j->slot = slot;
            s->reserved += j->bytes;
            s->peak = std::max(s->peak, s->reserved);
            s->active++;
        }
        auto t0 = Clock::now();
        const double queued = std::chrono::duration<double>(t0 - j->submitted).count();
        if (j->linear) run_linear_job(ctx, j);
        else run_job(s, ctx, j);
        const double ran = std::chrono::duration<double>(Clock::now() - t0).count();
        (j->linear ? j->lres.queued_s : j->result.queued_s) = queued;
        (j->linear ? j->lres.run_s : j->result.run_s) = ran;
        {
            std::lock_guard<std::mutex> lock(s->mu);
            s->reserved -= j->bytes;
            s->active--;
            if (j->status()) s->failed++;
            else s->completed++;
            j->done = true;
            // a cancel that came for this request ends with it: the slot's next request runs
            fw_ctx_request_cancel(ctx, 0);
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

}  // namespace

using namespace fw;

extern "C" {

int fw_server_estimate(const fw_syn_request* req, uint64_t* bytes) {
    FW_CHECK(req && bytes, "null argument");
    return estimate(req, bytes);
}

int fw_server_create(int device, uint64_t hbm_budget, int32_t slots, fw_server** out) {
    FW_CHECK(out && slots >= 1 && slots <= 64, "serve: 1..=64 slots");
    *out = nullptr;
    fw_server* s = new fw_server();
    s->device = device;
    s->slots = slots;
    for (int i = 0; i < slots; ++i) {
        fw_ctx* c = nullptr;
        int rc = fw_ctx_create(device, &c);
        if (!rc) rc = ensure_scratch(c, SLOT_PARTIALS + (size_t)(1 << 20));
        if (rc) {
            if (c) fw_ctx_destroy(c);
            for (auto* x : s->ctxs) fw_ctx_destroy(x);
            delete s;
            return rc;
        }
        s->ctxs.push_back(c);
    }
    if (hbm_budget == 0) {
        size_t f = 0, t = 0;
        cudaMemGetInfo(&f, &t);
        hbm_budget = (uint64_t)(0.9 * (double)f);
    }
    s->budget = hbm_budget;
    cudaEventCreate(&s->epoch);
    for (int i = 0; i < slots; ++i) s->threads.emplace_back(worker, s, i);
    *out = s;
    return 0;
}

int fw_server_submit(fw_server* s, const fw_syn_request* req, uint64_t* ticket) {
    FW_CHECK(s && req && ticket, "null argument");
    const int C = req->recipe.channels;
    FW_CHECK(C >= 1 && C <= FW_MAX_CHANNELS, "serve: 1..=4 channels");
    bool host = req->fixed && req->moving;
    bool dev = req->fixed_dev && req->moving_dev;
    FW_CHECK(host != dev, "serve: give either host or device images");
    FW_CHECK(!(req->fixed_mask && req->fixed_mask_dev) && !(req->moving_mask && req->moving_mask_dev),
             "serve: give a mask either as host data or as a device image");
    uint64_t bytes = 0;
    FW_TRY(estimate(req, &bytes));
    if (bytes > s->budget)
        return fail(FW_ERR_MEMORY, "serve: the request needs " + std::to_string(bytes) +
                                       " bytes of device memory, more than the budget of " +
                                       std::to_string(s->budget));
    Job* j = new Job();
    j->req = *req;
    j->bytes = bytes;
    HostGrid fg, mg;
    int rc = make_grid(&req->fixed_grid, fg);
    if (!rc) rc = make_grid(&req->moving_grid, mg);
    if (rc) {
        delete j;
        return rc;
    }
    if (host) {
        j->fixed_bytes = sizeof(float) * (size_t)fg.count();
        j->moving_bytes = sizeof(float) * (size_t)mg.count();
        for (int c = 0; c < C; ++c) {
            float* a = static_cast<float*>(pinned().get(j->fixed_bytes));
            float* b = static_cast<float*>(pinned().get(j->moving_bytes));
            if (a) j->fixed_host.push_back(a);
            if (b) j->moving_host.push_back(b);
            if (!a || !b) {
                for (auto* p : j->fixed_host) pinned().put(p, j->fixed_bytes);
                for (auto* p : j->moving_host) pinned().put(p, j->moving_bytes);
                delete j;
                return fail(FW_ERR_MEMORY, "serve: pinned host staging allocation failed");
            }
            std::memcpy(a, req->fixed[c], j->fixed_bytes);
            std::memcpy(b, req->moving[c], j->moving_bytes);
        }
    } else {
        for (int c = 0; c < C; ++c) {
            j->fixed_dev.push_back(req->fixed_dev[c]);
            j->moving_dev.push_back(req->moving_dev[c]);
        }
    }
    const float* mask_src[2] = {req->fixed_mask, req->moving_mask};
    const fw_grid* mask_grid[2] = {&req->fixed_mask_grid, &req->moving_mask_grid};
    for (int k = 0; k < 2; ++k) {
        if (!mask_src[k]) continue;
        HostGrid mgk;
        int mrc = make_grid(mask_grid[k], mgk);
        if (!mrc) {
            j->mask_bytes[k] = sizeof(float) * (size_t)mgk.count();
            j->mask_host[k] = static_cast<float*>(pinned().get(j->mask_bytes[k]));
            if (!j->mask_host[k]) mrc = fail(FW_ERR_MEMORY, "serve: pinned host staging allocation failed");
        }
        if (mrc) {
            for (auto* p : j->fixed_host) pinned().put(p, j->fixed_bytes);
            for (auto* p : j->moving_host) pinned().put(p, j->moving_bytes);
            for (int q = 0; q < 2; ++q) pinned().put(j->mask_host[q], j->mask_bytes[q]);
            delete j;
            return mrc;
        }
        std::memcpy(j->mask_host[k], mask_src[k], j->mask_bytes[k]);
    }
    j->req.fixed = j->req.moving = nullptr;
    j->req.fixed_dev = j->req.moving_dev = nullptr;
    j->req.fixed_mask = j->req.moving_mask = nullptr;
    j->submitted = Clock::now();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        j->ticket = s->next_ticket++;
        s->jobs[j->ticket] = j;
        s->queue.push_back(j);
        s->submitted++;
    }
    s->cv_work.notify_all();
    *ticket = j->ticket;
    return 0;
}

int fw_server_wait(fw_server* s, uint64_t ticket, double timeout_s, fw_syn_result* out) {
    FW_CHECK(s && out, "null argument");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return fail(FW_ERR_INVALID, "serve: unknown or already taken ticket");
    Job* j = it->second;
    if (j->linear) return fail(FW_ERR_INVALID, "serve: the ticket is a linear-stage request");
    auto ready = [&] { return j->done; };
    if (timeout_s < 0) {
        s->cv_done.wait(lock, ready);
    } else if (!s->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), ready)) {
        return fail(FW_ERR_TIMEOUT, "serve: the request is not done yet");
    }
    *out = j->result;
    s->jobs.erase(it);
    delete j;
    return 0;
}

int fw_server_cancel(fw_server* s, uint64_t ticket) {
    FW_CHECK(s, "null server");
    {
        std::lock_guard<std::mutex> lock(s->mu);
        auto it = s->jobs.find(ticket);
        if (it == s->jobs.end()) return fail(FW_ERR_INVALID, "serve: unknown or already taken ticket");
        Job* j = it->second;
        if (j->done) return 0;  // finished already: its result stands
        if (j->slot >= 0) {
            // running: the slot's context flag stops its level graph after the iteration in
            // flight; the slot clears the flag when the request ends
            return fw_ctx_request_cancel(s->ctxs[j->slot], 1);
        }
        // queued: it ends here without running
        for (auto q = s->queue.begin(); q != s->queue.end(); ++q)
            if (*q == j) {
                s->queue.erase(q);
                break;
            }
        for (auto* p : j->fixed_host) pinned().put(p, j->fixed_bytes);
        for (auto* p : j->moving_host) pinned().put(p, j->moving_bytes);
        j->fixed_host.clear();
        j->moving_host.clear();
        for (int k = 0; k < 2; ++k) {
            pinned().put(j->mask_host[k], j->mask_bytes[k]);
            j->mask_host[k] = nullptr;
        }
        const char* why = "registration cancelled";
        if (j->linear) {
            j->lres.tag = j->lreq.tag;
            j->lres.status = FW_ERR_CANCELLED;
            std::strncpy(j->lres.error, why, sizeof(j->lres.error) - 1);
        } else {
            j->result.tag = j->req.tag;
            j->result.status = FW_ERR_CANCELLED;
            std::strncpy(j->result.error, why, sizeof(j->result.error) - 1);
        }
        j->done = true;
        s->failed++;
    }
    s->cv_done.notify_all();
    return 0;
}

int fw_server_estimate_linear(const fw_linear_request* req, uint64_t* bytes) {
    FW_CHECK(req && bytes, "null argument");
    return estimate_linear(req, bytes);
}

int fw_server_submit_linear(fw_server* s, const fw_linear_request* req, uint64_t* ticket) {
    FW_CHECK(s && req && ticket, "null argument");
    const bool host = req->fixed && req->moving;
    const bool dev = req->fixed_dev && req->moving_dev;
    FW_CHECK(host != dev, "serve: give either host or device images");
    uint64_t bytes = 0;
    FW_TRY(estimate_linear(req, &bytes));
    if (bytes > s->budget)
        return fail(FW_ERR_MEMORY, "serve: the request needs " + std::to_string(bytes) +
                                       " bytes of device memory, more than the budget of " +
                                       std::to_string(s->budget));
    HostGrid fg, mg;
    FW_TRY(make_grid(&req->fixed_grid, fg));
    FW_TRY(make_grid(&req->moving_grid, mg));
    Job* j = new Job();
    j->linear = true;
    j->lreq = *req;
    j->bytes = bytes;
    if (host) {
        j->fixed_bytes = sizeof(float) * (size_t)fg.count();
        j->moving_bytes = sizeof(float) * (size_t)mg.count();
        float* a = static_cast<float*>(pinned().get(j->fixed_bytes));
        float* b = static_cast<float*>(pinned().get(j->moving_bytes));
        if (!a || !b) {
            pinned().put(a, j->fixed_bytes);
            pinned().put(b, j->moving_bytes);
            delete j;
            return fail(FW_ERR_MEMORY, "serve: pinned host staging allocation failed");
        }
        std::memcpy(a, req->fixed, j->fixed_bytes);
        std::memcpy(b, req->moving, j->moving_bytes);
        j->fixed_host.push_back(a);
        j->moving_host.push_back(b);
    } else {
        j->fixed_dev.push_back(req->fixed_dev);
        j->moving_dev.push_back(req->moving_dev);
    }
    j->lreq.fixed = j->lreq.moving = nullptr;
    j->lreq.fixed_dev = j->lreq.moving_dev = nullptr;
    j->submitted = Clock::now();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        j->ticket = s->next_ticket++;
        s->jobs[j->ticket] = j;
        s->queue.push_back(j);
        s->submitted++;
    }
    s->cv_work.notify_all();
    *ticket = j->ticket;
    return 0;
}

int fw_server_wait_linear(fw_server* s, uint64_t ticket, double timeout_s,
                          fw_linear_result* out) {
    FW_CHECK(s && out, "null argument");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return fail(FW_ERR_INVALID, "serve: unknown or already taken ticket");
    Job* j = it->second;
    if (!j->linear) return fail(FW_ERR_INVALID, "serve: the ticket is a SyN request");
    auto ready = [&] { return j->done; };
    if (timeout_s < 0) {
        s->cv_done.wait(lock, ready);
    } else if (!s->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), ready)) {
        return fail(FW_ERR_TIMEOUT, "serve: the request is not done yet");
    }
    *out = j->lres;
    s->jobs.erase(it);
    delete j;
    return 0;
}

void fw_server_result_free(fw_syn_result* r) {
    if (!r) return;
    const size_t bytes =
        3 * sizeof(float) * (size_t)(r->grid.size[0] * r->grid.size[1] * r->grid.size[2]);
    pinned().put(r->warp, bytes);
    pinned().put(r->inverse_warp, bytes);
    r->warp = r->inverse_warp = nullptr;
}

int fw_server_mark(fw_server* s) {
    FW_CHECK(s, "null server");
    cudaSetDevice(s->device);
    std::lock_guard<std::mutex> lock(s->mu);
    FW_CUDA(cudaEventRecord(s->epoch, s->ctxs[0]->stream));
    FW_CUDA(cudaEventSynchronize(s->epoch));
    s->epoch_set = true;
    return 0;
}

int fw_server_stats_get(fw_server* s, fw_server_stats* out) {
    FW_CHECK(s && out, "null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->failed = s->failed;
    out->active = s->active;
    out->queued = s->queue.size();
    out->reserved_bytes = s->reserved;
    out->peak_reserved_bytes = s->peak;
    out->budget_bytes = s->budget;
    out->kernel_launches = out->graph_launches = 0;
    for (auto* c : s->ctxs) {
        out->kernel_launches += c->stats.kernel_launches;
        out->graph_launches += c->stats.graph_launches;
    }
    return 0;
}

void fw_server_destroy(fw_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stopping = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->threads) t.join();
    for (auto& kv : s->jobs) {
        fw_server_result_free(&kv.second->result);
        fw_field_free(kv.second->result.warp_dev);
        fw_field_free(kv.second->result.inverse_dev);
        delete kv.second;
    }
    if (s->epoch) cudaEventDestroy(s->epoch);
    for (auto* c : s->ctxs) fw_ctx_destroy(c);
    delete s;
}

}  // extern "C"

extern "C" size_t fw_abi_struct_size(const char* name) {
    if (!name) return 0;
    const std::string n(name);
    if (n == "fw_grid") return sizeof(fw_grid);
    if (n == "fw_affine") return sizeof(fw_affine);
    if (n == "fw_invert_params") return sizeof(fw_invert_params);
    if (n == "fw_invert_stats") return sizeof(fw_invert_stats);
    if (n == "fw_mi_binning") return sizeof(fw_mi_binning);
    if (n == "fw_linear_transform") return sizeof(fw_linear_transform);
    if (n == "fw_syn_recipe") return sizeof(fw_syn_recipe);
    if (n == "fw_syn_iteration") return sizeof(fw_syn_iteration);
    if (n == "fw_stats") return sizeof(fw_stats);
    if (n == "fw_syn_request") return sizeof(fw_syn_request);
    if (n == "fw_syn_result") return sizeof(fw_syn_result);
    if (n == "fw_server_stats") return sizeof(fw_server_stats);
    if (n == "fw_cg_settings") return sizeof(fw_cg_settings);
    if (n == "fw_cg_trace") return sizeof(fw_cg_trace);
    if (n == "fw_transform_elem") return sizeof(fw_transform_elem);
    if (n == "fw_linear_recipe") return sizeof(fw_linear_recipe);
    if (n == "fw_linear_level_trace") return sizeof(fw_linear_level_trace);
    if (n == "fw_linear_request") return sizeof(fw_linear_request);
    if (n == "fw_linear_chain_result") return sizeof(fw_linear_chain_result);
    if (n == "fw_linear_result") return sizeof(fw_linear_result);
    if (n == "fw_batch_subject") return sizeof(fw_batch_subject);
    if (n == "fw_batch_tuning") return sizeof(fw_batch_tuning);
    if (n == "fw_batch_report") return sizeof(fw_batch_report);
    return 0;
}
