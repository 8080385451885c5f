// The serving form: frames from many callers (camera streams), detected by
// continuous batching. Each of `workers` threads owns a detector (its own
// stream and device arenas, the families' tables resident); whenever a
// worker is free it takes every frame that has arrived, oldest first, up to
// max_batch frames and its share of the device-memory budget, and runs them
// as one batch. With two or more workers, frames that arrive while a batch
// is on the GPU go into the next batch, which overlaps the first on the
// device. Each frame's detections are exactly what at_detect gives for it
// alone. The reference has no counterpart (it detects one frame per call,
// fast/detector.c:246-335); the detection itself is at_detect_batch.
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "apriltag_fast.h"

// internal, in at_detector.cu
extern "C" at_detector *at_detector_clone(const at_detector *src);
extern "C" int64_t at_detector_arena_bytes(const at_detector *td);  // bytes the last call needed

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
    uint64_t ticket, user;
    at_frame frame;
    double t_submit;
    int64_t est;  // device bytes it is expected to need
};

}  // namespace

struct at_server {
    at_server_config cfg;
    std::vector<int> dev_of;  // each worker's GPU
    std::vector<at_detector *> dets;
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request> pending;
    std::deque<at_server_result> done;
    bool stop = false;
    uint64_t next_ticket = 1;
    double bytes_per_pixel = 64.0;  // device bytes per input pixel, learned from the batches
    int64_t queued_bytes = 0;       // estimated device bytes of the pending and running frames
    at_server_stats st{};
};

static void worker(at_server *s, int w) {
    cudaSetDevice(s->dev_of[w]);
    at_detector *td = s->dets[w];
    const int64_t share = s->cfg.memory_budget / (s->cfg.workers > 0 ? s->cfg.workers : 1);
    std::vector<Request> batch;
    std::vector<at_frame> frames;
    std::vector<at_frame_result> res;
    for (;;) {
        batch.clear();
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stop || !s->pending.empty(); });
            if (s->stop && s->pending.empty()) return;
            int64_t bytes = 0;
            while (!s->pending.empty() && (int64_t)batch.size() < s->cfg.max_batch) {
                const Request &r = s->pending.front();
                if (!batch.empty() && bytes + r.est > share) break;
                bytes += r.est;
                batch.push_back(r);
                s->pending.pop_front();
            }
            if (batch.empty()) continue;
            s->st.batches++;
            s->st.in_flight += (int64_t)batch.size();
        }
        frames.resize(batch.size());
        res.resize(batch.size());
        int64_t px = 0;
        for (size_t i = 0; i < batch.size(); i++) {
            frames[i] = batch[i].frame;
            px += batch[i].frame.width * batch[i].frame.height;
        }
        const double t_start = now_s();
        at_detect_batch(td, frames.data(), (int64_t)frames.size(), res.data());
        const double t_done = now_s();
        const int status = at_detector_last_error(td, nullptr);
        const int64_t arena = at_detector_arena_bytes(td);
        std::vector<at_server_result> out(batch.size());
        for (size_t i = 0; i < batch.size(); i++) {
            at_server_result &o = out[i];
            memset(&o, 0, sizeof o);
            o.ticket = batch[i].ticket;
            o.user = batch[i].user;
            o.status = status;
            o.nquads = res[i].nquads;
            o.ndetections = res[i].count;
            o.batch_frames = (int32_t)batch.size();
            o.worker = w;
            if (res[i].count > 0) {
                o.detections = (at_detection *)malloc(sizeof(at_detection) * res[i].count);
                memcpy(o.detections, td->detections + res[i].first, sizeof(at_detection) * res[i].count);
            }
            o.t_submit = batch[i].t_submit;
            o.t_start = t_start;
            o.t_done = t_done;
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            for (auto &o : out) s->done.push_back(o);
            for (auto &r : batch) s->queued_bytes -= r.est;
            s->st.completed += (int64_t)batch.size();
            s->st.in_flight -= (int64_t)batch.size();
            if (px > 0 && (double)arena / (double)px > s->bytes_per_pixel) s->bytes_per_pixel = (double)arena / (double)px;
            if (arena > s->st.peak_arena_bytes) s->st.peak_arena_bytes = arena;
        }
        s->cv_done.notify_all();
    }
}

extern "C" {

at_server *at_server_create(const at_detector *params, const at_server_config *cfg) {
    if (params == nullptr) return nullptr;
    at_server *s = new at_server();
    at_server_config c{};
    c.workers = 2;
    c.max_batch = 16;
    c.memory_budget = (int64_t)24 << 30;
    if (cfg) {
        if (cfg->workers > 0) c.workers = cfg->workers;
        if (cfg->max_batch > 0) c.max_batch = cfg->max_batch;
        if (cfg->memory_budget > 0) c.memory_budget = cfg->memory_budget;
    }
    // the GPUs: the current one, or those of the mask (one detector replica
    // per worker, workers dealt out over the GPUs in turn; frames are
    // independent, so nothing passes between the replicas)
    int cur = 0, ndev = 0;
    cudaGetDevice(&cur);
    cudaGetDeviceCount(&ndev);
    std::vector<int> devs;
    const uint32_t mask = cfg ? cfg->device_mask : 0u;
    if (mask == 0) devs.push_back(cur);
    for (int d = 0; d < 32 && d < ndev; d++)
        if (mask & (1u << d)) devs.push_back(d);
    if (devs.empty()) {
        delete s;
        return nullptr;
    }
    c.device_mask = mask;
    s->cfg = c;
    for (int w = 0; w < c.workers; w++) {
        s->dev_of.push_back(devs[w % devs.size()]);
        cudaSetDevice(s->dev_of[w]);
        s->dets.push_back(at_detector_clone(params));
    }
    cudaSetDevice(cur);
    for (int w = 0; w < c.workers; w++) s->threads.emplace_back(worker, s, w);
    return s;
}

uint64_t at_server_submit(at_server *s, const at_frame *frame, uint64_t user) {
    if (s == nullptr || frame == nullptr || frame->pixels == nullptr || frame->width <= 0 || frame->height <= 0)
        return 0;
    std::lock_guard<std::mutex> lk(s->mu);
    const int64_t est = (int64_t)(s->bytes_per_pixel * (double)(frame->width * frame->height));
    const int64_t share = s->cfg.memory_budget / s->cfg.workers;
    // a frame is admitted while the device bytes of everything pending or
    // running, this frame included, stay within the budget (and it fits
    // one worker's share on its own)
    if (s->stop || est > share || s->queued_bytes + est > s->cfg.memory_budget) {
        s->st.rejected++;
        return 0;
    }
    Request r{s->next_ticket++, user, *frame, now_s(), est};
    s->pending.push_back(r);
    s->queued_bytes += est;
    s->st.admitted++;
    s->cv_work.notify_one();
    return r.ticket;
}

int at_server_worker_device(const at_server *s, int32_t worker) {
    if (s == nullptr || worker < 0 || worker >= (int32_t)s->dev_of.size()) return -1;
    return s->dev_of[worker];
}

int at_server_cancel(at_server *s, uint64_t ticket) {
    if (s == nullptr) return 0;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (auto it = s->pending.begin(); it != s->pending.end(); ++it) {
            if (it->ticket != ticket) continue;
            at_server_result o;
            memset(&o, 0, sizeof o);
            o.ticket = it->ticket;
            o.user = it->user;
            o.status = AT_SERVER_CANCELLED;
            o.worker = -1;
            o.t_submit = it->t_submit;
            o.t_start = o.t_done = now_s();
            s->queued_bytes -= it->est;
            s->pending.erase(it);
            s->done.push_back(o);
            s->st.cancelled++;
            s->cv_done.notify_all();
            return 1;
        }
    }
    return 0;
}

int64_t at_server_poll(at_server *s, at_server_result *out, int64_t max, int32_t wait_ms) {
    if (s == nullptr || out == nullptr || max <= 0) return 0;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && wait_ms > 0)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->done.empty(); });
    int64_t n = 0;
    while (n < max && !s->done.empty()) {
        out[n++] = s->done.front();
        s->done.pop_front();
    }
    return n;
}

void at_server_free_result(at_server_result *r) {
    if (r == nullptr) return;
    free(r->detections);
    r->detections = nullptr;
    r->ndetections = 0;
}

void at_server_get_stats(at_server *s, at_server_stats *out) {
    if (s == nullptr || out == nullptr) return;
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->st;
    out->pending = (int64_t)s->pending.size();
    out->bytes_per_pixel = s->bytes_per_pixel;
}

void at_server_destroy(at_server *s) {
    if (s == nullptr) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto &t : s->threads) t.join();
    int cur = 0;
    cudaGetDevice(&cur);
    for (size_t w = 0; w < s->dets.size(); w++) {  // each replica on its own GPU
        cudaSetDevice(s->dev_of[w]);
        at_detector_destroy(s->dets[w]);
    }
    cudaSetDevice(cur);
    for (auto &r : s->done) free(r.detections);
    delete s;
}

}  // extern "C"
