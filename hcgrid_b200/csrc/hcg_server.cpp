// Request loop for serving gridding jobs (continuous batching).
//
// Clients submit jobs (a resident field, a target and device output
// buffers) as they arrive. A dispatcher thread hands pending jobs to one of
// `lanes` worker lanes while their HBM footprint fits the budget. A job whose
// channel sums fill the GPU by themselves (2^20 target pixels or more, or at
// least one channel-sum item per SM) runs alone, with the GPU to itself,
// through hcg_grid; smaller jobs run in batches (at most `max_batch`, through
// hcg_grid_batch's persistent kernels). The oldest pending job decides what
// runs next. If it is small, every pending small job joins its batch in
// arrival order, large ones skipped, so large jobs between them do not split
// the batch. If it is large, it waits for the GPU to be idle; meanwhile the
// small jobs queued behind it may pass it on a free lane, at most kMaxPasses
// batches, so a large job is not starved. Each lane owns its own context
// (stream + captured batch graphs) on the same device, so a batch that
// arrives while another batch is on the GPU is launched right away and the
// two overlap on the device. When a lane finishes, its footprint is released
// and the dispatcher admits more jobs. Every job records submit, start and
// finish times (host steady clock), from which the latency percentiles are
// taken.
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "hcgrid_c.h"

namespace hcg {  // hcg_capi.cu
bool job_fills_gpu(const hcg_job &job, int nsm);            // the job's channel sums fill the GPU alone
hcg_status grid_job(hcg_context *ctx, const hcg_job &job);  // hcg_grid of one job on a lane's context
int device_sms(int device);                                 // streaming multiprocessors of a device
}

namespace {

using Clock = std::chrono::steady_clock;
constexpr uint32_t kMaxPasses = 2;  // batches that may pass a waiting large job

struct Pending {
    uint64_t ticket;
    hcg_job job;
    uint64_t bytes;
    double t_submit;
    bool large;
    uint32_t passed = 0;  // batches dispatched while this job waited at the queue's head
};

struct Done {
    double t_submit = 0, t_start = 0, t_done = 0;
    hcg_status status = HCG_OK;
    uint32_t batch = 0;
    bool finished = false;
};

}  // namespace

struct hcg_server {
    hcg_context *primary = nullptr;
    std::vector<hcg_context *> lanes;
    uint64_t budget = 0, in_use = 0;
    uint32_t max_batch = 64;
    int nsm = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Pending> queue;
    std::unordered_map<uint64_t, Done> done;
    std::vector<bool> lane_busy;
    std::vector<std::thread> workers;
    std::thread dispatcher;
    std::vector<std::vector<Pending>> lane_batch;
    std::vector<char> lane_single;  // the lane's work is one large job (hcg_grid)
    bool stop = false;          // no more submissions; the dispatcher leaves once the queue is empty
    bool workers_stop = false;  // set after the dispatcher has left: lanes finish their work and leave
    uint64_t next_ticket = 1;
    uint32_t batches = 0;
    Clock::time_point t0 = Clock::now();
    std::string err;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

    void worker(size_t li) {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            cv_work.wait(lk, [&] { return workers_stop || !lane_batch[li].empty(); });
            if (lane_batch[li].empty() && workers_stop) return;
            std::vector<Pending> b;
            b.swap(lane_batch[li]);
            const bool single = lane_single[li];
            uint32_t bid = ++batches;
            lk.unlock();
            double ts = now();
            hcg_status st;
            if (single) {
                st = hcg::grid_job(lanes[li], b[0].job);
            } else {
                std::vector<hcg_job> jobs(b.size());
                for (size_t i = 0; i < b.size(); ++i) jobs[i] = b[i].job;
                st = hcg_grid_batch(lanes[li], (uint32_t)jobs.size(), jobs.data());
            }
            double td = now();
            lk.lock();
            for (auto &p : b) {
                Done &d = done[p.ticket];
                d.t_start = ts;
                d.t_done = td;
                d.status = st;
                d.batch = bid;
                d.finished = true;
                in_use -= std::min(in_use, p.bytes);
            }
            if (st != HCG_OK) err = hcg_last_error(lanes[li]);
            lane_busy[li] = false;
            cv_done.notify_all();
            cv_work.notify_all();
        }
    }

    void dispatch() {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            size_t busy = 0;
            bool busy_single = false;
            auto any_small = [&] {
                for (const Pending &p : queue)
                    if (!p.large) return true;
                return false;
            };
            cv_work.wait(lk, [&] {
                if (stop && queue.empty()) return true;
                if (queue.empty()) return false;
                busy = 0;
                busy_single = false;
                for (size_t i = 0; i < lanes.size(); ++i) {
                    busy += lane_busy[i] ? 1 : 0;
                    busy_single |= lane_busy[i] && lane_single[i];
                }
                if (busy_single || busy == lanes.size()) return false;
                const Pending &f = queue.front();
                if (!f.large || busy == 0) return true;
                return f.passed < kMaxPasses && any_small();
            });
            if (stop && queue.empty()) {
                cv_work.notify_all();
                return;
            }
            size_t li = 0;
            while (li < lanes.size() && lane_busy[li]) ++li;
            if (li == lanes.size()) continue;
            std::vector<Pending> b;
            const bool single = queue.front().large && busy == 0;
            if (single) {  // nothing else is resident: the budget holds it
                b.push_back(queue.front());
                in_use += b[0].bytes;
                queue.pop_front();
            } else {
                // the pending small jobs in arrival order, while the footprint
                // fits (one larger than the whole budget runs once nothing
                // else is resident)
                const bool passing = queue.front().large;
                std::deque<Pending> rest;
                bool full = false;
                for (Pending &p : queue) {
                    if (full || p.large || b.size() >= max_batch) {
                        rest.push_back(p);
                        continue;
                    }
                    if (in_use + p.bytes > budget && !(in_use == 0 && b.empty())) {
                        full = true;
                        rest.push_back(p);
                        continue;
                    }
                    in_use += p.bytes;
                    b.push_back(p);
                }
                queue.swap(rest);
                if (passing && !b.empty()) ++queue.front().passed;
            }
            if (b.empty()) {  // wait for memory to be released
                cv_done.wait(lk);
                continue;
            }
            lane_busy[li] = true;
            lane_single[li] = single;
            lane_batch[li] = std::move(b);
            cv_work.notify_all();
        }
    }
};

extern "C" {

hcg_status hcg_server_create(hcg_context *ctx, int device, uint32_t lanes, uint64_t hbm_budget_bytes,
                             uint32_t max_batch, hcg_server **out) {
    if (!ctx || !out || lanes == 0 || lanes > 8 || max_batch == 0) return HCG_EINVAL;
    hcg_server *s = new hcg_server();
    s->primary = ctx;
    s->budget = hbm_budget_bytes;
    s->max_batch = max_batch;
    s->nsm = hcg::device_sms(device);
    s->lanes.push_back(ctx);
    for (uint32_t i = 1; i < lanes; ++i) {
        hcg_context *c = nullptr;
        hcg_status st = hcg_context_create(device, nullptr, &c);
        if (st != HCG_OK) {
            for (size_t k = 1; k < s->lanes.size(); ++k) hcg_context_destroy(s->lanes[k]);
            delete s;
            return st;
        }
        s->lanes.push_back(c);
    }
    s->lane_busy.assign(lanes, false);
    s->lane_batch.resize(lanes);
    s->lane_single.assign(lanes, 0);
    for (uint32_t i = 0; i < lanes; ++i) s->workers.emplace_back([s, i] { s->worker(i); });
    s->dispatcher = std::thread([s] { s->dispatch(); });
    *out = s;
    return HCG_OK;
}

hcg_status hcg_server_submit(hcg_server *s, const hcg_job *job, uint64_t footprint_bytes, uint64_t *ticket) {
    if (!s || !job || !ticket) return HCG_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return HCG_ESTATE;
    Pending p{s->next_ticket++, *job, footprint_bytes, s->now(), hcg::job_fills_gpu(*job, s->nsm)};
    s->done[p.ticket].t_submit = p.t_submit;
    *ticket = p.ticket;
    s->queue.push_back(p);
    s->cv_work.notify_all();
    return HCG_OK;
}

hcg_status hcg_server_wait(hcg_server *s, uint64_t ticket, double *latency_s, double *queue_s) {
    if (!s) return HCG_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->done.find(ticket);
    if (it == s->done.end()) return HCG_EINVAL;
    s->cv_done.wait(lk, [&] { return s->done[ticket].finished; });
    const Done &d = s->done[ticket];
    if (latency_s) *latency_s = d.t_done - d.t_submit;
    if (queue_s) *queue_s = d.t_start - d.t_submit;
    return d.status;
}

hcg_status hcg_server_drain(hcg_server *s) {
    if (!s) return HCG_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait(lk, [&] {
        if (!s->queue.empty()) return false;
        for (bool b : s->lane_busy)
            if (b) return false;
        return true;
    });
    return s->err.empty() ? HCG_OK : HCG_EDEVICE;
}

/* Latency percentiles (seconds) over all finished jobs, and counts. */
hcg_status hcg_server_stats(hcg_server *s, double *p50, double *p99, uint64_t *jobs, uint32_t *batches) {
    if (!s) return HCG_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    std::vector<double> lat;
    for (auto &kv : s->done)
        if (kv.second.finished) lat.push_back(kv.second.t_done - kv.second.t_submit);
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double q) {
        if (lat.empty()) return 0.0;
        size_t i = (size_t)std::min<double>(lat.size() - 1, q * (lat.size() - 1) + 0.5);
        return lat[i];
    };
    if (p50) *p50 = pct(0.50);
    if (p99) *p99 = pct(0.99);
    if (jobs) *jobs = lat.size();
    if (batches) *batches = s->batches;
    return HCG_OK;
}

hcg_status hcg_server_destroy(hcg_server *s) {
    if (!s) return HCG_EINVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    s->dispatcher.join();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->workers_stop = true;
        s->cv_work.notify_all();
    }
    for (auto &w : s->workers) w.join();
    for (size_t k = 1; k < s->lanes.size(); ++k) hcg_context_destroy(s->lanes[k]);
    delete s;
    return HCG_OK;
}

}  // extern "C"
