// Batched and streamed Seed Check jobs: the scheduler that flattens jobs with different seed
// counts, rects and floors into shared phase-1 batches (wg_seed_check_jobs), and the job server
// built on it (wg_server_*: a worker thread with its own engine, continuous batching).
//
// The reference runs one job per process invocation (phase1_scan --worker, one request line at a
// time: engine/gpu/low54/phase1_scan.cu:1328-1387) or one lysh session per seed
// (engine/tools/lysh/src/eval.h:180-205); the results per job are the same as there.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "../../include/witchgpu.h"
#include "wg_device.cuh"
#include "wg_jobs.h"
#include "wg_queue.h"

namespace wg {

namespace {

constexpr uint64_t kMaxRectSide = 1ull << 24;
constexpr uint64_t kStageSeeds = 1ull << 21;   // pinned staging for the seeds of small jobs (16 MiB)

bool same_rules(const SchedJob &x, const SchedJob &y) {
    return x.salt == y.salt && x.opts.mc_1_18_2 == y.opts.mc_1_18_2 && x.opts.single_biome == y.opts.single_biome &&
           x.opts.pre_26_2 == y.opts.pre_26_2 && x.opts.large_biomes == y.opts.large_biomes;
}

bool candidate_order(const Candidate &x, const Candidate &y) {
    if (x.seed_index != y.seed_index) return x.seed_index < y.seed_index;
    if (x.rz != y.rz) return x.rz < y.rz;
    return x.rx < y.rx;
}

// Whether a job's climate coordinates are proved inside maintainPrecision's identity range.
bool job_small(const SchedJob &j) {
    const int64_t rh = (int64_t)(j.n_regions / (uint64_t)j.rw);
    return coords_small(std::min<int64_t>(j.rx0, j.rz0), std::max<int64_t>(j.rx0 + j.rw, j.rz0 + rh) - 1);
}

}  // namespace

int sched_job_init(SchedJob &j, const wg_job &spec, const wg_engine *eng) {
    if (spec.n_seeds == 0 || spec.rx1 <= spec.rx0 || spec.rz1 <= spec.rz0) return WG_ERR_ARG;
    const uint64_t rw = (uint64_t)((int64_t)spec.rx1 - spec.rx0), rh = (uint64_t)((int64_t)spec.rz1 - spec.rz0);
    if (rw > kMaxRectSide || rh > kMaxRectSide) return WG_ERR_ARG;
    j.opts = spec.opts;
    j.salt = spec.salt ? spec.salt : 14357620;
    j.max_height = spec.max_height;
    j.rx0 = spec.rx0;
    j.rz0 = spec.rz0;
    j.rw = (int)rw;
    j.n_regions = rw * rh;
    j.win = job_window(eng, j.n_regions);
    j.n_win = (j.n_regions + j.win - 1) / j.win;
    if (spec.n_seeds > ~0ull / j.n_win) return WG_ERR_ARG;
    j.units = spec.n_seeds * j.n_win;
    try {
        j.seeds.resize(spec.n_seeds);
    } catch (...) {
        return WG_ERR_NOMEM;
    }
    if (spec.seeds) std::memcpy(j.seeds.data(), spec.seeds, sizeof(int64_t) * spec.n_seeds);
    else
        for (uint64_t i = 0; i < spec.n_seeds; i++) j.seeds[i] = (int64_t)splitmix64(spec.gen_base + i);
    return WG_OK;
}

Scheduler::Scheduler(wg_engine *eng, uint64_t arena_seeds, uint64_t step_work)
    : eng_(eng), arena_cap_(std::max<uint64_t>(arena_seeds, 1)), step_work_(std::max<uint64_t>(step_work, 1)) {}

Scheduler::~Scheduler() {
    cudaFree(d_arena_);
    cudaFree(d_table_);
    cudaFreeHost(h_table_);
    cudaFreeHost(h_stage_);
}

int Scheduler::init() {
    cudaError_t e = cudaMalloc(&d_arena_, sizeof(int64_t) * arena_cap_);
    if (e != cudaSuccess) return eng_->fail(WG_ERR_NOMEM, "job seed arena", e);
    stage_cap_ = std::min<uint64_t>(arena_cap_, kStageSeeds);
    e = cudaMallocHost(&h_stage_, sizeof(int64_t) * stage_cap_);
    if (e != cudaSuccess) return eng_->fail(WG_ERR_NOMEM, "seed staging buffer", e);
    free_.clear();
    free_[0] = arena_cap_;
    return WG_OK;
}

uint64_t Scheduler::alloc(uint64_t n) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {   // first fit
        if (it->second < n) continue;
        const uint64_t off = it->first, len = it->second;
        free_.erase(it);
        if (len > n) free_[off + n] = len - n;
        return off;
    }
    return ~0ull;
}

void Scheduler::release(uint64_t off, uint64_t n) {
    auto it = free_.emplace(off, n).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {   // merge with the next range
        it->second += next->second;
        free_.erase(next);
    }
    if (it != free_.begin()) {   // and with the previous one
        auto prev = std::prev(it);
        if (prev->first + prev->second == it->first) {
            prev->second += it->second;
            free_.erase(it);
        }
    }
}

int Scheduler::flush_uploads() {
    // runs that continue each other in both buffers go up as one copy
    size_t i = 0;
    while (i < runs_.size()) {
        Run r = runs_[i++];
        while (i < runs_.size() && runs_[i].arena_off == r.arena_off + r.n && runs_[i].stage_off == r.stage_off + r.n)
            r.n += runs_[i++].n;
        cudaError_t e = cudaMemcpyAsync(d_arena_ + r.arena_off, h_stage_ + r.stage_off, sizeof(int64_t) * r.n,
                                        cudaMemcpyHostToDevice, eng_->stream);
        if (e != cudaSuccess) return eng_->fail(WG_ERR_CUDA, "upload job seeds", e);
    }
    runs_.clear();
    return WG_OK;
}

bool Scheduler::admit(SchedJob *j, int *rc) {
    *rc = WG_OK;
    const uint64_t n = j->seeds.size();
    const uint64_t off = alloc(n);
    if (off == ~0ull) return false;
    cudaError_t e = cudaSuccess;
    if (n > stage_cap_ / 4) {
        // a large job goes straight from its (pageable) host copy, read before the call returns
        e = cudaMemcpyAsync(d_arena_ + off, j->seeds.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice,
                            eng_->stream);
    } else {
        if (stage_used_ + n > stage_cap_) {   // staging full: send what it holds and reuse it
            *rc = flush_uploads();
            if (*rc == WG_OK) e = cudaStreamSynchronize(eng_->stream);
            stage_used_ = 0;
        }
        if (*rc == WG_OK && e == cudaSuccess) {
            std::memcpy(h_stage_ + stage_used_, j->seeds.data(), sizeof(int64_t) * n);
            runs_.push_back(Run{off, stage_used_, n});
            stage_used_ += n;
        }
    }
    if (*rc == WG_OK && e != cudaSuccess) *rc = eng_->fail(WG_ERR_CUDA, "upload job seeds", e);
    if (*rc) {
        release(off, n);
        return false;
    }
    j->arena_off = off;
    order_.insert(j);
    return true;
}

int Scheduler::step(std::vector<SchedJob *> &finished, std::vector<SchedJob *> &members) {
    members.clear();
    last_suspect_ = nullptr;
    if (order_.empty()) return WG_OK;
    SchedJob *alone = suspects_.empty() ? nullptr : *suspects_.begin();   // a suspect runs by itself
    last_suspect_ = alone;
    int rc = flush_uploads();   // the staged seeds of newly admitted jobs
    if (rc) return rc;
    const SchedJob &lead = alone ? *alone : **order_.begin();
    uint64_t budget = step_work_;
    if (lead.opts.single_biome)   // every region survives the climate stage
        budget = std::min<uint64_t>(budget, kCapSurv / 2);
    std::vector<JobGeom> &table = table_;
    table.clear();
    std::vector<uint64_t> took;
    uint64_t units = 0;
    int misses = 0;   // consecutive jobs whose windows no longer fit the budget
    for (SchedJob *j : order_) {
        if (units >= kMaxUnits || budget == 0 || misses >= 64) break;
        if (!same_rules(*j, lead) || (alone && j != alone)) continue;
        uint64_t k = std::min<uint64_t>(j->units - j->dispatched, kMaxUnits - units);
        uint64_t kb = budget / j->win;
        if (kb == 0) {
            if (units) {
                misses++;
                continue;
            }
            kb = 1;
        }
        misses = 0;
        k = std::min(k, kb);
        JobGeom g;
        std::memset(&g, 0, sizeof g);
        g.unit0 = units;
        g.first = j->dispatched;
        g.seed0 = j->arena_off;
        g.n_win = j->n_win;
        g.n_regions = j->n_regions;
        g.win = j->win;
        g.rx0 = j->rx0;
        g.rz0 = j->rz0;
        g.rw = j->rw;
        g.max_height = j->max_height;
        table.push_back(g);
        took.push_back(k);
        members.push_back(j);
        units += k;
        budget -= std::min(budget, k * (uint64_t)j->win);
    }
    // the table: pinned host copy (rewritten only after the batch's closing sync) -> device
    if (table.size() > table_cap_) {
        cudaFree(d_table_);
        cudaFreeHost(h_table_);
        d_table_ = nullptr;
        h_table_ = nullptr;
        table_cap_ = 0;
        const uint32_t cap = (uint32_t)std::max<size_t>(table.size() * 2, 256);
        cudaError_t e = cudaMalloc(&d_table_, sizeof(JobGeom) * cap);
        if (e == cudaSuccess) e = cudaMallocHost(&h_table_, sizeof(JobGeom) * cap);
        if (e != cudaSuccess) return eng_->fail(WG_ERR_NOMEM, "job table", e);
        table_cap_ = cap;
    }
    std::memcpy(h_table_, table.data(), sizeof(JobGeom) * table.size());
    cudaError_t e = cudaMemcpyAsync(d_table_, h_table_, sizeof(JobGeom) * table.size(), cudaMemcpyHostToDevice,
                                    eng_->stream);
    if (e != cudaSuccess) return eng_->fail(WG_ERR_CUDA, "upload job table", e);

    if (fail_job)
        for (const SchedJob *j : members)
            if (j->id == fail_job) return eng_->fail(WG_ERR_CUDA, "injected batch failure");

    BatchArgs a = base_args(eng_, lead.opts, lead.salt);
    a.seeds = d_arena_;
    a.jobs = d_table_;
    a.n_jobs = (uint32_t)table.size();
    a.small_coords = 1;
    for (const SchedJob *j : members) a.small_coords &= job_small(*j) ? 1 : 0;
    found_.clear();
    Sink sink;
    sink.host = &found_;
    rc = run_batch(eng_, a, 0, (uint32_t)units, sink, stats);
    stage_used_ = 0;   // the batch's closing sync also ended the staged copies
    if (rc) return rc;
    if (alone) suspects_.erase(alone);   // it passed by itself: an ordinary job again
    last_suspect_ = nullptr;

    // survivors back to their jobs: seed_index is an arena slot until here
    std::vector<std::pair<uint64_t, size_t>> by_off(members.size());
    for (size_t i = 0; i < members.size(); i++) by_off[i] = {members[i]->arena_off, i};
    std::sort(by_off.begin(), by_off.end());
    for (Candidate c : found_) {
        auto it = std::upper_bound(by_off.begin(), by_off.end(), std::make_pair(c.seed_index, ~(size_t)0));
        if (it == by_off.begin()) continue;   // not reachable: every slot belongs to a member
        --it;
        SchedJob *j = members[it->second];
        c.seed_index -= j->arena_off;
        if (c.seed_index >= j->seeds.size()) continue;
        j->found.push_back(c);
    }
    for (size_t i = 0; i < members.size(); i++) {
        SchedJob *j = members[i];
        order_.erase(j);   // its key changes
        j->dispatched += took[i];
        if (j->dispatched < j->units) {
            order_.insert(j);
            continue;
        }
        std::sort(j->found.begin(), j->found.end(), candidate_order);
        release(j->arena_off, j->seeds.size());
        stats.scanned += (int64_t)(j->seeds.size() * j->n_regions);
        stats.accepted += (int64_t)j->found.size();
        finished.push_back(j);
    }
    return WG_OK;
}

void Scheduler::fail_all(int rc, std::vector<SchedJob *> &finished) {
    cudaStreamSynchronize(eng_->stream);   // no staged copy may still read the staging buffer
    for (SchedJob *j : order_) {
        j->status = rc;
        release(j->arena_off, j->seeds.size());
        finished.push_back(j);
    }
    order_.clear();
    suspects_.clear();
    last_suspect_ = nullptr;
    runs_.clear();
    stage_used_ = 0;
}

void Scheduler::isolate(const std::vector<SchedJob *> &members) {
    for (SchedJob *j : members) suspects_.insert(j);
}

void Scheduler::fail_suspect(int rc, std::vector<SchedJob *> &finished) {
    SchedJob *j = last_suspect_;
    last_suspect_ = nullptr;
    if (!j) return;
    cudaStreamSynchronize(eng_->stream);   // no staged copy may still read the staging buffer
    order_.erase(j);
    suspects_.erase(j);
    j->status = rc;
    release(j->arena_off, j->seeds.size());
    finished.push_back(j);
}

// Whether an engine can run more batches after a failure: a non-sticky error is cleared here; a
// broken context fails the synchronisation.
bool engine_usable(wg_engine *eng) {
    cudaGetLastError();
    return cudaStreamSynchronize(eng->stream) == cudaSuccess && cudaGetLastError() == cudaSuccess;
}

}  // namespace wg

using namespace wg;

namespace {

// The jobs through the device work queue: every job's seeds resident at once, one job table per
// rule set, one graph launch per table (wg_queue.cu).  Returns WG_ERR_CAPACITY when the jobs do not
// fit (the caller then takes the host batch loop).
int jobs_on_device_queue(wg_engine *eng, std::vector<SchedJob> &js, uint64_t total_seeds, wg_scan_stats &st) {
    constexpr uint64_t kQueueSeeds = 1ull << 27;
    if (total_seeds > kQueueSeeds) return WG_ERR_CAPACITY;
    int64_t *d_seeds = nullptr;
    JobGeom *d_table = nullptr;
    std::vector<int64_t> all;
    std::vector<uint64_t> off(js.size());
    all.reserve(total_seeds);
    for (size_t i = 0; i < js.size(); i++) {
        off[i] = all.size();
        all.insert(all.end(), js[i].seeds.begin(), js[i].seeds.end());
    }
    std::vector<char> done(js.size(), 0);
    int rc = [&]() -> int {
        cudaError_t e = cudaMalloc(&d_seeds, sizeof(int64_t) * std::max<size_t>(all.size(), 1));
        if (e == cudaSuccess) e = cudaMalloc(&d_table, sizeof(JobGeom) * js.size());
        if (e != cudaSuccess) return eng->fail(WG_ERR_NOMEM, "job queue buffers", e);
        e = cudaMemcpyAsync(d_seeds, all.data(), sizeof(int64_t) * all.size(), cudaMemcpyHostToDevice, eng->stream);
        if (e != cudaSuccess) return eng->fail(WG_ERR_CUDA, "upload job seeds", e);
        for (size_t lead = 0; lead < js.size(); lead++) {
            if (done[lead]) continue;
            // one table: the lead's rule set
            std::vector<JobGeom> table;
            std::vector<size_t> member;
            uint64_t units = 0;
            uint32_t min_win = ~0u;
            for (size_t i = lead; i < js.size(); i++) {
                if (done[i] || !same_rules(js[i], js[lead])) continue;
                JobGeom g;
                std::memset(&g, 0, sizeof g);
                g.unit0 = units;
                g.seed0 = off[i];
                g.n_win = js[i].n_win;
                g.n_regions = js[i].n_regions;
                g.win = js[i].win;
                g.rx0 = js[i].rx0;
                g.rz0 = js[i].rz0;
                g.rw = js[i].rw;
                g.max_height = js[i].max_height;
                table.push_back(g);
                member.push_back(i);
                units += js[i].units;
                min_win = std::min(min_win, js[i].win);
                done[i] = 1;
            }
            e = cudaMemcpyAsync(d_table, table.data(), sizeof(JobGeom) * table.size(), cudaMemcpyHostToDevice,
                                eng->stream);
            if (e != cudaSuccess) return eng->fail(WG_ERR_CUDA, "upload job table", e);
            const uint64_t budget = eng->tuned_budget ? eng->tuned_budget : kWorkPerBatch;
            const uint64_t by_budget = (budget + min_win - 1) / min_win;
            const uint32_t max_units = (uint32_t)std::min<uint64_t>({(uint64_t)kMaxUnits, units, std::max<uint64_t>(by_budget, 1)});
            BatchArgs a = base_args(eng, js[lead].opts, js[lead].salt);
            a.seeds = d_seeds;
            a.jobs = d_table;
            a.n_jobs = (uint32_t)table.size();
            a.small_coords = 1;
            for (size_t k : member) a.small_coords &= job_small(js[k]) ? 1 : 0;
            std::vector<Candidate> found;
            const uint64_t slice = js[lead].opts.single_biome ? std::min<uint64_t>(budget, kCapSurv / 2) : budget;
            int r = run_queue(eng, a, units, max_units, slice, found, st);
            if (r) return r;
            // survivors back to their jobs: seed_index is a slot of the concatenated seed list
            std::vector<std::pair<uint64_t, size_t>> by_off(member.size());
            for (size_t k = 0; k < member.size(); k++) by_off[k] = {off[member[k]], member[k]};
            std::sort(by_off.begin(), by_off.end());
            for (Candidate c : found) {
                auto it = std::upper_bound(by_off.begin(), by_off.end(), std::make_pair(c.seed_index, ~(size_t)0));
                if (it == by_off.begin()) continue;
                --it;
                SchedJob &j = js[it->second];
                c.seed_index -= it->first;
                if (c.seed_index >= j.seeds.size()) continue;
                j.found.push_back(c);
            }
        }
        return WG_OK;
    }();
    cudaFree(d_seeds);
    cudaFree(d_table);
    if (rc) return rc;
    for (SchedJob &j : js) {
        std::sort(j.found.begin(), j.found.end(), candidate_order);
        st.scanned += (int64_t)(j.seeds.size() * j.n_regions);
        st.accepted += (int64_t)j.found.size();
    }
    return WG_OK;
}

}  // namespace

extern "C" int wg_seed_check_jobs(wg_engine *eng, const wg_job *jobs, uint64_t n_jobs, wg_candidate *out,
                                  uint64_t cap, uint64_t *n_out, uint64_t *job_found, wg_scan_stats *stats) {
    if (!eng || (n_jobs && !jobs) || (cap && !out)) return WG_ERR_ARG;
    const auto t0 = Clock::now();
    cudaError_t e = cudaSetDevice(eng->device);
    if (e != cudaSuccess) return eng->fail(WG_ERR_CUDA, "cudaSetDevice", e);
    std::vector<SchedJob> js(n_jobs);
    uint64_t total = 0, largest = 0;
    for (uint64_t i = 0; i < n_jobs; i++) {
        const int rc = sched_job_init(js[i], jobs[i], eng);
        if (rc) return eng->fail(rc, rc == WG_ERR_NOMEM ? "job seeds" : "job: empty or oversized");
        js[i].id = i;
        total += js[i].seeds.size();
        largest = std::max<uint64_t>(largest, js[i].seeds.size());
    }
    if (eng->job_queue && n_jobs) {
        wg_scan_stats qst{};
        e = cudaEventRecord(eng->ev0, eng->stream);
        if (e != cudaSuccess) return eng->fail(WG_ERR_CUDA, "event", e);
        int rc = jobs_on_device_queue(eng, js, total, qst);
        if (rc == WG_OK) {
            e = cudaEventRecord(eng->ev1, eng->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(eng->ev1);
            if (e != cudaSuccess) return eng->fail(WG_ERR_CUDA, "event", e);
            uint64_t w = 0, all = 0;
            for (uint64_t i = 0; i < n_jobs; i++) {
                if (job_found) job_found[i] = js[i].found.size();
                for (const Candidate &c : js[i].found) {
                    if (w < cap) std::memcpy(&out[w++], &c, sizeof c);
                    all++;
                }
            }
            if (n_out) *n_out = all;
            if (stats) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, eng->ev0, eng->ev1);
                qst.gpu_ms = ms;
                qst.wall_ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
                *stats = qst;
            }
            return WG_OK;
        }
        if (rc != WG_ERR_CAPACITY) return rc;
        // too large for one resident queue: the host batch loop below
        for (SchedJob &j : js) j.found.clear();
    }
    // seeds resident on the device at once: all of them, up to 2^27 (1 GiB), and the largest job
    Scheduler sched(eng, std::min<uint64_t>(std::max<uint64_t>(total, 1), std::max<uint64_t>(largest, 1ull << 27)),
                    kWorkPerBatch);
    int rc = sched.init();
    if (rc) return rc;
    e = cudaEventRecord(eng->ev0, eng->stream);
    if (e != cudaSuccess) return eng->fail(WG_ERR_CUDA, "event", e);
    std::vector<SchedJob *> finished, members;
    uint64_t next = 0, n_done = 0;
    while (n_done < n_jobs) {
        while (next < n_jobs && sched.admit(&js[next], &rc)) next++;
        if (rc) return rc;
        rc = sched.step(finished, members);
        if (rc) return rc;
        n_done += finished.size();
        finished.clear();
        if (sched.idle() && next < n_jobs && n_done < n_jobs && members.empty())
            return eng->fail(WG_ERR_CAPACITY, "job does not fit the seed arena");
    }
    e = cudaEventRecord(eng->ev1, eng->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(eng->ev1);
    if (e != cudaSuccess) return eng->fail(WG_ERR_CUDA, "event", e);
    uint64_t w = 0, all = 0;
    for (uint64_t i = 0; i < n_jobs; i++) {
        if (job_found) job_found[i] = js[i].found.size();
        for (const Candidate &c : js[i].found) {
            if (w < cap) std::memcpy(&out[w++], &c, sizeof c);
            all++;
        }
    }
    if (n_out) *n_out = all;
    if (stats) {
        wg_scan_stats st = sched.stats;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, eng->ev0, eng->ev1);
        st.gpu_ms = ms;
        st.wall_ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
        *stats = st;
    }
    return WG_OK;
}

// ---------------------------------------------------------------------------------------------
// Job server: submitters queue jobs; one worker thread admits them into the scheduler as seed
// slots free up (FIFO) and runs batch after batch, so jobs that arrive while others are on the
// device join the next batch.  Fields of a job that poll/take read are written under the lock.
// ---------------------------------------------------------------------------------------------
struct wg_server {
    int device = 0;
    wg_engine *eng = nullptr;
    std::unique_ptr<Scheduler> sched;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<SchedJob *> queue;
    std::unordered_map<uint64_t, std::unique_ptr<SchedJob>> jobs;
    uint64_t next_id = 1, queued_seeds = 0, max_queued = 0;
    bool stop = false;
    wg_scan_stats stats{};
};

namespace {

void server_loop(wg_server *s) {
    cudaSetDevice(s->device);
    Scheduler &sched = *s->sched;
    std::vector<SchedJob *> finished, members;
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty() || !sched.idle(); });
            if (s->stop) return;
        }
        // admit in arrival order while the seed arena has room (only this thread pops the queue);
        // a job whose admission fails (its seed upload) ends alone with that status
        for (;;) {
            SchedJob *j = nullptr;
            {
                std::lock_guard<std::mutex> lk(s->mu);
                if (s->queue.empty()) break;
                j = s->queue.front();
            }
            int arc = WG_OK;
            const bool in = sched.admit(j, &arc);
            if (!in && arc == WG_OK) break;   // no room yet
            std::lock_guard<std::mutex> lk(s->mu);
            s->queue.pop_front();
            s->queued_seeds -= j->seeds.size();
            if (!in) {
                j->status = arc;
                j->t_start = j->t_done = Clock::now();
                j->started = j->done = true;
                std::vector<int64_t>().swap(j->seeds);
                s->cv_done.notify_all();
            }
        }
        const auto t_step = Clock::now();
        int rc = sched.step(finished, members);
        bool broken = false;
        if (rc) {
            // Failure isolation: while the engine still works, a failed batch fails no job by
            // itself; its jobs run again one at a time, and only a job that fails alone ends
            // with the error.  A broken context ends every job, queued ones included.
            if (!engine_usable(s->eng)) {
                sched.fail_all(rc, finished);
                broken = true;
            } else if (sched.last_was_suspect()) {
                sched.fail_suspect(rc, finished);
            } else {
                sched.isolate(members);
            }
        }
        const auto t_end = Clock::now();
        std::lock_guard<std::mutex> lk(s->mu);
        for (SchedJob *j : members) {
            if (!j->started) {
                j->started = true;
                j->t_start = t_step;
            }
            j->batch_jobs = std::max<uint64_t>(j->batch_jobs, members.size());
        }
        for (SchedJob *j : finished) {
            if (!j->started) {
                j->started = true;
                j->t_start = t_step;
            }
            j->t_done = t_end;
            j->done = true;
            std::vector<int64_t>().swap(j->seeds);
        }
        if (broken) {   // a broken engine also fails the jobs still queued behind it
            for (SchedJob *j : s->queue) {
                j->status = rc;
                j->t_start = j->t_done = t_end;
                j->started = j->done = true;
            }
            s->queue.clear();
            s->queued_seeds = 0;
        }
        s->stats = sched.stats;
        finished.clear();
        s->cv_done.notify_all();
    }
}

}  // namespace

extern "C" {

int wg_server_open_config(int device, const wg_server_config *cfg, wg_server **out) {
    if (!out) return WG_ERR_ARG;
    *out = nullptr;
    wg_server_config c{};
    if (cfg) c = *cfg;
    auto s = std::make_unique<wg_server>();
    s->device = device;
    int rc = wg_engine_open(device, &s->eng);
    if (rc) return rc;
    // seeds resident on the device: a quarter of the free HBM, at most 2^28 (2 GiB)
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 1ull << 30;
    const uint64_t arena = c.arena_seeds ? c.arena_seeds
                                         : std::max<uint64_t>(1ull << 20, std::min<uint64_t>(free_b / 4 / sizeof(int64_t), 1ull << 28));
    s->max_queued = c.max_queued_seeds ? c.max_queued_seeds : (1ull << 30);
    // small batches keep a short job's wait behind the batch in flight short
    s->sched = std::make_unique<Scheduler>(s->eng, arena, c.batch_checks ? c.batch_checks : kWorkPerBatch / 4);
    s->sched->fail_job = c.fail_job;
    rc = s->sched->init();
    if (rc) {
        s->sched.reset();
        wg_engine_close(s->eng);
        return rc;
    }
    s->worker = std::thread(server_loop, s.get());
    *out = s.release();
    return WG_OK;
}

int wg_server_open(int device, uint64_t max_queued_seeds, wg_server **out) {
    wg_server_config c{};
    c.max_queued_seeds = max_queued_seeds;
    return wg_server_open_config(device, &c, out);
}

int wg_server_submit(wg_server *s, const wg_job *job, uint64_t *job_id) {
    if (!s || !job) return WG_ERR_ARG;
    const auto t = Clock::now();
    auto j = std::make_unique<SchedJob>();
    int rc = sched_job_init(*j, *job, s->eng);
    if (rc) return rc;
    if (j->seeds.size() > s->sched->arena_seeds()) return WG_ERR_CAPACITY;
    j->t_submit = t;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return WG_ERR_ARG;
    if (s->queued_seeds + j->seeds.size() > s->max_queued) return WG_ERR_CAPACITY;
    j->id = s->next_id++;
    if (job_id) *job_id = j->id;
    s->queued_seeds += j->seeds.size();
    s->queue.push_back(j.get());
    s->jobs.emplace(j->id, std::move(j));
    s->cv_work.notify_one();
    return WG_OK;
}

int wg_server_poll(wg_server *s, uint64_t job_id, int wait_ms, wg_job_status *st) {
    if (!s || !st) return WG_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return WG_ERR_ARG;
    SchedJob *j = it->second.get();
    if (wait_ms > 0 && !j->done)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return j->done; });
    std::memset(st, 0, sizeof *st);
    st->done = j->done ? 1 : 0;
    st->status = j->status;
    st->batch_jobs = j->batch_jobs;
    if (j->started) st->queue_ms = std::chrono::duration<double, std::milli>(j->t_start - j->t_submit).count();
    if (j->done) {
        st->found = j->found.size();
        st->latency_ms = std::chrono::duration<double, std::milli>(j->t_done - j->t_submit).count();
    }
    return WG_OK;
}

int wg_server_take(wg_server *s, uint64_t job_id, wg_candidate *out, uint64_t cap, uint64_t *n_out) {
    if (!s || (cap && !out)) return WG_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end() || !it->second->done) return WG_ERR_ARG;
    SchedJob *j = it->second.get();
    if (j->status) return j->status;
    const uint64_t n = j->found.size(), w = std::min<uint64_t>(n, cap);
    if (w) std::memcpy(out, j->found.data(), sizeof(Candidate) * w);
    if (n_out) *n_out = n;
    if (w == n) s->jobs.erase(it);
    return WG_OK;
}

int wg_server_stats(wg_server *s, wg_scan_stats *st) {
    if (!s || !st) return WG_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    *st = s->stats;
    return WG_OK;
}

void wg_server_close(wg_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    s->sched.reset();
    wg_engine_close(s->eng);
    delete s;
}

int wg_engine_set_job_queue(wg_engine *eng, int device_queue) {
    if (!eng || (device_queue != 0 && device_queue != 1)) return WG_ERR_ARG;
    eng->job_queue = device_queue;
    return WG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Autotuner of the batched-job settings: per job class (regions per seed), the regions per unit
// (more regions per unit build fewer Perlin tables per region, fewer give more independent units),
// then the (seed, region) checks per queue slice, each by timing the candidates on the device on
// probe jobs of that class (seed counts log-uniform 1..4,096 as in the uneven-jobs workload, from a
// splitmix64 stream).  The reference tunes its scanner per GPU the same way (a measured sweep of
// launch settings, kept per card).
// ---------------------------------------------------------------------------------------------
namespace {

constexpr int kTuneSides[4] = {3, 13, 41, 129};   // probe rect side of each class (9 .. 16,641 regions)
constexpr int kTuneJobs = 256;

std::vector<wg_job> probe_jobs(int cls, uint64_t stream) {
    std::vector<wg_job> jobs;
    uint64_t k = 0;
    const int side = kTuneSides[cls], r0 = -(side / 2);
    for (int i = 0; i < kTuneJobs; i++) {
        const double u = (double)(splitmix64(stream + k++) >> 11) * 0x1.0p-53;
        const uint64_t n = std::max<uint64_t>(1, (uint64_t)std::floor(std::pow(4096.0, u)));
        wg_job j{};
        j.gen_base = splitmix64(stream + k++);
        j.n_seeds = n;
        j.rx0 = r0;
        j.rx1 = r0 + side;
        j.rz0 = r0;
        j.rz1 = r0 + side;
        j.max_height = -50;
        wg_parse_version("1.19.x~26.1", &j.opts);
        jobs.push_back(j);
    }
    return jobs;
}

// Device time of one device-queue run of the jobs under the engine's current settings.
int time_jobs(wg_engine *eng, const std::vector<wg_job> &spec, double &ms) {
    std::vector<SchedJob> js(spec.size());
    uint64_t total = 0;
    for (size_t i = 0; i < spec.size(); i++) {
        const int rc = sched_job_init(js[i], spec[i], eng);
        if (rc) return eng->fail(rc, "tune: probe job");
        js[i].id = i;
        total += js[i].seeds.size();
    }
    wg_scan_stats st{};
    cudaError_t e = cudaEventRecord(eng->ev0, eng->stream);
    if (e != cudaSuccess) return eng->fail(WG_ERR_CUDA, "event", e);
    const int rc = jobs_on_device_queue(eng, js, total, st);
    if (rc) return rc;
    e = cudaEventRecord(eng->ev1, eng->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(eng->ev1);
    if (e != cudaSuccess) return eng->fail(WG_ERR_CUDA, "event", e);
    float f = 0.f;
    cudaEventElapsedTime(&f, eng->ev0, eng->ev1);
    ms = f;
    return WG_OK;
}

// Best of `reps` device-queue runs: one slow run (another tenant's burst on a shared GPU) must
// not decide the tuning.
int time_jobs_best(wg_engine *eng, const std::vector<wg_job> &spec, int reps, double &ms) {
    ms = 0.0;
    for (int i = 0; i < reps; i++) {
        double t = 0.0;
        const int rc = time_jobs(eng, spec, t);
        if (rc) return rc;
        if (i == 0 || t < ms) ms = t;
    }
    return WG_OK;
}

}  // namespace

extern "C" int wg_engine_tune(wg_engine *eng, wg_tune_report *rep) {
    if (!eng) return WG_ERR_ARG;
    cudaError_t e = cudaSetDevice(eng->device);
    if (e != cudaSuccess) return eng->fail(WG_ERR_CUDA, "cudaSetDevice", e);
    wg_tune_report r;
    std::memset(&r, 0, sizeof r);
    const uint32_t saved_win[4] = {eng->tuned_win[0], eng->tuned_win[1], eng->tuned_win[2], eng->tuned_win[3]};
    const uint64_t saved_budget = eng->tuned_budget;
    std::vector<wg_job> all;
    int rc = WG_OK;
    eng->tuned_budget = 0;
    for (int c = 0; c < 4 && rc == WG_OK; c++) {
        const uint64_t R = (uint64_t)kTuneSides[c] * kTuneSides[c];
        r.max_regions[c] = (uint32_t)std::min<uint64_t>(kJobClassMax[c], 0xFFFFFFFFull);
        // candidates: the whole seed per unit, and splits of it (large rects: 1,024 .. 16,384)
        uint32_t cand[4] = {0, 0, 0, 0};
        if (c < 3) {
            cand[0] = (uint32_t)R;
            cand[1] = (uint32_t)((R + 1) / 2);
        } else {
            cand[0] = 2048;
            cand[1] = 4096;
            cand[2] = 8192;
            cand[3] = 16384;
        }
        const std::vector<wg_job> jobs = probe_jobs(c, 0x7E57000000000000ull + (uint64_t)c * 0x10000ull);
        all.insert(all.end(), jobs.begin(), jobs.end());
        double best = 0.0;
        for (int q = 0; q < 4 && cand[q] && rc == WG_OK; q++) {
            eng->tuned_win[c] = cand[q];
            double ms = 0.0;
            rc = time_jobs(eng, jobs, ms);                 // warm-up of this setting
            if (rc == WG_OK) rc = time_jobs_best(eng, jobs, 3, ms);
            r.window_candidates[c][q] = cand[q];
            r.window_ms[c][q] = ms;
            if (rc == WG_OK && (q == 0 || ms < best)) {
                best = ms;
                r.window[c] = cand[q];
            }
        }
        eng->tuned_win[c] = r.window[c];
    }
    const uint64_t budgets[3] = {1ull << 25, 1ull << 26, 1ull << 27};
    double best = 0.0;
    for (int q = 0; q < 3 && rc == WG_OK; q++) {
        eng->tuned_budget = budgets[q];
        double ms = 0.0;
        rc = time_jobs_best(eng, all, 2, ms);
        r.budget_candidates[q] = budgets[q];
        r.budget_ms[q] = ms;
        if (rc == WG_OK && (q == 0 || ms < best)) {
            best = ms;
            r.budget = budgets[q];
        }
    }
    if (rc) {   // keep the settings the engine had
        for (int c = 0; c < 4; c++) eng->tuned_win[c] = saved_win[c];
        eng->tuned_budget = saved_budget;
        return rc;
    }
    eng->tuned_budget = r.budget;
    if (rep) *rep = r;
    return WG_OK;
}

extern "C" int wg_engine_set_tuning(wg_engine *eng, const uint32_t *window, uint64_t budget) {
    if (!eng) return WG_ERR_ARG;
    for (int c = 0; c < 4; c++) eng->tuned_win[c] = window ? window[c] : 0u;
    eng->tuned_budget = budget;
    return WG_OK;
}
