// Job scheduler behind wg_seed_check_jobs and the job server (wg_jobs.cu): many Seed Check jobs,
// each with its own seeds, rect and floor, flattened into shared phase-1 batches through the job
// table of the kernels' jobs mode (JobGeom).
#pragma once

#include <chrono>
#include <cstdint>
#include <map>
#include <set>
#include <vector>

#include "wg_engine_impl.h"

namespace wg {

using Clock = std::chrono::steady_clock;

struct SchedJob {
    uint64_t id = 0;
    wg_opts opts{};
    int salt = 0;
    int max_height = 0;
    int rx0 = 0, rz0 = 0, rw = 0;
    std::vector<int64_t> seeds;     // host copy (a generator job is expanded at submit)
    uint64_t n_regions = 0, n_win = 0, units = 0;
    uint32_t win = 0;
    uint64_t dispatched = 0;        // units handed to batches so far
    uint64_t arena_off = ~0ull;     // first seed in the device seed arena (~0: not admitted)
    std::vector<Candidate> found;   // survivors so far; seed_index = position in the job
    int status = WG_OK;
    bool started = false, done = false;
    uint64_t batch_jobs = 0;        // most jobs that shared a batch with this one
    Clock::time_point t_submit, t_start, t_done;

    uint64_t remaining_work() const { return (units - dispatched) * (uint64_t)win; }
};

// Fills a SchedJob's geometry and host seeds from a public job description (the window from the
// engine's tuned settings when eng is given); WG_ERR_ARG if the job is empty or its rect is out
// of range.
int sched_job_init(SchedJob &j, const wg_job &spec, const wg_engine *eng);

// Runs the admitted jobs of one engine batch by batch.  Not thread-safe: one thread drives it.
class Scheduler {
   public:
    // arena_seeds: device seed slots (jobs wait for admission while it is full); step_work:
    // (seed, region) checks per batch.
    Scheduler(wg_engine *eng, uint64_t arena_seeds, uint64_t step_work);
    ~Scheduler();
    int init();
    // Admits a job when its seeds fit in the arena (uploads them); returns false if they do not.
    bool admit(SchedJob *j, int *rc);
    // One batch over the admitted jobs (the rule set of the job with the least remaining work,
    // then every admitted job with the same rules and salt, least remaining work first).  Jobs
    // whose last units ran are moved to `finished`.
    // `members` receives the jobs that had units in the batch.
    int step(std::vector<SchedJob *> &finished, std::vector<SchedJob *> &members);
    // Ends every admitted job with status rc (after a failed step) and frees their seed slots.
    void fail_all(int rc, std::vector<SchedJob *> &finished);
    // After a failed step whose engine is still usable: the step's members become suspects, and
    // the following steps run one suspect at a time; a suspect whose own step fails ends with
    // that status (its seed slots freed), the others go on as before.  Units of the failed step
    // were not marked dispatched, so they run again.
    void isolate(const std::vector<SchedJob *> &members);
    // Whether the last failed step ran a single suspect (its failure is that job's own).
    bool last_was_suspect() const { return last_suspect_ != nullptr; }
    // Ends the suspect of the last failed step with status rc.
    void fail_suspect(int rc, std::vector<SchedJob *> &finished);
    bool idle() const { return order_.empty(); }
    uint64_t arena_seeds() const { return arena_cap_; }
    // Host-side fault injection (tests): every step holding the job with this id fails with
    // WG_ERR_CUDA before its kernels are launched (0 = none).
    uint64_t fail_job = 0;
    wg_scan_stats stats{};

   private:
    struct ByWork {   // least remaining work first, then submission order
        bool operator()(const SchedJob *x, const SchedJob *y) const {
            const uint64_t wx = x->remaining_work(), wy = y->remaining_work();
            return wx != wy ? wx < wy : x->id < y->id;
        }
    };
    uint64_t alloc(uint64_t n);
    void release(uint64_t off, uint64_t n);
    int flush_uploads();

    wg_engine *eng_;
    uint64_t arena_cap_, step_work_;
    int64_t *d_arena_ = nullptr;
    JobGeom *d_table_ = nullptr, *h_table_ = nullptr;
    uint32_t table_cap_ = 0;
    std::map<uint64_t, uint64_t> free_;   // free arena ranges: offset -> length
    std::set<SchedJob *, ByWork> order_;   // the admitted jobs (keys change only while out of the set)
    std::vector<Candidate> found_;
    std::vector<JobGeom> table_;
    std::set<SchedJob *> suspects_;       // members of a failed step, run alone until they pass
    SchedJob *last_suspect_ = nullptr;    // the suspect the last step ran alone
    // Seeds of small jobs are gathered in a pinned staging buffer and copied to the arena in
    // runs of consecutive slots before the next batch.
    int64_t *h_stage_ = nullptr;
    uint64_t stage_cap_ = 0, stage_used_ = 0;
    struct Run {
        uint64_t arena_off, stage_off, n;
    };
    std::vector<Run> runs_;
};

}  // namespace wg
