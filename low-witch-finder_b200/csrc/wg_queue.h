// Device work queue of batched Seed Check jobs (wg_queue.cu).
#pragma once

#include <cstdint>
#include <vector>

#include "wg_engine_impl.h"

namespace wg {

// Runs units [0, total_units) of a jobs-mode batch prototype (proto.jobs: the job table of every
// job, proto.seeds their seeds) as one graph launch whose while-loop takes slices of at most
// `budget` (seed, region) checks and max_units units off a device-side queue.  Survivors are
// appended to `found` (seed_index = the seed's slot in proto.seeds); the funnel, slice count and
// device time go to st.
int run_queue(wg_engine *eng, const BatchArgs &proto, uint64_t total_units, uint32_t max_units, uint64_t budget,
              std::vector<Candidate> &found, wg_scan_stats &st);

// Frees the queue's device state of an engine (called by wg_engine_close).
void queue_release(wg_engine *eng);

}  // namespace wg
