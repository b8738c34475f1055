// Device work queue for batched Seed Check jobs: the whole job list's units, in one job table, run
// as one CUDA graph launch.  The graph's body is a conditional while-node: a plan kernel takes the
// next slice of units off the queue (up to a budget of (seed, region) checks), the three phase-1
// kernels run that slice (reading its range from device memory, BatchArgs::dyn), and a commit
// kernel appends the slice's survivors to the output, adds its funnel, and either moves the queue
// on or, when a work list overflowed, halves the budget and runs the slice again; it then sets the
// loop condition.  No host synchronisation between slices.  An iteration limit ends the loop in
// any case (error status), so a bug cannot keep the GPU busy.
//
// The reference has no batched-job path (one request per phase1_scan invocation,
// engine/gpu/low54/phase1_scan.cu:1328-1387); the per-job results equal running each job alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/witchgpu.h"
#include "wg_engine_impl.h"
#include "wg_queue.h"

namespace wg {

struct QueueState {
    uint64_t dyn[2];              // unit0, n_units of the slice in flight (BatchArgs::dyn)
    uint64_t cursor, total;       // next unit of the queue, units in it
    uint64_t budget, max_budget;  // checks per slice (halved after an overflow, grown back after)
    uint64_t max_units;           // units per slice at most (the launch geometry)
    uint64_t slice_work;          // checks of the slice in flight (by whole windows)
    uint64_t n_out;               // survivors found (may exceed the output capacity)
    uint64_t iters, max_iters;
    uint64_t slices, retries;
    uint64_t climate_survivors, deep, rechecks, records;
    unsigned long long hist[P1_KINDS + kTiers];
    uint32_t error;               // 1 iteration limit, 2 a list full for a one-unit slice
    uint32_t n_jobs;
};

namespace {

// The last job-table entry whose first unit is <= u.
__device__ uint32_t entry_of(const JobGeom *jobs, uint32_t n, uint64_t u) {
    uint32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (jobs[mid].unit0 <= u) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void queue_plan_kernel(QueueState *q, const JobGeom *jobs, uint32_t *counters, unsigned long long *hist) {
    const int t = threadIdx.x;
    if (t < CNT_WORDS) counters[t] = 0;
    if (t < P1_KINDS + kTiers) hist[t] = 0;
    if (t != 0) return;
    // units from the cursor until the slice's checks reach the budget (a unit counts its window)
    const uint64_t u0 = q->cursor;
    uint64_t n = 0, work = 0;
    uint32_t e = entry_of(jobs, q->n_jobs, u0);
    while (u0 + n < q->total && n < q->max_units) {
        const uint64_t end = e + 1 < q->n_jobs ? jobs[e + 1].unit0 : q->total;
        const uint64_t per = jobs[e].win;
        uint64_t k = (q->budget - work) / per;
        if (k == 0) {
            if (n) break;
            k = 1;   // a slice holds at least one unit
        }
        k = min(k, end - (u0 + n));
        k = min(k, q->max_units - n);
        n += k;
        work += k * per;
        if (u0 + n < end || work >= q->budget) break;
        e++;
    }
    q->dyn[0] = u0;
    q->dyn[1] = n;
    q->slice_work = work;
}

__global__ void queue_commit_kernel(QueueState *q, const uint32_t *counters, const unsigned long long *hist,
                                    const Candidate *slice_out, Candidate *out, uint64_t cap,
                                    cudaGraphConditionalHandle cond) {
    __shared__ int advance;
    __shared__ uint64_t base;
    __shared__ uint32_t nf;
    const int t = threadIdx.x;
    if (t == 0) {
        q->iters++;
        advance = 0;
        if (counters[CNT_OVERFLOW]) {   // a work list was full: the same slice again, half as large
            q->retries++;
            if (q->dyn[1] <= 1) q->error = 2;
            else q->budget = max(1ull, (unsigned long long)(q->slice_work / 2));
        } else {
            advance = 1;
            nf = counters[CNT_FINAL];
            base = q->n_out;
            q->n_out += nf;
            q->climate_survivors += counters[CNT_SURVIVORS];
            q->deep += counters[CNT_DEEP];
            q->rechecks += counters[CNT_RECHECK];
            q->records += counters[CNT_RECORDS];
            q->cursor += q->dyn[1];
            q->slices++;
            if (q->budget < q->max_budget) q->budget = min(q->max_budget, q->budget * 2);
        }
    }
    __syncthreads();
    if (advance) {
        for (uint32_t k = t; k < nf; k += blockDim.x)
            if (base + k < cap) out[base + k] = slice_out[k];
        if (t < P1_KINDS + kTiers) q->hist[t] += hist[t];
    }
    if (t == 0) {
        if (q->iters >= q->max_iters && q->cursor < q->total) q->error = 1;
        cudaGraphSetConditional(cond, (q->cursor < q->total && q->error == 0) ? 1u : 0u);
    }
}

}  // namespace

struct QueueRes {
    QueueState *q = nullptr;
    Candidate *out = nullptr;
    uint64_t cap = 0;
};

void queue_release(wg_engine *eng) {
    if (!eng->queue) return;
    cudaFree(eng->queue->q);
    cudaFree(eng->queue->out);
    delete eng->queue;
    eng->queue = nullptr;
}

#define QUEUE_CUDA(call, what)                                          \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return eng->fail(WG_ERR_CUDA, what, e_); \
    } while (0)

int run_queue(wg_engine *eng, const BatchArgs &proto, uint64_t total_units, uint32_t max_units, uint64_t budget,
              std::vector<Candidate> &found, wg_scan_stats &st) {
    if (total_units == 0) return WG_OK;
    if (!eng->queue) {
        eng->queue = new (std::nothrow) QueueRes();
        if (!eng->queue) return eng->fail(WG_ERR_NOMEM, "queue state");
        QUEUE_CUDA(cudaMalloc(&eng->queue->q, sizeof(QueueState)), "queue state");
        eng->queue->cap = kCapOut;
        QUEUE_CUDA(cudaMalloc(&eng->queue->out, sizeof(Candidate) * eng->queue->cap), "queue output");
    }
    QueueRes &R = *eng->queue;
    cudaStream_t s = eng->stream;
    QueueState h;
    std::memset(&h, 0, sizeof h);
    h.total = total_units;
    h.budget = h.max_budget = std::max<uint64_t>(budget, 1);
    h.max_units = max_units;
    h.n_jobs = proto.n_jobs;
    // every iteration either advances the cursor or halves the slice, so a correct run takes far
    // fewer; the limit only bounds a faulty one (which then reports an error)
    h.max_iters = 1u << 20;
    QUEUE_CUDA(cudaMemcpyAsync(R.q, &h, sizeof h, cudaMemcpyHostToDevice, s), "queue upload");

    BatchArgs a = proto;
    a.unit0 = 0;
    a.n_units = max_units;   // the launch geometry; the slice range comes from dyn
    a.dyn = R.q->dyn;
    prepare_phase1_launches();

    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int rc = [&]() -> int {
        QUEUE_CUDA(cudaGraphCreate(&graph, 0), "graph create");
        cudaGraphConditionalHandle cond;
        QUEUE_CUDA(cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault), "graph condition");
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        QUEUE_CUDA(cudaGraphAddNode(&node, graph, nullptr, 0, &cp), "graph while node");
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        QUEUE_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed),
                   "capture");
        queue_plan_kernel<<<1, 32, 0, s>>>(R.q, proto.jobs, a.counters, a.hist);
        launch_climate(a, s);
        launch_entrance(a, 0, s);
        launch_ladder(a, 0, s);
        queue_commit_kernel<<<1, 256, 0, s>>>(R.q, a.counters, a.hist, a.out, R.out, R.cap, cond);
        cudaGraph_t captured = nullptr;
        QUEUE_CUDA(cudaStreamEndCapture(s, &captured), "capture end");
        QUEUE_CUDA(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
        QUEUE_CUDA(cudaEventRecord(eng->kev[0], s), "event");
        QUEUE_CUDA(cudaGraphLaunch(exec, s), "graph launch");
        QUEUE_CUDA(cudaEventRecord(eng->kev[1], s), "event");
        QUEUE_CUDA(cudaMemcpyAsync(&h, R.q, sizeof h, cudaMemcpyDeviceToHost, s), "queue read");
        QUEUE_CUDA(cudaStreamSynchronize(s), "queue run");
        return WG_OK;
    }();
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (rc) return rc;
    if (h.error == 1) return eng->fail(WG_ERR_CUDA, "device queue: iteration limit reached");
    if (h.error == 2) return eng->fail(WG_ERR_CAPACITY, "device queue: a work list stayed full for one unit");
    if (h.n_out > R.cap) return eng->fail(WG_ERR_CAPACITY, "device queue: more survivors than the output holds");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, eng->kev[0], eng->kev[1]);
    const size_t at = found.size();
    found.resize(at + h.n_out);
    if (h.n_out)
        QUEUE_CUDA(cudaMemcpy(found.data() + at, R.out, sizeof(Candidate) * h.n_out, cudaMemcpyDeviceToHost),
                   "queue survivors");
    for (int i = 0; i < P1_KINDS; i++) st.reject_hist[i] += (int64_t)h.hist[i];
    for (int i = 0; i < kTiers; i++) st.tier_hist[i] += (int64_t)h.hist[P1_KINDS + i];
    st.climate_survivors += (int64_t)h.climate_survivors;
    st.deep_candidates += (int64_t)h.deep;
    st.rechecks += (int64_t)h.rechecks;
    st.records += (int64_t)h.records;
    st.batches += (int64_t)h.slices;
    st.retries += (int64_t)h.retries;
    for (int k = 0; k < 3; k++) st.kernel_launches[k] += (int64_t)(h.slices + h.retries);
    st.kernel_ms[0] += ms;   // one graph: its time is booked on the climate kernel's line
    return WG_OK;
}

}  // namespace wg
