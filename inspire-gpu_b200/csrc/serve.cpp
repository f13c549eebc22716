// serve.cpp -- continuous-batching serving loop over resident databases
// (the ipir_serve_* entry points).  The reference has no counterpart: its
// batch entry point answers one caller-formed batch per blocking call
// (src/gpu_protocol.cu:1414-1535, src/capi.h:84-89).
//
// Requests enter pinned request slots (submit copies the query there and
// returns a ticket).  One worker thread owns every device call: for each
// database it admits waiting requests, oldest first and at most max_batch
// at a time, into a free lane -- a set of per-batch device buffers with its
// own stream.  A batch has two phases: the DB-bound one (mat-vec and tensor
// pass stream the whole database and the precomputed tensors) and the
// latency-bound Horner chains.  A database's next batch is admitted as soon
// as its previous batch has left the DB-bound phase, so the next DB pass
// overlaps only the previous batch's Horner (two DB passes at once would
// just share the memory bandwidth), and requests that arrive meanwhile
// still join it.  Lanes of different databases run concurrently.
// A lane batch is: one H2D copy per query, one replay of each phase's CUDA
// graph captured for that batch size (an event between them), one D2H copy
// per response straight into its request slot, the error word, and an
// event the worker polls (a host
// function per batch was tried first: on B200 with driver 580 its callbacks
// stalled for ~40 ms every ~2 s on an otherwise idle GPU).  Everything is
// allocated at create; the request path allocates nothing.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "inspire_b200.h"
#include "server_internal.h"

namespace ipb {
namespace {

using Clock = std::chrono::steady_clock;

enum SlotState : int { kFree = 0, kFilling, kQueued, kRunning, kDone, kFailed, kCollecting };

struct ReqSlot {
    uint64_t ticket = 0;
    int state = kFree;
    size_t db = 0;
    uint64_t* q = nullptr;     // pinned flat query (the database's qstride words)
    uint64_t* resp = nullptr;  // pinned response
    Clock::time_point t_submit, t_issue, t_done;
};

struct Engine;

struct LaneRun {
    Lane lane;
    cudaStream_t st = nullptr;
    std::vector<cudaGraphExec_t> graphs_db, graphs_horner;  // [batch size], index 0 unused
    bool busy = false;
    std::vector<uint32_t> slots;
    int* h_err = nullptr;  // pinned device-error word of the last batch
    cudaEvent_t ev_start = nullptr, ev_db = nullptr, ev_end = nullptr;
    int64_t t_issue0 = 0, t_issue1 = 0;  // steady-clock ns around the last issue()
    uint16_t db_index = 0, lane_index = 0;
    Engine* eng = nullptr;
};

// Cyclic shared scan (ipir_serve_config.scan_segments = ns > 1): a
// database's DB and tensor passes run as ns segments in rotation on one lane
// (segment k: DB columns [k C/ns, (k + 1) C/ns) and the tensor pass's
// (limb, slot) indices [k 2N/ns, (k + 1) 2N/ns), all groups).  The requests
// waiting when a segment is enqueued join the rotation there, as one group
// of contiguous lane query slots; each segment's kernels serve every active
// query at once (one read of that part of the DB and tensors), writing
// per-slot partial results.  After a group's ns-th segment its finalize
// runs, then its Horner chains and response copies on a higher-priority
// stream while the rotation goes on.  A request waits for the rest of the
// running segment instead of the rest of a whole DB pass.
struct ScanGroup {
    size_t s0 = 0, k = 0;        // lane query slots [s0, s0 + k)
    int left = 0;                // segments still to run
    std::vector<uint32_t> req;   // request slots, in lane-slot order
    cudaEvent_t ev_start = nullptr, ev_end = nullptr;
    int* h_err = nullptr;        // pinned copy of the device error word after its Horner chains
    int64_t t_issue0 = 0;        // steady-clock ns when its admission was enqueued
    int64_t issue_ns = 0;        // host time spent enqueueing its admission, Horner chains and copies
};

struct ScanState {
    int ns = 0;
    int next_seg = 0;
    size_t cap = 0;              // lane query slots (<= 32: one pass per segment)
    std::vector<char> used;
    std::deque<ScanGroup> active, finishing;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_free;
    std::vector<int*> err_free;
    int* pinned_err = nullptr;
    cudaEvent_t ev_next = nullptr;     // the last segment's mat-vec ran: time to enqueue the next one
    cudaEvent_t ev_seg_end = nullptr;
    cudaStream_t hst = nullptr;        // Horner chains and response copies
    bool stepped = false;
    uint32_t* keys_pos = nullptr;      // keys of the active queries in pass order (lane arena)
    std::vector<cudaEvent_t> all_events;
    ~ScanState() {
        if (hst) cudaStreamSynchronize(hst);
        for (auto e : all_events) cudaEventDestroy(e);
        if (hst) cudaStreamDestroy(hst);
        if (pinned_err) cudaFreeHost(pinned_err);
    }
};

struct DbState {
    Server* S = nullptr;
    size_t scan_ns = 0;               // > 1: cyclic scan in this many segments, else lane batches
    std::unique_ptr<ScanState> scan;  // cyclic scan mode, else lane batches
    size_t max_batch = 0;
    std::vector<Sched> sched;
    std::vector<std::unique_ptr<LaneRun>> lanes;
    std::deque<uint32_t> pending;
    int last_lane = -1;  // lane of the most recently issued batch
    uint64_t batches = 0, queries = 0;
    Server* swap_to = nullptr;  // next generation, installed once the lanes are idle
    bool swap_done = false;
    std::string swap_err;
};

struct Engine {
    std::vector<std::unique_ptr<DbState>> dbs;
    size_t q_words = 0, r_words = 0;  // per request slot
    std::vector<ReqSlot> slots;
    std::vector<uint32_t> free_slots;
    uint64_t* pinned_q = nullptr;
    uint64_t* pinned_r = nullptr;
    int* pinned_err = nullptr;
    bool use_graphs = true;
    bool overlap_db = false;  // admit without waiting for the previous DB phase
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_swap;
    std::thread worker;
    bool stop = false;
    bool failed = false;
    std::string fail_text;
    uint64_t next_seq = 1;
    uint64_t submitted = 0, completed = 0, n_failed = 0, batches = 0, batched = 0, max_seen = 0;
    double max_notice_ms = 0;  // batch end on the device -> completion handled by the worker (bound)
    std::vector<ipir_serve_batch_record> trace;  // ring of the last batches
    uint64_t trace_n = 0;

    ~Engine();
    void run();
    void issue(DbState& d, LaneRun& r);
    void finish(DbState& d, LaneRun& r);
    void fail_all_locked(const std::string& why);
    void swap_locked(DbState& d, std::unique_lock<std::mutex>& lk);
    void scan_step(DbState& d, std::unique_lock<std::mutex>& lk);
    void scan_poll(DbState& d, bool& any_busy, std::string& poll_err);
    void scan_finish(DbState& d, ScanGroup& g);
    void scan_fail_locked(DbState& d);
};

void Engine::issue(DbState& d, LaneRun& r) {
    const Server& S = *d.S;
    Lane& L = r.lane;
    const size_t n = r.slots.size();
    IPB_CK(cudaSetDevice(S.device));
    IPB_CK(cudaEventRecord(r.ev_start, r.st));
    for (size_t i = 0; i < n; ++i) stage_query_flat(S, L, i, slots[r.slots[i]].q, r.st);
    if (runs_chunked(S, d.sched[n], n)) {
        // One pipeline with the Horner chain trailing the DB pass in chunks;
        // ev_db is recorded inside, after the last chunk's finalize.
        if (use_graphs)
            IPB_CK(cudaGraphLaunch(r.graphs_db[n], r.st));
        else
            run_pipeline(S, L, d.sched[n], n, r.st, nullptr, kPhaseAll, 6, r.ev_db);
    } else {
        if (use_graphs)
            IPB_CK(cudaGraphLaunch(r.graphs_db[n], r.st));
        else
            run_pipeline(S, L, d.sched[n], n, r.st, nullptr, kPhaseDb);
        IPB_CK(cudaEventRecord(r.ev_db, r.st));
        if (use_graphs)
            IPB_CK(cudaGraphLaunch(r.graphs_horner[n], r.st));
        else
            run_pipeline(S, L, d.sched[n], n, r.st, nullptr, kPhaseHorner);
    }
    const size_t rb = S.resp_qstride * 8;
    for (size_t i = 0; i < n; ++i)
        IPB_CK(cudaMemcpyAsync(slots[r.slots[i]].resp, L.resp + i * S.resp_qstride, rb, cudaMemcpyDeviceToHost,
                               r.st));
    IPB_CK(cudaMemcpyAsync(r.h_err, L.d_err, sizeof(int), cudaMemcpyDeviceToHost, r.st));
    IPB_CK(cudaMemsetAsync(L.d_err, 0, sizeof(int), r.st));
    IPB_CK(cudaEventRecord(r.ev_end, r.st));
}

// Called with the lock held, once the lane's end event completed.
void Engine::finish(DbState& d, LaneRun& r) {
    const int err = *r.h_err;
    const auto now = Clock::now();
    float dev_ms = 0.f;
    if (cudaEventElapsedTime(&dev_ms, r.ev_start, r.ev_end) != cudaSuccess) dev_ms = -1.f;
    // Upper bound on the delay between the batch's end and this call: wall
    // time since the enqueue began, less the device time.
    const double notice = std::max(0.0, (now.time_since_epoch().count() - r.t_issue0) * 1e-6 - dev_ms);
    max_notice_ms = std::max(max_notice_ms, notice);
    if (!trace.empty()) {
        ipir_serve_batch_record& t = trace[trace_n++ % trace.size()];
        t.t_issue_s = r.t_issue0 * 1e-9;
        t.issue_ms = (float)((r.t_issue1 - r.t_issue0) * 1e-6);
        t.device_ms = dev_ms;
        t.notice_ms = (float)notice;
        t.db = r.db_index;
        t.lane = r.lane_index;
        t.count = (uint32_t)r.slots.size();
        t.failed = err != 0;
    }
    for (uint32_t s : r.slots) {
        slots[s].state = err ? kFailed : kDone;
        slots[s].t_done = now;
    }
    if (err) {
        n_failed += r.slots.size();
        fail_text = "device pipeline wait timed out (code " + std::to_string(err) + ")";
    } else {
        completed += r.slots.size();
    }
    ++d.batches;
    d.queries += r.slots.size();
    ++batches;
    batched += r.slots.size();
    max_seen = std::max<uint64_t>(max_seen, r.slots.size());
    r.slots.clear();
    r.busy = false;
    cv_done.notify_all();
}

void Engine::fail_all_locked(const std::string& why) {
    failed = true;
    fail_text = why;
    for (auto& d : dbs)
        if (d->scan) scan_fail_locked(*d);
    for (auto& d : dbs) {
        for (uint32_t s : d->pending) slots[s].state = kFailed;
        n_failed += d->pending.size();
        d->pending.clear();
    }
    cv_done.notify_all();
}

// Enqueue one segment of d's rotation (lock held on entry and exit):
// admit the waiting requests as a new group, run the segment for every
// active group, and start the Horner chains of the groups it completes.
void Engine::scan_step(DbState& d, std::unique_lock<std::mutex>& lk) {
    ScanState& sc = *d.scan;
    LaneRun& r = *d.lanes[0];
    size_t n_active = 0;
    for (auto& g : sc.active) n_active += g.k;
    bool admit = false;
    if (!d.swap_to && !d.pending.empty() && n_active < sc.cap && !sc.ev_free.empty() && !sc.err_free.empty()) {
        const size_t want = std::min(d.pending.size(), sc.cap - n_active);
        size_t best_s = 0, best_k = 0;  // longest run of free lane slots (first that fits)
        for (size_t i = 0; i < sc.cap && best_k < want;) {
            if (sc.used[i]) {
                ++i;
                continue;
            }
            size_t j = i;
            while (j < sc.cap && !sc.used[j]) ++j;
            if (j - i > best_k) {
                best_k = j - i;
                best_s = i;
            }
            i = j;
        }
        const size_t k = std::min(want, best_k);
        if (k > 0) {
            ScanGroup g;
            g.s0 = best_s;
            g.k = k;
            g.left = sc.ns;
            std::tie(g.ev_start, g.ev_end) = sc.ev_free.back();
            sc.ev_free.pop_back();
            g.h_err = sc.err_free.back();
            sc.err_free.pop_back();
            *g.h_err = 0;
            const auto now = Clock::now();
            for (size_t i = 0; i < k; ++i) {
                const uint32_t s = d.pending.front();
                d.pending.pop_front();
                slots[s].state = kRunning;
                slots[s].t_issue = now;
                g.req.push_back(s);
                sc.used[best_s + i] = 1;
            }
            sc.active.push_back(std::move(g));
            admit = true;
        }
    }
    if (sc.active.empty()) return;
    std::vector<SlotRun> runs;
    for (auto& g : sc.active) runs.push_back(SlotRun{g.s0, g.k});
    const int seg = sc.next_seg;
    sc.next_seg = (seg + 1) % sc.ns;
    for (auto& g : sc.active) --g.left;
    std::vector<ScanGroup> done;  // groups this segment completes (oldest first)
    while (!sc.active.empty() && sc.active.front().left == 0) {
        done.push_back(std::move(sc.active.front()));
        sc.active.pop_front();
    }
    ScanGroup* fresh = admit ? &sc.active.back() : nullptr;  // ns > 1: not completed yet
    sc.stepped = true;
    const Server& S = *d.S;
    lk.unlock();
    std::string err;
    try {
        Lane& L = r.lane;
        IPB_CK(cudaSetDevice(S.device));
        if (fresh) {
            fresh->t_issue0 = Clock::now().time_since_epoch().count();
            IPB_CK(cudaEventRecord(fresh->ev_start, r.st));
            for (size_t i = 0; i < fresh->k; ++i)
                IPB_CK(cudaMemcpyAsync(L.qraw + (fresh->s0 + i) * S.qstride, slots[fresh->req[i]].q, S.qstride * 8,
                                       cudaMemcpyHostToDevice, r.st));
            enqueue_qprep_slots(S, L, fresh->s0, fresh->k, r.st);
            fresh->issue_ns = Clock::now().time_since_epoch().count() - fresh->t_issue0;
        }
        enqueue_scan_segment(S, L, sc.keys_pos, runs, seg, sc.ns, r.st, sc.ev_next);
        if (!done.empty()) {
            for (auto& g : done) enqueue_scan_finalize(S, L, SlotRun{g.s0, g.k}, r.st);
            IPB_CK(cudaEventRecord(sc.ev_seg_end, r.st));
            IPB_CK(cudaStreamWaitEvent(sc.hst, sc.ev_seg_end, 0));
            for (auto& g : done) {
                const int64_t t0 = Clock::now().time_since_epoch().count();
                enqueue_horner(S, d.sched[g.k], L.packed_b + g.s0 * S.pb_qstride, L.rgsw32 + g.s0 * kRgswStride,
                               L.resp + g.s0 * S.resp_qstride, g.k, L.d_err, sc.hst);
                for (size_t i = 0; i < g.k; ++i)
                    IPB_CK(cudaMemcpyAsync(slots[g.req[i]].resp, L.resp + (g.s0 + i) * S.resp_qstride,
                                           S.resp_qstride * 8, cudaMemcpyDeviceToHost, sc.hst));
                IPB_CK(cudaMemcpyAsync(g.h_err, L.d_err, sizeof(int), cudaMemcpyDeviceToHost, sc.hst));
                IPB_CK(cudaEventRecord(g.ev_end, sc.hst));
                g.issue_ns += Clock::now().time_since_epoch().count() - t0;
            }
        }
    } catch (const std::exception& e) {
        err = e.what();
    }
    lk.lock();
    for (auto& g : done) sc.finishing.push_back(std::move(g));
    if (!err.empty()) {
        lk.unlock();
        cudaStreamSynchronize(r.st);
        cudaStreamSynchronize(sc.hst);
        lk.lock();
        fail_all_locked(err);
    }
}

// Fails every request of d's rotation and returns its slots and events.
void Engine::scan_fail_locked(DbState& d) {
    ScanState& sc = *d.scan;
    for (auto* q : {&sc.active, &sc.finishing}) {
        for (auto& g : *q) {
            for (uint32_t s : g.req) {
                slots[s].state = kFailed;
                slots[s].t_done = Clock::now();
            }
            n_failed += g.req.size();
            for (size_t i = 0; i < g.k; ++i) sc.used[g.s0 + i] = 0;
            sc.ev_free.emplace_back(g.ev_start, g.ev_end);
            sc.err_free.push_back(g.h_err);
        }
        q->clear();
    }
    cv_done.notify_all();
}

// Groups complete in order on the Horner stream (lock held).
void Engine::scan_poll(DbState& d, bool& any_busy, std::string& poll_err) {
    ScanState& sc = *d.scan;
    while (!sc.finishing.empty()) {
        ScanGroup& g = sc.finishing.front();
        const cudaError_t q = cudaEventQuery(g.ev_end);
        if (q == cudaErrorNotReady) {
            any_busy = true;
            break;
        }
        if (q != cudaSuccess) {
            poll_err = std::string("CUDA error while waiting for a batch: ") + cudaGetErrorString(q);
            return;
        }
        scan_finish(d, g);
        sc.finishing.pop_front();
    }
    if (!sc.active.empty()) any_busy = true;
}

void Engine::scan_finish(DbState& d, ScanGroup& g) {
    ScanState& sc = *d.scan;
    const int err = *g.h_err;
    const auto now = Clock::now();
    float dev_ms = 0.f;
    if (cudaEventElapsedTime(&dev_ms, g.ev_start, g.ev_end) != cudaSuccess) dev_ms = -1.f;
    // Upper bound on the delay between the group's end and this call: wall
    // time since its admission was enqueued, less its device time.
    const double notice = std::max(0.0, (now.time_since_epoch().count() - g.t_issue0) * 1e-6 - dev_ms);
    max_notice_ms = std::max(max_notice_ms, notice);
    if (!trace.empty()) {
        ipir_serve_batch_record& t = trace[trace_n++ % trace.size()];
        t.t_issue_s = g.t_issue0 * 1e-9;
        t.issue_ms = (float)(g.issue_ns * 1e-6);
        t.device_ms = dev_ms;
        t.notice_ms = (float)notice;
        t.db = 0;
        for (size_t i = 0; i < dbs.size(); ++i)
            if (dbs[i].get() == &d) t.db = (uint16_t)i;
        t.lane = 0;
        t.count = (uint32_t)g.k;
        t.failed = err != 0;
    }
    for (uint32_t s : g.req) {
        slots[s].state = err ? kFailed : kDone;
        slots[s].t_done = now;
    }
    if (err) {
        n_failed += g.req.size();
        fail_text = "device pipeline wait timed out (code " + std::to_string(err) + ")";
    } else {
        completed += g.req.size();
    }
    ++d.batches;
    d.queries += g.req.size();
    ++batches;
    batched += g.req.size();
    max_seen = std::max<uint64_t>(max_seen, g.req.size());
    for (size_t i = 0; i < g.k; ++i) sc.used[g.s0 + i] = 0;
    sc.ev_free.emplace_back(g.ev_start, g.ev_end);
    sc.err_free.push_back(g.h_err);
    cv_done.notify_all();
}

void Engine::run() {
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        bool any_busy = false;
        std::string poll_err;
        for (auto& dp : dbs)
            if (dp->scan) scan_poll(*dp, any_busy, poll_err);
        for (auto& dp : dbs)
            for (auto& r : dp->lanes)
                if (r->busy) {
                    const cudaError_t q = cudaEventQuery(r->ev_end);
                    if (q == cudaSuccess) {
                        finish(*dp, *r);
                    } else if (q == cudaErrorNotReady) {
                        any_busy = true;
                    } else {
                        for (uint32_t s : r->slots) slots[s].state = kFailed;
                        n_failed += r->slots.size();
                        r->slots.clear();
                        r->busy = false;
                        poll_err = std::string("CUDA error while waiting for a batch: ") + cudaGetErrorString(q);
                    }
                }
        if (!poll_err.empty()) fail_all_locked(poll_err);
        for (auto& dp : dbs) {
            if (!dp->swap_to) continue;
            bool idle = true;
            for (auto& r : dp->lanes) idle &= !r->busy;
            if (dp->scan)
                idle = dp->scan->active.empty() && dp->scan->finishing.empty() &&
                       cudaStreamQuery(dp->lanes[0]->st) == cudaSuccess;
            if (idle) swap_locked(*dp, lk);
            else any_busy = true;
        }
        // Scan rotations keep turning while they hold requests, also after
        // stop (admitting none then: stop fails the waiting requests below).
        if (!failed)
            for (auto& dp : dbs) {
                DbState& d = *dp;
                if (!d.scan) continue;
                ScanState& sc = *d.scan;
                const bool work = !sc.active.empty() || (!stop && !d.pending.empty() && !d.swap_to);
                if (work) {
                    const cudaError_t q = sc.stepped ? cudaEventQuery(sc.ev_next) : cudaSuccess;
                    if (q == cudaSuccess) {
                        scan_step(d, lk);
                    } else if (q != cudaErrorNotReady) {
                        fail_all_locked(std::string("CUDA error in the scan rotation: ") + cudaGetErrorString(q));
                    }
                }
                if (!sc.active.empty() || !sc.finishing.empty()) any_busy = true;
            }
        if (stop && !any_busy) break;
        if (!stop && !failed) {
            for (auto& dp : dbs) {
                DbState& d = *dp;
                if (d.scan) continue;
                if (d.pending.empty() || d.swap_to) continue;
                if (!overlap_db && d.last_lane >= 0 && d.lanes[d.last_lane]->busy) {
                    const cudaError_t q = cudaEventQuery(d.lanes[d.last_lane]->ev_db);
                    if (q == cudaErrorNotReady) continue;  // previous DB pass still running
                }
                for (size_t li = 0; li < d.lanes.size(); ++li) {
                    auto& r = d.lanes[li];
                    if (d.pending.empty()) break;
                    if (r->busy) continue;
                    const size_t n = std::min(d.max_batch, d.pending.size());
                    const auto t_issue = Clock::now();
                    for (size_t i = 0; i < n; ++i) {
                        const uint32_t s = d.pending.front();
                        d.pending.pop_front();
                        slots[s].state = kRunning;
                        slots[s].t_issue = t_issue;
                        r->slots.push_back(s);
                    }
                    r->busy = true;
                    any_busy = true;
                    d.last_lane = (int)li;
                    lk.unlock();
                    std::string err;
                    r->t_issue0 = Clock::now().time_since_epoch().count();
                    try {
                        issue(d, *r);
                    } catch (const std::exception& e) {
                        err = e.what();
                    }
                    r->t_issue1 = Clock::now().time_since_epoch().count();
                    lk.lock();
                    if (!err.empty()) {
                        // The lane's stream may hold part of the batch: wait for
                        // it outside the lock, then fail everything.
                        lk.unlock();
                        cudaStreamSynchronize(r->st);
                        lk.lock();
                        for (uint32_t s : r->slots) slots[s].state = kFailed;
                        n_failed += r->slots.size();
                        r->slots.clear();
                        r->busy = false;
                        fail_all_locked(err);
                    }
                    if (!overlap_db) break;  // one DB pass at a time per database
                }
            }
        }
        if (stop) {
            for (auto& d : dbs) {
                for (uint32_t s : d->pending) slots[s].state = kFailed;
                n_failed += d->pending.size();
                d->pending.clear();
            }
            cv_done.notify_all();
        }
        if (any_busy) {
            cv_work.wait_for(lk, std::chrono::microseconds(20));
        } else {
            bool work = false;
            for (auto& d : dbs) work |= !d->pending.empty();
            if (!work && !stop) cv_work.wait_for(lk, std::chrono::milliseconds(20));
        }
    }
}

Engine::~Engine() {
    for (auto& dp : dbs) {
        DbState& d = *dp;
        cudaSetDevice(d.S->device);
        if (d.scan && d.scan->hst) cudaStreamSynchronize(d.scan->hst);
        for (auto& r : d.lanes) {
            if (r->st) cudaStreamSynchronize(r->st);
            if (r->ev_start) cudaEventDestroy(r->ev_start);
            if (r->ev_db) cudaEventDestroy(r->ev_db);
            if (r->ev_end) cudaEventDestroy(r->ev_end);
            for (auto g : r->graphs_db)
                if (g) cudaGraphExecDestroy(g);
            for (auto g : r->graphs_horner)
                if (g) cudaGraphExecDestroy(g);
            if (r->st) cudaStreamDestroy(r->st);
            r->lane.arena.free_all();
        }
    }
    if (pinned_q) cudaFreeHost(pinned_q);
    if (pinned_r) cudaFreeHost(pinned_r);
    if (pinned_err) cudaFreeHost(pinned_err);
}

cudaGraphExec_t capture_phase(DbState& d, LaneRun& r, size_t c, int phase, cudaEvent_t db_done = nullptr) {
    cudaGraph_t g = nullptr;
    IPB_CK(cudaStreamBeginCapture(r.st, cudaStreamCaptureModeThreadLocal));
    try {
        run_pipeline(*d.S, r.lane, d.sched[c], c, r.st, nullptr, phase, 6, db_done);
    } catch (...) {
        cudaStreamEndCapture(r.st, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    IPB_CK(cudaStreamEndCapture(r.st, &g));
    cudaGraphExec_t ge = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    IPB_CK(e);
    return ge;
}

void capture_graphs(DbState& d, LaneRun& r, bool warm = true) {
    for (auto g : r.graphs_db)
        if (g) cudaGraphExecDestroy(g);
    for (auto g : r.graphs_horner)
        if (g) cudaGraphExecDestroy(g);
    r.graphs_db.assign(d.max_batch + 1, nullptr);
    r.graphs_horner.assign(d.max_batch + 1, nullptr);
    for (size_t c = 1; c <= d.max_batch; ++c) {
        // An eager run first: kernel attributes are set outside the capture.
        if (warm) run_pipeline(*d.S, r.lane, d.sched[c], c, r.st, nullptr);
        if (runs_chunked(*d.S, d.sched[c], c)) {
            r.graphs_db[c] = capture_phase(d, r, c, kPhaseAll, r.ev_db);  // the whole chunked pipeline
        } else {
            r.graphs_db[c] = capture_phase(d, r, c, kPhaseDb);
            r.graphs_horner[c] = capture_phase(d, r, c, kPhaseHorner);
        }
    }
    IPB_CK(cudaStreamSynchronize(r.st));
}

// Called by the worker with the lock held once every lane of d is idle:
// point d at the next generation and re-capture its graphs (same geometry,
// so the lane buffers and schedules carry over; kernels are already set up).
void Engine::swap_locked(DbState& d, std::unique_lock<std::mutex>& lk) {
    Server* next = d.swap_to;
    d.S = next;  // under the lock: collectors read the response size through d.S
    lk.unlock();
    std::string err;
    try {
        IPB_CK(cudaSetDevice(next->device));
        if (use_graphs && !d.scan)
            for (auto& r : d.lanes) capture_graphs(d, *r, false);
    } catch (const std::exception& e) {
        err = e.what();
    }
    lk.lock();
    d.swap_to = nullptr;
    d.swap_err = err;
    d.swap_done = true;
    if (!err.empty()) fail_all_locked(err);
    cv_swap.notify_all();
}

}  // namespace
}  // namespace ipb

struct ipir_serve {
    ipb::Engine* e;
};

namespace {
template <class F>
int serve_guarded(F&& f, int fail_code) {
    ipb::DeviceRestore keep_device;
    try {
        return f();
    } catch (const std::exception& e) {
        ipb::set_last_error(e.what());
    } catch (...) {
        ipb::set_last_error("unknown error");
    }
    return fail_code;
}
}  // namespace

extern "C" {

ipir_serve* ipir_serve_create(ipir_server* const* dbs, size_t n_dbs, const ipir_serve_config* cfg_in) {
    if (!dbs || n_dbs == 0) {
        ipb::set_last_error("ipir_serve_create: no databases");
        return nullptr;
    }
    ipir_serve_config cfg{};
    if (cfg_in) cfg = *cfg_in;
    if (!cfg.max_batch) cfg.max_batch = 64;
    if (!cfg.lanes_per_db) cfg.lanes_per_db = 2;
    if (!cfg.queue_slots) cfg.queue_slots = 256;
    ipir_serve* out = nullptr;
    serve_guarded(
        [&]() -> int {
            auto E = std::make_unique<ipb::Engine>();
            E->use_graphs = cfg.disable_graphs == 0;
            E->overlap_db = cfg.overlap_db_passes != 0;
            for (size_t i = 0; i < n_dbs; ++i) {
                if (!dbs[i] || !dbs[i]->s) throw std::invalid_argument("ipir_serve_create: null database handle");
                auto d = std::make_unique<ipb::DbState>();
                d->S = dbs[i]->s;
                E->dbs.push_back(std::move(d));
            }
            // Size lanes by the HBM budget: halve the batch, then the lane
            // count, until every database's lanes fit.
            IPB_CK(cudaSetDevice(E->dbs[0]->S->device));
            size_t budget = cfg.hbm_budget_bytes;
            if (!budget) {
                size_t fr = 0, tot = 0;
                IPB_CK(cudaMemGetInfo(&fr, &tot));
                const size_t reserve = (size_t)2 << 30;
                budget = fr > reserve ? fr - reserve : 0;
            }
            // Cyclic scan for databases whose columns split into scan_segments
            // parts of whole 128-column tiles (the tensor pass splits its
            // 2N (limb, slot) indices the same way, in multiples of 32).
            // scan_segments < 0: per database, from its own plain answer.
            auto splits = [](const ipb::Server& S, size_t ns) {
                return ns > 1 && S.pp.db_cols % (128 * ns) == 0 && (2 * ipb::kN) % (32 * ns) == 0;
            };
            for (auto& dp : E->dbs) {
                ipb::DbState& d = *dp;
                if (cfg.scan_segments > 1) {
                    d.scan_ns = splits(*d.S, (size_t)cfg.scan_segments) ? (size_t)cfg.scan_segments : 0;
                } else if (cfg.scan_segments < 0) {
                    size_t ns = ipb::auto_scan_segments(ipb::time_plain_answer(*d.S));
                    while (ns > 1 && !splits(*d.S, ns)) ns /= 2;
                    d.scan_ns = ns > 1 ? ns : 0;
                }
            }
            auto scan_ok = [&](const ipb::DbState& d) { return d.scan_ns > 1; };
            size_t mb = cfg.max_batch, lanes = cfg.lanes_per_db;
            auto need = [&](size_t b, size_t l) {
                size_t t = 0;
                for (auto& d : E->dbs) {
                    if (scan_ok(*d)) {
                        const size_t c = std::min<size_t>(b, 32);
                        t += ipb::lane_bytes(*d->S, c, ipb::lane_gt_pass(*d->S, c)) + c * ipb::kKeyStride * 4;
                    } else {
                        t += l * ipb::lane_bytes(*d->S, b, ipb::lane_gt_pass(*d->S, b));
                    }
                }
                return t;
            };
            while (need(mb, lanes) > budget) {
                if (mb > 1) mb /= 2;
                else if (lanes > 1) --lanes;
                else throw std::runtime_error("ipir_serve_create: one lane per database exceeds the HBM budget");
            }
            size_t q_words = 0, r_words = 0;
            for (auto& dp : E->dbs) {
                ipb::DbState& d = *dp;
                const bool scan = scan_ok(d);
                d.max_batch = scan ? std::min<size_t>(mb, 32) : mb;
                q_words = std::max(q_words, d.S->qstride);
                r_words = std::max(r_words, d.S->resp_qstride);
                for (size_t k = 0; k < (scan ? 1 : lanes); ++k) {
                    auto r = std::make_unique<ipb::LaneRun>();
                    r->eng = E.get();
                    r->db_index = (uint16_t)(&dp - &E->dbs[0]);
                    r->lane_index = (uint16_t)k;
                    IPB_CK(cudaSetDevice(d.S->device));
                    IPB_CK(cudaStreamCreateWithFlags(&r->st, cudaStreamNonBlocking));
                    IPB_CK(cudaEventCreate(&r->ev_start));
                    IPB_CK(cudaEventCreate(&r->ev_end));
                    IPB_CK(cudaEventCreateWithFlags(&r->ev_db, cudaEventDisableTiming));
                    ipb::alloc_lane(*d.S, r->lane, d.max_batch, ipb::lane_gt_pass(*d.S, d.max_batch));
                    d.lanes.push_back(std::move(r));
                }
                d.sched = !cfg.disable_autotune ? ipb::autotune(*d.S, d.lanes[0]->lane, d.lanes[0]->st)
                                       : ipb::default_sched(*d.S, d.max_batch, d.lanes[0]->lane.gt_pass);
                if (scan) {
                    auto sc = std::make_unique<ipb::ScanState>();
                    sc->ns = (int)d.scan_ns;
                    sc->cap = d.max_batch;
                    sc->used.assign(sc->cap, 0);
                    sc->keys_pos = d.lanes[0]->lane.arena.alloc<uint32_t>(sc->cap * ipb::kKeyStride);
                    int lo = 0, hi = 0;
                    IPB_CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
                    IPB_CK(cudaStreamCreateWithPriority(&sc->hst, cudaStreamNonBlocking, hi));
                    auto mk = [&](unsigned flags) {
                        cudaEvent_t e = nullptr;
                        IPB_CK(cudaEventCreateWithFlags(&e, flags));
                        sc->all_events.push_back(e);
                        return e;
                    };
                    sc->ev_next = mk(cudaEventDisableTiming);
                    sc->ev_seg_end = mk(cudaEventDisableTiming);
                    IPB_CK(cudaMallocHost(&sc->pinned_err, sc->cap * sizeof(int)));
                    for (size_t i = 0; i < sc->cap; ++i) {
                        sc->ev_free.emplace_back(mk(cudaEventDefault), mk(cudaEventDefault));
                        sc->err_free.push_back(sc->pinned_err + i);
                    }
                    d.scan = std::move(sc);
                } else if (E->use_graphs) {
                    for (auto& r : d.lanes) ipb::capture_graphs(d, *r);
                }
            }
            E->q_words = q_words;
            E->r_words = r_words;
            const size_t Q = cfg.queue_slots;
            IPB_CK(cudaMallocHost(&E->pinned_q, Q * q_words * 8));
            IPB_CK(cudaMallocHost(&E->pinned_r, Q * r_words * 8));
            size_t n_lanes = 0;
            for (auto& d : E->dbs) n_lanes += d->lanes.size();
            IPB_CK(cudaMallocHost(&E->pinned_err, n_lanes * sizeof(int)));
            size_t li = 0;
            for (auto& d : E->dbs)
                for (auto& r : d->lanes) {
                    r->h_err = E->pinned_err + li++;
                    *r->h_err = 0;
                }
            E->trace.resize(4096);
            E->slots.resize(Q);
            for (size_t s = 0; s < Q; ++s) {
                E->slots[s].q = E->pinned_q + s * q_words;
                E->slots[s].resp = E->pinned_r + s * r_words;
                E->free_slots.push_back((uint32_t)(Q - 1 - s));
            }
            ipb::Engine* raw = E.get();
            E->worker = std::thread([raw] {
                cudaSetDevice(raw->dbs[0]->S->device);
                raw->run();
            });
            out = new ipir_serve{E.release()};
            return 0;
        },
        1);
    return out;
}

int ipir_serve_submit(ipir_serve* sv, size_t db, const ipir_query_view* q, uint64_t* ticket) {
    if (!sv || !q || !ticket) return 1;
    ipb::Engine& E = *sv->e;
    if (db >= E.dbs.size()) return 1;
    if (!q->lwe_b_limb0 || !q->lwe_b_limb1 || !q->ksk5_b || !q->kskneg1_b || !q->rgsw) return 3;
    uint32_t s;
    {
        std::lock_guard<std::mutex> lk(E.mu);
        if (E.failed) {
            ipb::set_last_error(E.fail_text.c_str());
            return 4;
        }
        if (E.free_slots.empty()) return 6;
        s = E.free_slots.back();
        E.free_slots.pop_back();
        ipb::ReqSlot& r = E.slots[s];
        r.state = ipb::kFilling;
        r.db = db;
        r.ticket = E.next_seq++ * E.slots.size() + s;
        *ticket = r.ticket;
    }
    const ipb::Server& S = *E.dbs[db]->S;
    const size_t R = S.pp.db_rows, B = ipb::kBlk;
    uint64_t* d = E.slots[s].q;
    std::memcpy(d, q->lwe_b_limb0, R * 8);
    std::memcpy(d + R, q->lwe_b_limb1, R * 8);
    std::memcpy(d + 2 * R, q->ksk5_b, B * 8);
    std::memcpy(d + 2 * R + B, q->kskneg1_b, B * 8);
    std::memcpy(d + 2 * R + 2 * B, q->rgsw, 4 * B * 8);
    {
        std::lock_guard<std::mutex> lk(E.mu);
        ipb::ReqSlot& r = E.slots[s];
        r.t_submit = ipb::Clock::now();
        if (E.failed) {
            r.state = ipb::kFailed;
            ++E.n_failed;
        } else {
            r.state = ipb::kQueued;
            E.dbs[db]->pending.push_back(s);
            ++E.submitted;
        }
    }
    E.cv_work.notify_one();
    return 0;
}

namespace {
// Collects a finished slot: 0 done, 1 pending, 2 unknown ticket, 4 failed.
int collect(ipb::Engine& E, std::unique_lock<std::mutex>& lk, uint64_t ticket, uint64_t* out, double* lat,
            double* queue) {
    const size_t s = (size_t)(ticket % E.slots.size());
    ipb::ReqSlot& r = E.slots[s];
    if (r.ticket != ticket || r.state == ipb::kFree || r.state == ipb::kCollecting) return 2;
    if (r.state == ipb::kFailed) {
        ipb::set_last_error(E.fail_text.empty() ? "request failed" : E.fail_text.c_str());
        r.state = ipb::kFree;
        E.free_slots.push_back((uint32_t)s);
        return 4;
    }
    if (r.state != ipb::kDone) return 1;
    if (lat) *lat = std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count();
    if (queue) *queue = std::chrono::duration<double, std::milli>(r.t_issue - r.t_submit).count();
    r.state = ipb::kCollecting;
    const size_t words = E.dbs[r.db]->S->resp_qstride;
    lk.unlock();
    if (out) std::memcpy(out, r.resp, words * 8);
    lk.lock();
    r.state = ipb::kFree;
    E.free_slots.push_back((uint32_t)s);
    return 0;
}
}  // namespace

int ipir_serve_poll(ipir_serve* sv, uint64_t ticket, uint64_t* out_resp, double* latency_ms, double* queue_ms) {
    if (!sv) return 1;
    std::unique_lock<std::mutex> lk(sv->e->mu);
    return collect(*sv->e, lk, ticket, out_resp, latency_ms, queue_ms);
}

int ipir_serve_wait(ipir_serve* sv, uint64_t ticket, double timeout_s, uint64_t* out_resp, double* latency_ms,
                    double* queue_ms) {
    if (!sv) return 1;
    ipb::Engine& E = *sv->e;
    const auto deadline = ipb::Clock::now() + std::chrono::duration_cast<ipb::Clock::duration>(
                                                  std::chrono::duration<double>(std::max(0.0, timeout_s)));
    std::unique_lock<std::mutex> lk(E.mu);
    for (;;) {
        const int rc = collect(E, lk, ticket, out_resp, latency_ms, queue_ms);
        if (rc != 1) return rc;
        if (E.cv_done.wait_until(lk, deadline) == std::cv_status::timeout) {
            const int rc2 = collect(E, lk, ticket, out_resp, latency_ms, queue_ms);
            return rc2 == 1 ? 5 : rc2;
        }
    }
}

int ipir_serve_stats(ipir_serve* sv, ipir_serve_counters* out) {
    if (!sv || !out) return 1;
    ipb::Engine& E = *sv->e;
    std::lock_guard<std::mutex> lk(E.mu);
    out->submitted = E.submitted;
    out->completed = E.completed;
    out->failed = E.n_failed;
    out->batches = E.batches;
    out->batched_queries = E.batched;
    out->max_batch_seen = E.max_seen;
    size_t q = 0;
    for (auto& d : E.dbs) q += d->pending.size();
    out->queued = q;
    out->free_slots = E.free_slots.size();
    out->max_notice_ms = E.max_notice_ms;
    return 0;
}

int ipir_serve_db_info(ipir_serve* sv, size_t db, size_t* lanes, size_t* max_batch, ipir_serve_schedule* sched,
                       size_t sched_len) {
    if (!sv) return 1;
    ipb::Engine& E = *sv->e;
    if (db >= E.dbs.size()) return 1;
    const ipb::DbState& d = *E.dbs[db];
    if (lanes) *lanes = d.lanes.size();
    if (max_batch) *max_batch = d.max_batch;
    if (sched)
        for (size_t c = 1; c < sched_len && c <= d.max_batch; ++c) {
            sched[c].matvec_tc = d.sched[c].matvec_tc;
            sched[c].tp_pass = d.sched[c].tp_pass;
            sched[c].horner_cluster = d.sched[c].horner_cluster;
            sched[c].tp_sms = d.sched[c].tp_sms;
            sched[c].slice = d.sched[c].slice;
            sched[c].hchunks = d.sched[c].hchunks;
        }
    return 0;
}

int ipir_serve_replace_db(ipir_serve* sv, size_t db, ipir_server* next) {
    if (!sv || !next || !next->s) return 1;
    ipb::Engine& E = *sv->e;
    if (db >= E.dbs.size()) return 1;
    ipb::DbState& d = *E.dbs[db];
    const ipb::Server& a = *d.S;
    const ipb::Server& b = *next->s;
    if (a.device != b.device || a.pp.db_rows != b.pp.db_rows || a.pp.db_cols != b.pp.db_cols ||
        a.pp.n_packed != b.pp.n_packed || a.pp.D != b.pp.D || a.pp.num_cts != b.pp.num_cts ||
        a.qstride != b.qstride || a.mv_qstride != b.mv_qstride || a.tc_kchunk_rows != b.tc_kchunk_rows ||
        a.mv_chunks != b.mv_chunks) {
        ipb::set_last_error("ipir_serve_replace_db: the new generation must have the same geometry and device");
        return 2;
    }
    std::unique_lock<std::mutex> lk(E.mu);
    if (E.failed) {
        ipb::set_last_error(E.fail_text.c_str());
        return 4;
    }
    if (d.swap_to) {
        ipb::set_last_error("ipir_serve_replace_db: a swap of this database is in progress");
        return 6;
    }
    if (d.S == next->s) return 0;
    d.swap_to = next->s;
    d.swap_done = false;
    E.cv_work.notify_one();
    E.cv_swap.wait(lk, [&] { return d.swap_done || E.stop; });
    if (!d.swap_done) return 4;
    if (!d.swap_err.empty()) {
        ipb::set_last_error(d.swap_err.c_str());
        return 4;
    }
    return 0;
}

size_t ipir_serve_trace(ipir_serve* sv, ipir_serve_batch_record* out, size_t max_records) {
    if (!sv || !out) return 0;
    ipb::Engine& E = *sv->e;
    std::lock_guard<std::mutex> lk(E.mu);
    const size_t cap = E.trace.size();
    const size_t avail = (size_t)std::min<uint64_t>(E.trace_n, cap);
    const size_t n = std::min(avail, max_records);
    for (size_t i = 0; i < n; ++i) out[i] = E.trace[(E.trace_n - n + i) % cap];
    return n;
}

void ipir_serve_destroy(ipir_serve* sv) {
    if (!sv) return;
    ipb::DeviceRestore keep_device;  // the engine's destructor switches to its device
    ipb::Engine* E = sv->e;
    {
        std::lock_guard<std::mutex> lk(E->mu);
        E->stop = true;
    }
    E->cv_work.notify_all();
    if (E->worker.joinable()) E->worker.join();
    delete E;
    delete sv;
}

}  // extern "C"
