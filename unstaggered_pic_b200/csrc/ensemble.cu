// Ensembles of independent explicit-method runs advanced together by one
// CUDA graph (upic_ensemble_*): every run keeps its own context, grid size,
// particle count, tiling and re-sort cadence; one graph holds `period` steps
// of every run, each run's chain of kernels on its own stream forked from
// and joined to the ensemble's stream, so the runs proceed concurrently and
// one launch advances all of them.  A graph freezes the host-side state its
// kernels were recorded with: the history ring slot, the re-sort counter
// and which of the two particle buffers is current (a re-sort swaps them).
// The period is a common multiple of 5 (the BDF history ring) and twice
// every re-sort interval, so a recorded period returns every run to the
// state it started from; replaying is valid while every run is in the state
// the graph was captured at and no call has since reallocated or reset it
// (the context's generation count), otherwise the next step call captures
// again.
//
// Implicit-method runs (CN_ORBIT, CN_ORBIT_NONREL) decide their outer
// iteration count on the host after every map evaluation, so their steps
// cannot be recorded; an ensemble of them advances each run on a pool of
// host threads instead (every run on its own stream), so that the small
// kernels and synchronisations of different runs overlap on the GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "context.h"

using namespace upic_host;

struct upic_ensemble {
    std::vector<upic_ctx*> runs;
    cudaStream_t master = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int period = 0;
    bool implicit = false;
    // per run: history head, re-sort counter and current particle buffer
    // where the graph starts and where it ends
    std::vector<int> head0, count0, cur0, head1, count1, cur1;
    // per run: state generation the graph was recorded in (a later particle
    // upload, start-up, state load or stream change makes it stale)
    std::vector<long> gen;
    long captures = 0, launches = 0;
};

namespace {

int phase_count(const upic_ctx* c) {
    // the re-sort counter only matters up to the interval (runs without
    // particles never re-sort)
    if (c->np <= 0) return 0;
    return c->steps_since_sort < c->sort_interval ? c->steps_since_sort : c->sort_interval;
}

void drop_graph(upic_ensemble* e) {
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    e->exec = nullptr;
    e->graph = nullptr;
}

int ens_fail(upic_ensemble* e, int code, const std::string& msg) {
    return fail(e->runs.empty() ? nullptr : e->runs[0], code, msg);
}

// Capture `period` steps of every run into one graph (the host-side step
// counters advance as the launches are recorded; the work runs when the
// graph is launched).
int capture(upic_ensemble* e) {
    drop_graph(e);
    const size_t n = e->runs.size();
    // host counters before recording: restored if the recording fails, so
    // that no run counts steps that never ran
    struct Saved {
        int head, cur, since;
        long steps;
    };
    std::vector<Saved> saved(n);
    for (size_t r = 0; r < n; ++r) {
        const upic_ctx* c = e->runs[r];
        saved[r] = {c->head, c->cur, c->steps_since_sort, c->steps};
    }
    auto restore = [&]() {
        for (size_t r = 0; r < n; ++r) {
            upic_ctx* c = e->runs[r];
            c->head = saved[r].head;
            c->cur = saved[r].cur;
            c->steps_since_sort = saved[r].since;
            c->steps = saved[r].steps;
        }
    };
    for (size_t r = 0; r < n; ++r) {
        e->head0[r] = e->runs[r]->head;
        e->count0[r] = phase_count(e->runs[r]);
        e->cur0[r] = e->runs[r]->cur;
        e->gen[r] = e->runs[r]->generation;
    }
    cudaError_t ce = cudaStreamBeginCapture(e->master, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) return ens_fail(e, UPIC_ERR_CUDA, std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(ce));
    int rc = 0;
    if ((ce = cudaEventRecord(e->fork, e->master)) != cudaSuccess) rc = UPIC_ERR_CUDA;
    for (size_t r = 0; r < n && rc == 0; ++r) {
        upic_ctx* c = e->runs[r];
        if ((ce = cudaStreamWaitEvent(c->st, e->fork, 0)) != cudaSuccess) {
            rc = UPIC_ERR_CUDA;
            break;
        }
        if ((rc = explicit_advance(c, e->period, 0, nullptr, false))) break;
        if ((ce = cudaEventRecord(e->join[r], c->st)) != cudaSuccess ||
            (ce = cudaStreamWaitEvent(e->master, e->join[r], 0)) != cudaSuccess)
            rc = UPIC_ERR_CUDA;
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(e->master, &g);
    if (rc || ee != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        restore();
        if (rc == UPIC_ERR_CUDA || rc == 0)
            return ens_fail(e, UPIC_ERR_CUDA,
                            std::string("ensemble capture: ") + cudaGetErrorString(ce != cudaSuccess ? ce : ee));
        return rc;
    }
    e->graph = g;
    if ((ce = cudaGraphInstantiate(&e->exec, e->graph, 0)) != cudaSuccess) {
        drop_graph(e);
        restore();
        return ens_fail(e, UPIC_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ce));
    }
    for (size_t r = 0; r < n; ++r) {
        e->head1[r] = e->runs[r]->head;
        e->count1[r] = phase_count(e->runs[r]);
        e->cur1[r] = e->runs[r]->cur;
    }
    ++e->captures;
    return 0;
}

bool at_capture_phase(const upic_ensemble* e) {
    for (size_t r = 0; r < e->runs.size(); ++r)
        if (e->runs[r]->head != e->head0[r] || phase_count(e->runs[r]) != e->count0[r] ||
            e->runs[r]->cur != e->cur0[r] || e->runs[r]->generation != e->gen[r])
            return false;
    return true;
}

int sync_all(upic_ensemble* e) {
    cudaError_t ce = cudaStreamSynchronize(e->master);
    for (upic_ctx* c : e->runs) {
        const cudaError_t c2 = cudaStreamSynchronize(c->st);
        if (ce == cudaSuccess) ce = c2;
    }
    if (ce != cudaSuccess) return ens_fail(e, UPIC_ERR_CUDA, std::string("ensemble step: ") + cudaGetErrorString(ce));
    return 0;
}

}  // namespace

extern "C" int upic_step_implicit(upic_ctx* c, int nsteps, double* diag, double* info, double* step_diag);

namespace {

// Implicit runs: a pool of host threads, each taking the next run and
// advancing it by nsteps with upic_step_implicit.  Runs are handed out
// largest first (longest-processing-time order), so that the last runs to
// start are the short ones and the threads finish together; each run's
// result does not depend on the order.
int step_threads(upic_ensemble* e, int nsteps) {
    const int n = (int)e->runs.size();
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int T = std::max(1, std::min({n, hw, 64}));
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return e->runs[a]->np > e->runs[b]->np; });
    std::atomic<int> next{0};
    std::vector<int> rc(n, 0);
    auto work = [&]() {
        for (int k = next++; k < n; k = next++) {
            const int i = order[k];
            upic_ctx* c = e->runs[i];
            if (cudaSetDevice(c->device) != cudaSuccess) {
                rc[i] = UPIC_ERR_CUDA;
                continue;
            }
            rc[i] = upic_step_implicit(c, nsteps, nullptr, nullptr, nullptr);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < T; ++t) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    for (int i = 0; i < n; ++i)
        if (rc[i]) {
            if (i == 0) return rc[0];
            return ens_fail(e, rc[i], "ensemble run " + std::to_string(i) + ": " + e->runs[i]->err);
        }
    return 0;
}

}  // namespace

extern "C" {

int upic_ensemble_create(upic_ctx* const* runs, int nruns, upic_ensemble** out) {
    if (!out || !runs || nruns < 1) return fail(nullptr, UPIC_ERR_ARGUMENT, "upic_ensemble_create: no runs");
    *out = nullptr;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(nullptr, UPIC_ERR_CUDA, "cudaGetDevice failed");
    std::vector<upic_ctx*> v(runs, runs + nruns);
    long period = 5;  // BDF history ring (kHistSlots)
    for (int r = 0; r < nruns; ++r) {
        upic_ctx* c = v[r];
        if (!c) return fail(nullptr, UPIC_ERR_ARGUMENT, "upic_ensemble_create: null run");
        for (int q = 0; q < r; ++q)
            if (v[q] == c) return fail(nullptr, UPIC_ERR_ARGUMENT, "upic_ensemble_create: a run appears twice");
        if ((c->imp != nullptr) != (v[0]->imp != nullptr))
            return fail(nullptr, UPIC_ERR_ARGUMENT,
                        "upic_ensemble_create: runs of explicit and implicit methods cannot share an ensemble");
        if (!c->fields_ready) return fail(nullptr, UPIC_ERR_STATE, "upic_ensemble_create: upic_init_fields first");
        if (c->profiling) return fail(nullptr, UPIC_ERR_STATE, "upic_ensemble_create: a run has profiling enabled");
        if (c->device != dev) return fail(nullptr, UPIC_ERR_ARGUMENT, "upic_ensemble_create: runs on another device");
        period = std::lcm(period, 2L * std::max(1, c->sort_interval));
        if (period > 1024) return fail(nullptr, UPIC_ERR_ARGUMENT, "upic_ensemble_create: re-sort intervals too unlike");
    }
    upic_ensemble* e = new upic_ensemble();
    e->runs = v;
    e->implicit = v[0]->imp != nullptr;
    e->period = e->implicit ? 1 : (int)period;
    e->join.assign(nruns, nullptr);
    e->head0.assign(nruns, 0);
    e->count0.assign(nruns, 0);
    e->head1.assign(nruns, 0);
    e->count1.assign(nruns, 0);
    e->cur0.assign(nruns, 0);
    e->cur1.assign(nruns, 0);
    e->gen.assign(nruns, -1);
    bool ok = cudaStreamCreateWithFlags(&e->master, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) == cudaSuccess;
    for (int r = 0; r < nruns && ok; ++r)
        ok = cudaEventCreateWithFlags(&e->join[r], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        upic_ensemble_destroy(e);
        return fail(nullptr, UPIC_ERR_CUDA, "upic_ensemble_create: stream or event creation failed");
    }
    *out = e;
    return UPIC_OK;
}

int upic_ensemble_period(const upic_ensemble* e, int* period) {
    if (!e || !period) return UPIC_ERR_ARGUMENT;
    *period = e->period;
    return UPIC_OK;
}

int upic_ensemble_step(upic_ensemble* e, int nsteps) {
    if (!e) return UPIC_ERR_ARGUMENT;
    if (nsteps < 0) return ens_fail(e, UPIC_ERR_ARGUMENT, "upic_ensemble_step: nsteps < 0");
    for (upic_ctx* c : e->runs)
        if (!c->fields_ready || c->profiling || (c->imp != nullptr) != e->implicit)
            return ens_fail(e, UPIC_ERR_STATE, "upic_ensemble_step: a run was reset or has profiling enabled");
    if (e->implicit) return step_threads(e, nsteps);
    int rc, left = nsteps;
    // work queued before on the runs' own streams is complete: every API
    // call that queues work on a run synchronises before it returns
    while (left >= e->period) {
        bool fresh = false;
        if (!e->exec || !at_capture_phase(e)) {
            if ((rc = capture(e))) return rc;
            fresh = true;
        }
        const cudaError_t ce = cudaGraphLaunch(e->exec, e->master);
        if (ce != cudaSuccess) return ens_fail(e, UPIC_ERR_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(ce));
        ++e->launches;
        if (!fresh) {
            // the recorded steps advanced the host counters only at capture
            for (size_t r = 0; r < e->runs.size(); ++r) {
                upic_ctx* c = e->runs[r];
                c->head = e->head1[r];
                c->cur = e->cur1[r];
                if (c->np > 0) c->steps_since_sort = e->count1[r];
                else c->steps_since_sort += e->period;
                c->steps += e->period;
            }
        }
        left -= e->period;
    }
    if (left > 0) {
        // the rest with ordinary launches, after the graph
        if (e->launches > 0) {
            const cudaError_t ce = cudaEventRecord(e->fork, e->master);
            if (ce != cudaSuccess) return ens_fail(e, UPIC_ERR_CUDA, "cudaEventRecord failed");
        }
        for (upic_ctx* c : e->runs) {
            if (e->launches > 0 && cudaStreamWaitEvent(c->st, e->fork, 0) != cudaSuccess)
                return ens_fail(e, UPIC_ERR_CUDA, "cudaStreamWaitEvent failed");
            if ((rc = explicit_advance(c, left, 0, nullptr, false))) return rc;
        }
    }
    return sync_all(e);
}

int upic_ensemble_destroy(upic_ensemble* e) {
    if (!e) return UPIC_OK;
    drop_graph(e);
    for (cudaEvent_t ev : e->join)
        if (ev) cudaEventDestroy(ev);
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->master) {
        cudaStreamSynchronize(e->master);
        cudaStreamDestroy(e->master);
    }
    delete e;
    return UPIC_OK;
}

}  // extern "C"
