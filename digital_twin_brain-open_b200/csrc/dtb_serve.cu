// Serving form: many resident networks under an HBM cap, a stream of
// simulate-window requests, and two policies to serve it.
//
// The reference serves one network per process group: every Run RPC
// (snn.proto:63-92, dist_simulator.cpp:3217-3451) is executed alone, in arrival
// order, on the network that Init loaded.  Here a Server holds a pool of
// networks (each an Engine) and replays a request trace in real time:
//
//   * policy DTB_SERVE_BATCHED -- continuous batching: between slices of
//     `slice_steps` steps, finished requests leave and arrived ones join; every
//     slice advances all requests in flight with ONE launch of each per-step
//     kernel (the Batch of dtb_batch.cu, membership reset in place);
//   * policy DTB_SERVE_SEQUENTIAL -- the plain path: one request at a time, in
//     arrival order, each a dtb_run of its network.
//
// A request carries its network, its step count, new per-population OU
// parameters (Updateoubackgroundparam before the Run) and a host buffer for the
// per-step population spike counts (RunResponse.freq).  A network holds at most
// one request in flight; later requests for it wait in arrival order.
//
// Networks whose device memory would push the resident total above the cap are
// evicted to the host (state blob + their last OU parameters; the CSR is rebuilt
// from the spec or the npz file on return), least recently used first, never
// one with a request in flight.  Restoring gives bit-identical continuations:
// the OU parameters are re-applied, then the state blob (V, J, OU current,
// t_last, spike bitmaps, clock) is loaded, and the device noise is keyed by
// (seed, step, neuron).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>

#include "dtb_batch.h"

namespace dtb {

using WallClock = std::chrono::steady_clock;

struct ServedNet {
    // how to rebuild it
    bool structured = true;
    std::string npz;
    dtb_options opt{};
    dtb_structured_spec spec{};
    std::vector<uint32_t> sizes, exc;
    std::vector<uint64_t> cdf;
    std::vector<float> prop;
    // residency
    Engine* eng = nullptr;
    std::vector<uint8_t> saved;          // state blob while evicted (empty before the first eviction)
    uint64_t bytes = 0;                  // device bytes when resident (0 until first built)
    uint64_t last_use = 0;
    int busy = -1;                       // request in flight on it
    // identity and the OU parameters last set (re-applied after a restore)
    uint32_t P = 0;
    std::vector<uint32_t> pop_ids;
    std::vector<float> ou_mean, ou_sigma, ou_tau;
};

// A request submitted to the online scheduler (dtb_server_submit): the caller's
// struct receives the outputs; the OU parameters are copied at submission.
struct Job {
    dtb_request* r = nullptr;
    uint64_t ticket = 0;
    std::vector<float> ou_mean, ou_sigma, ou_tau;
    std::vector<int32_t> scratch;        // per-step counts when the caller passed no buffer
    uint32_t done_steps = 0;
    bool finished = false;
};

class Server {
public:
    ~Server();
    dtb_server_options o{};
    std::deque<ServedNet> nets;           // stable addresses: engines are reached through references
    uint64_t resident_bytes = 0;
    uint64_t clock = 0;                   // LRU clock
    dtb_server_stats stats{};
    Batch* batch = nullptr;

    int add(ServedNet&& sn, uint32_t* id);
    int build(ServedNet& sn);
    int evict(ServedNet& sn);
    int make_resident(uint32_t id, bool* ok);
    int begin_request(dtb_request& r);
    int play(uint32_t n, dtb_request* reqs, uint32_t policy);
    int play_sequential(uint32_t n, dtb_request* reqs);
    int play_batched(uint32_t n, dtb_request* reqs);

    // ---- online serving: a scheduler thread admits submitted requests as slots and
    // device memory free up, between slices of the requests in flight
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread worker;
    bool running = false, stopping = false;
    uint32_t online_policy = DTB_SERVE_BATCHED;
    int worker_status = DTB_OK;
    std::string worker_error;
    uint64_t next_ticket = 1;
    std::deque<Job*> submitted;                       // not yet admitted, arrival order
    std::map<uint64_t, std::unique_ptr<Job>> jobs;    // every job until its result is collected
    WallClock::time_point t0_online;
    int start(uint32_t policy);
    int submit(dtb_request* r, uint64_t* ticket);
    int poll(uint64_t ticket, uint32_t wait_ms, int32_t* done);
    int stop();
    void serve_online();
    int online_slice(std::vector<Job*>& inflight, bool& changed, std::vector<Engine*>& members);
};

Server::~Server() {
    stop();
    delete batch;
    for (ServedNet& sn : nets) delete sn.eng;
}

int Server::build(ServedNet& sn) {
    auto* e = new Engine();
    int st = sn.structured ? e->create_structured(sn.spec, sn.opt) : e->create_from_npz(sn.npz, sn.opt);
    // parameters first: a population's first OU configuration resets its OU
    // current to the mean, which the saved state must then overwrite
    if (st == DTB_OK && !sn.ou_mean.empty())
        st = e->set_ou(sn.P, sn.pop_ids.data(), sn.ou_mean.data(), sn.ou_sigma.data(), sn.ou_tau.data());
    if (st == DTB_OK && !sn.saved.empty()) st = e->load_state(sn.saved.data(), sn.saved.size());
    if (st != DTB_OK) {
        delete e;
        return st;
    }
    e->autotune = o.autotune != 0;     // plain-path runs tune (or not) like the batch
    sn.eng = e;
    sn.bytes = e->dev_bytes;
    resident_bytes += sn.bytes;
    sn.saved.clear();
    sn.saved.shrink_to_fit();
    return DTB_OK;
}

int Server::evict(ServedNet& sn) {
    sn.saved.resize(sn.eng->state_size());
    DTB_TRY(sn.eng->save_state(sn.saved.data(), sn.saved.size()));
    resident_bytes -= sn.bytes;
    delete sn.eng;
    sn.eng = nullptr;
    ++stats.evictions;
    return DTB_OK;
}

// Device memory kept free beyond a network's own bytes when it is rebuilt (the
// device CSR build sorts through temporary buffers).
constexpr uint64_t kRebuildReserve = 1ull << 30;

// Bring network `id` into HBM.  It is admitted when the resident networks stay
// within the cap AND the device has the bytes free (cudaMemGetInfo: other engines
// and other processes count too); idle networks are evicted, least recently used
// first, until both hold.  *ok = false when only networks with requests in flight
// stand in the way (the caller retries after a slice).
int Server::make_resident(uint32_t id, bool* ok) {
    ServedNet& sn = nets[id];
    *ok = true;
    sn.last_use = ++clock;
    if (sn.eng) return DTB_OK;
    const uint64_t need = sn.bytes;
    auto fits = [&](bool* yes) -> int {
        size_t free_b = 0, total_b = 0;
        DTB_CU(cudaMemGetInfo(&free_b, &total_b));
        *yes = resident_bytes + need <= o.hbm_cap_bytes && free_b >= need + kRebuildReserve;
        return DTB_OK;
    };
    bool yes = false;
    DTB_TRY(fits(&yes));
    while (!yes) {
        ServedNet* victim = nullptr;
        for (ServedNet& c : nets)
            if (c.eng && c.busy < 0 && &c != &sn && (!victim || c.last_use < victim->last_use)) victim = &c;
        if (!victim) {
            *ok = false;
            return DTB_OK;
        }
        DTB_TRY(evict(*victim));
        DTB_TRY(fits(&yes));
    }
    DTB_TRY(build(sn));
    ++stats.restores;
    return DTB_OK;
}

int Server::add(ServedNet&& sn_in, uint32_t* id) {
    {
        std::lock_guard<std::mutex> lk(mu);
        if (running) return fail(DTB_UNSUPPORTED, "networks are added before dtb_server_start or after dtb_server_stop");
    }
    nets.push_back(std::move(sn_in));
    ServedNet& sn = nets.back();
    if (sn.structured) {
        sn.spec.pop_sizes = sn.sizes.data();
        sn.spec.pop_exc = sn.exc.data();
        sn.spec.src_cdf = sn.cdf.data();
        sn.spec.pop_property = sn.prop.data();
    }
    // first build: make room the same way a restore does, then record the size
    const uint32_t nid = static_cast<uint32_t>(nets.size() - 1);
    int st = build(sn);
    if (st != DTB_OK) {
        nets.pop_back();
        return st;
    }
    sn.last_use = ++clock;
    sn.P = sn.eng->P;
    sn.pop_ids = sn.eng->pop_ids;
    if (sn.bytes > o.hbm_cap_bytes) {
        resident_bytes -= sn.bytes;
        delete sn.eng;
        nets.pop_back();
        return fail(DTB_OUT_OF_MEMORY, "network larger than the HBM cap");
    }
    while (resident_bytes > o.hbm_cap_bytes) {
        ServedNet* victim = nullptr;
        for (ServedNet& c : nets)
            if (c.eng && c.busy < 0 && &c != &sn && (!victim || c.last_use < victim->last_use)) victim = &c;
        if (!victim) break;
        DTB_TRY(evict(*victim));
    }
    *id = nid;
    return DTB_OK;
}

// Updateoubackgroundparam of the request (kept on the host for restores).
int Server::begin_request(dtb_request& r) {
    ServedNet& sn = nets[r.net];
    if (r.ou_mean) {
        sn.ou_mean.assign(r.ou_mean, r.ou_mean + sn.P);
        sn.ou_sigma.assign(r.ou_sigma, r.ou_sigma + sn.P);
        sn.ou_tau.assign(r.ou_tau, r.ou_tau + sn.P);
        DTB_TRY(sn.eng->set_ou(sn.P, sn.pop_ids.data(), r.ou_mean, r.ou_sigma, r.ou_tau));
    }
    r.events = 0;
    return DTB_OK;
}

static double seconds_since(WallClock::time_point t0) {
    return std::chrono::duration<double>(WallClock::now() - t0).count();
}

static void wait_until(WallClock::time_point t0, double s) {
    const double dt = s - seconds_since(t0);
    if (dt > 0) std::this_thread::sleep_for(std::chrono::duration<double>(dt));
}

int Server::play_sequential(uint32_t n, dtb_request* reqs) {
    const WallClock::time_point t0 = WallClock::now();
    const uint32_t flags = o.flags | DTB_RUN_FREQ;
    for (uint32_t i = 0; i < n; ++i) {
        dtb_request& r = reqs[i];
        wait_until(t0, r.arrival_s);
        bool ok = false;
        DTB_TRY(make_resident(r.net, &ok));
        if (!ok) return fail(DTB_OUT_OF_MEMORY, "no room for the network under the HBM cap");
        ServedNet& sn = nets[r.net];
        DTB_TRY(begin_request(r));
        r.start_s = seconds_since(t0);
        std::vector<int32_t> scratch;
        int32_t* fr = r.freqs;
        if (!fr) {
            scratch.resize(static_cast<size_t>(r.iters) * sn.P);
            fr = scratch.data();
        }
        dtb_run_request rq{r.iters, flags, DTB_PROP_THRESHOLD, o.syn_mode, 1, {0, 0, 0}};
        dtb_run_output out{};
        out.freqs = fr;
        r.status = sn.eng->run(rq, out);
        DTB_TRY(r.status);
        r.events = out.events;
        r.finish_s = seconds_since(t0);
        ++stats.slices;
        stats.batch_members_sum += 1;
    }
    return DTB_OK;
}

int Server::play_batched(uint32_t n, dtb_request* reqs) {
    const WallClock::time_point t0 = WallClock::now();
    const uint32_t flags = o.flags | DTB_RUN_FREQ;
    std::deque<uint32_t> pending;          // arrived, not admitted, arrival order
    std::vector<uint32_t> inflight;        // admitted
    std::vector<uint32_t> done_steps(n, 0);
    std::vector<std::vector<int32_t>> scratch(n);
    std::vector<Engine*> members;
    bool changed = true;
    uint32_t next = 0, completed = 0;
    while (completed < n) {
        const double now = seconds_since(t0);
        while (next < n && reqs[next].arrival_s <= now) pending.push_back(next++);
        // admit in arrival order; a request waits while its network is busy
        for (auto it = pending.begin(); it != pending.end() && inflight.size() < o.max_batch;) {
            dtb_request& r = reqs[*it];
            if (nets[r.net].busy >= 0) { ++it; continue; }
            bool ok = false;
            DTB_TRY(make_resident(r.net, &ok));
            if (!ok) break;
            nets[r.net].busy = static_cast<int>(*it);
            DTB_TRY(begin_request(r));
            r.start_s = seconds_since(t0);
            if (!r.freqs) scratch[*it].resize(static_cast<size_t>(r.iters) * nets[r.net].P);
            inflight.push_back(*it);
            it = pending.erase(it);
            changed = true;
        }
        if (inflight.empty()) {
            if (next < n) wait_until(t0, reqs[next].arrival_s);
            continue;
        }
        uint32_t slice = o.slice_steps;
        for (uint32_t q : inflight) slice = std::min(slice, reqs[q].iters - done_steps[q]);
        if (changed) {
            members.clear();
            for (uint32_t q : inflight) members.push_back(nets[reqs[q].net].eng);
            if (!batch) {
                batch = new Batch();
                DTB_TRY(batch->create(members.data(), static_cast<uint32_t>(members.size())));
                batch->push_cfg = PushCfg{PUSH_REG, 8, 32};
                batch->autotune = o.autotune != 0;
            } else {
                DTB_TRY(batch->set_members(members.data(), static_cast<uint32_t>(members.size())));
            }
            changed = false;
        }
        std::vector<dtb_run_output> outs(inflight.size());
        for (size_t i = 0; i < inflight.size(); ++i) {
            const uint32_t q = inflight[i];
            int32_t* fr = reqs[q].freqs ? reqs[q].freqs : scratch[q].data();
            outs[i] = dtb_run_output{};
            outs[i].freqs = fr + static_cast<size_t>(done_steps[q]) * nets[reqs[q].net].P;
        }
        dtb_run_request rq{slice, flags, DTB_PROP_THRESHOLD, o.syn_mode, 1, {0, 0, 0}};
        DTB_TRY(batch->run(rq, outs.data()));
        ++stats.slices;
        stats.batch_members_sum += inflight.size();
        const double t_end = seconds_since(t0);
        for (size_t i = 0; i < inflight.size();) {
            const uint32_t q = inflight[i];
            done_steps[q] += slice;
            reqs[q].events += outs[i].events;
            nets[reqs[q].net].last_use = ++clock;
            if (done_steps[q] == reqs[q].iters) {
                reqs[q].finish_s = t_end;
                reqs[q].status = DTB_OK;
                nets[reqs[q].net].busy = -1;
                ++completed;
                inflight.erase(inflight.begin() + i);
                outs.erase(outs.begin() + i);
                changed = true;
            } else {
                ++i;
            }
        }
    }
    return DTB_OK;
}

int Server::start(uint32_t policy) {
    if (policy > DTB_SERVE_SEQUENTIAL) return fail(DTB_INVALID_PARAMETER, "unknown serving policy");
    std::lock_guard<std::mutex> lk(mu);
    if (running) return fail(DTB_INVALID_PARAMETER, "the server is already serving");
    for (ServedNet& sn : nets) sn.busy = -1;
    online_policy = policy;
    stopping = false;
    worker_status = DTB_OK;
    worker_error.clear();
    t0_online = WallClock::now();
    int dev = 0;
    DTB_CU(cudaGetDevice(&dev));
    running = true;
    worker = std::thread([this, dev] {
        cudaSetDevice(dev);
        serve_online();
    });
    return DTB_OK;
}

int Server::submit(dtb_request* r, uint64_t* ticket) {
    if (!r || !ticket) return fail(DTB_INVALID_PARAMETER, "NULL argument");
    std::lock_guard<std::mutex> lk(mu);
    if (!running || stopping) return fail(DTB_INVALID_PARAMETER, "the server is not serving (dtb_server_start)");
    if (r->net >= nets.size()) return fail(DTB_INVALID_PARAMETER, "request for an unknown network");
    if (r->iters == 0) return fail(DTB_INVALID_PARAMETER, "request with zero steps");
    if (r->ou_mean && (!r->ou_sigma || !r->ou_tau)) return fail(DTB_INVALID_PARAMETER, "OU mean without sigma or tau");
    auto job = std::make_unique<Job>();
    job->r = r;
    job->ticket = next_ticket++;
    const uint32_t P = nets[r->net].P;
    if (r->ou_mean) {
        job->ou_mean.assign(r->ou_mean, r->ou_mean + P);
        job->ou_sigma.assign(r->ou_sigma, r->ou_sigma + P);
        job->ou_tau.assign(r->ou_tau, r->ou_tau + P);
    }
    if (!r->freqs) job->scratch.resize(static_cast<size_t>(r->iters) * P);
    r->status = -1;
    r->arrival_s = seconds_since(t0_online);
    r->start_s = r->finish_s = 0.0;
    r->events = 0;
    *ticket = job->ticket;
    submitted.push_back(job.get());
    jobs[job->ticket] = std::move(job);
    cv_work.notify_one();
    return DTB_OK;
}

int Server::poll(uint64_t ticket, uint32_t wait_ms, int32_t* done) {
    if (!done) return fail(DTB_INVALID_PARAMETER, "NULL argument");
    std::unique_lock<std::mutex> lk(mu);
    auto it = jobs.find(ticket);
    if (it == jobs.end()) return fail(DTB_INVALID_PARAMETER, "unknown ticket (never submitted, or already collected)");
    Job* j = it->second.get();
    cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return j->finished || !running; });
    *done = j->finished ? 1 : 0;
    if (j->finished) {
        jobs.erase(it);      // collected: the caller's struct holds the outputs
        return DTB_OK;
    }
    if (!running && worker_status != DTB_OK) return fail(worker_status, worker_error);
    return DTB_OK;
}

int Server::stop() {
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!running) return DTB_OK;
        stopping = true;
        cv_work.notify_all();
    }
    if (worker.joinable()) worker.join();
    std::lock_guard<std::mutex> lk(mu);
    running = false;
    cv_done.notify_all();
    if (worker_status != DTB_OK) return fail(worker_status, worker_error);
    return DTB_OK;
}

// One pass of the scheduler: admit waiting requests in arrival order (a network
// holds one request at a time; room under the cap and in free device memory),
// then advance every request in flight by one slice (batched) or run the oldest
// to completion (sequential), and hand back the finished ones.
int Server::online_slice(std::vector<Job*>& inflight, bool& changed, std::vector<Engine*>& members) {
    std::vector<Job*> waiting;
    {
        std::lock_guard<std::mutex> lk(mu);
        waiting.assign(submitted.begin(), submitted.end());
    }
    const uint32_t cap = online_policy == DTB_SERVE_SEQUENTIAL ? 1u : o.max_batch;
    std::vector<Job*> admitted;
    for (Job* j : waiting) {
        if (inflight.size() >= cap) break;
        dtb_request& r = *j->r;
        if (nets[r.net].busy >= 0) continue;
        bool ok = false;
        DTB_TRY(make_resident(r.net, &ok));
        if (!ok) break;
        ServedNet& sn = nets[r.net];
        sn.busy = static_cast<int>(j->ticket & 0x7FFFFFFF);
        if (!j->ou_mean.empty()) {
            sn.ou_mean = j->ou_mean;
            sn.ou_sigma = j->ou_sigma;
            sn.ou_tau = j->ou_tau;
            DTB_TRY(sn.eng->set_ou(sn.P, sn.pop_ids.data(), j->ou_mean.data(), j->ou_sigma.data(), j->ou_tau.data()));
        }
        r.start_s = seconds_since(t0_online);
        inflight.push_back(j);
        admitted.push_back(j);
        changed = true;
    }
    if (!admitted.empty()) {
        std::lock_guard<std::mutex> lk(mu);
        for (Job* j : admitted) submitted.erase(std::find(submitted.begin(), submitted.end(), j));
    }
    if (inflight.empty()) return DTB_OK;
    const uint32_t flags = o.flags | DTB_RUN_FREQ;
    std::vector<Job*> finished;
    if (online_policy == DTB_SERVE_SEQUENTIAL) {
        Job* j = inflight.front();
        dtb_request& r = *j->r;
        ServedNet& sn = nets[r.net];
        dtb_run_request rq{r.iters, flags, DTB_PROP_THRESHOLD, o.syn_mode, 1, {0, 0, 0}};
        dtb_run_output out{};
        out.freqs = r.freqs ? r.freqs : j->scratch.data();
        DTB_TRY(sn.eng->run(rq, out));
        r.events = out.events;
        j->done_steps = r.iters;
        sn.last_use = ++clock;
        finished.push_back(j);
        inflight.clear();
        ++stats.slices;
        stats.batch_members_sum += 1;
    } else {
        uint32_t slice = o.slice_steps;
        for (Job* j : inflight) slice = std::min(slice, j->r->iters - j->done_steps);
        if (changed) {
            members.clear();
            for (Job* j : inflight) members.push_back(nets[j->r->net].eng);
            if (!batch) {
                batch = new Batch();
                DTB_TRY(batch->create(members.data(), static_cast<uint32_t>(members.size())));
                batch->push_cfg = PushCfg{PUSH_REG, 8, 32};
                batch->autotune = o.autotune != 0;
            } else {
                DTB_TRY(batch->set_members(members.data(), static_cast<uint32_t>(members.size())));
            }
            changed = false;
        }
        std::vector<dtb_run_output> outs(inflight.size());
        for (size_t i = 0; i < inflight.size(); ++i) {
            Job* j = inflight[i];
            int32_t* fr = j->r->freqs ? j->r->freqs : j->scratch.data();
            outs[i] = dtb_run_output{};
            outs[i].freqs = fr + static_cast<size_t>(j->done_steps) * nets[j->r->net].P;
        }
        dtb_run_request rq{slice, flags, DTB_PROP_THRESHOLD, o.syn_mode, 1, {0, 0, 0}};
        DTB_TRY(batch->run(rq, outs.data()));
        ++stats.slices;
        stats.batch_members_sum += inflight.size();
        for (size_t i = 0; i < inflight.size();) {
            Job* j = inflight[i];
            j->done_steps += slice;
            j->r->events += outs[i].events;
            nets[j->r->net].last_use = ++clock;
            if (j->done_steps == j->r->iters) {
                finished.push_back(j);
                inflight.erase(inflight.begin() + static_cast<long>(i));
                outs.erase(outs.begin() + static_cast<long>(i));
                changed = true;
            } else {
                ++i;
            }
        }
    }
    if (!finished.empty()) {
        const double t = seconds_since(t0_online);
        std::lock_guard<std::mutex> lk(mu);
        for (Job* j : finished) {
            nets[j->r->net].busy = -1;
            j->r->finish_s = t;
            j->r->status = DTB_OK;
            j->finished = true;
        }
        cv_done.notify_all();
    }
    return DTB_OK;
}

void Server::serve_online() {
    std::vector<Job*> inflight;
    std::vector<Engine*> members;
    bool changed = true;
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] { return stopping || !submitted.empty() || !inflight.empty(); });
            if (stopping && submitted.empty() && inflight.empty()) break;
        }
        const int st = online_slice(inflight, changed, members);
        if (st != DTB_OK) {
            // a failure ends the scheduler: every unfinished request carries the status
            std::lock_guard<std::mutex> lk(mu);
            worker_status = st;
            worker_error = last_error();
            for (auto& kv : jobs) {
                if (kv.second->finished) continue;
                kv.second->r->status = st;
                kv.second->finished = true;
            }
            for (ServedNet& sn : nets) sn.busy = -1;
            submitted.clear();
            cv_done.notify_all();
            break;
        }
    }
}

int Server::play(uint32_t n, dtb_request* reqs, uint32_t policy) {
    {
        std::lock_guard<std::mutex> lk(mu);
        if (running) return fail(DTB_INVALID_PARAMETER, "the server is serving online (dtb_server_stop first)");
    }
    for (uint32_t i = 0; i < n; ++i) {
        dtb_request& r = reqs[i];
        if (r.net >= nets.size()) return fail(DTB_INVALID_PARAMETER, "request for an unknown network");
        if (r.iters == 0) return fail(DTB_INVALID_PARAMETER, "request with zero steps");
        if (i > 0 && r.arrival_s < reqs[i - 1].arrival_s) return fail(DTB_INVALID_PARAMETER, "arrival times must be non-decreasing");
        if (r.ou_mean && (!r.ou_sigma || !r.ou_tau)) return fail(DTB_INVALID_PARAMETER, "OU mean without sigma or tau");
        r.status = -1;
        r.start_s = r.finish_s = 0.0;
        r.events = 0;
    }
    for (ServedNet& sn : nets) sn.busy = -1;
    if (policy == DTB_SERVE_SEQUENTIAL) return play_sequential(n, reqs);
    if (policy == DTB_SERVE_BATCHED) return play_batched(n, reqs);
    return fail(DTB_INVALID_PARAMETER, "unknown serving policy");
}

}  // namespace dtb

using dtb::Server;

namespace {

template <class F>
int32_t server_guarded(F&& f) {
    try {
        return static_cast<int32_t>(f());
    } catch (const std::bad_alloc&) {
        return dtb::fail(DTB_OUT_OF_MEMORY, "host allocation failed");
    }
}

}  // namespace

extern "C" {

void dtb_server_default_options(dtb_server_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->hbm_cap_bytes = 150ull * 1000 * 1000 * 1000;
    o->slice_steps = 100;
    o->max_batch = 64;
    o->syn_mode = DTB_SYN_PUSH;
    o->flags = DTB_RUN_USE_OU;
    o->autotune = 1;
}

int32_t dtb_server_create(const dtb_server_options* opt, void** server) {
    if (!opt || !server) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    if (opt->slice_steps == 0 || opt->max_batch == 0) return dtb::fail(DTB_INVALID_PARAMETER, "slice_steps and max_batch must be positive");
    if (opt->syn_mode > DTB_SYN_PUSH_FIXED) return dtb::fail(DTB_INVALID_PARAMETER, "unknown syn_mode");
    return server_guarded([&] {
        auto* s = new Server();
        s->o = *opt;
        *server = s;
        return DTB_OK;
    });
}

int32_t dtb_server_destroy(void* server) {
    if (!server) return dtb::fail(DTB_INVALID_PARAMETER, "NULL server");
    delete static_cast<Server*>(server);
    return DTB_OK;
}

int32_t dtb_server_add_structured(void* server, const dtb_structured_spec* spec, const dtb_options* opt, uint32_t* net_id) {
    if (!server || !spec || !opt || !net_id) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    if (spec->n_pops == 0 || !spec->pop_sizes || !spec->pop_exc || !spec->src_cdf || !spec->pop_property)
        return dtb::fail(DTB_INVALID_PARAMETER, "structured spec incomplete");
    return server_guarded([&] {
        dtb::ServedNet sn;
        const uint32_t P = spec->n_pops;
        sn.structured = true;
        sn.opt = *opt;
        sn.spec = *spec;
        sn.sizes.assign(spec->pop_sizes, spec->pop_sizes + P);
        sn.exc.assign(spec->pop_exc, spec->pop_exc + P);
        sn.cdf.assign(spec->src_cdf, spec->src_cdf + static_cast<size_t>(P) * P);
        sn.prop.assign(spec->pop_property, spec->pop_property + static_cast<size_t>(P) * 22);
        return static_cast<Server*>(server)->add(std::move(sn), net_id);
    });
}

int32_t dtb_server_add_npz(void* server, const char* path, const dtb_options* opt, uint32_t* net_id) {
    if (!server || !path || !opt || !net_id) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    return server_guarded([&] {
        dtb::ServedNet sn;
        sn.structured = false;
        sn.npz = path;
        sn.opt = *opt;
        return static_cast<Server*>(server)->add(std::move(sn), net_id);
    });
}

int32_t dtb_server_play(void* server, uint32_t n, dtb_request* reqs, uint32_t policy) {
    if (!server || (n && !reqs)) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    return server_guarded([&] { return static_cast<Server*>(server)->play(n, reqs, policy); });
}

int32_t dtb_server_start(void* server, uint32_t policy) {
    if (!server) return dtb::fail(DTB_INVALID_PARAMETER, "NULL server");
    return server_guarded([&] { return static_cast<Server*>(server)->start(policy); });
}

int32_t dtb_server_submit(void* server, dtb_request* req, uint64_t* ticket) {
    if (!server) return dtb::fail(DTB_INVALID_PARAMETER, "NULL server");
    return server_guarded([&] { return static_cast<Server*>(server)->submit(req, ticket); });
}

int32_t dtb_server_poll(void* server, uint64_t ticket, uint32_t wait_ms, int32_t* done) {
    if (!server) return dtb::fail(DTB_INVALID_PARAMETER, "NULL server");
    return server_guarded([&] { return static_cast<Server*>(server)->poll(ticket, wait_ms, done); });
}

int32_t dtb_server_stop(void* server) {
    if (!server) return dtb::fail(DTB_INVALID_PARAMETER, "NULL server");
    return server_guarded([&] { return static_cast<Server*>(server)->stop(); });
}

int32_t dtb_server_info(void* server, dtb_server_stats* info) {
    if (!server || !info) return dtb::fail(DTB_INVALID_PARAMETER, "NULL argument");
    const Server* s = static_cast<const Server*>(server);
    *info = s->stats;
    info->n_nets = static_cast<uint32_t>(s->nets.size());
    info->resident = 0;
    for (const dtb::ServedNet& sn : s->nets) info->resident += sn.eng != nullptr;
    info->resident_bytes = s->resident_bytes;
    return DTB_OK;
}

}  // extern "C"
