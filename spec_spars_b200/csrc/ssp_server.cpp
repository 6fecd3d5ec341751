// ssp_server.cpp -- a persistent request loop for sparsification on one device.
//
// The reference runs one graph per process (sparsify_dataset, lib.rs:158-168; InputStream::run_stream,
// stream.rs:40-64).  Here requests of uneven size arrive from any host thread (ssp_submit) and are served by
// `slots` worker threads, each owning one ssp_context (its own stream and grow-only workspace), so the
// admitted requests run concurrently on the device.
// Admission: a free slot takes the oldest pending request whose estimated device footprint fits beside the
// footprints in flight (the HBM budget).  A younger request may go ahead of an older one that does not fit
// yet, until the older one has waited FRONT_AGE_MS; from then on admission is strictly first come, first
// served, so a large request is not starved.  A request whose footprint alone exceeds the budget is refused
// at submit.
// Batching (continuous): the slot then adds the other pending requests that can share its run -- the same
// factor seed, precision, PCG options and reweighting, the same epsilon, and dense_threshold = 0 (each keeps
// its own truncation, fixed or autotuned) -- up to max_batch requests and the slot's share of the
// budget, and runs them as one ssp_sparsify_batch: one factorization and one PCG over their disjoint union.
// Requests that arrive while batches run are picked up by the next free slot, so their work overlaps on the
// device.  A request that cannot be batched runs the same ssp_sparsify as a lone call; a batched one equals
// its lone result to the solve's rounding (ssp_sparsify_batch).  If a batch fails as a whole, its requests are
// run one by one.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/specspars.h"

namespace ssp {
double spmm_slab_mb();  // ssp_pcg.cu
}

namespace ssp {
void set_last_error(const std::string& msg);
}

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

constexpr double FRONT_AGE_MS = 500.0;  // after this wait the oldest request is admitted strictly first

struct Job {
    uint64_t ticket = 0;
    int64_t n = 0;
    std::vector<int64_t> colptr;
    std::vector<int32_t> rowidx;
    std::vector<double> values;
    ssp_params params;
    int32_t check_probes = 0;
    std::string output_file;
    int64_t est_bytes = 0;
    Clock::time_point t_submit, t_admit, t_done;
    bool done = false;
    int32_t status = SSP_OK;
    std::string error;
    ssp_csc_out out;
    ssp_stats stats;
    int32_t slot = -1;
    int32_t batch = 0;  // requests in the run that served this one
    // inline check (a15)
    bool checked = false;
    ssp_probe_result probe{};
    int64_t cc_graph = 0, cc_sparsifier = 0;
    double check_ms = 0.0;
};

// x^T L_H x against x^T L_G x on the request's own graph, and the component counts of both (a15)
int check_result(ssp_context* ctx, const ssp_csc& g, const ssp_params& prm, int32_t probes, const ssp_csc_out& out,
                 Job* j) {
    int64_t m = 0, lnnz = 0;
    int rc = ssp_stage_graph(ctx, &g, &m, &lnnz, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    if (rc != SSP_OK) return rc;
    std::vector<int32_t> v1(m + 1), v2(m + 1), ri(lnnz + 1);
    std::vector<double> w(m + 1), va(lnnz + 1);
    std::vector<int64_t> cp(g.n + 1);
    rc = ssp_stage_graph(ctx, &g, &m, &lnnz, v1.data(), v2.data(), w.data(), cp.data(), ri.data(), va.data());
    if (rc != SSP_OK) return rc;
    ssp_csc lg{g.n, lnnz, cp.data(), ri.data(), va.data(), SSP_MEM_HOST};
    ssp_csc lh{out.n, out.nnz, out.colptr, out.rowidx, out.values, SSP_MEM_HOST};
    rc = ssp_probe_quadratic_form(ctx, &lg, &lh, prm.epsilon, probes, prm.sampling_seed, &j->probe);
    if (rc != SSP_OK) return rc;
    rc = ssp_connected_components(ctx, &g, SSP_MEM_HOST, nullptr, &j->cc_graph);
    if (rc != SSP_OK) return rc;
    return ssp_connected_components(ctx, &lh, SSP_MEM_HOST, nullptr, &j->cc_sparsifier);
}

int fail(int code, const std::string& msg) {
    ssp::set_last_error(msg);
    return code;
}

bool batchable(const ssp_params& p) { return p.dense_threshold == 0 && p.factor_max_degree >= -1; }

bool same_batch(const ssp_params& a, const ssp_params& b) {
    return a.epsilon == b.epsilon && a.factor_seed == b.factor_seed && a.precision == b.precision &&
           a.pcg_tol == b.pcg_tol && a.pcg_abs_tol == b.pcg_abs_tol && a.pcg_max_iters == b.pcg_max_iters &&
           a.reweight == b.reweight && batchable(a) && batchable(b);
}

// device footprint of a batch: its union's n x ld blocks use the largest k of the batch for every row
int64_t batch_footprint(const std::vector<Job*>& js) {
    if (js.size() == 1) return js[0]->est_bytes;
    int64_t ld = 0, n = 0, nnz = 0;
    for (const Job* j : js) {
        const int64_t k = ssp_params_jl_dim(&j->params, j->n);
        ld = std::max<int64_t>(ld, (k + 31) / 32 * 32);
        n += j->n;
        nnz += (int64_t)j->values.size();
    }
    const double blocks = js[0]->params.precision == SSP_PRECISION_MIXED ? 6.0 + 2.5 + 1.0 : 6.0;
    return (int64_t)(blocks * 8.0 * (double)n * (double)ld) + 200 * nnz + 96 * n + (16ll << 20);
}

}  // namespace

struct ssp_server {
    ssp_server_opts opts;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Job*> pending;
    std::unordered_map<uint64_t, std::unique_ptr<Job>> jobs;
    uint64_t next_ticket = 1;
    int32_t inflight = 0, peak_inflight = 0, peak_batch = 0;
    int64_t batches = 0;
    int64_t inflight_bytes = 0, peak_inflight_bytes = 0;
    int64_t submitted = 0, completed = 0, failed = 0, rejected = 0;
    int32_t waiters = 0;  // threads inside ssp_wait; destroy lets them leave before the server goes
    bool stopping = false;
    std::vector<ssp_context*> ctxs;
    std::vector<std::thread> workers;

    // Under the lock: the requests a free slot runs next (empty: none can be admitted now).
    std::vector<Job*> take() {
        std::vector<Job*> run;
        if (pending.empty()) return run;
        const Clock::time_point now = Clock::now();
        auto fits = [&](int64_t bytes) { return inflight == 0 || inflight_bytes + bytes <= opts.hbm_budget_bytes; };
        size_t lead = pending.size();
        if (fits(pending.front()->est_bytes)) {
            lead = 0;
        } else if (ms_between(pending.front()->t_submit, now) < FRONT_AGE_MS) {
            for (size_t i = 1; i < pending.size(); i++)
                if (fits(pending[i]->est_bytes)) {
                    lead = i;
                    break;
                }
        }
        if (lead == pending.size()) return run;
        run.push_back(pending[lead]);
        if (opts.max_batch > 1 && batchable(run[0]->params)) {
            const int64_t share = opts.hbm_budget_bytes / std::max(1, opts.slots);
            for (size_t i = lead + 1; i < pending.size() && (int32_t)run.size() < opts.max_batch; i++) {
                if (!same_batch(pending[i]->params, run[0]->params)) continue;
                run.push_back(pending[i]);
                const int64_t b = batch_footprint(run);
                if (b > share || !fits(b)) run.pop_back();
            }
        }
        for (Job* j : run) pending.erase(std::find(pending.begin(), pending.end(), j));
        return run;
    }

    void run_alone(ssp_context* ctx, Job* j) {
        ssp_csc g{j->n, (int64_t)j->values.size(), j->colptr.data(), j->rowidx.data(), j->values.data(), SSP_MEM_HOST};
        j->params.output_file = j->output_file.c_str();
        memset(&j->out, 0, sizeof(j->out));
        memset(&j->stats, 0, sizeof(j->stats));
        const int rc = ssp_sparsify(ctx, &g, &j->params, SSP_MEM_HOST, &j->out, &j->stats);
        j->status = rc;
        j->error = rc == SSP_OK ? std::string() : std::string(ssp_last_error());
    }

    void run_batch(ssp_context* ctx, const std::vector<Job*>& run) {
        const size_t cnt = run.size();
        std::vector<ssp_csc> gs(cnt);
        std::vector<ssp_params> ps(cnt);
        std::vector<ssp_csc_out> outs(cnt);
        std::vector<ssp_stats> sts(cnt);
        for (size_t i = 0; i < cnt; i++) {
            Job* j = run[i];
            j->params.output_file = j->output_file.c_str();
            gs[i] = ssp_csc{j->n, (int64_t)j->values.size(), j->colptr.data(), j->rowidx.data(), j->values.data(),
                            SSP_MEM_HOST};
            ps[i] = j->params;
        }
        const int rc = ssp_sparsify_batch(ctx, (int32_t)cnt, gs.data(), ps.data(), outs.data(), sts.data());
        if (rc != SSP_OK) {  // the batch as a whole failed: run its requests one by one
            for (Job* j : run) run_alone(ctx, j);
            return;
        }
        for (size_t i = 0; i < cnt; i++) {
            run[i]->out = outs[i];
            run[i]->stats = sts[i];
            run[i]->status = SSP_OK;
            run[i]->error.clear();
        }
    }

    void worker(int slot) {
        ssp_context* ctx = ctxs[slot];
        const int64_t keep_ws = opts.hbm_budget_bytes / std::max(1, opts.slots);
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            std::vector<Job*> run;
            // a request that must wait for capacity is re-examined when anything finishes, or when it ages
            cv_work.wait_for(lk, std::chrono::milliseconds((int64_t)FRONT_AGE_MS), [&] {
                if (stopping) return true;
                run = take();
                return !run.empty();
            });
            if (stopping) return;
            if (run.empty()) continue;
            const int64_t bytes = batch_footprint(run);
            inflight += (int32_t)run.size();
            inflight_bytes += bytes;
            peak_inflight = std::max(peak_inflight, inflight);
            peak_inflight_bytes = std::max(peak_inflight_bytes, inflight_bytes);
            peak_batch = std::max(peak_batch, (int32_t)run.size());
            batches++;
            const Clock::time_point t_admit = Clock::now();
            for (Job* j : run) {
                j->t_admit = t_admit;
                j->slot = slot;
                j->batch = (int32_t)run.size();
            }
            lk.unlock();

            if (run.size() == 1) run_alone(ctx, run[0]);
            else run_batch(ctx, run);
            for (Job* j : run) {
                if (j->status == SSP_OK && j->check_probes > 0) {
                    ssp_csc g{j->n, (int64_t)j->values.size(), j->colptr.data(), j->rowidx.data(), j->values.data(),
                              SSP_MEM_HOST};
                    const Clock::time_point t0 = Clock::now();
                    const int crc = check_result(ctx, g, j->params, j->check_probes, j->out, j);
                    j->check_ms = ms_between(t0, Clock::now());
                    if (crc == SSP_OK) {
                        j->checked = true;
                    } else {
                        j->status = crc;
                        j->error = std::string("inline check: ") + ssp_last_error();
                        ssp_csc_free(&j->out);
                    }
                }
            }
            // keep the slot's cached workspace within its share of the budget (batches are sized to that share,
            // so this frees only after a request larger than the share ran alone)
            if (ssp_context_workspace_bytes(ctx) > keep_ws) ssp_context_release_workspace(ctx);
            for (Job* j : run) {  // the input copies are no longer needed
                std::vector<int64_t>().swap(j->colptr);
                std::vector<int32_t>().swap(j->rowidx);
                std::vector<double>().swap(j->values);
            }

            lk.lock();
            const Clock::time_point t_done = Clock::now();
            for (Job* j : run) {
                j->t_done = t_done;
                j->done = true;
                if (j->status == SSP_OK) completed++;
                else failed++;
            }
            inflight -= (int32_t)run.size();
            inflight_bytes -= bytes;
            cv_done.notify_all();
            cv_work.notify_all();
        }
    }

    void fill(Job* j, ssp_result* r) {
        memset(r, 0, sizeof(*r));
        r->status = j->status;
        snprintf(r->error, sizeof r->error, "%s", j->error.c_str());
        r->out = j->out;
        r->stats = j->stats;
        r->est_bytes = j->est_bytes;
        r->queue_ms = ms_between(j->t_submit, j->t_admit);
        r->run_ms = ms_between(j->t_admit, j->t_done);
        r->latency_ms = ms_between(j->t_submit, j->t_done);
        r->slot = j->slot;
        r->batch = j->batch;
        r->checked = j->checked ? 1 : 0;
        r->probe_upper_violations = j->probe.upper_bound_violations;
        r->probe_lower_violations = j->probe.lower_bound_violations;
        r->probe_mean_relative_error = j->probe.mean_relative_error;
        r->probe_max_relative_error = j->probe.max_relative_error;
        r->components_graph = j->cc_graph;
        r->components_sparsifier = j->cc_sparsifier;
        r->check_ms = j->check_ms;
    }
};

extern "C" {

void ssp_server_opts_default(ssp_server_opts* o) {
    memset(o, 0, sizeof(*o));
    o->device = 0;
    o->slots = 4;
    o->hbm_budget_bytes = 0;  // 85% of the device memory free at creation
    o->max_pending = 0;       // unbounded
    o->max_batch = 32;        // requests that may share one run (ssp_sparsify_batch)
}

int64_t ssp_request_footprint(const ssp_csc* graph, const ssp_params* params) {
    if (!graph || !params || graph->n <= 0) return -1;
    const int64_t n = graph->n, nnz = graph->nnz;
    const int64_t k = ssp_params_jl_dim(params, n);
    const int64_t ld = (k + 31) / 32 * 32;  // whole 32-column tiles
    // n x ld blocks: sketch + x, r, z, p, q in FP64 (+ five FP32 blocks and an FP64 increment when mixed);
    // graph, Laplacian, factor pools and sampling arrays per stored entry; the SpMM's column-slab copy of
    // the Laplacian when slabs are on and the graph has more rows than one slab holds (256-byte rows, at
    // most 16 slabs); a fixed allowance
    const double blocks = params->precision == SSP_PRECISION_MIXED ? 6.0 + 2.5 + 1.0 : 6.0;
    const int64_t slab_rows = std::max<int64_t>(1, (int64_t)(ssp::spmm_slab_mb() * 1048576.0 / 256));
    const int64_t slabs = ssp::spmm_slab_mb() > 0 && n > slab_rows
                              ? std::min<int64_t>(16, (n + slab_rows - 1) / slab_rows) : 0;
    const int64_t slab_bytes = slabs ? 12 * (nnz + n) + 12 * slabs * n : 0;
    return (int64_t)(blocks * 8.0 * (double)n * (double)ld) + 200 * nnz + 96 * n + slab_bytes + (16ll << 20);
}

int ssp_server_create(const ssp_server_opts* opts, ssp_server** out) {
    if (!out) return fail(SSP_ERR_INVALID, "ssp_server_create: out is NULL");
    *out = nullptr;
    ssp_server_opts o;
    if (opts) o = *opts;
    else ssp_server_opts_default(&o);
    if (o.slots < 1 || o.slots > 64) return fail(SSP_ERR_INVALID, "ssp_server_create: slots must be in [1, 64]");
    if (o.max_batch < 0 || o.max_batch > 4096)
        return fail(SSP_ERR_INVALID, "ssp_server_create: max_batch must be in [0, 4096]");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(SSP_ERR_NO_DEVICE, "no CUDA device visible");
    }
    if (o.device < 0 || o.device >= count) return fail(SSP_ERR_INVALID, "ssp_server_create: device out of range");
    if (o.hbm_budget_bytes <= 0) {
        size_t fr = 0, tot = 0;
        if (cudaSetDevice(o.device) != cudaSuccess || cudaMemGetInfo(&fr, &tot) != cudaSuccess)
            return fail(SSP_ERR_CUDA, "ssp_server_create: cannot query device memory");
        o.hbm_budget_bytes = (int64_t)(0.85 * (double)fr);
    }
    std::unique_ptr<ssp_server> s(new ssp_server());
    s->opts = o;
    for (int i = 0; i < o.slots; i++) {
        ssp_context* c = nullptr;
        const int rc = ssp_context_create(o.device, &c);
        if (rc != SSP_OK) {
            const std::string msg = ssp_last_error();
            for (auto* x : s->ctxs) ssp_context_destroy(x);
            return fail(rc, msg);
        }
        s->ctxs.push_back(c);
    }
    for (int i = 0; i < o.slots; i++) s->workers.emplace_back([srv = s.get(), i] { srv->worker(i); });
    *out = s.release();
    return SSP_OK;
}

int ssp_submit(ssp_server* s, const ssp_request* req, uint64_t* ticket) {
    if (!s || !req || !ticket) return fail(SSP_ERR_INVALID, "ssp_submit: bad arguments");
    if (req->kind != SSP_REQ_SPARSIFY) return fail(SSP_ERR_INVALID, "ssp_submit: unknown request kind");
    const ssp_csc& g = req->graph;
    if (g.mem != SSP_MEM_HOST || g.n <= 0 || g.nnz < 0 || !g.colptr || (g.nnz > 0 && (!g.rowidx || !g.values)) ||
        g.colptr[0] != 0 || g.colptr[g.n] != g.nnz)
        return fail(SSP_ERR_INVALID, "ssp_submit: the graph must be a valid host CSC");
    const int64_t est = ssp_request_footprint(&g, &req->params);
    std::unique_ptr<Job> j(new Job());
    j->n = g.n;
    j->colptr.assign(g.colptr, g.colptr + g.n + 1);
    j->rowidx.assign(g.rowidx, g.rowidx + g.nnz);
    j->values.assign(g.values, g.values + g.nnz);
    j->params = req->params;
    j->check_probes = req->check_probes;
    j->output_file = req->params.output_file ? req->params.output_file : "";
    j->est_bytes = est;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) return fail(SSP_ERR_INVALID, "ssp_submit: server is shutting down");
    if (est > s->opts.hbm_budget_bytes) {
        s->rejected++;
        return fail(SSP_ERR_CAPACITY, "ssp_submit: estimated footprint " + std::to_string(est) +
                                          " bytes exceeds the HBM budget " + std::to_string(s->opts.hbm_budget_bytes));
    }
    if (s->opts.max_pending > 0 && (int64_t)s->pending.size() >= s->opts.max_pending) {
        s->rejected++;
        return fail(SSP_ERR_CAPACITY, "ssp_submit: pending queue is full");
    }
    j->ticket = s->next_ticket++;
    j->t_submit = Clock::now();
    *ticket = j->ticket;
    s->pending.push_back(j.get());
    s->jobs.emplace(j->ticket, std::move(j));
    s->submitted++;
    s->cv_work.notify_one();
    return SSP_OK;
}

// On completion the result (including ownership of res->out) moves to the caller and the ticket is retired.
// Several threads may wait on one ticket: the first to see it done collects it, the others get
// SSP_ERR_INVALID (the job is looked up again after every wake-up, never through a pointer kept across one).
int ssp_wait(ssp_server* s, uint64_t ticket, int64_t timeout_ms, ssp_result* res) {
    if (!s || !res) return fail(SSP_ERR_INVALID, "ssp_wait: bad arguments");
    std::unique_lock<std::mutex> lk(s->mu);
    struct Waiting {  // counted while inside; the last to leave wakes a destroy that waits for it
        ssp_server* s;
        explicit Waiting(ssp_server* sv) : s(sv) { s->waiters++; }
        ~Waiting() {
            s->waiters--;
            s->cv_done.notify_all();
        }
    } waiting(s);
    if (s->jobs.find(ticket) == s->jobs.end())
        return fail(SSP_ERR_INVALID, "ssp_wait: unknown or already collected ticket");
    auto ready = [&] {
        auto f = s->jobs.find(ticket);
        return f == s->jobs.end() || f->second->done;
    };
    if (timeout_ms < 0) s->cv_done.wait(lk, ready);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
        return SSP_ERR_PENDING;
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return fail(SSP_ERR_INVALID, "ssp_wait: the ticket was collected by another caller");
    s->fill(it->second.get(), res);
    s->jobs.erase(it);
    s->cv_done.notify_all();  // other waiters of this ticket re-check and leave
    return SSP_OK;
}

int ssp_poll(ssp_server* s, uint64_t ticket, ssp_result* res) { return ssp_wait(s, ticket, 0, res); }

int ssp_server_info_get(ssp_server* s, ssp_server_info* info) {
    if (!s || !info) return fail(SSP_ERR_INVALID, "ssp_server_info_get: bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    memset(info, 0, sizeof(*info));
    info->submitted = s->submitted;
    info->completed = s->completed;
    info->failed = s->failed;
    info->rejected = s->rejected;
    info->pending = (int64_t)s->pending.size();
    info->inflight = s->inflight;
    info->peak_inflight = s->peak_inflight;
    info->peak_inflight_bytes = s->peak_inflight_bytes;
    info->budget_bytes = s->opts.hbm_budget_bytes;
    info->slots = s->opts.slots;
    info->waiters = s->waiters;
    info->batches = s->batches;
    info->peak_batch = s->peak_batch;
    return SSP_OK;
}

// Requests still pending are dropped: they complete with SSP_ERR_INVALID, so threads waiting on them return.
// Admitted ones finish first, and threads inside ssp_wait leave before the server is freed.  Uncollected
// results are freed.
int ssp_server_destroy(ssp_server* s) {
    if (!s) return SSP_OK;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        const Clock::time_point now = Clock::now();
        for (Job* j : s->pending) {
            j->status = SSP_ERR_INVALID;
            j->error = "dropped: the server was destroyed before the request was admitted";
            j->t_admit = j->t_done = now;
            j->done = true;
            s->failed++;
        }
        s->pending.clear();
        s->cv_done.notify_all();
        s->cv_done.wait(lk, [&] { return s->inflight == 0 && s->waiters == 0; });
        s->stopping = true;
        s->cv_work.notify_all();
    }
    for (auto& t : s->workers) t.join();
    for (auto& kv : s->jobs)
        if (kv.second->done && kv.second->status == SSP_OK) ssp_csc_free(&kv.second->out);
    for (auto* c : s->ctxs) ssp_context_destroy(c);
    delete s;
    return SSP_OK;
}

}  // extern "C"
