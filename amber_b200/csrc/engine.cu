// Request engine: many realisations estimated together on one GPU.
//
// The estimator's own batch is one realisation (one gridded cube, its rings and
// channels, all its closed triangles).  Ensembles of realisations (noise or
// simulation sets for error bars) and streams of estimation requests are the
// same problem: many such batches of uneven size.  This engine runs them
// together:
//
//  * amber_cuda_enqueue copies a request's inputs into library memory and puts
//    it in a FIFO; a worker thread of the context does all GPU work.
//  * Admission by HBM footprint: a request is admitted when its estimated
//    device footprint (cube, calCR maps, lag arrays, one batch of ring maps of
//    its largest r1 group and the map builder's intermediate) fits beside the
//    admitted ones in the context's budget.  Its cube and maps then stay
//    resident on the device until it completes.
//  * Rounds: each round builds the next map-set batch of every admitted request
//    and contracts all of their triangles together in the persistent int8
//    kernel (small jobs of many requests share one launch).  A request that
//    arrives while a round runs is admitted at the next round boundary, so its
//    work overlaps on the device with the requests already running
//    (continuous batching).  Finished requests leave after their round.
//  * A job's result depends on the job only (chunking, reduction grouping), so
//    a request's lag arrays are the same alone and in any mix.
//
// The owning context's own device buffers (partial tiles, job lists) serve the
// contraction; each request holds a child context for its realisation state.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"

namespace amber {

namespace {

double now_ms()
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
    int64_t id = 0;
    // inputs (library copies)
    long N1 = 0, nc = 0;
    double Du = 0;
    int flag_key = 0;
    std::vector<double> re_im, ntig;
    std::vector<double> ulow, uhigh;
    int nc10 = 0;
    std::vector<int> uf;
    int want_v2 = 0;
    const double *d_re_im = nullptr, *d_ntig = nullptr;  // caller-owned device cube (read in place)
    bool want_cyl = false;  // cylindrical bispectra of every triangle as well
    amber_cuda_cylbs_params cyl{};
    // plan
    std::vector<int> tri;  // closed triangles (host enumeration, as calCR)
    size_t footprint = 0;
    // state
    enum { QUEUED, ADMITTED, DONE, FAILED } state = QUEUED;
    int rc = AMBER_OK;
    std::string err;
    amber_cuda_ctx *sub = nullptr;
    RunState run;
    bool started = false;
    // results (host)
    std::vector<double> rdata, bldnu, numtri, cyl_out;
    std::vector<int64_t> counts;
    double t_enqueue = 0, t_admit = 0, t_done = 0;
};

}  // namespace

struct Engine {
    amber_cuda_ctx *owner = nullptr;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> queue;
    std::vector<Request *> active;
    std::map<int64_t, std::unique_ptr<Request>> reqs;
    int64_t next_id = 1;
    size_t budget = 0, in_use = 0;
    bool stop = false;
    amber_cuda_engine_info info{};

    void loop();
    int setup(Request *r);
    void finish(Request *r);
    void fail_req(Request *r, int rc, const std::string &msg);
};

namespace {

// Upper bound of a request's device bytes: what its child context may hold.
size_t footprint_of(const Request &r, int precision, long nslots_max)
{
    const size_t cells = (size_t)r.N1 * (size_t)(r.N1 / 2 + 1);
    const size_t grid = sizeof(double) * 3 * cells * r.nc;         // double2 grid + double mask
    const size_t staging = r.d_re_im ? 0 : sizeof(double) * 3 * cells * r.nc;  // raw sums + counts on upload
    const size_t Nr = r.ulow.size();
    const size_t calcr_maps = sizeof(double) * Nr * (size_t)r.N1 * r.N1;
    const int nclen = 2 * r.nc10 + 1;
    const size_t ntri = std::max<size_t>(1, r.tri.size() / 3);
    const size_t results = sizeof(double) * 2 * (size_t)nclen * nclen * ntri;
    long ng_max = 0;
    for (size_t t = 0; t < ntri && !r.tri.empty(); ++t) ng_max = std::max(ng_max, ring_ng1(r.uhigh[r.tri[3 * t]], r.Du));
    const size_t maps = (size_t)nslots_max * map_slot_bytes(precision, ng_max, r.nc, r.want_v2);
    // FP64 paths contract in the child context: its partial tiles (anchors × k-splits × lag cells)
    const size_t partial = precision == AMBER_PREC_MIXED ? 0 : sizeof(double) * (size_t)r.nc * 64 * nclen * nclen;
    // the mask maps grow calCR's map buffer; D maps and the builder's intermediate come on top
    const size_t cyl = r.want_cyl ? cyl_bs_bytes(r.nc10, r.cyl.n_cut, (int)ntri) : 0;
    return grid + std::max(staging, partial) + calcr_maps + maps + results + cyl + ((size_t)192 << 20);
}

// Ring slots one batch of the request's largest r1 group would like (all of its rings).
long slots_wanted(const Request &r)
{
    std::map<int, std::set<int>> rings;
    for (size_t t = 0; t + 2 < r.tri.size(); t += 3) {
        auto &s = rings[r.tri[t]];
        s.insert(r.tri[t]);
        s.insert(r.tri[t + 1]);
        s.insert(r.tri[t + 2]);
    }
    long m = 3;
    for (auto &kv : rings) m = std::max<long>(m, (long)kv.second.size());
    return m;
}

bool run_finished(const RunState &st)
{
    for (size_t g = st.gi; g < st.groups.size(); ++g)
        if ((g == st.gi ? st.ti : 0) < st.groups[g].tris.size()) return false;
    return true;
}

}  // namespace

void Engine::fail_req(Request *r, int rc, const std::string &msg)
{
    if (r->sub) {
        amber_cuda_destroy(r->sub);
        r->sub = nullptr;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (r->state == Request::ADMITTED) in_use -= r->footprint;
    r->state = Request::FAILED;
    r->rc = rc;
    r->err = msg;
    r->t_done = now_ms();
    active.erase(std::remove(active.begin(), active.end(), r), active.end());
    cv_done.notify_all();
}

int Engine::setup(Request *r)
{
    amber_cuda_opts o;
    amber_cuda_default_opts(&o);
    o.device = owner->device;
    o.precision = owner->fp64_abs ? AMBER_PREC_FP64_ABS : owner->precision;
    o.hbm_budget = r->footprint;
    o.stream = owner->stream;
    o.chunk_px = owner->chunk_px;
    int rc = amber_cuda_create(&o, &r->sub);
    if (rc) return rc;
    amber_cuda_ctx *s = r->sub;
    s->contracts_elsewhere = owner->precision == AMBER_PREC_MIXED;
    if ((rc = r->d_re_im ? amber_cuda_load_grid_device(s, r->N1, r->nc, r->Du, r->flag_key, r->d_re_im, r->d_ntig)
                         : amber_cuda_load_grid_packed(s, r->N1, r->nc, r->Du, r->flag_key, r->re_im.data(),
                                                       r->ntig.data())))
        return rc;
    // the host copies are no longer needed once the cube is on the device
    std::vector<double>().swap(r->re_im);
    std::vector<double>().swap(r->ntig);
    if ((rc = amber_cuda_set_rings(s, (int)r->ulow.size(), r->ulow.data(), r->uhigh.data()))) return rc;
    if ((rc = amber_cuda_set_channels(s, r->nc10, r->flag_key == 1 ? (int)r->uf.size() : 0,
                                      r->uf.empty() ? nullptr : r->uf.data())))
        return rc;
    const int ntri = (int)r->tri.size() / 3;
    r->rdata.assign((size_t)4 * std::max(1, ntri), 0.0);
    int rcount = 0;
    if ((rc = amber_cuda_calcr(s, ntri, &rcount, r->rdata.data()))) return rc;
    if (rcount != ntri) return fail(s, AMBER_ERR_STATE, "calCR found %d triangles, the plan %d", rcount, ntri);
    if ((rc = run_begin(s, r->run, ntri, r->tri.data(), r->want_v2))) return rc;
    r->started = true;
    return AMBER_OK;
}

void Engine::finish(Request *r)
{
    amber_cuda_ctx *s = r->sub;
    const int ntri = (int)r->tri.size() / 3;
    const long ncsize = (long)(2 * r->nc10 + 1) * (2 * r->nc10 + 1);
    std::vector<double> res((size_t)2 * ncsize * std::max(1, ntri));
    int rc = AMBER_OK;
    if (ntri > 0)
        rc = cuda_check(s, cudaMemcpyAsync(res.data(), s->results.p, sizeof(double) * res.size(), cudaMemcpyDeviceToHost,
                                           s->stream),
                        "results download");
    if (!rc) rc = cuda_check(s, cudaStreamSynchronize(s->stream), "results download");
    if (rc) {
        fail_req(r, rc, s->err);
        return;
    }
    r->bldnu.resize((size_t)ncsize * ntri);
    if (r->want_v2) r->numtri.resize((size_t)ncsize * ntri);
    for (int t = 0; t < ntri; ++t) {
        std::copy(res.begin() + (size_t)t * 2 * ncsize, res.begin() + (size_t)t * 2 * ncsize + ncsize,
                  r->bldnu.begin() + (size_t)t * ncsize);
        if (r->want_v2)
            std::copy(res.begin() + (size_t)t * 2 * ncsize + ncsize, res.begin() + (size_t)(t + 1) * 2 * ncsize,
                      r->numtri.begin() + (size_t)t * ncsize);
    }
    if (r->want_cyl && ntri > 0) {
        // the reference's analysis chains: v1 files are read back divided by Num
        // (amber.c:193-202, mabs_funcs.py:172-187), v2 files as written
        std::vector<double> num;
        if (r->cyl.denominator == 0)
            for (int t = 0; t < ntri; ++t) {
                const double gfact = (1. * ring_ng1(r->uhigh[r->tri[3 * t]], r->Du)) / (1. * r->N1);
                num.push_back(gfact * gfact * r->rdata[4 * t + 3]);
            }
        s->last_ntri = ntri;
        s->last_v2 = r->want_v2;
        const long n = 2 * (r->nc10 + 1 - r->cyl.n_cut) - 1;
        r->cyl_out.assign((size_t)ntri * n * n, 0.0);
        if ((rc = amber_cuda_cyl_bs(s, &r->cyl, num.empty() ? nullptr : num.data(), r->cyl_out.data()))) {
            fail_req(r, rc, s->err);
            return;
        }
    }
    r->counts = s->counts;
    const double products = s->last_products;
    amber_cuda_destroy(s);
    r->sub = nullptr;
    std::lock_guard<std::mutex> lk(mu);
    info.products += products;
    in_use -= r->footprint;
    r->state = Request::DONE;
    r->t_done = now_ms();
    info.requests_done += 1;
    active.erase(std::remove(active.begin(), active.end(), r), active.end());
    cv_done.notify_all();
}

void Engine::loop()
{
    cudaSetDevice(owner->device);
    while (true) {
        std::vector<Request *> round;
        {
            std::unique_lock<std::mutex> lk(mu);
            // admission, first come first served: the head waits until its footprint fits
            while (!queue.empty()) {
                Request *r = queue.front();
                if (r->footprint > budget) {
                    queue.pop_front();
                    r->state = Request::FAILED;
                    r->rc = AMBER_ERR_OOM;
                    r->err = "request footprint exceeds the engine's HBM budget";
                    r->t_done = now_ms();
                    cv_done.notify_all();
                    continue;
                }
                if (in_use + r->footprint > budget) break;
                queue.pop_front();
                in_use += r->footprint;
                r->state = Request::ADMITTED;
                r->t_admit = now_ms();
                active.push_back(r);
            }
            info.peak_bytes = std::max(info.peak_bytes, in_use);
            info.max_active = std::max<long>(info.max_active, (long)active.size());
            if (active.empty()) {
                if (stop) return;
                cv_work.wait(lk);
                continue;
            }
            round = active;
        }
        const double t0 = now_ms();
        // this round's share of the statistics, published under the lock at its end
        double setup_ms = 0, maps_ms = 0, contract_ms = 0, finish_ms = 0, kernel_ms = 0;
        long launches = 0, all_launches = 0;
        owner->phase_used = 0;  // per-phase timing events are reused round after round
        // one map-set batch of every active request
        std::vector<I8Job> jobs;
        std::vector<Request *> in_round;
        for (Request *r : round) {
            int rc = AMBER_OK;
            double ta = now_ms();
            if (!r->started) {
                rc = setup(r);
                if (r->sub) all_launches += r->sub->launches;  // grid normalisation and calCR of the new request
            }
            setup_ms += now_ms() - ta;
            if (!rc && run_finished(r->run)) {
                finish(r);  // no triangles at all
                continue;
            }
            if (!rc) {
                ta = now_ms();
                const long launched = r->sub->launches, contracted = r->sub->contractions;
                r->sub->phase_used = 0;
                rc = run_next_batch(r->sub, r->run, &jobs);
                all_launches += r->sub->launches - launched;
                launches += r->sub->contractions - contracted;
                // contractions that ran inside the request's own context (the FP64 paths): their
                // kernel time, from the phase events around each launch
                for (size_t i = 0; i < r->sub->phase_used; ++i)
                    if (r->sub->phase_ev[i].phase == 1 && cudaEventSynchronize(r->sub->phase_ev[i].b) == cudaSuccess) {
                        float ms = 0;
                        if (cudaEventElapsedTime(&ms, r->sub->phase_ev[i].a, r->sub->phase_ev[i].b) == cudaSuccess)
                            kernel_ms += ms;
                    }
                cudaGetLastError();
                rc = rc < 0 ? rc : AMBER_OK;
                maps_ms += now_ms() - ta;
            }
            if (rc) {
                fail_req(r, rc, r->sub ? r->sub->err : std::string("context creation failed"));
                continue;
            }
            in_round.push_back(r);
        }
        int rc = AMBER_OK;
        double tc = now_ms();
        if (!jobs.empty()) {
            const long before = owner->contractions, launched = owner->launches;
            rc = contract_i8_jobs(owner, jobs);  // synchronises the stream
            launches += owner->contractions - before;
            all_launches += owner->launches - launched;
            for (size_t i = 0; i < owner->phase_used; ++i)
                if (owner->phase_ev[i].phase == 1) {
                    float ms = 0;
                    if (cudaEventElapsedTime(&ms, owner->phase_ev[i].a, owner->phase_ev[i].b) == cudaSuccess)
                        kernel_ms += ms;
                }
            cudaGetLastError();
        }
        contract_ms = now_ms() - tc;
        tc = now_ms();
        if (rc) {
            const std::string msg = owner->err;
            for (Request *r : in_round) fail_req(r, rc, msg);
        } else {
            for (Request *r : in_round)
                if (run_finished(r->run)) finish(r);
        }
        finish_ms = now_ms() - tc;
        std::lock_guard<std::mutex> lk(mu);
        info.setup_ms += setup_ms;
        info.maps_ms += maps_ms;
        info.contract_ms += contract_ms;
        info.finish_ms += finish_ms;
        info.contraction_launches += launches;
        info.kernel_launches += all_launches;
        info.contract_kernel_ms += kernel_ms;
        info.rounds += 1;
        info.busy_ms += now_ms() - t0;
    }
}

Engine *engine_of(amber_cuda_ctx *c)
{
    if (!c->engine) {
        Engine *e = new Engine();
        e->owner = c;
        // the contraction's own buffers (partial tiles of one launch, job lists) come first
        const size_t own = std::max<size_t>((size_t)512 << 20, std::min<size_t>((size_t)8 << 30, c->budget / 8)) +
                           ((size_t)1 << 30);
        e->budget = c->budget > own ? c->budget - own : 0;
        c->engine = e;
        e->worker = std::thread([e] { e->loop(); });
    }
    return c->engine;
}

void engine_shutdown(amber_cuda_ctx *c)
{
    Engine *e = c->engine;
    if (!e) return;
    {
        std::lock_guard<std::mutex> lk(e->mu);
        e->stop = true;
        // queued requests are dropped; admitted ones finish their current round
        for (Request *r : e->queue) {
            r->state = Request::FAILED;
            r->rc = AMBER_ERR_STATE;
        }
        e->queue.clear();
    }
    e->cv_work.notify_all();
    // the worker returns once no request is active
    e->worker.join();
    for (auto &kv : e->reqs)
        if (kv.second->sub) amber_cuda_destroy(kv.second->sub);
    delete e;
    c->engine = nullptr;
}

}  // namespace amber

using amber::Engine;
using amber::Request;

extern "C" {

int amber_cuda_enqueue(amber_cuda_ctx *c, const amber_cuda_request *q, int64_t *ticket)
{
    if (!c || !q || !ticket) return AMBER_ERR_ARG;
    if (q->N1 <= 0 || q->N1 % 2 || q->nc <= 5 || q->Du <= 0 || !q->re_im || !q->ntig || q->Nr <= 0 || !q->ULow ||
        !q->UHigh || q->nc10 < 0 || q->nc10 >= q->nc || (q->flag_key == 1 && (q->uf_nc <= 0 || !q->uf_chans)))
        return amber::fail(c, AMBER_ERR_ARG, "enqueue: bad request (N1 even > 0, nc > 5, 0 <= nc10 < nc, rings, "
                                             "and the unflagged channel list when flag_key is 1)");
    for (int i = 0; i < q->Nr; ++i)
        if (!(q->ULow[i] >= 0 && q->ULow[i] < q->UHigh[i] && q->UHigh[i] <= q->N1 / 2))
            return amber::fail(c, AMBER_ERR_ARG, "enqueue: ring %d edges outside 0 <= ULow < UHigh <= N1/2", i);
    auto r = std::make_unique<Request>();
    r->N1 = q->N1;
    r->nc = q->nc;
    r->Du = q->Du;
    r->flag_key = q->flag_key;
    const size_t cells = (size_t)q->N1 * (size_t)(q->N1 / 2 + 1);
    if (q->inputs_on_device) {
        r->d_re_im = q->re_im;
        r->d_ntig = q->ntig;
    } else {
        r->re_im.assign(q->re_im, q->re_im + 2 * cells * q->nc);
        r->ntig.assign(q->ntig, q->ntig + cells * q->nc);
    }
    r->ulow.assign(q->ULow, q->ULow + q->Nr);
    r->uhigh.assign(q->UHigh, q->UHigh + q->Nr);
    r->nc10 = q->nc10;
    if (q->flag_key == 1) r->uf.assign(q->uf_chans, q->uf_chans + q->uf_nc);
    r->want_v2 = q->want_v2 ? 1 : 0;
    if (q->cylbs) {
        if (const char *why = amber::cyl_bs_invalid(q->cylbs, q->nc10, r->want_v2))
            return amber::fail(c, AMBER_ERR_ARG, "enqueue: cylindrical bispectrum parameters: %s", why);
        r->want_cyl = true;
        r->cyl = *q->cylbs;
    }
    r->tri = amber::closed_triangles(r->ulow, r->uhigh);
    const int prec = c->precision;
    r->footprint = amber::footprint_of(*r, prec, amber::slots_wanted(*r));
    Engine *e = amber::engine_of(c);
    // a footprint beyond the budget with all of the largest group's rings: settle for fewer slots
    for (long sl = amber::slots_wanted(*r); sl > 3 && r->footprint > e->budget; --sl)
        r->footprint = amber::footprint_of(*r, prec, sl);
    r->t_enqueue = amber::now_ms();
    std::lock_guard<std::mutex> lk(e->mu);
    r->id = e->next_id++;
    *ticket = r->id;
    e->queue.push_back(r.get());
    e->reqs[r->id] = std::move(r);
    e->cv_work.notify_all();
    return AMBER_OK;
}

int amber_cuda_wait(amber_cuda_ctx *c, int64_t ticket, int timeout_ms, int *ntri)
{
    if (!c || !c->engine) return AMBER_ERR_ARG;
    Engine *e = c->engine;
    std::unique_lock<std::mutex> lk(e->mu);
    auto it = e->reqs.find(ticket);
    if (it == e->reqs.end()) return AMBER_ERR_ARG;
    Request *r = it->second.get();
    auto done = [&] { return r->state == Request::DONE || r->state == Request::FAILED; };
    if (timeout_ms < 0)
        e->cv_done.wait(lk, done);
    else if (!e->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done))
        return AMBER_ERR_TIMEOUT;
    if (ntri) *ntri = (int)r->tri.size() / 3;
    if (r->state == Request::FAILED) {
        c->err = "request " + std::to_string(ticket) + ": " + r->err;
        return r->rc ? r->rc : AMBER_ERR_STATE;
    }
    return AMBER_OK;
}

int amber_cuda_result(amber_cuda_ctx *c, int64_t ticket, int max_tri, double *rdata, double *bldnu, int64_t *numdnu,
                      double *numtri, double *latency_ms, double *cyl_bs)
{
    if (!c || !c->engine) return AMBER_ERR_ARG;
    Engine *e = c->engine;
    std::unique_ptr<Request> r;
    {
        std::lock_guard<std::mutex> lk(e->mu);
        auto it = e->reqs.find(ticket);
        if (it == e->reqs.end()) return AMBER_ERR_ARG;
        if (it->second->state == Request::FAILED) {
            // a failed request is forgotten here too, with its copied inputs: nothing else
            // frees them before the context is destroyed
            const int rc = it->second->rc ? it->second->rc : AMBER_ERR_STATE;
            c->err = "request " + std::to_string(ticket) + ": " + it->second->err;
            e->reqs.erase(it);
            return rc;
        }
        if (it->second->state != Request::DONE) return AMBER_ERR_STATE;
        const int ntri = (int)it->second->tri.size() / 3;
        if (ntri > max_tri) return amber::fail(c, AMBER_ERR_ARG, "result: %d triangles, room for %d", ntri, max_tri);
        r = std::move(it->second);
        e->reqs.erase(it);
    }
    const int ntri = (int)r->tri.size() / 3;
    const size_t ncsize = (size_t)(2 * r->nc10 + 1) * (2 * r->nc10 + 1);
    if (rdata) std::copy(r->rdata.begin(), r->rdata.begin() + (size_t)4 * ntri, rdata);
    if (bldnu) std::copy(r->bldnu.begin(), r->bldnu.end(), bldnu);
    if (numtri && r->want_v2) std::copy(r->numtri.begin(), r->numtri.end(), numtri);
    if (numdnu)
        for (int t = 0; t < ntri; ++t) std::copy(r->counts.begin(), r->counts.end(), numdnu + (size_t)t * ncsize);
    if (cyl_bs && r->want_cyl) std::copy(r->cyl_out.begin(), r->cyl_out.end(), cyl_bs);
    if (latency_ms) *latency_ms = r->t_done - r->t_enqueue;
    return AMBER_OK;
}

int amber_cuda_engine_stats(amber_cuda_ctx *c, amber_cuda_engine_info *info)
{
    if (!c || !info) return AMBER_ERR_ARG;
    if (!c->engine) {
        *info = amber_cuda_engine_info{};
        return AMBER_OK;
    }
    std::lock_guard<std::mutex> lk(c->engine->mu);
    *info = c->engine->info;
    info->budget_bytes = c->engine->budget;
    info->queued = (long)c->engine->queue.size();
    info->active = (long)c->engine->active.size();
    return AMBER_OK;
}

}  // extern "C"
