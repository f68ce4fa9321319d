// Site-optimisation eigensolve server: continuous batching of H_eff eigensolves on one GPU.
//
// No counterpart in the reference (DMRG++ solves one site problem at a time on the calling thread,
// solver_primme.cpp:298-517).  Requests are queued; `max_inflight` worker threads (slots), each with its
// own CUDA stream and its own arena operator, take the first queued request that fits into the remaining
// device-memory budget (first-fit admission, so a small request is not stuck behind one that does not fit
// yet), bind it to the arena (environments copied onto the device, resident for the whole solve), run the
// eigensolver and copy the result out.  The arena keeps every device buffer from one request to the next
// and grows only when a request needs more, so once it has grown to the stream's sizes a request costs no
// cudaMalloc or cudaFree: those synchronise the whole device and would stall every other slot's stream.
// The budget counts what the arenas hold (idle ones included); an idle slot gives its arena back when a
// queued request does not fit otherwise.  Requests that arrive while others are on the GPU are admitted
// as soon as a slot and memory free up; their kernels overlap on the device.  Every kernel on the path
// reduces in a fixed order, so a request's result does not depend on what else is running or on which
// slot ran it.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "eig.cuh"
#include "gemm_i8.cuh"
#include "op.cuh"
#include "runtime.cuh"

struct heff_server {
    heff_server_config                cfg{};
    std::mutex                        mu;
    std::condition_variable           cv_work, cv_done;
    struct Item {
        int64_t          id;
        heff_request     req;
        heff::ArenaBytes need;  // per-buffer bytes this request needs in an arena
        double           t_submit;
    };
    struct Slot {
        heff_op *op   = nullptr;  // arena operator (op_create_arena), owned by the slot's worker thread
        size_t   held = 0;        // bytes its arena holds (counted in `used`)
    };
    std::vector<Slot>                 slots;
    std::deque<Item>                  queue;
    std::map<int64_t, heff_response>  done;
    std::vector<double>               latencies;
    std::vector<std::thread>          workers;
    size_t                            used = 0, peak_used = 0;
    int                               inflight = 0, peak_inflight = 0;
    int64_t                           next_id = 1, completed = 0, failed = 0, arena_grows = 0;
    double                            t_first = -1, t_last = 0, busy_overlap = 0;
    bool                              stop = false;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace heff {

// Slack per arena for the few small buffers the estimate does not itemise (row maxima of the INT8 engine's
// accumulators, flags).
static constexpr size_t kArenaSlack = (size_t)4 << 20;

static bool request_dims_ok(const heff_request &r) { return r.spin > 0 && r.chiL > 0 && r.chiR > 0 && r.mpoL > 0 && r.mpoR > 0; }

// Device memory one request holds while it runs (operator copies + matvec scratch + mixed-precision
// split operands or INT8-engine digit planes + eigensolver basis + start/result vectors): the per-buffer sizes
// the arena allocates for it (arena_need, computed by the same functions that size the buffers).
size_t request_bytes(const heff_request &r, int max_basis) {
    if(!request_dims_ok(r)) return 0;
    return arena_need(r, max_basis).total() + kArenaSlack;
}

static int server_basis(const heff_server *srv) { return srv->cfg.max_basis > 0 ? srv->cfg.max_basis : 24; }

static void run_request(heff_server *srv, heff_server::Item &it, heff_op *op, heff_response &out) {
    const heff_request &r      = it.req;
    cudaStream_t        stream = op->stream;
    out.id                     = it.id;
    out.t_submit               = it.t_submit;
    out.t_start                = srv->now();
    void *vec                  = nullptr;
    int   rc                   = op_arena_bind(op, r, server_basis(srv), &vec);
    if(rc == HEFF_OK) {
        heff_eig_config cfg;
        heff_eig_config_default(&cfg);
        cfg.ritz      = r.ritz;
        cfg.target    = r.target;
        cfg.tol       = r.tol > 0 ? r.tol : 1e-10;
        cfg.mixed     = r.precision == HEFF_PREC_MIXED;
        cfg.max_basis = server_basis(srv);
        const size_t es   = r.dtype == HEFF_C128 ? 16 : 8;
        const size_t nb   = (size_t)op->d.size_mps() * es;
        void        *xout = vec;
        void        *x0   = nullptr;
        if(r.theta0) {
            x0 = reinterpret_cast<char *>(vec) + nb;
            if(cudaMemcpyAsync(x0, r.theta0, nb, cudaMemcpyDefault, stream) != cudaSuccess) rc = HEFF_CUDA_ERROR;
        }
        heff_eig_result er;
        std::memset(&er, 0, sizeof(er));
        if(rc == HEFF_OK) rc = eigs(op, &cfg, x0, xout, &er);
        if((rc == HEFF_OK || rc == HEFF_NOT_CONVERGED) && r.theta_out)
            if(cudaMemcpyAsync(r.theta_out, xout, nb, cudaMemcpyDeviceToHost, stream) != cudaSuccess || cudaStreamSynchronize(stream) != cudaSuccess)
                rc = HEFF_CUDA_ERROR;
        out.eigval       = er.eigval;
        out.resnorm      = er.resnorm;
        out.num_mv       = er.num_mv;
        out.num_mv_mixed = er.num_mv_mixed;
        out.converged    = er.converged;
    }
    out.status = rc;
    out.t_done = srv->now();
}

static void worker_main(heff_server *srv, int k) {
    cudaSetDevice(srv->cfg.device);
    cudaStream_t stream = nullptr;
    cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    heff_server::Slot &slot = srv->slots[k];
    op_create_arena(&slot.op, stream);
    std::unique_lock<std::mutex> lock(srv->mu);
    while(true) {
        auto   fit      = srv->queue.end();
        size_t new_held = 0;
        for(auto itq = srv->queue.begin(); itq != srv->queue.end(); ++itq) {
            const size_t t = arena_held(slot.op).max_with(itq->need).total() + kArenaSlack;
            if(srv->used - slot.held + t <= srv->cfg.hbm_budget_bytes) {
                fit      = itq;
                new_held = t;
                break;
            }
        }
        if(fit == srv->queue.end()) {
            if(srv->stop && srv->queue.empty()) break;
            if(!srv->queue.empty() && slot.held > 0) {
                // memory pressure: nothing queued fits next to what the arenas hold, so this idle slot gives its arena back
                heff_op *old = slot.op;
                srv->used -= slot.held;
                slot.held = 0;
                slot.op   = nullptr;
                lock.unlock();
                heff_op_destroy(old);
                op_create_arena(&slot.op, stream);
                lock.lock();
                srv->cv_work.notify_all();
                continue;
            }
            srv->cv_work.wait(lock);
            continue;
        }
        heff_server::Item it = *fit;
        srv->queue.erase(fit);
        srv->used += new_held - slot.held;
        slot.held = new_held;
        srv->inflight++;
        srv->peak_used     = std::max(srv->peak_used, srv->used);
        srv->peak_inflight = std::max(srv->peak_inflight, srv->inflight);
        const size_t before = arena_held(slot.op).total();
        lock.unlock();
        heff_response resp;
        std::memset(&resp, 0, sizeof(resp));
        run_request(srv, it, slot.op, resp);
        const size_t after  = arena_held(slot.op).total();
        const size_t actual = after + kArenaSlack;
        lock.lock();
        if(after > before) srv->arena_grows++;
        if(actual > slot.held) {  // the estimate missed a buffer: count what the arena really holds
            srv->used += actual - slot.held;
            slot.held      = actual;
            srv->peak_used = std::max(srv->peak_used, srv->used);
        }
        srv->inflight--;
        if(resp.status == HEFF_OK || resp.status == HEFF_NOT_CONVERGED) {
            srv->completed++;
            srv->latencies.push_back(resp.t_done - resp.t_submit);
            srv->t_last = std::max(srv->t_last, resp.t_done);
        } else {
            srv->failed++;
        }
        srv->done[it.id] = resp;
        srv->cv_done.notify_all();
        srv->cv_work.notify_all();
    }
    srv->used -= slot.held;
    slot.held = 0;
    lock.unlock();
    heff_op_destroy(slot.op);
    slot.op = nullptr;
    cudaStreamDestroy(stream);
}

}  // namespace heff

using namespace heff;

extern "C" void heff_server_config_default(heff_server_config *cfg) {
    if(!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->hbm_budget_bytes = (size_t)64 << 30;
    cfg->max_inflight     = 4;
    cfg->device           = 0;
    cfg->max_basis        = 24;
}

extern "C" int heff_server_create(const heff_server_config *cfg, heff_server **out) {
    if(!out) return HEFF_BAD_ARG;
    heff_server *srv = new heff_server();
    heff_server_config_default(&srv->cfg);
    if(cfg) srv->cfg = *cfg;
    if(srv->cfg.max_inflight < 1 || srv->cfg.max_inflight > 64 || srv->cfg.hbm_budget_bytes == 0) {
        delete srv;
        return HEFF_BAD_ARG;
    }
    srv->slots.resize(srv->cfg.max_inflight);
    for(int i = 0; i < srv->cfg.max_inflight; i++) srv->workers.emplace_back(worker_main, srv, i);
    *out = srv;
    return HEFF_OK;
}

extern "C" size_t heff_request_bytes(const heff_request *req, int max_basis) { return req ? request_bytes(*req, max_basis > 0 ? max_basis : 24) : 0; }

extern "C" int heff_server_submit(heff_server *srv, const heff_request *req, int64_t *id) {
    if(!srv || !req || !id || !req->mpo || !req->envL || !req->envR) return HEFF_BAD_ARG;
    if(!request_dims_ok(*req)) return HEFF_BAD_SHAPE;
    if(req->dtype != HEFF_F64 && req->dtype != HEFF_C128) return HEFF_BAD_ARG;
    const ArenaBytes need  = arena_need(*req, server_basis(srv));
    const size_t     bytes = need.total() + kArenaSlack;
    std::lock_guard<std::mutex> lock(srv->mu);
    if(srv->stop) return HEFF_BAD_ARG;
    *id = srv->next_id++;
    if(bytes > srv->cfg.hbm_budget_bytes) {
        heff_response resp;
        std::memset(&resp, 0, sizeof(resp));
        resp.id                = *id;
        resp.status            = HEFF_OOM;
        resp.t_submit = resp.t_start = resp.t_done = srv->now();
        srv->done[*id]         = resp;
        srv->failed++;
        srv->cv_done.notify_all();
        return HEFF_OK;  // the request is answered (status HEFF_OOM), the server stays up
    }
    heff_server::Item it{*id, *req, need, srv->now()};
    if(srv->t_first < 0) srv->t_first = it.t_submit;
    srv->queue.push_back(it);
    srv->cv_work.notify_one();
    return HEFF_OK;
}

extern "C" int heff_server_wait(heff_server *srv, int64_t id, double timeout_s, heff_response *resp) {
    if(!srv || !resp) return HEFF_BAD_ARG;
    std::unique_lock<std::mutex> lock(srv->mu);
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 1e9);
    while(srv->done.find(id) == srv->done.end()) {
        if(srv->cv_done.wait_until(lock, deadline) == std::cv_status::timeout && srv->done.find(id) == srv->done.end()) return HEFF_TIMEOUT;
    }
    *resp = srv->done[id];
    return HEFF_OK;
}

extern "C" int heff_server_get_stats(heff_server *srv, heff_server_stats *st) {
    if(!srv || !st) return HEFF_BAD_ARG;
    std::lock_guard<std::mutex> lock(srv->mu);
    std::memset(st, 0, sizeof(*st));
    st->completed     = srv->completed;
    st->failed        = srv->failed;
    st->queued        = (int64_t)srv->queue.size();
    st->inflight      = srv->inflight;
    st->peak_inflight = srv->peak_inflight;
    st->peak_bytes    = srv->peak_used;
    st->arena_bytes   = srv->used;
    st->arena_grows   = srv->arena_grows;
    std::vector<double> l = srv->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) { return l.empty() ? 0.0 : l[std::min(l.size() - 1, (size_t)(p * (l.size() - 1) + 0.5))]; };
    st->p50_latency_s = pct(0.50);
    st->p99_latency_s = pct(0.99);
    st->max_latency_s = l.empty() ? 0.0 : l.back();
    const double span = srv->t_last - (srv->t_first < 0 ? 0 : srv->t_first);
    st->solves_per_s  = span > 0 ? (double)srv->completed / span : 0.0;
    return HEFF_OK;
}

extern "C" int heff_server_destroy(heff_server *srv) {
    if(!srv) return HEFF_OK;
    {
        std::lock_guard<std::mutex> lock(srv->mu);
        srv->stop = true;
    }
    srv->cv_work.notify_all();
    for(auto &t : srv->workers) t.join();
    delete srv;
    return HEFF_OK;
}
