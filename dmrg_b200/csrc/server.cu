// Site-optimisation eigensolve server: continuous batching of H_eff eigensolves on one GPU.
//
// No counterpart in the reference (DMRG++ solves one site problem at a time on the calling thread,
// solver_primme.cpp:298-517).  Requests are queued; `max_inflight` worker threads, each with its own
// CUDA stream, take the first queued request that fits into the remaining device-memory budget
// (first-fit admission, so a small request is not stuck behind one that does not fit yet), build its
// operator (environments resident on the device for the whole solve), run the eigensolver and copy
// the result out.  Requests that arrive while others are on the GPU are admitted as soon as a slot
// and memory free up; their kernels overlap on the device.  Every kernel on the path reduces in a
// fixed order, so a request's result does not depend on what else is running.
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
        int64_t      id;
        heff_request req;
        size_t       bytes;
        double       t_submit;
    };
    std::deque<Item>                  queue;
    std::map<int64_t, heff_response>  done;
    std::vector<double>               latencies;
    std::vector<std::thread>          workers;
    size_t                            used = 0, peak_used = 0;
    int                               inflight = 0, peak_inflight = 0;
    int64_t                           next_id = 1, completed = 0, failed = 0;
    double                            t_first = -1, t_last = 0, busy_overlap = 0;
    bool                              stop = false;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace heff {

static int64_t r64(int64_t v) { return (v + 63) / 64 * 64; }

// Device memory one request holds while it runs (operator copies + matvec scratch + mixed-precision
// split operands or INT8-engine digit planes + eigensolver basis), matching the allocations in op.cu,
// mixed.cu, emu.cu and eig.cu.
size_t request_bytes(const heff_request &r, int max_basis) {
    const int64_t es = r.dtype == HEFF_C128 ? 16 : 8, cf = r.dtype == HEFF_C128 ? 2 : 1;
    const int64_t S = r.spin, cL = r.chiL, cR = r.chiR, DL = r.mpoL, DR = r.mpoR;
    const int64_t n = S * cL * cR;
    auto          pad = [](int64_t v) { return (v + 31) / 32 * 32; };
    int64_t       b   = es * (cL * cL * DL + 2 * cR * cR * DR + DL * DR * S * S);  // L, R' (+ transient R), W
    b += es * (pad(n) + pad(DL * n) + pad(DR * n));                                 // x', T1, T2
    b += (int64_t)matvec_split_bytes((size_t)(es * (pad(n) + pad(DL * n) + pad(DR * n))));  // GEMM tail-split partials
    const bool mixed = r.precision == HEFF_PREC_MIXED;
    if(mixed) {
        const int64_t nseg = r.dtype == HEFF_C128 ? 6 : 3;
        b += 2 * (cL * DL) * nseg * r64(cL) + 2 * cf * (S * cR) * nseg * r64(cL);      // A1, B1
        b += 2 * (S * cL) * nseg * r64(cR * DR) + 2 * cf * cR * nseg * r64(cR * DR);   // A2, B2
        b += 4 * (cL * DL) * cf * (S * cR);                                            // T1 (fp32)
    }
    if(r.fp64_engine == HEFF_FP64_INT8) b += (int64_t)emu_bytes(S, cL, cR, DL, DR, r.dtype == HEFF_C128, Z_DEFAULT_SLICES);  // digit planes
    const int64_t vec = (es * n + 255) / 256 * 256;
    b += vec * (2 * (max_basis + 1) + 2 * max_basis + 4 + (mixed ? 5 : 0)) + (int64_t)(es * 128 * 131) + 8 * 512 * 128 * 4;
    return (size_t)b + (size_t)(4 << 20);
}

static void run_request(heff_server *srv, heff_server::Item &it, cudaStream_t stream, heff_response &out) {
    const heff_request &r = it.req;
    out.id                = it.id;
    out.t_submit          = it.t_submit;
    out.t_start           = srv->now();
    const void   *mp[1]   = {r.mpo};
    const int64_t md[4]   = {r.mpoL, r.mpoR, r.spin, r.spin};
    const int64_t ld[3]   = {r.chiL, r.chiL, r.mpoL};
    const int64_t rd[3]   = {r.chiR, r.chiR, r.mpoR};
    heff_op      *op      = nullptr;
    int rc = heff_op_create(&op, (heff_dtype)r.dtype, 1, mp, md, r.envL, ld, r.envR, rd, (heff_mem)r.env_where, (heff_precision)r.precision, stream);
    if(rc == HEFF_OK && r.fp64_engine != HEFF_FP64_DMMA) rc = heff_op_set_fp64_engine(op, r.fp64_engine, 0);
    if(rc == HEFF_OK) {
        heff_eig_config cfg;
        heff_eig_config_default(&cfg);
        cfg.ritz   = r.ritz;
        cfg.target = r.target;
        cfg.tol    = r.tol > 0 ? r.tol : 1e-10;
        cfg.mixed  = r.precision == HEFF_PREC_MIXED;
        cfg.max_basis = srv->cfg.max_basis > 0 ? srv->cfg.max_basis : 24;
        const size_t es   = r.dtype == HEFF_C128 ? 16 : 8;
        const size_t nb   = (size_t)op->d.size_mps() * es;
        void        *x0   = nullptr;
        void        *xout = nullptr;
        if(cudaMalloc(&xout, 2 * nb) != cudaSuccess) rc = HEFF_OOM;
        if(rc == HEFF_OK && r.theta0) {
            x0 = reinterpret_cast<char *>(xout) + nb;
            if(cudaMemcpyAsync(x0, r.theta0, nb, cudaMemcpyDefault, stream) != cudaSuccess)
                rc = HEFF_CUDA_ERROR;
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
        if(xout) cudaFree(xout);
        heff_op_destroy(op);
    }
    out.status = rc;
    out.t_done = srv->now();
}

static void worker_main(heff_server *srv) {
    cudaSetDevice(srv->cfg.device);
    cudaStream_t stream = nullptr;
    cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    std::unique_lock<std::mutex> lock(srv->mu);
    while(true) {
        auto fit = srv->queue.end();
        for(auto itq = srv->queue.begin(); itq != srv->queue.end(); ++itq)
            if(srv->used + itq->bytes <= srv->cfg.hbm_budget_bytes) {
                fit = itq;
                break;
            }
        if(fit == srv->queue.end()) {
            if(srv->stop && srv->queue.empty()) break;
            srv->cv_work.wait(lock);
            continue;
        }
        heff_server::Item it = *fit;
        srv->queue.erase(fit);
        srv->used += it.bytes;
        srv->inflight++;
        srv->peak_used     = std::max(srv->peak_used, srv->used);
        srv->peak_inflight = std::max(srv->peak_inflight, srv->inflight);
        lock.unlock();
        heff_response resp;
        std::memset(&resp, 0, sizeof(resp));
        run_request(srv, it, stream, resp);
        lock.lock();
        srv->used -= it.bytes;
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
    lock.unlock();
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
    for(int i = 0; i < srv->cfg.max_inflight; i++) srv->workers.emplace_back(worker_main, srv);
    *out = srv;
    return HEFF_OK;
}

extern "C" size_t heff_request_bytes(const heff_request *req, int max_basis) { return req ? request_bytes(*req, max_basis > 0 ? max_basis : 24) : 0; }

extern "C" int heff_server_submit(heff_server *srv, const heff_request *req, int64_t *id) {
    if(!srv || !req || !id || !req->mpo || !req->envL || !req->envR) return HEFF_BAD_ARG;
    if(req->spin <= 0 || req->chiL <= 0 || req->chiR <= 0 || req->mpoL <= 0 || req->mpoR <= 0) return HEFF_BAD_SHAPE;
    const size_t bytes = request_bytes(*req, srv->cfg.max_basis > 0 ? srv->cfg.max_basis : 24);
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
    heff_server::Item it{*id, *req, bytes, srv->now()};
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
