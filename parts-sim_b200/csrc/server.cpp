// Continuous-batching request loop for many independent voxel solves on one GPU.
//
// The reference runs one structural job at a time behind a global GPU lock
// (native/src/gpu/gpu.hpp:43, gpu_fea.cpp:256). Here requests arrive at any time and:
//   1. builder threads (host cores) build each request's multigrid hierarchy and stage its load
//      vector and result buffer in pinned memory;
//   2. one scheduler thread admits built requests in arrival order while their estimated device
//      footprint fits the HBM budget and an active slot is free; uploader threads put each
//      admitted hierarchy on the GPU and start its solve on its own stream (the solve is a
//      non-blocking state machine), so uploads never hold up the running solves;
//   3. the scheduler polls every active solve without waiting, launches their next iteration
//      batches, retires finished ones (device memory back to the stream-ordered pool at once,
//      which keeps it for the next request instead of returning it to the driver) and back-fills
//      from the queue.
// Solves of different requests therefore overlap on the device; each result is computed exactly
// as a lone solve of the same model would be (same kernels, same launch shapes, deterministic
// reductions).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "host_util.hpp"
#include "ps_fea.h"
#include "solver.hpp"

namespace psfea {
namespace {

using Clock = std::chrono::steady_clock;

double secs(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

struct Request {
    int64_t id = 0;
    int32_t dims[3] = {0, 0, 0};
    std::vector<float> density;
    std::vector<uint8_t> bc;
    std::vector<double> fHost;  // until staged
    double nu = 0.3;
    int64_t coarsest = 300;
    ps_solve_opts opts{};
    int64_t nDof = 0;
    double* fPinned = nullptr;
    double* uPinned = nullptr;
    std::unique_ptr<Hierarchy> hier;
    std::unique_ptr<Solver> solver;
    int64_t need = 0;
    enum State { QUEUED, BUILT, ADMITTED, ACTIVE, DONE } state = QUEUED;
    ps_status status = PS_OK;
    std::string error;
    ps_solve_result res{};
    Clock::time_point tSubmit, tBuilt, tAdmit, tDone;
};

}  // namespace
}  // namespace psfea

struct ps_server {
    int64_t budget = 0;
    int maxActive = 0;
    int device = 0;
    std::mutex mu;
    std::condition_variable cvBuild, cvSched, cvDone, cvUpload;
    std::deque<psfea::Request*> buildQueue;
    std::deque<psfea::Request*> ready;  // built, in arrival order
    std::deque<psfea::Request*> uploads;  // admitted, waiting for an uploader
    int uploading = 0;
    std::vector<psfea::Request*> active;
    std::vector<std::thread> uploaders;
    std::map<int64_t, std::unique_ptr<psfea::Request>> all;
    std::vector<std::thread> builders;
    std::thread scheduler;
    bool stop = false;
    int64_t nextId = 1;
    int64_t used = 0, peakUsed = 0;
    int peakActive = 0;
    int64_t completed = 0;
};

namespace psfea {
namespace {

void fail(ps_server* S, Request* R, ps_status st, const std::string& msg) {
    R->status = st;
    R->error = msg;
    R->state = Request::DONE;
    R->tDone = Clock::now();
    S->completed++;
}

void builderLoop(ps_server* S) {
    cudaSetDevice(S->device);
    // PSFEA_SERVER_GALERKIN=1: each build thread forms the Galerkin coarse matrices of its requests
    // on the device (bitwise the host's) for levels of at least PSFEA_SERVER_GALERKIN_MIN (64)
    // classes of child patterns. Off by default: on the 512-request stream it made builds slower
    // (p50 3.9 -> 6.4 s) and the stream 21.3 -> 18.7 MDOF/s; the solves, not the builds, hold the
    // requests back, and the products' round trips share the device with them.
    std::unique_ptr<GalerkinEngine> engine;
    {
        const char* e = std::getenv("PSFEA_SERVER_GALERKIN");
        const char* m = std::getenv("PSFEA_SERVER_GALERKIN_MIN");
        if (e && std::atoi(e) != 0) {
            try {
                engine = makeDeviceGalerkin(m ? std::atoll(m) : 64);
            } catch (const Error&) {
                engine.reset();  // no device for the engine: the requests' builds stay on the host
            }
        }
    }
    for (;;) {
        Request* R = nullptr;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cvBuild.wait(lk, [&] { return S->stop || !S->buildQueue.empty(); });
            if (S->stop) return;
            R = S->buildQueue.front();
            S->buildQueue.pop_front();
        }
        ps_status st = PS_OK;
        std::string err;
        try {
            auto h = std::make_unique<Hierarchy>(buildHierarchy(R->dims, R->density.data(), R->nu, R->bc.data(), R->coarsest, nullptr,
                                                                engine.get()));
            R->need = estimateDeviceBytes(*h);
            R->hier = std::move(h);
            R->density.clear();
            R->density.shrink_to_fit();
            if (cudaMallocHost(&R->fPinned, size_t(R->nDof) * 8) != cudaSuccess || cudaMallocHost(&R->uPinned, size_t(R->nDof) * 8) != cudaSuccess) {
                cudaGetLastError();
                throw Error(PS_EOOM, "pinned host memory exhausted");
            }
            std::memcpy(R->fPinned, R->fHost.data(), size_t(R->nDof) * 8);
            R->fHost.clear();
            R->fHost.shrink_to_fit();
        } catch (const Error& e) {
            st = e.status;
            err = e.what();
        } catch (const std::exception& e) {
            st = PS_EOOM;
            err = e.what();
        }
        {
            std::lock_guard<std::mutex> lk(S->mu);
            R->tBuilt = Clock::now();
            if (st != PS_OK) {
                fail(S, R, st, err);
                S->cvDone.notify_all();
            } else {
                R->state = Request::BUILT;
                // keep arrival order among the built ones
                auto it = std::find_if(S->ready.begin(), S->ready.end(), [&](Request* o) { return o->id > R->id; });
                S->ready.insert(it, R);
                S->cvSched.notify_all();
            }
        }
    }
}

// an admitted request's hierarchy to the GPU and its solve started; then it is active
void uploaderLoop(ps_server* S) {
    cudaSetDevice(S->device);
    for (;;) {
        Request* R = nullptr;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cvUpload.wait(lk, [&] { return S->stop || !S->uploads.empty(); });
            if (S->stop) return;
            R = S->uploads.front();
            S->uploads.pop_front();
        }
        try {
            R->solver = std::make_unique<Solver>(std::move(*R->hier));
            R->hier.reset();
            R->solver->begin(R->fPinned, R->opts, R->uPinned);
            std::lock_guard<std::mutex> lk(S->mu);
            R->state = Request::ACTIVE;
            S->uploading--;
            S->active.push_back(R);
            S->peakActive = std::max(S->peakActive, int(S->active.size()));
        } catch (const Error& e) {
            R->solver.reset();
            std::lock_guard<std::mutex> lk(S->mu);
            S->uploading--;
            S->used -= R->need;
            fail(S, R, e.status, e.what());
            S->cvDone.notify_all();
        }
        S->cvSched.notify_all();
    }
}

void schedulerLoop(ps_server* S) {
    cudaSetDevice(S->device);
    for (;;) {
        bool admitted = false;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            if (S->stop) return;
            // admission: arrival order, HBM footprint and slots; an oversized request runs alone
            while (!S->ready.empty() && int(S->active.size()) + S->uploading < S->maxActive) {
                Request* R = S->ready.front();
                const bool alone = S->active.empty() && S->uploading == 0;
                if (S->used + R->need > S->budget && !alone) break;
                S->ready.pop_front();
                S->used += R->need;
                S->peakUsed = std::max(S->peakUsed, S->used);
                R->state = Request::ADMITTED;
                R->tAdmit = Clock::now();
                S->uploading++;
                S->uploads.push_back(R);
                admitted = true;
            }
            if (admitted) S->cvUpload.notify_all();
            if (S->active.empty()) {
                S->cvSched.wait_for(lk, std::chrono::milliseconds(admitted ? 0 : 2));
                continue;
            }
        }
        bool progressed = admitted;
        std::vector<Request*> act;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            act = S->active;
        }
        for (Request* R : act) {
            ps_solve_result res{};
            bool finished = false;
            ps_status st = PS_OK;
            std::string err;
            try {
                finished = R->solver->poll(res);
            } catch (const Error& e) {
                finished = true;
                st = e.status;
                err = e.what();
            }
            if (!finished) continue;
            progressed = true;
            R->solver.reset();  // frees its device memory
            std::lock_guard<std::mutex> lk(S->mu);
            S->active.erase(std::find(S->active.begin(), S->active.end(), R));
            S->used -= R->need;
            if (st != PS_OK) fail(S, R, st, err);
            else {
                R->res = res;
                R->status = ps_status(res.status);
                R->state = Request::DONE;
                R->tDone = Clock::now();
                S->completed++;
            }
            S->cvDone.notify_all();
        }
        if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

void fillResult(const Request* R, ps_request_result* out) {
    std::memset(out, 0, sizeof *out);
    out->id = R->id;
    out->status = R->status;
    out->iterations = R->res.iterations;
    out->converged = R->res.converged;
    out->residual = R->res.residual;
    out->n_dof = R->nDof;
    out->u = R->uPinned;
    out->build_s = secs(R->tSubmit, R->tBuilt);
    out->wait_s = R->tAdmit.time_since_epoch().count() ? secs(R->tBuilt, R->tAdmit) : 0;
    out->solve_s = R->tAdmit.time_since_epoch().count() ? secs(R->tAdmit, R->tDone) : 0;
    out->total_s = secs(R->tSubmit, R->tDone);
}

}  // namespace
}  // namespace psfea

using psfea::Request;

extern "C" {

ps_status ps_server_create(int64_t device_budget_bytes, int32_t max_active, int32_t build_threads, ps_server_t** out) {
    if (!out) return PS_EINVAL;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return PS_ENODEV;
    }
    auto* S = new ps_server;
    cudaGetDevice(&S->device);
    size_t freeB = 0, totalB = 0;
    cudaMemGetInfo(&freeB, &totalB);
    S->budget = device_budget_bytes > 0 ? device_budget_bytes : int64_t(double(freeB) * 0.8);
    S->maxActive = max_active > 0 ? max_active : 4;
    // freed device memory stays in the stream-ordered allocator's pool for the next request (the
    // default would hand it back to the driver at every synchronisation)
    cudaMemPool_t pool = nullptr;
    if (cudaDeviceGetDefaultMemPool(&pool, S->device) == cudaSuccess) {
        uint64_t keep = uint64_t(S->budget);
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    const int nb = build_threads > 0 ? build_threads : int(std::max(1u, psfea::hostThreads() / 2));
    for (int t = 0; t < nb; t++) S->builders.emplace_back(psfea::builderLoop, S);
    for (int t = 0; t < 2; t++) S->uploaders.emplace_back(psfea::uploaderLoop, S);
    S->scheduler = std::thread(psfea::schedulerLoop, S);
    *out = S;
    return PS_OK;
}

ps_status ps_server_submit(ps_server_t* S, const ps_request* q, int64_t* id) {
    if (!S || !q || !id || !q->density || !q->bc || !q->f) return PS_EINVAL;
    if (q->dims[0] < 1 || q->dims[1] < 1 || q->dims[2] < 1) return PS_EINVAL;
    auto R = std::make_unique<Request>();
    std::memcpy(R->dims, q->dims, sizeof R->dims);
    const int64_t nE = int64_t(q->dims[0]) * q->dims[1] * q->dims[2];
    R->nDof = 3 * int64_t(q->dims[0] + 1) * (q->dims[1] + 1) * (q->dims[2] + 1);
    for (int64_t i = 0; i < R->nDof; i++)
        if (!std::isfinite(q->f[i])) return PS_ENONFINITE;
    R->density.assign(q->density, q->density + nE);
    R->bc.assign(q->bc, q->bc + R->nDof);
    R->fHost.assign(q->f, q->f + R->nDof);
    R->nu = q->nu;
    R->coarsest = q->coarsest_max_dof > 0 ? q->coarsest_max_dof : 300;
    ps_solve_opts_default(&R->opts);
    R->opts.tol = q->tol > 0 ? q->tol : 1e-8;
    R->opts.max_iter = q->max_iter > 0 ? q->max_iter : 5000;
    R->opts.precision = q->precision;
    R->opts.smoother_degree = q->smoother_degree;
    R->tSubmit = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> lk(S->mu);
    R->id = S->nextId++;
    *id = R->id;
    S->buildQueue.push_back(R.get());
    S->all[R->id] = std::move(R);
    S->cvBuild.notify_one();
    return PS_OK;
}

ps_status ps_server_poll(ps_server_t* S, int64_t id, ps_request_result* out) {
    if (!S || !out) return PS_EINVAL;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->all.find(id);
    if (it == S->all.end()) return PS_EINVAL;
    if (it->second->state != Request::DONE) return PS_PENDING;
    psfea::fillResult(it->second.get(), out);
    return PS_OK;
}

ps_status ps_server_wait(ps_server_t* S, int64_t id, ps_request_result* out) {
    if (!S || !out) return PS_EINVAL;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->all.find(id);
    if (it == S->all.end()) return PS_EINVAL;
    Request* R = it->second.get();
    S->cvDone.wait(lk, [&] { return R->state == Request::DONE; });
    psfea::fillResult(R, out);
    return PS_OK;
}

ps_status ps_server_release(ps_server_t* S, int64_t id) {
    if (!S) return PS_EINVAL;
    std::unique_ptr<Request> R;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        auto it = S->all.find(id);
        if (it == S->all.end() || it->second->state != Request::DONE) return PS_EINVAL;
        R = std::move(it->second);
        S->all.erase(it);
    }
    if (R->fPinned) cudaFreeHost(R->fPinned);
    if (R->uPinned) cudaFreeHost(R->uPinned);
    return PS_OK;
}

ps_status ps_server_get_stats(ps_server_t* S, ps_server_stats* out) {
    if (!S || !out) return PS_EINVAL;
    std::lock_guard<std::mutex> lk(S->mu);
    out->queued = int64_t(S->buildQueue.size() + S->ready.size());
    out->active = int64_t(S->active.size());
    out->completed = S->completed;
    out->device_bytes_in_use = S->used;
    out->peak_device_bytes = S->peakUsed;
    out->peak_active = S->peakActive;
    out->budget_bytes = S->budget;
    return PS_OK;
}

void ps_server_destroy(ps_server_t* S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cvBuild.notify_all();
    S->cvSched.notify_all();
    S->cvUpload.notify_all();
    for (auto& t : S->builders) t.join();
    for (auto& t : S->uploaders) t.join();
    S->scheduler.join();
    for (auto& kv : S->all) {
        kv.second->solver.reset();
        if (kv.second->fPinned) cudaFreeHost(kv.second->fPinned);
        if (kv.second->uPinned) cudaFreeHost(kv.second->uPinned);
    }
    delete S;
}

}  // extern "C"
