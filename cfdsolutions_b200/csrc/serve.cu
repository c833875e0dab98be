// Serving loop: steady-solve requests admitted against an HBM budget and run
// concurrently on one GPU.
//
// A server owns a FIFO of requests and a fixed set of worker threads, each
// with its own non-blocking CUDA stream.  A worker takes the head request as
// soon as the request's memory estimate fits in what the budget has left,
// then builds its mesh on the host (while the other workers' solves keep the
// GPU busy), creates a context on its stream, sets the seeded initial state,
// and runs the implicit steady solve to the request's residual drop.  Device
// memory of a worker is allocated stream-ordered on its stream, so no worker
// synchronises the device and solves of different sizes overlap; their
// kernels interleave on the GPU, filling it where one small solve alone is
// latency bound.  Every kernel of the solve is deterministic (fixed summation
// orders, no floating-point atomics), so a request's result does not depend on
// what runs beside it.
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "cfd_internal.h"
#include "ctx.cuh"

namespace {

using Clock = std::chrono::steady_clock;

uint64_t splitmix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

// U[-1, 1) from (seed, counter): 53 random bits of a counter-based hash.
double unit_pm1(uint64_t seed, uint64_t k) {
    const uint64_t z = splitmix64(seed ^ splitmix64(k));
    return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// Device bytes of one request, from the box dimensions (the mesh is built
// after admission): per node the state, residuals, gradients, limiters (two
// buffers), geometry, incidence and (restart+1)+5 Krylov/work vectors; per block of the
// Jacobian its stored copies, the preconditioner factors (three times their
// size: the factors and the triangular solves' padded packed copy) and the
// ordering lists.  A tet-split box has ~7 interior edges per node, blocks = N + 2E.
double estimate_bytes(const cfd_serve_request &r) {
    const double N = (double)(r.nx + 1) * (r.ny + 1) * (r.nz + 1);
    const double nnzb = N * 15.5;
    const int gp = r.opts.gmres.precision & ~CFD_PREC_LOW_ONLY;
    const bool low_only = (r.opts.gmres.precision & CFD_PREC_LOW_ONLY) != 0 && r.opts.linear_solver == 1;
    double a = low_only ? 0.0 : 200.0;
    if (r.opts.linear_solver == 1) a += gp == CFD_PREC_FP32 ? 100.0 : gp == CFD_PREC_BF16 ? 50.0 : 0.0;
    const double m = r.opts.linear_solver == 1 ? 3.0 * (gp == CFD_PREC_FP64 ? 200.0 : 100.0) : 0.0;
    const double krylov = r.opts.linear_solver == 1 ? 40.0 * (r.opts.gmres.restart + 1 + 5) : 240.0;
    return 1.2 * (N * (1644.0 + krylov) + nnzb * (a + m + 60.0)) + (16 << 20);
}

struct Job {
    cfd_serve_request req{};
    cfd_serve_result res{};
    std::vector<double> state;
    bool done = false;
};

// Fuses the interior residual launches and the block SpMV launches of the
// requests being solved side by side into one k_residual_gather_batch /
// k_bspmv_batch launch over a request table.  A worker's cfd_residual (or
// GMRES SpMV) hands its job to submit(), which records an event on the
// worker's stream and waits until the batcher has launched a batch that
// contains the job; the batcher waits for the events of the batch's jobs on
// its own stream, launches, records each job's completion event, and the
// worker's stream waits for that event before its next kernel.  A batch takes
// the jobs of the first job's kernel (key) queued until as many jobs as
// requests in their solves are waiting, or `window` after the first, up to
// kBatchMax.  Each node's residual and each row's product are computed by the
// same code as in the request's own launch, so results do not depend on the
// batching.
struct Batcher {
    struct Pend {
        int key;
        cfd::GatherJob gather;  // key < kSpmvKey
        cfd::SpmvJob spmv;      // key >= kSpmvKey
        cudaEvent_t ev_in, ev_out;
        bool launched;
        int status;
    };
    int device = 0;
    std::chrono::duration<double> window{50e-6};
    std::atomic<int> solving{0};  // requests inside their solves: jobs worth waiting for
    std::mutex mu;
    std::condition_variable cv_sub, cv_done;
    std::deque<Pend *> q;
    bool stop = false, dead = false;
    uint64_t batches[2] = {0, 0}, jobs[2] = {0, 0};  // [residual, SpMV]
    std::thread th;

    int launch(int key, const std::vector<Pend *> &take, cudaStream_t s) {
        if (key >= cfd::kSpmvKey) {
            cfd::SpmvBatch b;
            b.njobs = (int)take.size();
            int blk = 0;
            for (int k = 0; k < b.njobs; k++) {
                b.job[k] = take[k]->spmv;
                b.job[k].block_begin = blk;
                blk += (int)((5 * (int64_t)b.job[k].nrow + 159) / 160);
            }
            return cfd::launch_spmv_batch(key, b, s);
        }
        cfd::GatherBatch b;
        b.njobs = (int)take.size();
        int blk = 0;
        for (int k = 0; k < b.njobs; k++) {
            b.job[k] = take[k]->gather;
            b.job[k].block_begin = blk;
            blk += (b.job[k].nnode + 127) / 128;
        }
        return cfd::launch_gather_batch(key, b, s);
    }

    void run() {
        cudaSetDevice(device);
        cudaStream_t s = nullptr;
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
            std::lock_guard<std::mutex> lk(mu);
            dead = true;
            for (Pend *p : q) { p->status = CFD_ERR_CUDA; p->launched = true; }
            q.clear();
            cv_done.notify_all();
            return;
        }
        for (;;) {
            std::vector<Pend *> take;
            int key;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_sub.wait(lk, [&] { return stop || !q.empty(); });
                if (q.empty()) break;  // stop with nothing queued
                const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(window);
                cv_sub.wait_until(lk, deadline, [&] {
                    return stop || (int)q.size() >= std::min(cfd::kBatchMax, std::max(1, solving.load()));
                });
                key = q.front()->key;
                for (auto it = q.begin(); it != q.end() && (int)take.size() < cfd::kBatchMax;) {
                    if ((*it)->key == key) {
                        take.push_back(*it);
                        it = q.erase(it);
                    } else {
                        ++it;
                    }
                }
            }
            int st = CFD_OK;
            for (Pend *p : take)
                if (cudaStreamWaitEvent(s, p->ev_in, 0) != cudaSuccess) st = CFD_ERR_CUDA;
            if (st == CFD_OK) st = launch(key, take, s);
            for (Pend *p : take)
                if (st == CFD_OK && cudaEventRecord(p->ev_out, s) != cudaSuccess) st = CFD_ERR_CUDA;
            {
                std::lock_guard<std::mutex> lk(mu);
                for (Pend *p : take) {
                    p->status = st;
                    p->launched = true;
                }
                const int kind = key >= cfd::kSpmvKey ? 1 : 0;
                batches[kind]++;
                jobs[kind] += take.size();
            }
            cv_done.notify_all();
        }
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
};

// per worker thread: the events of its fused jobs
thread_local cudaEvent_t tl_ev_in = nullptr, tl_ev_out = nullptr;

int batch_submit(void *b, cfd_ctx *c, int key, const void *job) {
    Batcher *B = static_cast<Batcher *>(b);
    if (!tl_ev_in) {
        CFD_CUDA(cudaEventCreateWithFlags(&tl_ev_in, cudaEventDisableTiming));
        CFD_CUDA(cudaEventCreateWithFlags(&tl_ev_out, cudaEventDisableTiming));
    }
    CFD_CUDA(cudaEventRecord(tl_ev_in, c->stream));
    Batcher::Pend p{};
    p.key = key;
    if (key >= cfd::kSpmvKey) p.spmv = *static_cast<const cfd::SpmvJob *>(job);
    else p.gather = *static_cast<const cfd::GatherJob *>(job);
    p.ev_in = tl_ev_in;
    p.ev_out = tl_ev_out;
    p.launched = false;
    p.status = CFD_OK;
    {
        std::unique_lock<std::mutex> lk(B->mu);
        if (B->dead || B->stop) {
            cfd::set_error("launch batcher: not running");
            return CFD_ERR_STATE;
        }
        B->q.push_back(&p);
        B->cv_sub.notify_one();
        B->cv_done.wait(lk, [&] { return p.launched; });
    }
    if (p.status) {
        cfd::set_error("launch batcher: fused launch failed (%d)", p.status);
        return p.status;
    }
    CFD_CUDA(cudaStreamWaitEvent(c->stream, tl_ev_out, 0));
    return CFD_OK;
}

}  // namespace

struct cfd_server {
    int device = 0;
    Batcher *batcher = nullptr;  // fuser of the requests' residual launches
    bool batching = true;        // requests use it (cfd_server_set_batching)
    double budget = 0.0, reserved = 0.0, peak = 0.0;
    int active = 0;
    bool stop = false;
    int64_t next_id = 1;
    Clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv;       // queue / admission changes
    std::condition_variable done_cv;  // a job finished
    std::deque<int64_t> queue;
    std::unordered_map<int64_t, Job> jobs;
    std::vector<std::thread> workers;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
    void run_worker();
};

namespace {

// One request on the calling worker (its stream is already current for
// allocation).  Returns the first failing status.
int run_job(int device, cudaStream_t s, const cfd_serve_request &r, cfd_serve_result &res, std::vector<double> &keep,
            const cfd_server &srv) {
    cfd_mesh *mesh = nullptr;
    int st = cfd_mesh_box(r.nx, r.ny, r.nz, r.lx, r.ly, r.lz, r.jitter, r.mesh_seed, r.numbering, r.face_bc, &mesh);
    if (st) return st;
    cfd_ctx *ctx = nullptr;
    std::vector<double> Q;
    do {
        if ((st = cfd_create(device, &ctx))) break;
        if ((st = cfd_set_stream(ctx, s))) break;
        if (srv.batcher && srv.batching) {
            ctx->batcher = srv.batcher;
            ctx->batch_submit = batch_submit;
        }
        if ((st = cfd_set_params(ctx, &r.params))) break;
        if ((st = cfd_set_mesh_from(ctx, mesh))) break;
        res.nnode = mesh->m.nnode;
        res.nghost = mesh->m.nghost;
        Q.resize((size_t)5 * (res.nnode + res.nghost));
        const cfd_params &p = r.params;
        const double noise[3] = {r.noise, r.noise, r.noise};
        if ((st = cfd_initial_state(mesh, &p, noise, r.state_seed, Q.data()))) break;
        if ((st = cfd_set_state(ctx, Q.data()))) break;
        if (r.opts.linear_solver == 1 && r.opts.gmres.precond == CFD_PC_ILU0_MC &&
            (st = cfd_ilu_mc_order(ctx, nullptr, nullptr)))
            break;
        res.t_start_solve = srv.now();
        Batcher *fuse = ctx->batcher ? srv.batcher : nullptr;
        if (fuse) fuse->solving++;
        st = cfd_solve_steady(ctx, &r.opts, &res.stats);
        if (fuse) fuse->solving--;
        if (st) break;
        if (r.keep_state) {
            keep.resize(Q.size());
            if ((st = cfd_get_state(ctx, keep.data()))) break;
        }
    } while (false);
    if (ctx) cfd_destroy(ctx);
    cudaStreamSynchronize(s);  // the stream-ordered frees have completed
    cfd_mesh_free(mesh);
    return st;
}

}  // namespace

void cfd_server::run_worker() {
    cudaSetDevice(device);
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return;
    cfd::g_alloc_async = true;
    cfd::g_host_threads = 2;  // mesh builds share the host with the other workers
    cfd::g_alloc_stream = s;
    for (;;) {
        int64_t id;
        Job *job;
        double est;
        {
            std::unique_lock<std::mutex> lk(mu);
            // FIFO admission: the head request waits until its estimate fits
            cv.wait(lk, [&] {
                if (stop) return true;
                if (queue.empty()) return false;
                const double e = jobs[queue.front()].res.bytes_estimate;
                return reserved + e <= budget || active == 0;
            });
            if (stop) break;
            id = queue.front();
            queue.pop_front();
            job = &jobs[id];
            est = job->res.bytes_estimate;
            reserved += est;
            peak = std::max(peak, reserved);
            active++;
            job->res.t_admit = now();
        }
        cfd_serve_result res = job->res;
        std::vector<double> keep;
        res.status = run_job(device, s, job->req, res, keep, *this);
        if (res.status) std::snprintf(res.message, sizeof(res.message), "%s", cfd_last_error());
        res.t_done = now();
        {
            std::lock_guard<std::mutex> lk(mu);
            job->res = res;
            job->state.swap(keep);
            job->done = true;
            reserved -= est;
            active--;
        }
        cv.notify_all();
        done_cv.notify_all();
    }
    cfd::g_alloc_async = false;
    cfd::g_alloc_stream = nullptr;
    if (tl_ev_in) {
        cudaEventDestroy(tl_ev_in);
        cudaEventDestroy(tl_ev_out);
        tl_ev_in = tl_ev_out = nullptr;
    }
    cudaStreamDestroy(s);
}

extern "C" {

int cfd_perturbed_freestream(const cfd_mesh *m, double gamma, double mach, double alpha_deg, double beta_deg,
                             double noise, uint64_t seed, double *Q) {
    cfd_params p;
    cfd_params_default(&p);
    p.gamma = gamma;
    p.mach = p.mach_min = mach;
    p.alpha_deg = alpha_deg;
    p.beta_deg = beta_deg;
    const double nz[3] = {noise, noise, noise};
    return cfd_initial_state(m, &p, nz, seed, Q);
}

int cfd_initial_state(const cfd_mesh *m, const cfd_params *p, const double noise[3], uint64_t seed, double *Q) {
    if (!m || !p || !noise || !Q || !(p->gamma > 1.0) || !(p->pinf >= 0.0)) return CFD_ERR_ARG;
    const double gamma = p->gamma, pinf = p->pinf;
    const int64_t N = m->m.nnode, n = N + m->m.nghost;
    // rho = 1, p = 1: c^2 = gamma (1 + pinf)
    const double c = pinf != 0.0 ? std::sqrt(gamma * (1.0 + pinf)) : std::sqrt(gamma);
    const double deg = 3.14159265358979323846 / 180.0;
    const double a = p->alpha_deg * deg, b = p->beta_deg * deg, mach = p->mach;
    const double u0[3] = {mach * c * std::cos(a) * std::cos(b), mach * c * std::sin(a),
                          mach * c * std::sin(b) * std::cos(a)};
    for (int64_t i = 0; i < n; i++) {
        const bool phys = i < N;
        const double rho = 1.0 * (phys ? 1.0 + noise[0] * unit_pm1(seed, (uint64_t)i) : 1.0);
        double v[3];
        for (int d = 0; d < 3; d++)
            v[d] = u0[d] * (phys ? 1.0 + noise[1] * unit_pm1(seed, (uint64_t)((1 + d) * N + i)) : 1.0);
        const double pr = 1.0 * (phys ? 1.0 + noise[2] * unit_pm1(seed, (uint64_t)(4 * N + i)) : 1.0);
        Q[i] = rho;
        if (p->variables == CFD_VARS_RUP) {
            Q[n + i] = v[0];
            Q[2 * n + i] = v[1];
            Q[3 * n + i] = v[2];
            Q[4 * n + i] = pr;
            continue;
        }
        const double et = (pr + gamma * pinf) / ((gamma - 1.0) * rho) + 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        Q[n + i] = rho * v[0];
        Q[2 * n + i] = rho * v[1];
        Q[3 * n + i] = rho * v[2];
        Q[4 * n + i] = rho * et;
    }
    return CFD_OK;
}

int cfd_server_create(int device, int workers, double budget_bytes, cfd_server **out) {
    if (!out || workers < 1 || workers > 256 || !(budget_bytes > 0.0)) {
        cfd::set_error("cfd_server_create: workers in [1,256] and a positive budget");
        return CFD_ERR_ARG;
    }
    *out = nullptr;
    int ndev = 0;
    CFD_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) { cfd::set_error("cfd_server_create: device %d of %d", device, ndev); return CFD_ERR_ARG; }
    CFD_CUDA(cudaSetDevice(device));
    // keep freed blocks in the device pool for the next request
    cudaMemPool_t pool;
    CFD_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t thr = UINT64_MAX;
    CFD_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    cfd_server *srv = new cfd_server();
    srv->device = device;
    srv->budget = budget_bytes;
    srv->t0 = Clock::now();
    srv->batcher = new Batcher();
    srv->batcher->device = device;
    srv->batcher->th = std::thread([b = srv->batcher] { b->run(); });
    for (int w = 0; w < workers; w++) srv->workers.emplace_back([srv] { srv->run_worker(); });
    *out = srv;
    return CFD_OK;
}

int cfd_server_submit(cfd_server *srv, const cfd_serve_request *req, int64_t *id) {
    if (!srv || !req || !id) return CFD_ERR_ARG;
    if (req->nx < 1 || req->ny < 1 || req->nz < 1 || !(req->lx > 0) || !(req->ly > 0) || !(req->lz > 0)) {
        cfd::set_error("cfd_server_submit: box of at least one hex with positive extents");
        return CFD_ERR_ARG;
    }
    if (req->opts.max_iterations < 1) { cfd::set_error("cfd_server_submit: max_iterations < 1"); return CFD_ERR_ARG; }
    const double est = estimate_bytes(*req);
    std::lock_guard<std::mutex> lk(srv->mu);
    if (est > srv->budget) {
        cfd::set_error("cfd_server_submit: request needs ~%.3g GB, more than the %.3g GB budget", est / 1e9,
                       srv->budget / 1e9);
        return CFD_ERR_RANGE;
    }
    if (srv->stop) { cfd::set_error("cfd_server_submit: server is shutting down"); return CFD_ERR_STATE; }
    const int64_t k = srv->next_id++;
    Job &j = srv->jobs[k];
    j.req = *req;
    j.res.status = CFD_PENDING;
    j.res.t_submit = srv->now();
    j.res.bytes_estimate = est;
    srv->queue.push_back(k);
    *id = k;
    srv->cv.notify_all();
    return CFD_OK;
}

int cfd_server_wait(cfd_server *srv, int64_t id, double timeout_s, cfd_serve_result *out) {
    if (!srv) return CFD_ERR_ARG;
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->jobs.find(id);
    if (it == srv->jobs.end()) { cfd::set_error("cfd_server_wait: unknown request %lld", (long long)id); return CFD_ERR_ARG; }
    auto ready = [&] { return srv->jobs[id].done; };
    if (timeout_s < 0) srv->done_cv.wait(lk, ready);
    else if (!srv->done_cv.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) return CFD_PENDING;
    if (out) *out = srv->jobs[id].res;
    return CFD_OK;
}

int cfd_server_state(cfd_server *srv, int64_t id, double *Q) {
    if (!srv || !Q) return CFD_ERR_ARG;
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->jobs.find(id);
    if (it == srv->jobs.end() || !it->second.done) { cfd::set_error("cfd_server_state: request not finished"); return CFD_ERR_STATE; }
    if (it->second.state.empty()) { cfd::set_error("cfd_server_state: request did not keep its state"); return CFD_ERR_STATE; }
    std::memcpy(Q, it->second.state.data(), sizeof(double) * it->second.state.size());
    return CFD_OK;
}

int cfd_server_release(cfd_server *srv, int64_t id) {
    if (!srv) return CFD_ERR_ARG;
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->jobs.find(id);
    if (it == srv->jobs.end() || !it->second.done) return CFD_ERR_STATE;
    srv->jobs.erase(it);
    return CFD_OK;
}

int cfd_server_stats(cfd_server *srv, double out[5]) {
    if (!srv || !out) return CFD_ERR_ARG;
    std::lock_guard<std::mutex> lk(srv->mu);
    out[0] = srv->active;
    out[1] = (double)srv->queue.size();
    out[2] = srv->reserved;
    out[3] = srv->peak;
    out[4] = srv->now();
    return CFD_OK;
}

int cfd_server_destroy(cfd_server *srv) {
    if (!srv) return CFD_OK;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stop = true;  // queued requests are not started; running ones finish
    }
    srv->cv.notify_all();
    for (auto &t : srv->workers) t.join();
    if (srv->batcher) {
        {
            std::lock_guard<std::mutex> lk(srv->batcher->mu);
            srv->batcher->stop = true;
        }
        srv->batcher->cv_sub.notify_all();
        srv->batcher->th.join();
        delete srv->batcher;
    }
    delete srv;
    return CFD_OK;
}

int cfd_server_set_batching(cfd_server *srv, int enable, double window_us) {
    if (!srv || !srv->batcher || !(window_us >= 0.0) || window_us > 1e6) {
        cfd::set_error("cfd_server_set_batching: a server and a window in [0, 1e6] us");
        return CFD_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->active > 0 || !srv->queue.empty()) {
        cfd::set_error("cfd_server_set_batching: set it before submitting requests");
        return CFD_ERR_STATE;
    }
    srv->batching = enable != 0;
    srv->batcher->window = std::chrono::duration<double>(window_us * 1e-6);
    return CFD_OK;
}

int cfd_server_batch_stats(cfd_server *srv, double out[4]) {
    if (!srv || !out) return CFD_ERR_ARG;
    std::lock_guard<std::mutex> lk(srv->batcher->mu);
    for (int k = 0; k < 2; k++) {
        out[2 * k] = (double)srv->batcher->batches[k];
        out[2 * k + 1] = (double)srv->batcher->jobs[k];
    }
    return CFD_OK;
}

}  // extern "C"
