// Continuous-batching server for independent ADMP evaluations on one GPU (dmffb_server_*).
//
// A pool of engines ("slots"), each with its own CUDA streams, created once at the largest
// request size and re-pointed at every request with dmffb_admp_reconfigure, and one host worker
// thread per slot.  Requests queue in arrival order; a worker admits the head request when its
// arrival time has passed and the device footprint of everything in flight plus its own fits
// the budget.  Workers run their requests through dmffb_admp_compute_host on their own streams,
// so the GPU interleaves the kernels of all admitted requests: many small, launch-bound boxes
// overlap, while the footprint budget keeps only a few large ones in flight.  With several slots
// the engines run the per-pass dipole solve (short kernels that interleave); a single slot uses
// the persistent solve for small requests.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/dmffb200.h"

struct dmffb_server {
    dmffb_server_desc d;
    int device = 0;
    std::vector<dmffb_engine*> eng;
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<dmffb_request*> pending;
    int64_t in_flight_bytes = 0;
    int64_t submitted = 0, completed = 0;
    bool stop = false;
    std::chrono::steady_clock::time_point t0;
};

namespace {

double now_s(const dmffb_server* s) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - s->t0).count();
}

dmffb_admp_desc request_desc(const dmffb_server* s, const dmffb_request* r) {
    dmffb_admp_desc a;
    memset(&a, 0, sizeof(a));
    a.n_atoms = r->n_atoms;
    a.lmax = s->d.lmax;
    a.lpol = s->d.lpol;
    a.lpme = 1;
    a.precision = s->d.precision;
    a.rc = r->rc;
    a.kappa = r->kappa;
    for (int k = 0; k < 3; ++k) a.K[k] = r->K[k];
    a.axis_types = r->axis_types;
    a.axis_indices = r->axis_indices;
    a.n_cov = r->n_cov;
    a.cov_rows = r->cov_rows;
    for (int k = 0; k < 6; ++k) {
        a.mscales[k] = s->d.mscales[k];
        a.pscales[k] = s->d.pscales[k];
        a.dscales[k] = s->d.dscales[k];
    }
    a.solver = s->d.solver;
    a.cg_tol = s->d.cg_tol;
    a.max_iter = s->d.max_iter;
    return a;
}

// one request on one slot; returns the evaluation status
int run_request(dmffb_server* s, int slot, dmffb_request* r) {
    dmffb_engine* h = s->eng[slot];
    dmffb_admp_desc a = request_desc(s, r);
    int st = dmffb_admp_reconfigure(h, &a);
    if (!st) st = dmffb_admp_set_params(h, r->Q_local, r->pol, r->thole);
    dmffb_admp_result res;
    memset(&res, 0, sizeof(res));
    if (!st) st = dmffb_admp_compute_host(h, r->pos, r->box, nullptr, 0, nullptr, r->forces_out, &res);
    r->energy = res.energy;
    for (int k = 0; k < 9; ++k) r->box_grad[k] = res.box_grad[k];
    r->n_iter = res.n_iter;
    return st;
}

void worker(dmffb_server* s, int slot) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        if (s->stop) return;
        if (s->pending.empty()) {
            s->cv.wait(lk);
            continue;
        }
        dmffb_request* r = s->pending.front();
        const double t = now_s(s);
        if (r->t_arrival > t) {  // not arrived yet: sleep until it does (or something changes)
            s->cv.wait_for(lk, std::chrono::duration<double>(r->t_arrival - t));
            continue;
        }
        const int64_t budget = s->d.hbm_budget_bytes;
        if (budget > 0 && s->in_flight_bytes > 0 && s->in_flight_bytes + r->footprint_bytes > budget) {
            s->cv.wait(lk);  // memory frees when a running request completes
            continue;
        }
        s->pending.pop_front();
        s->in_flight_bytes += r->footprint_bytes;
        lk.unlock();
        s->cv.notify_all();  // the next head may fit too
        r->slot = slot;
        r->t_start = now_s(s);
        const int st = run_request(s, slot, r);
        r->t_done = now_s(s);
        r->status = st;
        lk.lock();
        s->in_flight_bytes -= r->footprint_bytes;
        s->completed++;
        __atomic_store_n(&r->done, 1, __ATOMIC_RELEASE);
        s->cv.notify_all();
    }
}

}  // namespace

extern "C" {

int64_t dmffb_request_footprint(int32_t n_atoms, double rc, const int32_t K[3], double box_volume, int32_t lpol) {
    // accounting convention: per-atom engine arrays, neighbour rows + both-direction CSR with the
    // matvec pair tensors, and the mesh with its complex transform, cuFFT work area and (with
    // polarization) the second real grid of the dipole field pass
    const double n = n_atoms;
    const double dens = box_volume > 0 ? n / box_volume : 0.1;
    const double half_pairs = n * dens * (4.0 / 3.0) * M_PI * rc * rc * rc / 2.0;
    const double K3 = (double)K[0] * K[1] * K[2];
    const double bytes = n * (600.0 + (lpol ? 320.0 : 0.0)) + half_pairs * 92.0 + (lpol ? 20.0 : 16.0) * K3;
    return (int64_t)bytes;
}

int dmffb_server_create(const dmffb_server_desc* d, dmffb_server** out) {
    if (!d || !out || d->n_slots <= 0 || d->capacity_atoms <= 0) return DMFFB_BAD_ARG;
    *out = nullptr;
    dmffb_server* s = new dmffb_server();
    s->d = *d;
    s->t0 = std::chrono::steady_clock::now();
    cudaGetDevice(&s->device);
    // every slot starts as a minimal system of full capacity (no-axis atoms, an 8^3 mesh)
    const int n = d->capacity_atoms;
    std::vector<int32_t> at(n, DMFFB_NOAXISTYPE), ai(3 * (size_t)n, -1);
    dmffb_admp_desc a;
    memset(&a, 0, sizeof(a));
    a.n_atoms = n;
    a.lmax = d->lmax;
    a.lpol = d->lpol;
    a.lpme = 1;
    a.precision = d->precision;
    a.rc = 8.0;
    a.kappa = 0.3;
    a.K[0] = a.K[1] = a.K[2] = 8;
    a.axis_types = at.data();
    a.axis_indices = ai.data();
    for (int k = 0; k < 6; ++k) {
        a.mscales[k] = d->mscales[k];
        a.pscales[k] = d->pscales[k];
        a.dscales[k] = d->dscales[k];
    }
    a.solver = d->solver;
    a.cg_tol = d->cg_tol;
    a.max_iter = d->max_iter;
    for (int k = 0; k < d->n_slots; ++k) {
        dmffb_engine* h = nullptr;
        int st = dmffb_admp_create(&a, &h);
        if (st) {
            if (h) dmffb_destroy(h);
            dmffb_server_destroy(s);
            return st;
        }
        dmffb_set_graphs(h, d->use_graphs);
        // several slots: the per-pass solve, whose short kernels interleave with the other slots'
        // (a persistent solve holds its SMs for the whole solve, mostly waiting at barriers);
        // one slot: the engine's size rule, which shortens each small request
        dmffb_set_persistent_cg(h, d->n_slots > 1 ? 0 : 2);
        s->eng.push_back(h);
    }
    for (int k = 0; k < d->n_slots; ++k) s->workers.emplace_back(worker, s, k);
    *out = s;
    return DMFFB_OK;
}

int dmffb_server_submit(dmffb_server* s, dmffb_request* r) {
    if (!s || !r || r->n_atoms <= 0 || !r->pos || !r->Q_local || !r->forces_out) return DMFFB_BAD_ARG;
    if (r->n_atoms > s->d.capacity_atoms) return DMFFB_SCRATCH_TOO_SMALL;
    if (s->d.lpol && (!r->pol || !r->thole)) return DMFFB_BAD_ARG;
    const double V = fabs(r->box[0] * (r->box[4] * r->box[8] - r->box[5] * r->box[7]) -
                          r->box[1] * (r->box[3] * r->box[8] - r->box[5] * r->box[6]) +
                          r->box[2] * (r->box[3] * r->box[7] - r->box[4] * r->box[6]));
    r->footprint_bytes = dmffb_request_footprint(r->n_atoms, r->rc, r->K, V, s->d.lpol);
    r->done = 0;
    r->status = -1;
    r->slot = -1;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (!s->pending.empty() && r->t_arrival < s->pending.back()->t_arrival) return DMFFB_BAD_ARG;
        s->pending.push_back(r);
        s->submitted++;
    }
    s->cv.notify_all();
    return DMFFB_OK;
}

int dmffb_server_wait(dmffb_server* s, double timeout_s) {
    if (!s) return DMFFB_BAD_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    const bool ok = s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                   [&] { return s->completed == s->submitted; });
    return ok ? DMFFB_OK : DMFFB_CUDA_ERROR;
}

double dmffb_server_clock(const dmffb_server* s) { return s ? now_s(s) : 0.0; }

int dmffb_server_prewarm(dmffb_server* s, dmffb_request* reqs, int32_t n_reqs) {
    if (!s || (n_reqs > 0 && !reqs)) return DMFFB_BAD_ARG;
    {  // only while idle: the slots' engines are driven from this thread
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->completed != s->submitted) return DMFFB_BAD_ARG;
    }
    for (size_t k = 0; k < s->eng.size(); ++k)
        for (int32_t q = 0; q < n_reqs; ++q) {
            int st = run_request(s, (int)k, &reqs[q]);
            if (st && st != DMFFB_NOT_CONVERGED) return st;
        }
    return DMFFB_OK;
}

void dmffb_server_destroy(dmffb_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    for (auto& t : s->workers)
        if (t.joinable()) t.join();
    for (auto h : s->eng) dmffb_destroy(h);
    delete s;
}

}  // extern "C"
