// Serving loop: transport solves of different sizes admitted by device
// memory and advanced together with continuous batching.
//
// A request is one coupled transport solve (mesh, cell averages, face
// velocities, final time) -- what AdvancePhaseCoupled does for one
// configuration (src/couple/evolve.cpp:513-519). Requests are queued on
// submit; a loop thread owns a batch (batch.cu) and, before every step,
// admits queued requests while their device bytes fit the budget and the
// resident cells are below a target. The order is arrival (FIFO) or smallest
// estimated work first: work ~ cells * t_final * (cells per unit length),
// the step count of a CFL-limited solve scaling with the mesh resolution.
// The resident target keeps enough cells on the GPU to fill it while short
// requests pass long ones. Every step advances all resident requests at once (one launch per
// stage kernel for all of them), so work that arrives while others are on the
// GPU joins at the next step. A request leaves when it reaches its final time
// or fails; its result is copied out and its memory freed for the queue.
// State stays resident on the device between steps. A request on a general
// quad mesh joins the same batch as a quad instance (per-cell tables built
// on admission, its stage kernels batched over the quad instances).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.hpp"

extern "C" {
mp_status mp_batch_add_quads(mp_batch* b, const mp_mesh_desc* mesh, const double* xy, int* instance);
mp_status mp_batch_create(const mp_mesh_desc* meshes, int count, const mp_transport_opts* opts, mp_stream_t stream,
                          mp_batch** out);
void mp_batch_destroy(mp_batch* b);
mp_status mp_batch_add(mp_batch* b, const mp_mesh_desc* mesh, int* instance);
mp_status mp_batch_remove(mp_batch* b, int instance);
size_t mp_batch_instance_bytes(const mp_mesh_desc* mesh);
size_t mp_batch_bytes_in_use(const mp_batch* b);
int mp_batch_slots(const mp_batch* b);
mp_status mp_batch_set_face_velocity(mp_batch* b, int instance, const double* vs_n, const double* ud_n);
mp_status mp_batch_set_state(mp_batch* b, int instance, const double* H, const double* C, double time);
mp_status mp_batch_get_state(mp_batch* b, int instance, double* H, double* C, double* T, double* phi, double* time,
                             int* accepted, int* status);
mp_status mp_batch_step(mp_batch* b, int nsteps, mp_step_report* reports);
mp_status mp_batch_set_end_time(mp_batch* b, int instance, double t_end);
int mp_batch_finished(const mp_batch* b, int instance);
}

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    long long id = 0;
    mp_mesh_desc mesh{};
    size_t cells = 0, bytes = 0;
    std::vector<double> H, C, vs, ud;      // inputs (host copies)
    std::vector<double> oH, oC, oT, oP;    // results
    double t_final = 0;
    double work = 0;                       // admission-order estimate
    Clock::time_point submitted, admitted, finished;
    int slot = -1;
    bool quad = false;                     // general quad mesh
    std::vector<double> xy;                // its vertices until admission
    int status = 0;
    int accepted = 0;
    double time = 0;
    bool done = false;
};

}  // namespace

struct mp_server {
    mp_transport_opts opts{};
    int device = 0;
    size_t budget = 0;
    cudaStream_t stream = nullptr;
    mp_batch* batch = nullptr;
    std::thread loop;
    std::mutex m;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> queue;
    std::map<long long, std::shared_ptr<Request>> requests;
    std::vector<std::shared_ptr<Request>> active;
    long long next_id = 1;
    int order = MP_SERVE_SMALLEST_WORK;
    double resident_target = 1.0e6;        // cells; 0 = no limit
    double resident_cells = 0;
    bool stop = false;
    mp_status fatal = MP_OK;
    std::string fatal_msg;
    // statistics
    double cell_updates = 0;
    double busy_s = 0;
    long long steps = 0;
    Clock::time_point t0 = Clock::now();
};

namespace {

double seconds(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

// Admit queued requests (FIFO or smallest estimated work first) while they
// fit the memory budget and the resident cells are below the target. A
// request that does not fit waits; under FIFO nothing passes it.
void admit(mp_server* s) {
    for (;;) {
        std::shared_ptr<Request> r;
        {
            std::lock_guard<std::mutex> g(s->m);
            if (s->queue.empty()) return;
            if (s->resident_target > 0 && !s->active.empty() && s->resident_cells >= s->resident_target) return;
            auto pick = s->queue.begin();
            if (s->order == MP_SERVE_SMALLEST_WORK)
                for (auto it = s->queue.begin(); it != s->queue.end(); ++it)
                    if ((*it)->work < (*pick)->work) pick = it;
            r = *pick;
            if (mp_batch_bytes_in_use(s->batch) + r->bytes > s->budget) return;
            s->queue.erase(pick);
        }
        int slot = -1;
        mp_status st = r->quad ? mp_batch_add_quads(s->batch, &r->mesh, r->xy.data(), &slot)
                               : mp_batch_add(s->batch, &r->mesh, &slot);
        if (st == MP_OK) st = mp_batch_set_face_velocity(s->batch, slot, r->vs.data(), r->ud.data());
        if (st == MP_OK) st = mp_batch_set_state(s->batch, slot, r->H.data(), r->C.data(), 0.0);
        if (st == MP_OK) st = mp_batch_set_end_time(s->batch, slot, r->t_final);
        r->admitted = Clock::now();
        if (st != MP_OK) {
            if (slot >= 0) mp_batch_remove(s->batch, slot);
            std::lock_guard<std::mutex> g(s->m);
            r->status = st; r->done = true; r->finished = Clock::now();
            s->cv_done.notify_all();
            continue;
        }
        r->slot = slot;
        s->resident_cells += (double)r->cells;
        r->H.clear(); r->H.shrink_to_fit(); r->C.clear(); r->C.shrink_to_fit();
        r->vs.clear(); r->vs.shrink_to_fit(); r->ud.clear(); r->ud.shrink_to_fit();
        r->xy.clear(); r->xy.shrink_to_fit();
        std::lock_guard<std::mutex> g(s->m);
        s->active.push_back(r);
    }
}

// Copy out and release requests that reached their final time or failed.
void retire(mp_server* s) {
    std::vector<std::shared_ptr<Request>> keep;
    for (auto& r : s->active) {
        double time = 0;
        int acc = 0, status = 0;
        mp_batch_get_state(s->batch, r->slot, nullptr, nullptr, nullptr, nullptr, &time, &acc, &status);
        if (!status && !mp_batch_finished(s->batch, r->slot)) { keep.push_back(r); continue; }
        r->oH.resize(r->cells); r->oC.resize(r->cells); r->oT.resize(r->cells); r->oP.resize(r->cells);
        mp_batch_get_state(s->batch, r->slot, r->oH.data(), r->oC.data(), r->oT.data(), r->oP.data(), &r->time,
                           &r->accepted, &r->status);
        mp_batch_remove(s->batch, r->slot);
        std::lock_guard<std::mutex> g(s->m);
        s->resident_cells -= (double)r->cells;
        r->finished = Clock::now();
        r->done = true;
        s->cv_done.notify_all();
    }
    std::lock_guard<std::mutex> g(s->m);
    s->active.swap(keep);
}

void run(mp_server* s) {
    cudaSetDevice(s->device);
    while (true) {
        {
            std::unique_lock<std::mutex> lk(s->m);
            s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty() || !s->active.empty(); });
            if (s->stop) break;
        }
        admit(s);
        if (s->active.empty()) continue;
        // Cell-updates of this step: one per cell of every request that accepts it.
        std::vector<int> before(s->active.size());
        for (size_t k = 0; k < s->active.size(); ++k)
            mp_batch_get_state(s->batch, s->active[k]->slot, nullptr, nullptr, nullptr, nullptr, nullptr, &before[k], nullptr);
        const auto a = Clock::now();
        const mp_status st = mp_batch_step(s->batch, 1, nullptr);
        const auto b = Clock::now();
        if (st != MP_OK) {
            std::lock_guard<std::mutex> g(s->m);
            s->fatal = st;
            s->fatal_msg = mp_last_error_string();
            s->stop = true;
            s->cv_done.notify_all();
            break;
        }
        double upd = 0;
        for (size_t k = 0; k < s->active.size(); ++k) {
            int acc = 0;
            mp_batch_get_state(s->batch, s->active[k]->slot, nullptr, nullptr, nullptr, nullptr, nullptr, &acc, nullptr);
            upd += (double)(acc - before[k]) * (double)s->active[k]->cells;
        }
        {
            std::lock_guard<std::mutex> g(s->m);
            s->cell_updates += upd;
            s->busy_s += seconds(a, b);
            s->steps += 1;
        }
        retire(s);
    }
}

}  // namespace

extern "C" mp_status mp_serve_create(const mp_transport_opts* opts, size_t memory_budget, mp_server** out) {
    if (!opts || !out) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    if (opts->material.alpha0 != 0.0) {
        mp::set_error("served requests carry no cell-point velocities: the adiabatic source (alpha0 != 0) needs "
                      "mp_batch_set_cell_velocity or the single-instance path");
        return MP_ERR_ARG_WRONG;
    }
    auto* s = new mp_server;
    s->opts = *opts;
    s->budget = memory_budget;
    cudaGetDevice(&s->device);
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete s; return mp::cuda_status(e, "mp_serve_create"); }
    const mp_status st = mp_batch_create(nullptr, 0, opts, (mp_stream_t)s->stream, &s->batch);
    if (st != MP_OK) { cudaStreamDestroy(s->stream); delete s; return st; }
    s->loop = std::thread(run, s);
    *out = s;
    return MP_OK;
}

extern "C" void mp_serve_destroy(mp_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->m);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->loop.joinable()) s->loop.join();
    mp_batch_destroy(s->batch);
    cudaStreamDestroy(s->stream);
    delete s;
}

namespace {

mp_status submit_impl(mp_server* s, const mp_mesh_desc* mesh, const double* xy, const double* H, const double* C,
                      const double* vs_n, const double* ud_n, double t_final, long long* id) {
    if (!s || !mesh || !H || !C || !vs_n || !ud_n || !id) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    if (mesh->nx < 2 || mesh->ny < 2) { mp::set_error("Transport requires at least 2x2 cells"); return MP_ERR_ARG_SIZ; }
    if (mp::mesh_too_large(mesh->nx, mesh->ny)) { mp::set_error("mesh has 2^31 edges or more"); return MP_ERR_ARG_SIZ; }
    if (!(t_final > 0)) { mp::set_error("final time must be positive"); return MP_ERR_ARG_OUTOFRANGE; }
    auto r = std::make_shared<Request>();
    r->mesh = *mesh;
    r->cells = (size_t)mesh->nx * mesh->ny;
    const size_t edges = (size_t)mesh->nx * (mesh->ny + 1) + (size_t)(mesh->nx + 1) * mesh->ny;
    r->quad = xy != nullptr;
    r->bytes = r->quad ? mp_transport_instance_bytes(mesh, 1) : mp_batch_instance_bytes(mesh);
    if (r->bytes > s->budget) {
        mp::set_error("request needs %zu device bytes, above the server budget of %zu", r->bytes, s->budget);
        return MP_ERR_NOMEM;
    }
    if (r->quad) r->xy.assign(xy, xy + 2 * (size_t)(mesh->nx + 1) * (mesh->ny + 1));
    r->H.assign(H, H + r->cells);
    r->C.assign(C, C + r->cells);
    r->vs.assign(vs_n, vs_n + edges * 5);
    r->ud.assign(ud_n, ud_n + edges * 5);
    r->t_final = t_final;
    const double res = std::max(mesh->nx / std::fabs(mesh->x1 - mesh->x0), mesh->ny / std::fabs(mesh->y1 - mesh->y0));
    r->work = (double)r->cells * t_final * res;
    r->submitted = Clock::now();
    {
        std::lock_guard<std::mutex> g(s->m);
        if (s->stop) { mp::set_error("server stopped: %s", s->fatal_msg.c_str()); return s->fatal ? s->fatal : MP_ERR_ARG_WRONGSTATE; }
        r->id = s->next_id++;
        s->requests[r->id] = r;
        s->queue.push_back(r);
        *id = r->id;
    }
    s->cv_work.notify_all();
    return MP_OK;
}

}  // namespace

extern "C" mp_status mp_serve_submit(mp_server* s, const mp_mesh_desc* mesh, const double* H, const double* C,
                                     const double* vs_n, const double* ud_n, double t_final, long long* id) {
    return submit_impl(s, mesh, nullptr, H, C, vs_n, ud_n, t_final, id);
}

extern "C" mp_status mp_serve_submit_quads(mp_server* s, const mp_mesh_desc* mesh, const double* xy, const double* H,
                                           const double* C, const double* vs_n, const double* ud_n, double t_final,
                                           long long* id) {
    if (!xy) { mp::set_error("null vertex array"); return MP_ERR_ARG_WRONG; }
    return submit_impl(s, mesh, xy, H, C, vs_n, ud_n, t_final, id);
}

extern "C" mp_status mp_serve_wait(mp_server* s, long long id, double timeout_s, double* H, double* C, double* T,
                                   double* phi, mp_request_info* info) {
    if (!s) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    std::shared_ptr<Request> r;
    {
        std::unique_lock<std::mutex> lk(s->m);
        auto it = s->requests.find(id);
        if (it == s->requests.end()) { mp::set_error("unknown request %lld", id); return MP_ERR_ARG_OUTOFRANGE; }
        r = it->second;
        const auto pred = [&] { return r->done || s->stop; };
        if (timeout_s < 0) s->cv_done.wait(lk, pred);
        else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) {
            mp::set_error("request %lld not finished within %.3f s", id, timeout_s);
            return MP_ERR_TIMEOUT;
        }
        if (!r->done) { mp::set_error("server stopped: %s", s->fatal_msg.c_str()); return s->fatal ? s->fatal : MP_ERR_ARG_WRONGSTATE; }
        s->requests.erase(it);
    }
    const size_t n = r->cells;
    if (!r->oH.empty()) {
        if (H) std::copy(r->oH.begin(), r->oH.end(), H);
        if (C) std::copy(r->oC.begin(), r->oC.end(), C);
        if (T) std::copy(r->oT.begin(), r->oT.end(), T);
        if (phi) std::copy(r->oP.begin(), r->oP.end(), phi);
    }
    (void)n;
    if (info) {
        info->status = r->status;
        info->accepted = r->accepted;
        info->time = r->time;
        info->queue_s = seconds(r->submitted, r->admitted);
        info->latency_s = seconds(r->submitted, r->finished);
        info->cells = (double)r->cells;
    }
    return MP_OK;
}

extern "C" mp_status mp_serve_set_policy(mp_server* s, int order, double resident_cells_target) {
    if (!s) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    if (order != MP_SERVE_FIFO && order != MP_SERVE_SMALLEST_WORK) { mp::set_error("unknown admission order %d", order); return MP_ERR_ARG_OUTOFRANGE; }
    if (!(resident_cells_target >= 0)) { mp::set_error("resident target must be >= 0"); return MP_ERR_ARG_OUTOFRANGE; }
    {
        std::lock_guard<std::mutex> g(s->m);
        s->order = order;
        s->resident_target = resident_cells_target;
    }
    s->cv_work.notify_all();
    return MP_OK;
}

extern "C" mp_status mp_serve_stats(mp_server* s, double* cell_updates, double* busy_s, long long* steps,
                                    int* resident, int* queued) {
    if (!s) { mp::set_error("null argument"); return MP_ERR_ARG_WRONG; }
    std::lock_guard<std::mutex> g(s->m);
    if (cell_updates) *cell_updates = s->cell_updates;
    if (busy_s) *busy_s = s->busy_s;
    if (steps) *steps = s->steps;
    if (resident) *resident = (int)s->active.size();
    if (queued) *queued = (int)s->queue.size();
    return MP_OK;
}
