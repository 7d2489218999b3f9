// Serving: a request loop over device-resident pools (the "serving" section of
// include/gnn_coloring.h).  The reference has no counterpart; its runner colors one graph per
// process (src/runner.c:105-153).  The coloring arithmetic is the plain path's, unchanged: a job's
// colors are those of its graph colored alone by gc_priority + gc_color.
//
// Structure
//   lanes     W worker threads, each owning one context (its own stream), one batch slot (a
//             gc_batch with fixed capacity, allocated at start) and pinned staging buffers.  All
//             lanes run concurrently on the device, so work of different lanes overlaps.
//   pool      every device allocation of the lanes is stream-ordered from one memory pool
//             (cudaMallocFromPoolAsync), so a job's allocations never synchronise the device and
//             stall the other lanes' kernels.
//   admission the slots are charged to the HBM budget once, at start.  A job too large for a slot
//             (or with a heuristic batches do not offer) runs alone on the plain path and is
//             charged gc_batch_device_bytes(1, N, M, h) while it runs; it starts only when that
//             fits in what the budget has left.  Such jobs start in arrival order (one blocked by
//             the budget holds back the later ones, so none starves); small jobs never wait on
//             the budget.  A job that could never fit is refused at submission (GC_ERR_BUDGET).
//             With two or more lanes, at most lanes - 1 of them run such jobs at a time: one lane
//             always stays for small jobs, whose latency would otherwise queue behind seconds of
//             large-graph work.
//   batching  continuous: an idle lane takes the oldest pending job; if it is small, the lane also
//             takes every other pending small job of the same class (heuristic, layers, recolor)
//             that still fits its slot, and colors them all in one gc_batch_color_once pass.  Jobs
//             that arrive while the lanes are busy accumulate and join the next free lane's batch.
//   isolation a batch that fails (a malformed CSR of one job) is re-run job by job on the plain
//             path, so one bad job cannot fail its batch-mates.
//   resident  graphs registered once (gc_serve_register) stay in device memory, charged to the
//             budget until released; jobs on them skip the host-to-device copy: batched ones are
//             gathered into the slot by one kernel, the others wrap the resident CSR.
//   copies    a job's CSR from host memory goes up through two pinned chunks per lane, filled by
//             several host threads while the previous chunk's DMA runs (pageable copies through the
//             driver reach a fraction of the link's bandwidth); colors come back the same way.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "gc_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

double seconds_since(Clock::time_point t0, Clock::time_point t) {
    return std::chrono::duration<double>(t - t0).count();
}

// A CSR registered with the server: device-resident until released.
struct Reg {
    uint64_t id = 0;
    uint32_t N = 0, M = 0;
    uint32_t *dV = nullptr, *dE = nullptr;
    uint64_t bytes = 0;
    uint32_t refs = 0;  // jobs pending or running on it
};

struct Job {
    uint64_t id = 0;
    Reg *reg = nullptr;        // set for jobs on a registered graph (V, E are then unused)
    uint32_t N = 0, M = 0;
    const uint32_t *V = nullptr, *E = nullptr;
    int32_t *color_out = nullptr;
    gc_heuristic h = GC_FF;
    int layers = 0, recolor = 0;
    bool small = false;        // batched in a slot
    uint64_t bytes = 0;        // budget charge when run alone
    Clock::time_point t_submit, t_start, t_done;
    bool done = false;
    gc_status status = GC_OK;
    int colors = 0;
    uint32_t batch_jobs = 0;
    uint32_t lane = 0;
    std::string error;
};

struct Lane {
    uint32_t index = 0;
    gc_ctx *ctx = nullptr;
    gc_batch *slot = nullptr;
    gc_model *models[8] = {};    // by layer count
    uint32_t *h_voff = nullptr, *h_V = nullptr, *h_E = nullptr;
    int32_t *h_color = nullptr, *h_counts = nullptr;
    char *stage[2] = {nullptr, nullptr};  // pinned chunks of the copies of jobs run alone
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
    std::thread thread;
};

constexpr size_t STAGE_BYTES = 32u << 20;  // bytes per pinned chunk
constexpr int COPY_THREADS = 4;            // host threads filling / draining one chunk

}  // namespace

struct gc_server {
    gc_serve_config cfg{};
    int device = 0;
    cudaMemPool_t pool = nullptr;
    std::vector<Lane *> lanes;
    uint64_t slot_bytes = 0;     // charged once per lane
    bool have_model[8] = {};

    std::mutex mu;
    std::condition_variable cv_work;  // lanes wait for work
    std::condition_variable cv_done;  // callers wait for jobs
    std::deque<Job *> pending;
    std::unordered_map<uint64_t, Job *> jobs;  // every job not yet released by gc_serve_wait
    std::unordered_map<uint64_t, Reg *> regs;  // registered graphs
    uint64_t next_reg = 1;
    cudaStream_t reg_stream = nullptr;         // uploads and releases of registered graphs
    uint64_t next_id = 1;
    uint64_t reserved = 0, peak_reserved = 0;
    bool large_blocked = false;  // set during a pick when the oldest large job did not fit
    uint32_t large_running = 0;  // lanes running a job alone
    bool stop = false;
    bool started = false;        // first submission seen (models are fixed from then on)
    uint32_t inflight = 0;       // jobs taken by lanes and not yet complete

    // statistics since the last reset
    std::vector<double> latencies_ms;
    uint64_t st_submitted = 0, st_completed = 0, st_failed = 0, st_rejected = 0, st_edges = 0, st_launches = 0;
    uint64_t st_batched_jobs = 0;
    bool st_have_first = false;
    Clock::time_point st_first_submit, st_last_done;
    std::string last_error;
};

namespace {

// ---- work selection (called with the server lock held) ---------------------------------------------

struct Work {
    std::vector<Job *> jobs;
    bool batch = false;
};

bool same_class(const Job *a, const Job *b) {
    return a->h == b->h && a->layers == b->layers && a->recolor == b->recolor && (a->reg != nullptr) == (b->reg != nullptr);
}

Work pick_work(gc_server *s) {
    Work w;
    const gc_serve_config &c = s->cfg;
    bool large_seen_blocked = false;
    uint64_t nv = 0, ne = 0;
    for (auto it = s->pending.begin(); it != s->pending.end(); ++it) {
        Job *j = *it;
        if (w.jobs.empty()) {
            if (j->small) {
                w.batch = true;
                w.jobs.push_back(j);
                nv = j->N;
                ne = j->M;
                continue;
            }
            if (large_seen_blocked) continue;  // later large jobs wait behind the blocked one
            if (c.lanes > 1 && s->large_running >= c.lanes - 1) continue;  // a lane stays for small jobs
            if (s->reserved + j->bytes <= c.hbm_budget) {
                w.jobs.push_back(j);
                break;
            }
            large_seen_blocked = true;
            continue;
        }
        if (!w.batch) break;
        if (!j->small || !same_class(j, w.jobs[0])) continue;
        if (w.jobs.size() >= c.slot_graphs || nv + j->N > c.slot_vertices || ne + j->M > c.slot_edges) continue;
        w.jobs.push_back(j);
        nv += j->N;
        ne += j->M;
    }
    s->large_blocked = large_seen_blocked;
    if (!w.jobs.empty()) {
        // remove the chosen jobs from the queue, keeping the others' order
        std::deque<Job *> rest;
        size_t k = 0;
        for (Job *j : s->pending) {
            if (k < w.jobs.size() && std::find(w.jobs.begin(), w.jobs.end(), j) != w.jobs.end()) {
                k++;
                continue;
            }
            rest.push_back(j);
        }
        s->pending.swap(rest);
        if (!w.batch) {
            s->reserved += w.jobs[0]->bytes;
            s->peak_reserved = std::max(s->peak_reserved, s->reserved);
            s->large_running++;
        }
    }
    return w;
}

void complete(gc_server *s, Job *j, gc_status st, int colors, uint32_t batch_jobs, const std::string &err) {
    // called with the lock held
    j->status = st;
    j->colors = colors;
    j->batch_jobs = batch_jobs;
    j->error = err;
    j->t_done = Clock::now();
    j->done = true;
    if (j->reg) j->reg->refs--;
    if (st == GC_OK) {
        s->st_completed++;
        s->st_edges += j->M;
        s->latencies_ms.push_back(1e3 * seconds_since(j->t_submit, j->t_done));
        if (batch_jobs > 1) s->st_batched_jobs++;
        if (!s->st_have_first || j->t_done > s->st_last_done) s->st_last_done = j->t_done;
    } else {
        s->st_failed++;
        s->last_error = err;
    }
}

// ---- execution (no lock held) ----------------------------------------------------------------------

gc_model *lane_model(Lane *L, const Job *j) { return j->h == GC_GNN ? L->models[j->layers] : nullptr; }

// memcpy split over COPY_THREADS host threads (large copies only).
void copy_host(void *dst, const void *src, size_t bytes) {
    if (bytes < (4u << 20)) {
        memcpy(dst, src, bytes);
        return;
    }
    const size_t piece = (bytes + COPY_THREADS - 1) / COPY_THREADS;
#pragma omp parallel for num_threads(COPY_THREADS) schedule(static)
    for (int t = 0; t < COPY_THREADS; t++) {
        const size_t a = (size_t)t * piece;
        if (a < bytes) memcpy((char *)dst + a, (const char *)src + a, std::min(piece, bytes - a));
    }
}

// Host memory to device memory through the lane's two pinned chunks: chunk k is filled while the
// DMA of chunk k - 1 runs.
gc_status h2d_staged(Lane *L, void *dst, const void *src, size_t bytes) {
    gc_ctx *ctx = L->ctx;
    gc_status st = GC_OK;
    for (size_t off = 0, k = 0; off < bytes && st == GC_OK; off += STAGE_BYTES, k++) {
        const size_t n = std::min(STAGE_BYTES, bytes - off);
        const int b = (int)(k & 1);
        st = gc_check_cuda(ctx, cudaEventSynchronize(L->stage_ev[b]), "staging");
        if (st != GC_OK) break;
        copy_host(L->stage[b], (const char *)src + off, n);
        st = gc_check_cuda(ctx, cudaMemcpyAsync((char *)dst + off, L->stage[b], n, cudaMemcpyHostToDevice, ctx->stream),
                           "upload");
        if (st == GC_OK) st = gc_check_cuda(ctx, cudaEventRecord(L->stage_ev[b], ctx->stream), "staging");
    }
    return st;
}

// Device memory to host memory the same way: the DMA of chunk k + 1 runs while chunk k is copied out.
gc_status d2h_staged(Lane *L, void *dst, const void *src, size_t bytes) {
    gc_ctx *ctx = L->ctx;
    const size_t chunks = (bytes + STAGE_BYTES - 1) / STAGE_BYTES;
    auto issue = [&](size_t k) -> gc_status {
        const size_t off = k * STAGE_BYTES, n = std::min(STAGE_BYTES, bytes - off);
        const int b = (int)(k & 1);
        gc_status st = gc_check_cuda(ctx, cudaMemcpyAsync(L->stage[b], (const char *)src + off, n,
                                                          cudaMemcpyDeviceToHost, ctx->stream), "download");
        if (st == GC_OK) st = gc_check_cuda(ctx, cudaEventRecord(L->stage_ev[b], ctx->stream), "staging");
        return st;
    };
    gc_status st = chunks ? issue(0) : GC_OK;
    for (size_t k = 0; k < chunks && st == GC_OK; k++) {
        const int b = (int)(k & 1);
        if ((st = gc_check_cuda(ctx, cudaEventSynchronize(L->stage_ev[b]), "staging")) != GC_OK) break;
        if (k + 1 < chunks && (st = issue(k + 1)) != GC_OK) break;
        const size_t off = k * STAGE_BYTES;
        copy_host((char *)dst + off, L->stage[b], std::min(STAGE_BYTES, bytes - off));
    }
    return st;
}

// One job alone on the plain path: its CSR up (or the registered one wrapped), priority,
// coloring, colors back.
gc_status run_alone(Lane *L, Job *j, int *colors, std::string *err) {
    gc_ctx *ctx = L->ctx;
    gc_graph *g = nullptr;
    gc_status st;
    if (j->reg) {
        st = gc_graph_wrap_device(ctx, j->N, j->M, j->reg->dV, j->reg->dE, &g);
    } else {
        st = gc_graph_create(ctx, j->N, j->M, &g);
        if (st == GC_OK) st = h2d_staged(L, g->V, j->V, sizeof(uint32_t) * ((size_t)j->N + 1));
        if (st == GC_OK && j->M) st = h2d_staged(L, g->E, j->E, sizeof(uint32_t) * (size_t)j->M);
        if (st == GC_OK) {
            g->N = j->N;
            g->M = j->M;
            st = gc_graph_finish_upload(g);
        }
    }
    if (st == GC_OK) st = gc_priority(ctx, g, j->h, lane_model(L, j));
    if (st == GC_OK) st = gc_color(ctx, g, j->recolor, colors);
    if (st == GC_OK && j->color_out && j->N) st = d2h_staged(L, j->color_out, g->color, sizeof(int32_t) * (size_t)j->N);
    if (st != GC_OK) *err = gc_last_error(ctx);
    if (g) gc_graph_free(g);
    return st;
}

// Small jobs of one class as one batch: their CSRs into the lane's slot (staged through pinned
// memory, or gathered on the device for registered graphs), color, and scatter the colors back to
// each job's buffer.
gc_status run_batch(Lane *L, const std::vector<Job *> &jobs, std::string *err) {
    gc_ctx *ctx = L->ctx;
    const uint32_t G = (uint32_t)jobs.size();
    uint32_t nv = 0, ne = 0;
    L->h_voff[0] = 0;
    gc_status st;
    if (jobs[0]->reg) {
        std::vector<uint32_t> n(G), m(G);
        std::vector<const uint32_t *> dV(G), dE(G);
        for (uint32_t i = 0; i < G; i++) {
            const Reg *r = jobs[i]->reg;
            n[i] = r->N;
            m[i] = r->M;
            dV[i] = r->dV;
            dE[i] = r->dE;
            nv += r->N;
            L->h_voff[i + 1] = nv;
        }
        st = gc_batch_reupload_device_graphs(ctx, L->slot, G, n.data(), m.data(), dV.data(), dE.data());
    } else {
        L->h_V[0] = 0;
        for (uint32_t i = 0; i < G; i++) {
            const Job *j = jobs[i];
            for (uint32_t u = 0; u < j->N; u++) L->h_V[nv + u + 1] = ne + j->V[u + 1];
            if (j->M) memcpy(L->h_E + ne, j->E, sizeof(uint32_t) * j->M);
            nv += j->N;
            ne += j->M;
            L->h_voff[i + 1] = nv;
        }
        st = gc_batch_reupload(ctx, L->slot, G, L->h_voff, L->h_V, L->h_E);
    }
    const Job *j0 = jobs[0];
    if (st == GC_OK) st = gc_batch_color_once(ctx, L->slot, j0->h, lane_model(L, j0), j0->recolor, L->h_counts);
    bool any_out = false;
    for (const Job *j : jobs) any_out |= j->color_out != nullptr;
    if (st == GC_OK && any_out && nv) st = gc_batch_download_colors(ctx, L->slot, L->h_color);
    if (st != GC_OK) {
        *err = gc_last_error(ctx);
        return st;
    }
    for (uint32_t i = 0; i < G; i++) {
        Job *j = jobs[i];
        if (j->color_out && j->N) memcpy(j->color_out, L->h_color + L->h_voff[i], sizeof(int32_t) * j->N);
    }
    return GC_OK;
}

void lane_loop(gc_server *s, Lane *L) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        Work w;
        s->cv_work.wait(lk, [&] {
            if (s->stop) return true;
            if (s->pending.empty()) return false;
            w = pick_work(s);
            return !w.jobs.empty();
        });
        if (w.jobs.empty() && s->stop) return;
        const auto t_start = Clock::now();
        for (Job *j : w.jobs) {
            j->t_start = t_start;
            j->lane = L->index;
        }
        s->inflight += (uint32_t)w.jobs.size();
        s->st_launches++;
        if (!s->pending.empty()) s->cv_work.notify_one();  // another idle lane may take the rest
        lk.unlock();

        std::vector<gc_status> status(w.jobs.size(), GC_OK);
        std::vector<int> colors(w.jobs.size(), 0);
        std::vector<std::string> errors(w.jobs.size());
        if (w.batch) {
            std::string err;
            gc_status st = run_batch(L, w.jobs, &err);
            if (st == GC_OK) {
                for (size_t i = 0; i < w.jobs.size(); i++) colors[i] = L->h_counts[i];
            } else if (w.jobs.size() == 1) {
                status[0] = st;
                errors[0] = err;
            } else {
                // isolate the failing job: each one alone on the plain path
                for (size_t i = 0; i < w.jobs.size(); i++) status[i] = run_alone(L, w.jobs[i], &colors[i], &errors[i]);
            }
        } else {
            status[0] = run_alone(L, w.jobs[0], &colors[0], &errors[0]);
        }

        lk.lock();
        const uint32_t n = (uint32_t)w.jobs.size();
        for (size_t i = 0; i < w.jobs.size(); i++) complete(s, w.jobs[i], status[i], colors[i], n, errors[i]);
        if (!w.batch) {
            s->reserved -= w.jobs[0]->bytes;
            s->large_running--;
        }
        s->inflight -= n;
        s->cv_done.notify_all();
        s->cv_work.notify_all();  // budget freed, or more work may be pending
    }
}

gc_status fail(gc_server *s, gc_status st, const std::string &msg) {
    if (s) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->last_error = msg;
    }
    return st;
}

void destroy_lane(Lane *L) {
    if (L->slot) gc_batch_free(L->slot);
    for (gc_model *m : L->models)
        if (m) gc_model_free(m);
    if (L->h_voff) cudaFreeHost(L->h_voff);
    if (L->h_V) cudaFreeHost(L->h_V);
    if (L->h_E) cudaFreeHost(L->h_E);
    if (L->h_color) cudaFreeHost(L->h_color);
    if (L->h_counts) cudaFreeHost(L->h_counts);
    for (int b = 0; b < 2; b++) {
        if (L->stage[b]) cudaFreeHost(L->stage[b]);
        if (L->stage_ev[b]) cudaEventDestroy(L->stage_ev[b]);
    }
    if (L->ctx) gc_ctx_destroy(L->ctx);
    delete L;
}

gc_status submit_locked(gc_server *s, Reg *reg, uint32_t N, const uint32_t *V, const uint32_t *E, gc_heuristic h,
                        int layers, int recolor, int32_t *color_out, Clock::time_point now, uint64_t *job_id) {
    // argument checks that need no lock are done by the caller
    const gc_serve_config &c = s->cfg;
    Job *j = new Job();
    j->id = s->next_id++;
    j->reg = reg;
    j->N = reg ? reg->N : N;
    j->M = reg ? reg->M : V[N];
    N = j->N;
    j->V = V;
    j->E = E;
    j->color_out = color_out;
    j->h = h;
    j->layers = h == GC_GNN ? layers : 0;
    j->recolor = recolor;
    const bool batchable = h == GC_FF || h == GC_LF || h == GC_LLF || h == GC_GNN;
    j->small = batchable && N <= c.batch_max_job_vertices && j->M <= c.slot_edges && N <= c.slot_vertices;
    j->bytes = gc_batch_device_bytes(1, N, j->M, h);
    j->t_submit = now;
    if (!j->small && s->slot_bytes * s->lanes.size() + j->bytes > c.hbm_budget) {
        s->st_rejected++;
        s->last_error = "job needs " + std::to_string(j->bytes) + " device bytes; the budget leaves " +
                        std::to_string(c.hbm_budget - std::min<uint64_t>(c.hbm_budget, s->slot_bytes * s->lanes.size()));
        delete j;
        return GC_ERR_BUDGET;
    }
    if (!s->st_have_first) {
        s->st_have_first = true;
        s->st_first_submit = now;
    }
    s->started = true;
    s->st_submitted++;
    s->jobs[j->id] = j;
    s->pending.push_back(j);
    if (reg) reg->refs++;
    *job_id = j->id;
    return GC_OK;
}

gc_status check_kind(gc_server *s, gc_heuristic h, int layers, int recolor) {
    if (recolor < 0) return fail(s, GC_ERR_INVALID, "recolor must be >= 0");
    if ((int)h < GC_FF || (int)h > GC_GNN) return fail(s, GC_ERR_INVALID, "unknown heuristic");
    if (h == GC_GNN && (layers < 2 || layers > 7 || !s->have_model[layers]))
        return fail(s, GC_ERR_INVALID, "no GNN model with " + std::to_string(layers) + " layers was added");
    return GC_OK;
}

gc_status check_job(gc_server *s, uint32_t N, const uint32_t *V, const uint32_t *E, gc_heuristic h, int layers,
                    int recolor) {
    if (!V) return fail(s, GC_ERR_INVALID, "V is NULL");
    if (V[0] != 0) return fail(s, GC_ERR_INVALID, "V[0] must be 0");
    if (V[N] && !E) return fail(s, GC_ERR_INVALID, "E is NULL");
    if (N >= 0xffffffffu) return fail(s, GC_ERR_INVALID, "too many vertices");
    return check_kind(s, h, layers, recolor);
}

// Host-side check of a CSR to register: rows monotone and ending at M, ids below N.
bool csr_valid(uint32_t N, const uint32_t *V, const uint32_t *E) {
    if (V[0] != 0) return false;
    bool ok = true;
#pragma omp parallel for reduction(&& : ok) schedule(static)
    for (int64_t u = 0; u < (int64_t)N; u++) ok = ok && V[u] <= V[u + 1];
    if (!ok) return false;
    const int64_t M = V[N];
#pragma omp parallel for reduction(&& : ok) schedule(static)
    for (int64_t i = 0; i < M; i++) ok = ok && E[i] < N;
    return ok;
}

void free_reg(gc_server *s, Reg *r) {
    if (r->dV) cudaFreeAsync(r->dV, s->reg_stream);
    if (r->dE) cudaFreeAsync(r->dE, s->reg_stream);
    cudaStreamSynchronize(s->reg_stream);
    delete r;
}

void fill_info(const Job *j, gc_job_info *info) {
    if (!info) return;
    info->status = j->status;
    info->colors = j->colors;
    info->N = j->N;
    info->M = j->M;
    info->batch_jobs = j->batch_jobs;
    info->lane = j->lane;
    info->queue_ms = 1e3 * seconds_since(j->t_submit, j->t_start);
    info->run_ms = 1e3 * seconds_since(j->t_start, j->t_done);
    info->latency_ms = 1e3 * seconds_since(j->t_submit, j->t_done);
}

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    // nearest rank
    size_t k = (size_t)std::ceil(q * (double)v.size());
    if (k < 1) k = 1;
    if (k > v.size()) k = v.size();
    return v[k - 1];
}

}  // namespace

extern "C" {

void gc_serve_config_default(gc_serve_config *c) {
    if (!c) return;
    c->device = 0;
    c->lanes = 4;
    c->hbm_budget = 0;
    c->slot_graphs = 4096;
    c->slot_vertices = 1u << 22;
    c->slot_edges = 1u << 26;
    c->batch_max_job_vertices = 1u << 17;
}

gc_status gc_serve_create(const gc_serve_config *cfg_in, gc_server **out) {
    if (!out) return GC_ERR_INVALID;
    *out = nullptr;
    gc_serve_config cfg;
    gc_serve_config_default(&cfg);
    if (cfg_in) cfg = *cfg_in;
    if (cfg.lanes < 1 || cfg.lanes > 64 || cfg.slot_graphs < 1 || cfg.slot_vertices < 1 || cfg.slot_edges < 1)
        return GC_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return GC_ERR_NODEV;
    }
    if (cfg.device < 0 || cfg.device >= ndev) return GC_ERR_INVALID;
    if (cudaSetDevice(cfg.device) != cudaSuccess) return GC_ERR_CUDA;
    if (cfg.hbm_budget == 0) {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return GC_ERR_CUDA;
        cfg.hbm_budget = (uint64_t)(0.8 * (double)free_b);
    }
    gc_server *s = new gc_server();
    s->cfg = cfg;
    s->device = cfg.device;
    s->slot_bytes = gc_batch_device_bytes(cfg.slot_graphs, cfg.slot_vertices, cfg.slot_edges, GC_GNN);
    if (s->slot_bytes * cfg.lanes > cfg.hbm_budget) {
        delete s;
        return GC_ERR_BUDGET;
    }
    // one stream-ordered pool for every lane; freed memory is kept for reuse up to the budget, and
    // no lane's allocation waits on another lane's stream
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = cfg.device;
    gc_status st = GC_OK;
    if (cudaMemPoolCreate(&s->pool, &props) != cudaSuccess) {
        cudaGetLastError();
        delete s;
        return GC_ERR_CUDA;
    }
    uint64_t keep = cfg.hbm_budget;
    int no = 0;
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolReuseAllowInternalDependencies, &no);
    for (uint32_t i = 0; i < cfg.lanes && st == GC_OK; i++) {
        Lane *L = new Lane();
        L->index = i;
        s->lanes.push_back(L);
        if ((st = gc_ctx_create(cfg.device, &L->ctx)) != GC_OK) break;
        L->ctx->pool = s->pool;
        if ((st = gc_batch_create(L->ctx, cfg.slot_graphs, cfg.slot_vertices, cfg.slot_edges, &L->slot)) != GC_OK)
            break;
        const size_t bytes[] = {4ull * (cfg.slot_graphs + 1), 4ull * ((size_t)cfg.slot_vertices + 1),
                                4ull * (size_t)cfg.slot_edges, 4ull * (size_t)cfg.slot_vertices, 4ull * cfg.slot_graphs};
        void **bufs[] = {(void **)&L->h_voff, (void **)&L->h_V, (void **)&L->h_E, (void **)&L->h_color,
                         (void **)&L->h_counts};
        for (int k = 0; k < 5 && st == GC_OK; k++)
            if (cudaMallocHost(bufs[k], bytes[k]) != cudaSuccess) {
                cudaGetLastError();
                st = GC_ERR_NOMEM;
            }
        for (int b = 0; b < 2 && st == GC_OK; b++) {
            if (cudaMallocHost((void **)&L->stage[b], STAGE_BYTES) != cudaSuccess ||
                cudaEventCreateWithFlags(&L->stage_ev[b], cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                st = GC_ERR_NOMEM;
            }
        }
        if (st == GC_OK && cudaStreamSynchronize(L->ctx->stream) != cudaSuccess) st = GC_ERR_CUDA;
    }
    if (st == GC_OK && cudaStreamCreateWithFlags(&s->reg_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        st = GC_ERR_CUDA;
    }
    if (st != GC_OK) {
        for (Lane *L : s->lanes) destroy_lane(L);
        if (s->reg_stream) cudaStreamDestroy(s->reg_stream);
        cudaMemPoolDestroy(s->pool);
        delete s;
        return st;
    }
    s->reserved = s->slot_bytes * cfg.lanes;
    s->peak_reserved = s->reserved;
    for (Lane *L : s->lanes) L->thread = std::thread(lane_loop, s, L);
    *out = s;
    return GC_OK;
}

gc_status gc_serve_add_model(gc_server *s, int params, int md, const float *param) {
    if (!s || !param || params < 2 * 528 || params % 528) return GC_ERR_INVALID;
    const int layers = params / 528;
    if (layers > 7) return fail(s, GC_ERR_INVALID, "at most 7 layers");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->started) {
            s->last_error = "models must be added before the first submission";
            return GC_ERR_STATE;
        }
    }
    for (Lane *L : s->lanes) {
        gc_model *m = nullptr;
        gc_status st = gc_model_create(L->ctx, params, md, param, &m);
        if (st != GC_OK) return fail(s, st, gc_last_error(L->ctx));
        if (L->models[layers]) gc_model_free(L->models[layers]);
        L->models[layers] = m;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->have_model[layers] = true;
    return GC_OK;
}

gc_status gc_serve_submit(gc_server *s, uint32_t N, const uint32_t *V, const uint32_t *E, gc_heuristic h, int layers,
                          int recolor, int32_t *color_out, uint64_t *job) {
    if (!s || !job) return GC_ERR_INVALID;
    *job = 0;
    gc_status st = check_job(s, N, V, E, h, layers, recolor);
    if (st != GC_OK) return st;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return GC_ERR_STATE;
    st = submit_locked(s, nullptr, N, V, E, h, layers, recolor, color_out, Clock::now(), job);
    if (st == GC_OK) s->cv_work.notify_one();
    return st;
}

gc_status gc_serve_register(gc_server *s, uint32_t N, const uint32_t *V, const uint32_t *E, uint64_t *graph) {
    if (!s || !graph || !V) return GC_ERR_INVALID;
    *graph = 0;
    if (N >= 0xffffffffu) return fail(s, GC_ERR_INVALID, "too many vertices");
    const uint32_t M = V[N];
    if (M && !E) return fail(s, GC_ERR_INVALID, "E is NULL");
    if (!csr_valid(N, V, E)) return fail(s, GC_ERR_INVALID, "malformed CSR: rows not monotone or an id out of range");
    const uint64_t bytes = 4ull * ((uint64_t)N + 1) + 4ull * M;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->reserved + bytes > s->cfg.hbm_budget) {
            s->st_rejected++;
            s->last_error = "registering needs " + std::to_string(bytes) + " device bytes beyond the budget";
            return GC_ERR_BUDGET;
        }
        s->reserved += bytes;  // held while the copy runs
        s->peak_reserved = std::max(s->peak_reserved, s->reserved);
    }
    cudaSetDevice(s->device);
    Reg *r = new Reg();
    r->N = N;
    r->M = M;
    r->bytes = bytes;
    cudaError_t e = cudaMallocFromPoolAsync((void **)&r->dV, 4ull * ((size_t)N + 1), s->pool, s->reg_stream);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync((void **)&r->dE, 4ull * (M ? M : 1), s->pool, s->reg_stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(r->dV, V, 4ull * ((size_t)N + 1), cudaMemcpyHostToDevice, s->reg_stream);
    if (e == cudaSuccess && M) e = cudaMemcpyAsync(r->dE, E, 4ull * M, cudaMemcpyHostToDevice, s->reg_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->reg_stream);
    std::lock_guard<std::mutex> lk(s->mu);
    if (e != cudaSuccess) {
        cudaGetLastError();
        s->reserved -= bytes;
        s->last_error = std::string("register: ") + cudaGetErrorString(e);
        free_reg(s, r);
        return e == cudaErrorMemoryAllocation ? GC_ERR_NOMEM : GC_ERR_CUDA;
    }
    r->id = s->next_reg++;
    s->regs[r->id] = r;
    *graph = r->id;
    return GC_OK;
}

gc_status gc_serve_unregister(gc_server *s, uint64_t graph) {
    if (!s) return GC_ERR_INVALID;
    Reg *r = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->regs.find(graph);
        if (it == s->regs.end()) return GC_ERR_INVALID;
        if (it->second->refs) {
            s->last_error = "graph still has jobs pending or running";
            return GC_ERR_STATE;
        }
        r = it->second;
        s->regs.erase(it);
        s->reserved -= r->bytes;
    }
    cudaSetDevice(s->device);
    free_reg(s, r);
    return GC_OK;
}

gc_status gc_serve_submit_registered(gc_server *s, uint64_t graph, gc_heuristic h, int layers, int recolor,
                                     int32_t *color_out, uint64_t *job) {
    if (!s || !job) return GC_ERR_INVALID;
    *job = 0;
    gc_status st = check_kind(s, h, layers, recolor);
    if (st != GC_OK) return st;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return GC_ERR_STATE;
    auto it = s->regs.find(graph);
    if (it == s->regs.end()) {
        s->last_error = "unknown registered graph";
        return GC_ERR_INVALID;
    }
    st = submit_locked(s, it->second, 0, nullptr, nullptr, h, layers, recolor, color_out, Clock::now(), job);
    if (st == GC_OK) s->cv_work.notify_one();
    return st;
}

gc_status gc_serve_replay_registered(gc_server *s, uint32_t J, const double *arrive_s, const uint64_t *graph,
                                     const int *h, const int *layers, const int *recolor, int32_t *const *color_out,
                                     gc_job_info *info) {
    if (!s || (J && (!arrive_s || !graph || !h))) return GC_ERR_INVALID;
    std::vector<Reg *> regs(J, nullptr);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (uint32_t i = 0; i < J; i++) {
            auto it = s->regs.find(graph[i]);
            if (it == s->regs.end()) {
                s->last_error = "unknown registered graph";
                return GC_ERR_INVALID;
            }
            regs[i] = it->second;
        }
    }
    for (uint32_t i = 0; i < J; i++) {
        gc_status st = check_kind(s, (gc_heuristic)h[i], layers ? layers[i] : 0, recolor ? recolor[i] : 0);
        if (st != GC_OK) return st;
        if (i && arrive_s[i] < arrive_s[i - 1]) return fail(s, GC_ERR_INVALID, "arrival times must not decrease");
    }
    std::vector<uint64_t> ids(J, 0);
    std::vector<gc_status> sub(J, GC_OK);
    const auto t0 = Clock::now();
    for (uint32_t i = 0; i < J; i++) {
        const auto due = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrive_s[i]));
        for (;;) {
            const auto now = Clock::now();
            if (now >= due) break;
            const auto left = due - now;
            if (left > std::chrono::microseconds(200)) std::this_thread::sleep_for(left - std::chrono::microseconds(150));
        }
        std::lock_guard<std::mutex> lk(s->mu);
        if (!s->regs.count(graph[i])) {
            sub[i] = GC_ERR_INVALID;  // released meanwhile by another thread
            continue;
        }
        sub[i] = submit_locked(s, regs[i], 0, nullptr, nullptr, (gc_heuristic)h[i], layers ? layers[i] : 0,
                               recolor ? recolor[i] : 0, color_out ? color_out[i] : nullptr, due, &ids[i]);
        if (sub[i] == GC_OK) s->cv_work.notify_one();
    }
    gc_status worst = GC_OK;
    for (uint32_t i = 0; i < J; i++) {
        gc_status st = sub[i];
        if (st == GC_OK) st = gc_serve_wait(s, ids[i], info ? info + i : nullptr);
        else if (info) {
            memset(info + i, 0, sizeof(gc_job_info));
            info[i].status = st;
        }
        if (st != GC_OK && worst == GC_OK) worst = st;
    }
    return worst;
}

gc_status gc_serve_test(gc_server *s, uint64_t job, int *done) {
    if (!s || !done) return GC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job);
    if (it == s->jobs.end()) return GC_ERR_INVALID;
    *done = it->second->done ? 1 : 0;
    return GC_OK;
}

gc_status gc_serve_wait(gc_server *s, uint64_t job, gc_job_info *info) {
    if (!s) return GC_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job);
    if (it == s->jobs.end()) return GC_ERR_INVALID;
    Job *j = it->second;
    s->cv_done.wait(lk, [&] { return j->done; });
    fill_info(j, info);
    const gc_status st = j->status;
    if (st != GC_OK) s->last_error = j->error;
    s->jobs.erase(it);
    delete j;
    return st;
}

gc_status gc_serve_drain(gc_server *s) {
    if (!s) return GC_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait(lk, [&] { return s->pending.empty() && s->inflight == 0; });
    return GC_OK;
}

gc_status gc_serve_replay(gc_server *s, uint32_t J, const double *arrive_s, const uint32_t *N,
                          const uint32_t *const *V, const uint32_t *const *E, const int *h, const int *layers,
                          const int *recolor, int32_t *const *color_out, gc_job_info *info) {
    if (!s || (J && (!arrive_s || !N || !V || !E || !h))) return GC_ERR_INVALID;
    for (uint32_t i = 0; i < J; i++) {
        gc_status st = check_job(s, N[i], V[i], E[i], (gc_heuristic)h[i], layers ? layers[i] : 0,
                                 recolor ? recolor[i] : 0);
        if (st != GC_OK) return st;
        if (i && arrive_s[i] < arrive_s[i - 1]) return fail(s, GC_ERR_INVALID, "arrival times must not decrease");
    }
    std::vector<uint64_t> ids(J, 0);
    std::vector<gc_status> sub(J, GC_OK);
    const auto t0 = Clock::now();
    for (uint32_t i = 0; i < J; i++) {
        const auto due = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrive_s[i]));
        // sleep until shortly before the arrival, then spin (sleep granularity is ~50-100 us)
        for (;;) {
            const auto now = Clock::now();
            if (now >= due) break;
            const auto left = due - now;
            if (left > std::chrono::microseconds(200)) std::this_thread::sleep_for(left - std::chrono::microseconds(150));
        }
        std::lock_guard<std::mutex> lk(s->mu);
        sub[i] = submit_locked(s, nullptr, N[i], V[i], E[i], (gc_heuristic)h[i], layers ? layers[i] : 0,
                               recolor ? recolor[i] : 0, color_out ? color_out[i] : nullptr, due, &ids[i]);
        if (sub[i] == GC_OK) s->cv_work.notify_one();
    }
    gc_status worst = GC_OK;
    for (uint32_t i = 0; i < J; i++) {
        gc_status st = sub[i];
        if (st == GC_OK) st = gc_serve_wait(s, ids[i], info ? info + i : nullptr);
        else if (info) {
            memset(info + i, 0, sizeof(gc_job_info));
            info[i].status = st;
            info[i].N = N[i];
            info[i].M = V[i][N[i]];
        }
        if (st != GC_OK && worst == GC_OK) worst = st;
    }
    return worst;
}

gc_status gc_serve_read_stats(gc_server *s, gc_serve_stats *out) {
    if (!s || !out) return GC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    memset(out, 0, sizeof *out);
    out->submitted = s->st_submitted;
    out->completed = s->st_completed;
    out->failed = s->st_failed;
    out->rejected = s->st_rejected;
    out->edges = s->st_edges;
    out->launches = s->st_launches;
    out->batched_jobs = s->st_batched_jobs;
    out->p50_ms = percentile(s->latencies_ms, 0.50);
    out->p99_ms = percentile(s->latencies_ms, 0.99);
    double sum = 0, mx = 0;
    for (double v : s->latencies_ms) {
        sum += v;
        mx = std::max(mx, v);
    }
    out->mean_ms = s->latencies_ms.empty() ? 0.0 : sum / (double)s->latencies_ms.size();
    out->max_ms = mx;
    out->span_s = s->st_have_first && s->st_completed ? seconds_since(s->st_first_submit, s->st_last_done) : 0.0;
    out->edges_per_s = out->span_s > 0 ? (double)s->st_edges / out->span_s : 0.0;
    out->budget_bytes = s->cfg.hbm_budget;
    out->reserved_bytes = s->reserved;
    out->peak_reserved_bytes = s->peak_reserved;
    uint64_t used = 0;
    if (s->pool) cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrUsedMemHigh, &used);
    out->pool_peak_bytes = used;
    out->lanes = (uint32_t)s->lanes.size();
    return GC_OK;
}

void gc_serve_reset_stats(gc_server *s) {
    if (!s) return;
    std::lock_guard<std::mutex> lk(s->mu);
    s->latencies_ms.clear();
    s->st_submitted = s->st_completed = s->st_failed = s->st_rejected = s->st_edges = s->st_launches = 0;
    s->st_batched_jobs = 0;
    s->st_have_first = false;
    s->peak_reserved = s->reserved;
    uint64_t zero = 0;
    if (s->pool) cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrUsedMemHigh, &zero);
}

const char *gc_serve_last_error(gc_server *s) {
    if (!s) return "no server";
    std::lock_guard<std::mutex> lk(s->mu);
    thread_local std::string copy;
    copy = s->last_error;
    return copy.c_str();
}

void gc_serve_destroy(gc_server *s) {
    if (!s) return;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_done.wait(lk, [&] { return s->pending.empty() && s->inflight == 0; });
        s->stop = true;
        s->cv_work.notify_all();
    }
    for (Lane *L : s->lanes)
        if (L->thread.joinable()) L->thread.join();
    cudaSetDevice(s->device);
    for (Lane *L : s->lanes) destroy_lane(L);
    for (auto &kv : s->jobs) delete kv.second;
    for (auto &kv : s->regs) free_reg(s, kv.second);
    if (s->reg_stream) cudaStreamDestroy(s->reg_stream);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
}

}  // extern "C"
