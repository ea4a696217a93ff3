// qoa_server.cpp — the serving form: a request loop over the engine's C ABI.
//
// A request is one circuit (reference opcodes) with a depolarising noise level
// p, a number of Pauli trajectories and a number of shots per trajectory.
// Trajectory t of a request seeded s is fully determined by (s, t): its noise
// draws come from the counter-based generator on stream t (the engine's
// QuantumState::apply_noise restatement, quantum_state.rs:839-885), its shot
// uniforms from stream t ^ kShotStream. A result therefore does not depend on
// which worker ran it, on the other requests in flight or on their timing.
//
// Scheduling (continuous batching):
//  - requests queue in arrival order;
//  - a worker takes the next unit of work of the oldest admitted request, so
//    the work of several requests overlaps on the device. A unit is
//      * a chunk of trajectories run as one batch (qoa_batch_add_trajectory:
//        every trajectory a batch circuit, its shots sampled on the device),
//        for requests of unitary ops on up to kBatchMaxQubits qubits — a
//        chunk is one launch per pass round for all of its trajectories
//        instead of one launch per pass and trajectory; a noiseless request's
//        trajectories are one circuit, sampled with all of their uniforms;
//      * otherwise one trajectory on a pooled state handle of the worker's
//        size (its own stream), reused by later trajectories of that size;
//  - a unit starts when its memory (a state, or a chunk's states) fits in the
//    HBM budget beside the running ones (idle pooled states of other sizes are
//    freed to make room).
// Every finished request holds its outcomes until qoa_server_take_shots.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/qoa_cuda.h"

namespace qoa {
void note_global_error(const char* msg);
}

namespace {

constexpr uint32_t kShotStream = 0x73686f74u;  // "shot"
// Trajectory chunks: requests of up to this many qubits, chunks of up to
// kChunkBytes of states (and the budget) each.
constexpr uint32_t kBatchMaxQubits = 22;
constexpr size_t kChunkBytes = size_t(2) << 30;

struct Request {
    uint64_t id = 0;
    uint32_t n = 0;
    int precision = QOA_PREC_F64;
    std::vector<qoa_op> ops;
    std::vector<uint32_t> qlists;   // owned copies of every op's qubit list
    std::vector<double> matrices;   // and matrices
    double noise_p = 0.0;
    uint32_t trajectories = 1, shots = 1;
    uint64_t seed = 0;
    uint32_t next_traj = 0, started = 0, done_traj = 0;
    bool batched = false;   // trajectories run in chunks of `chunk` as batches
    uint32_t chunk = 1;
    int status = QOA_OK;
    std::string err;
    double t_submit = 0, t_admit = -1, t_start = -1, t_done = -1;
    std::vector<uint64_t> out;      // trajectories x shots outcomes
};

struct Slot {
    qoa_state_t h = nullptr;
    uint32_t n = 0;
    int precision = 0;
    size_t bytes = 0;
    bool busy = false;
    uint64_t last_use = 0;
};

size_t footprint(uint32_t n, int precision) {
    // state + sampling tree (FP64 per amplitude) + reduction scratch
    const size_t amps = (size_t)1 << n;
    const size_t esz = precision == QOA_PREC_F32 ? 8 : 16;
    return amps * (esz + 8) + ((size_t)1 << 20);
}

}  // namespace

struct qoa_server_s {
    qoa_server_config cfg{};
    int device = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    std::deque<Request*> queue;                        // not yet admitted
    std::list<Request*> admitted;                      // admission order
    std::map<uint64_t, std::unique_ptr<Request>> all;  // until the shots are taken
    std::deque<uint64_t> completed;                    // not yet polled
    std::list<Slot> slots;
    size_t bytes_reserved = 0, peak_bytes = 0;
    size_t chunk_bytes = 0;                            // reserved by running chunks
    uint64_t traj_batched = 0;
    uint64_t next_id = 1, use_clock = 0;
    uint64_t n_submitted = 0, n_done = 0, traj_running = 0;
    std::vector<std::thread> workers;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    // Effective precision of a request: the tensor-core block form needs
    // n >= 11 qubits; smaller requests then run in complex128.
    int prec_for(uint32_t n) const {
        if (cfg.precision != QOA_PREC_F32) return QOA_PREC_F64;
        return ((cfg.flags & QOA_FLAG_F32_TENSOR) && n < 11) ? QOA_PREC_F64 : QOA_PREC_F32;
    }

    size_t busy_bytes() const {
        size_t b = chunk_bytes;
        for (const Slot& s : slots)
            if (s.busy) b += s.bytes;
        return b;
    }

    // Memory a request's next unit needs.
    size_t unit_bytes(const Request* q) const {
        const size_t fp = footprint(q->n, q->precision);
        if (!q->batched) return fp;
        const uint32_t k = std::min(q->chunk, q->trajectories - q->next_traj);
        return q->noise_p > 0.0 ? fp * k : fp;  // a noiseless chunk is one circuit
    }

    // Under the lock: reserves `need` bytes for a chunk, freeing idle pooled
    // states (least recently used first); false when the budget does not
    // allow it now.
    bool acquire_bytes(size_t need, std::vector<qoa_state_t>& to_free) {
        while (bytes_reserved + need > cfg.hbm_budget_bytes) {
            auto victim = slots.end();
            for (auto it = slots.begin(); it != slots.end(); ++it)
                if (!it->busy && (victim == slots.end() || it->last_use < victim->last_use)) victim = it;
            if (victim == slots.end()) return false;
            if (victim->h) to_free.push_back(victim->h);
            bytes_reserved -= victim->bytes;
            slots.erase(victim);
        }
        bytes_reserved += need;
        chunk_bytes += need;
        peak_bytes = std::max(peak_bytes, bytes_reserved);
        return true;
    }

    // Under the lock: an idle state of (n, precision), or room for a new one
    // (freeing idle states of other sizes, least recently used first).
    // Returns the slot, or nullptr when the budget does not allow it now.
    Slot* acquire(uint32_t n, int prec, std::vector<qoa_state_t>& to_free) {
        for (Slot& s : slots)
            if (!s.busy && s.n == n && s.precision == prec) {
                s.busy = true;
                return &s;
            }
        const size_t need = footprint(n, prec);
        while (bytes_reserved + need > cfg.hbm_budget_bytes) {
            auto victim = slots.end();
            for (auto it = slots.begin(); it != slots.end(); ++it)
                if (!it->busy && (victim == slots.end() || it->last_use < victim->last_use)) victim = it;
            if (victim == slots.end()) return nullptr;
            if (victim->h) to_free.push_back(victim->h);
            bytes_reserved -= victim->bytes;
            slots.erase(victim);
        }
        bytes_reserved += need;
        peak_bytes = std::max(peak_bytes, bytes_reserved);
        slots.push_back(Slot{nullptr, n, prec, need, true, 0});
        return &slots.back();
    }

    // A unit of work: trajectories [t, t + count) of request r, on a pooled
    // state (slot) or, for a chunk, as a batch holding `bytes`.
    struct Unit {
        Request* r = nullptr;
        uint32_t t = 0, count = 1;
        Slot* slot = nullptr;
        size_t bytes = 0;
    };

    // Under the lock: the next unit to run.
    bool next_work(Unit& u, std::vector<qoa_state_t>& to_free) {
        for (;;) {
            for (Request* q : admitted) {
                if (q->next_traj >= q->trajectories) continue;
                if (q->batched) {
                    const size_t need = unit_bytes(q);
                    if (!acquire_bytes(need, to_free)) continue;
                    u.r = q;
                    u.t = q->next_traj;
                    u.count = std::min(q->chunk, q->trajectories - q->next_traj);
                    u.slot = nullptr;
                    u.bytes = need;
                    q->next_traj += u.count;
                    q->started += u.count;
                } else {
                    Slot* s = acquire(q->n, q->precision, to_free);
                    if (!s) continue;
                    u.r = q;
                    u.t = q->next_traj++;
                    u.count = 1;
                    u.slot = s;
                    u.bytes = 0;
                    q->started++;
                }
                if (q->t_start < 0) q->t_start = now();
                return true;
            }
            // nothing runnable among the admitted: admit the next arrival
            if (queue.empty()) return false;
            Request* q = queue.front();
            const size_t need = unit_bytes(q);
            if (need > cfg.hbm_budget_bytes) {
                queue.pop_front();
                q->status = QOA_E_OOM;
                q->err = "request state does not fit the HBM budget";
                q->t_admit = q->t_start = q->t_done = now();
                completed.push_back(q->id);
                n_done++;
                cv_done.notify_all();
                continue;
            }
            if (busy_bytes() + need > cfg.hbm_budget_bytes) return false;  // wait for memory
            queue.pop_front();
            q->t_admit = now();
            admitted.push_back(q);
        }
    }

    void finish_unit(const Unit& u, int rc, const std::string& msg) {
        Request* r = u.r;
        if (u.slot) {
            u.slot->busy = false;
            u.slot->last_use = ++use_clock;
        } else {
            bytes_reserved -= u.bytes;
            chunk_bytes -= u.bytes;
            traj_batched += u.count;
        }
        traj_running -= u.count;
        if (rc != QOA_OK && r->status == QOA_OK) {
            r->status = rc;
            r->err = msg;
            r->next_traj = r->trajectories;  // start none of its other trajectories
        }
        r->done_traj += u.count;
        if (r->next_traj >= r->trajectories && r->done_traj == r->started) {
            r->t_done = now();
            admitted.remove(r);
            completed.push_back(r->id);
            n_done++;
            cv_done.notify_all();
        }
    }

    int run_traj(Request* r, uint32_t t, Slot* slot) {
        int rc;
        if (!slot->h) {
            const uint32_t fl = slot->precision == QOA_PREC_F32 ? cfg.flags : (cfg.flags & ~QOA_FLAG_F32_TENSOR);
            rc = qoa_create(r->n, slot->precision, fl, &slot->h);
            if (rc) {
                slot->h = nullptr;
                return rc;
            }
        }
        qoa_state_t h = slot->h;
        if ((rc = qoa_seed(h, r->seed))) return rc;
        if ((rc = qoa_set_noise(h, r->noise_p > 0.0 ? 1 : 0, r->noise_p))) return rc;
        if ((rc = qoa_set_trajectory(h, t))) return rc;
        if ((rc = qoa_reset_all(h))) return rc;
        // out-of-range qubits are skipped ops, as in the reference: not fatal
        rc = qoa_apply(h, r->ops.data(), r->ops.size());
        if (rc && rc != QOA_E_RANGE) return rc;
        std::vector<double> u(r->shots);
        for (uint32_t k = 0; k < r->shots; ++k) u[k] = qoa_philox_uniform(r->seed, t ^ kShotStream, k, 0);
        return qoa_sample(h, u.data(), r->shots, 1, r->out.data() + (size_t)t * r->shots);
    }

    // Trajectories [t0, t0 + count) of r as one batch of worker-owned
    // handle b (reset after the run); their shots go to r->out.
    int run_chunk(Request* r, uint32_t t0, uint32_t count, qoa_batch_t b, std::string& msg) {
        int rc = QOA_OK;
        std::vector<double> u;
        auto fail = [&](int code) {
            const char* m = qoa_batch_last_error(b);
            msg = m ? m : "";
            qoa_batch_reset(b);
            return code;
        };
        // a noiseless request's trajectories share one final state: one
        // circuit, sampled with every trajectory's uniforms in order
        const bool one = !(r->noise_p > 0.0);
        const uint32_t ncirc = one ? 1 : count;
        const uint32_t per = one ? count * r->shots : r->shots;
        std::vector<uint32_t> ids(ncirc);
        for (uint32_t c = 0; c < ncirc; ++c) {
            u.resize(per);
            for (uint32_t k = 0; k < per; ++k) {
                const uint32_t t = one ? t0 + k / r->shots : t0 + c;
                const uint32_t shot = one ? k % r->shots : k;
                u[k] = qoa_philox_uniform(r->seed, t ^ kShotStream, shot, 0);
            }
            rc = qoa_batch_add_trajectory(b, r->n, r->ops.data(), r->ops.size(), r->seed, r->noise_p, t0 + c,
                                          u.data(), per, &ids[c]);
            if (rc && rc != QOA_E_RANGE) return fail(rc);  // out-of-range ops are skipped, as in the reference
        }
        if ((rc = qoa_batch_run(b))) return fail(rc);
        for (uint32_t c = 0; c < ncirc; ++c)
            if ((rc = qoa_batch_shots(b, ids[c], r->out.data() + (size_t)(t0 + c) * r->shots, per))) return fail(rc);
        qoa_batch_reset(b);
        return QOA_OK;
    }

    void worker() {
        cudaSetDevice(device);
        qoa_batch_t batches[2] = {nullptr, nullptr};  // this worker's chunk batches, by precision
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            Unit u;
            std::vector<qoa_state_t> to_free;
            while (!stop && !next_work(u, to_free)) {
                for (qoa_state_t h : to_free) qoa_destroy(h);
                to_free.clear();
                cv_work.wait(lk);
            }
            if (!u.r) break;  // stopping
            traj_running += u.count;
            lk.unlock();
            for (qoa_state_t h : to_free) qoa_destroy(h);
            int rc;
            std::string msg;
            if (u.slot) {
                rc = run_traj(u.r, u.t, u.slot);
                if (rc) {
                    const char* m = qoa_last_error(u.slot->h);
                    msg = m ? m : "";
                }
            } else {
                const int pi = u.r->precision == QOA_PREC_F32 ? 1 : 0;
                rc = QOA_OK;
                if (!batches[pi]) {
                    rc = qoa_batch_create(u.r->precision, cfg.flags & ~QOA_FLAG_F32_TENSOR, &batches[pi]);
                    if (!rc) {
                        qoa_batch_tuning tu;
                        qoa_batch_get_tuning(batches[pi], &tu);
                        tu.streams = 1;           // a chunk's circuits are one size: arena or small route
                        tu.jit = QOA_JIT_OFF;     // noisy trajectories rarely share a pass structure
                        qoa_batch_set_tuning(batches[pi], &tu);
                        qoa_batch_set_host_threads(batches[pi], 1);  // the workers are the parallelism
                    } else {
                        batches[pi] = nullptr;
                        const char* m = qoa_last_error(nullptr);
                        msg = m ? m : "";
                    }
                }
                if (!rc) rc = run_chunk(u.r, u.t, u.count, batches[pi], msg);
            }
            lk.lock();
            finish_unit(u, rc, msg);
            cv_work.notify_all();
        }
        lk.unlock();
        for (qoa_batch_t b : batches)
            if (b) qoa_batch_destroy(b);
    }
};

extern "C" {

double qoa_server_now(qoa_server_t s) { return s ? s->now() : 0.0; }

int qoa_server_create(const qoa_server_config* cfg, qoa_server_t* out) {
    if (!cfg || !out) {
        qoa::note_global_error("qoa_server_create: null argument");
        return QOA_E_ARG;
    }
    *out = nullptr;
    if ((cfg->precision != QOA_PREC_F64 && cfg->precision != QOA_PREC_F32) || cfg->workers < 1 ||
        cfg->workers > 256 || cfg->hbm_budget_bytes == 0) {
        qoa::note_global_error("qoa_server_create: bad configuration");
        return QOA_E_ARG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        qoa::note_global_error("qoa_server_create: no CUDA device");
        return QOA_E_NOGPU;
    }
    qoa_server_t s = new qoa_server_s();
    s->cfg = *cfg;
    cudaGetDevice(&s->device);
    for (uint32_t i = 0; i < cfg->workers; ++i) s->workers.emplace_back([s] { s->worker(); });
    *out = s;
    return QOA_OK;
}

int qoa_server_submit(qoa_server_t s, const qoa_request* req, uint64_t* id) {
    if (!s || !req || (!req->ops && req->nops)) {
        qoa::note_global_error("qoa_server_submit: null argument");
        return QOA_E_ARG;
    }
    if (req->n < 1 || req->n > 40 || req->trajectories < 1 || req->shots_per_trajectory < 1 ||
        !(req->noise_p >= 0.0 && req->noise_p <= 1.0)) {
        qoa::note_global_error("qoa_server_submit: bad request");
        return QOA_E_ARG;
    }
    auto r = std::make_unique<Request>();
    r->n = req->n;
    r->precision = s->prec_for(req->n);
    r->noise_p = req->noise_p;
    r->trajectories = req->trajectories;
    r->shots = req->shots_per_trajectory;
    r->seed = req->seed;
    r->ops.assign(req->ops, req->ops + req->nops);
    // deep copies of qubit lists and matrices (2x2 -> 8 doubles, 4x4 -> 32)
    size_t nq = 0, nm = 0;
    for (const qoa_op& o : r->ops) {
        if (o.qlist) nq += o.nq;
        if (o.matrix) nm += o.opcode == QOA_OP_U2 ? 32 : 8;
    }
    r->qlists.resize(nq);
    r->matrices.resize(nm);
    nq = nm = 0;
    for (qoa_op& o : r->ops) {
        if (o.qlist) {
            std::memcpy(r->qlists.data() + nq, o.qlist, o.nq * sizeof(uint32_t));
            o.qlist = r->qlists.data() + nq;
            nq += o.nq;
        }
        if (o.matrix) {
            const size_t k = o.opcode == QOA_OP_U2 ? 32 : 8;
            std::memcpy(r->matrices.data() + nm, o.matrix, k * sizeof(double));
            o.matrix = r->matrices.data() + nm;
            nm += k;
        }
    }
    r->out.assign((size_t)r->trajectories * r->shots, 0);
    // trajectory chunks for unitary requests of up to kBatchMaxQubits qubits
    // (the tensor-core block form keeps its per-state path); the chunk size
    // depends on the request and the configuration only, so a result does not
    // depend on the other requests
    int unitary = 0;
    const bool tensor = r->precision == QOA_PREC_F32 && (s->cfg.flags & QOA_FLAG_F32_TENSOR);
    if (r->n <= kBatchMaxQubits && !tensor &&
        qoa_ops_unitary(r->n, s->cfg.flags, r->ops.data(), r->ops.size(), &unitary) == QOA_OK && unitary) {
        const size_t fp = footprint(r->n, r->precision);
        const size_t cap = std::min(kChunkBytes, (size_t)s->cfg.hbm_budget_bytes);
        r->batched = true;
        r->chunk = (uint32_t)std::max<size_t>(1, std::min<size_t>(r->trajectories, cap / fp));
    }
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    r->t_submit = s->now();
    if (id) *id = r->id;
    s->queue.push_back(r.get());
    s->all[r->id] = std::move(r);
    s->n_submitted++;
    s->cv_work.notify_one();
    return QOA_OK;
}

int qoa_server_poll(qoa_server_t s, qoa_request_result* out, size_t cap, size_t* got, int timeout_ms) {
    if (!s || !got || (!out && cap)) {
        qoa::note_global_error("qoa_server_poll: null argument");
        return QOA_E_ARG;
    }
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->completed.empty() && timeout_ms != 0) {
        auto pred = [s] { return !s->completed.empty(); };
        if (timeout_ms < 0) s->cv_done.wait(lk, pred);
        else s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred);
    }
    size_t k = 0;
    while (k < cap && !s->completed.empty()) {
        const uint64_t id = s->completed.front();
        s->completed.pop_front();
        const Request* r = s->all[id].get();
        qoa_request_result& o = out[k++];
        o.id = id;
        o.status = r->status;
        o.n = r->n;
        o.precision = r->precision;
        o.t_submit = r->t_submit;
        o.t_admit = r->t_admit;
        o.t_start = r->t_start;
        o.t_done = r->t_done;
        o.shots = r->out.size();
    }
    *got = k;
    return QOA_OK;
}

int qoa_server_take_shots(qoa_server_t s, uint64_t id, uint64_t* out, size_t cap) {
    if (!s || (!out && cap)) {
        qoa::note_global_error("qoa_server_take_shots: null argument");
        return QOA_E_ARG;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end() || it->second->t_done < 0) {
        qoa::note_global_error("qoa_server_take_shots: no finished request with that id");
        return QOA_E_ARG;
    }
    Request* r = it->second.get();
    if (cap != r->out.size()) {
        qoa::note_global_error("qoa_server_take_shots: cap must equal trajectories x shots");
        return QOA_E_ARG;
    }
    if (cap) std::memcpy(out, r->out.data(), cap * sizeof(uint64_t));
    const int st = r->status;
    if (st != QOA_OK) qoa::note_global_error(r->err.c_str());
    s->all.erase(it);
    return st;
}

int qoa_server_get_stats(qoa_server_t s, qoa_server_stats* out) {
    if (!s || !out) {
        qoa::note_global_error("qoa_server_get_stats: null argument");
        return QOA_E_ARG;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    out->submitted = s->n_submitted;
    out->done = s->n_done;
    out->queued = s->queue.size();
    out->admitted = s->admitted.size();
    out->trajectories_running = s->traj_running;
    out->states_resident = s->slots.size();
    out->bytes_reserved = s->bytes_reserved;
    out->peak_bytes_reserved = s->peak_bytes;
    out->trajectories_batched = s->traj_batched;
    return QOA_OK;
}

int qoa_server_destroy(qoa_server_t s) {
    if (!s) return QOA_OK;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        // drain: wait for everything submitted to finish
        s->cv_done.wait(lk, [s] { return s->n_done == s->n_submitted; });
        s->stop = true;
        s->cv_work.notify_all();
    }
    for (std::thread& t : s->workers) t.join();
    for (Slot& sl : s->slots)
        if (sl.h) qoa_destroy(sl.h);
    delete s;
    return QOA_OK;
}

}  // extern "C"
