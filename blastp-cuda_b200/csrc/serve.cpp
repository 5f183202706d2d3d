// Serving loop: continuous batching of arriving queries against one resident
// database.
//
// The reference answers one blastp call at a time (gpu_blastp.cu:16-259); a
// server keeps the database on the device and takes queries as they come:
//  * submit() queues a request (any thread);
//  * a dispatcher thread admits queued requests in arrival order while the
//    device-memory budget allows (the request's neighbour table, its
//    per-subject outputs and its share of the HSP record buffer), builds
//    their tables and launches them as one batched persistent search on a
//    lane -- each lane's launch takes 1/lanes of the SMs, so a batch that
//    starts while another lane's is running overlaps it on the device (with
//    one lane, a batch of one request runs as the plain single-query search
//    instead, which takes every SM);
//  * a lane holds up to lane_depth batches, each in a slot with its own
//    engine (stream and scratch): the slot's stream waits for the lane's
//    previous batch (an event), so a lane runs its batches back to back in
//    admission order while the host builds the next batch's tables and
//    launches it behind them -- a request admitted while its lane is busy
//    waits for the batches ahead of it, not for a batch boundary;
//  * finished batches are noticed by polling their streams; results stay on
//    the device, in the batch's per-query segments, until the request is
//    released, which is when its memory returns to the budget;
//  * with `segments` > 1, a request is admitted on its own and searched as
//    that many jobs over consecutive subject ranges; each free slot takes the
//    next range of the request the admission policy picks (the oldest, or the
//    one with the least work left), so a short request arriving while a long
//    one runs waits for one range of it, not for all of it.  Its result stays
//    in pieces, one per range, and is read back (or digested) piece by piece.
// Every query's result is its single-query result (the batched kernel scans
// each (query, subject) pair exactly as the plain kernel does).
#include <string.h>

#include <algorithm>
#include <cmath>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "bp_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

double now_ms() {
    return std::chrono::duration<double, std::milli>(Clock::now().time_since_epoch()).count();
}

struct Job;

struct Req {
    uint64_t id = 0;
    std::vector<uint8_t> residues;
    double t_arrive = 0, t_start = 0, t_done = 0;
    int state = BP_REQ_QUEUED;
    bp_status status = BP_OK;
    int64_t bytes = 0;
    bp_query* query = nullptr;
    Job* job = nullptr;
    int index = -1;
    bool released = false;
    // segment mode: one job per subject range, launched in range order
    std::vector<Job*> segs;
    int seg_next = 0, seg_done = 0;
};

struct Job {
    int lane = 0;
    int slot = 0;             // lane * lane_depth + position
    bp_batch* batch = nullptr;
    std::vector<Req*> reqs;
    int live = 0;             // requests not yet released
    int64_t bytes = 0;
    bool done = false;
    int seg = -1;             // segment mode: the subject range searched
    bp_result* result = nullptr;   // a one-request job runs as the plain search instead of a batch
};

}  // namespace

struct bp_server {
    bp_engine* e = nullptr;
    const bp_db* db = nullptr;
    bp_server_options o{};
    int n_lanes = 0, depth = 1;
    std::vector<bp_engine*> slots;        // lane l's slots are l * depth .. l * depth + depth - 1
    std::vector<Job*> slot_job;
    std::vector<cudaEvent_t> lane_tail;   // recorded after the lane's latest batch
    std::vector<bool> lane_used;          // lane_tail has been recorded
    std::thread th;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req*> pending;
    std::vector<int32_t> seg_first;       // segment mode: range k is subjects [seg_first[k], seg_first[k + 1])
    std::vector<Req*> active;             // segment mode: admitted requests with ranges left to launch
    cudaStream_t readback = nullptr;      // digests of finished requests (with e's scratch)
    std::mutex readback_mu;
    std::unordered_map<uint64_t, Req*> reqs;
    uint64_t next_id = 1;
    int64_t mem_used = 0, mem_peak = 0;
    bool stop = false;
    // statistics
    std::vector<double> latency_ms;
    int64_t n_done = 0, n_failed = 0, n_batches = 0, batched_queries = 0;
    double t_first = -1, t_last = 0, resq = 0;
    int max_in_flight = 0, in_flight = 0;
};

namespace {

// Device bytes a request holds while admitted: its table (cell starts +
// entries, estimated from the query length), its per-subject outputs
// (counters, CSR offsets, fill cursor) and its expected HSP records.
int64_t request_bytes(const bp_server* s, int32_t qlen) {
    const int64_t n = s->db->n;
    const int64_t table = (BP_NC + 1) * 4 + (int64_t)qlen * 40 + 4096;
    const int64_t outputs = n * (12 + 8 + 4) + 8;
    const int64_t records = (int64_t)(3e-4 * 1.5 * (double)qlen / 500.0 * (double)s->db->nres) * 60;
    return table + outputs + records;
}

// A job's search is a batch of its requests or, for a single request, the
// plain search (the single-query scan kernel, no item schedule: 7-8 % faster
// than a batch of one on the serving database).
bp_status job_wait(Job* j) { return j->result ? bp_result_wait(j->result) : bp_batch_wait(j->batch); }

// A finished job's result for request `index`; synchronous copies on the
// legacy stream, which do not wait for what the slot's stream runs now.
bp_status job_copy(Job* j, int index, int32_t* counters, int64_t* hsp_off, bp_hsp* hsps, int64_t* n_hsps) {
    if (!j->result) return bp_batch_copy_query(j->batch, index, counters, hsp_off, hsps, n_hsps);
    bp_result* r = j->result;
    const bp_status st = bp_result_wait(r);
    if (st != BP_OK) return st;
    cudaError_t err = cudaSetDevice(r->e->device);
    if (n_hsps) *n_hsps = r->n_hsps;
    if (err == cudaSuccess && counters && r->n > 0)
        err = cudaMemcpy(counters, r->d_counters, (size_t)r->n * 3 * sizeof(int32_t), cudaMemcpyDeviceToHost);
    if (err == cudaSuccess && hsp_off)
        err = cudaMemcpy(hsp_off, r->d_hsp_off, ((size_t)r->n + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost);
    if (err == cudaSuccess && hsps && r->n_hsps > 0)
        err = cudaMemcpy(hsps, r->d_hsps, (size_t)r->n_hsps * sizeof(bp_hsp), cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return bp_set_cuda_error(r->e, err, "server result copy");
    return BP_OK;
}

// A finished job's digest sums for request `index`, as one piece of a
// result (bp_digest_sums), on the server's read-back stream.
bp_status job_digest_sums(bp_server* s, Job* j, int index, int64_t first, int64_t rec_base, bool last,
                          uint64_t sums[2]) {
    if (!j->result) return bp_batch_digest_sums(j->batch, index, s->e, s->readback, first, rec_base, last, sums);
    bp_result* r = j->result;
    const bp_status st = bp_result_wait(r);
    if (st != BP_OK) return st;
    return bp_digest_sums(s->e, s->readback, r->d_counters, r->n, r->d_hsp_off, r->d_hsps, first, rec_base, last,
                          sums);
}

// Frees a finished job's search, stream-ordered (the slot's stream may
// already run another job).
void job_free(Job* j) {
    bp_batch_destroy_finished(j->batch);
    j->batch = nullptr;
    if (j->result) bp_result_destroy(j->result);
    j->result = nullptr;
}

void fail_request(bp_server* s, Req* r, bp_status st) {
    r->state = BP_REQ_FAILED;
    r->status = st;
    r->t_done = now_ms();
    s->n_failed += 1;
}

// Builds tables and launches one batch on `lane` (called without the lock;
// the requests are already marked admitted and owned by the dispatcher).
void launch_job(bp_server* s, Job* job) {
    bp_engine* le = s->slots[job->slot];
    std::vector<const bp_query*> qs;
    bp_status st = BP_OK;
    for (Req* r : job->reqs) {
        st = bp_query_create(le, r->residues.data(), (int32_t)r->residues.size(), &s->o.params, &r->query);
        if (st != BP_OK) break;
        qs.push_back(r->query);
    }
    bp_batch_options bo;
    bp_batch_options_default(&bo);
    bo.chunk_residues = s->o.chunk_residues > 0 ? s->o.chunk_residues : (1 << 20);
    bo.schedule = s->o.schedule;
    bo.use_graph = 0;
    bo.ctas = std::max(1, le->sm_count / std::max(1, s->n_lanes));
    bo.plain_unpacked = s->n_lanes == 1 ? 1 : 0;   // (a plain scan takes every SM)
    std::vector<float> costs;
    if (st == BP_OK && bo.schedule == BP_SCHED_COSTS && !(qs.size() == 1 && s->n_lanes == 1)) {
        if (!s->o.model) {
            bo.schedule = BP_SCHED_STATIC;   // no model: the static schedule
        } else {
            int32_t nc = 0;
            st = bp_batch_plan(s->db, 0, -1, bo.chunk_residues, nullptr, &nc);
            std::vector<int32_t> first((size_t)nc + 1);
            if (st == BP_OK) st = bp_batch_plan(s->db, 0, -1, bo.chunk_residues, first.data(), &nc);
            costs.resize((size_t)qs.size() * nc);
            if (st == BP_OK)
                st = bp_batch_predict_costs(le, s->o.model, s->o.cost_weights, s->db, qs.data(), (int32_t)qs.size(),
                                            first.data(), nc, s->o.planted_density, costs.data());
            bo.item_costs = costs.data();
        }
    }
    // behind the lane's previous job on the device, then this one becomes the lane's tail
    const bool plain = qs.size() == 1 && s->n_lanes == 1;   // (a plain search takes every SM)
    if (st == BP_OK && plain) {
        if (s->lane_used[job->lane] && cudaStreamWaitEvent(le->stream, s->lane_tail[job->lane], 0) != cudaSuccess) {
            cudaGetLastError();
            st = BP_ERR_CUDA;
        }
        if (st == BP_OK) st = bp_search(le, s->db, qs[0], 0, -1, &job->result);
    } else if (st == BP_OK) {
        st = bp_search_batch_behind(le, s->db, qs.data(), (int32_t)qs.size(), &bo,
                                    s->lane_used[job->lane] ? s->lane_tail[job->lane] : nullptr, &job->batch);
    }
    if (st == BP_OK) {
        if (cudaEventRecord(s->lane_tail[job->lane], le->stream) == cudaSuccess) {
            s->lane_used[job->lane] = true;
        } else {
            cudaGetLastError();
            st = BP_ERR_CUDA;
        }
    }
    std::lock_guard<std::mutex> lock(s->mu);
    const double t = now_ms();
    for (size_t i = 0; i < job->reqs.size(); ++i) {
        Req* r = job->reqs[i];
        r->index = (int)i;
        if (st == BP_OK) {
            r->state = BP_REQ_RUNNING;
            r->t_start = t;
        } else {
            fail_request(s, r, st);
        }
    }
    if (st != BP_OK) {
        job->done = true;
        s->cv_done.notify_all();
    }
}

// The queued request to admit next, or pending.end() when none may go now
// (`extra`: bytes already taken by the batch being formed).  Arrival order:
// the oldest, when it fits the budget.  Shortest first: the shortest, when it
// fits together with every request queued before it -- so memory stays for
// the older requests it overtakes, and a client that waits for its requests
// in submission order (holding the results of later ones) cannot stall the
// server -- else the oldest.  A lone request on an idle server always goes.
std::deque<Req*>::iterator pick_pending(bp_server* s, int64_t extra) {
    auto oldest = s->pending.begin();
    if (oldest == s->pending.end()) return oldest;
    const int64_t room = s->o.device_memory_budget - s->mem_used - extra;
    const bool overdue = s->o.max_wait_ms > 0 && now_ms() - (*oldest)->t_arrive >= s->o.max_wait_ms;
    if (s->o.admission == BP_ADMIT_SHORTEST && !overdue) {
        auto best = oldest;
        for (auto it = s->pending.begin(); it != s->pending.end(); ++it)
            if ((*it)->residues.size() < (*best)->residues.size()) best = it;
        if (best != oldest) {
            int64_t need = (*best)->bytes;
            for (auto it = oldest; it != best; ++it) need += (*it)->bytes;
            if (need <= room) return best;
        }
    }
    if ((*oldest)->bytes <= room || (extra == 0 && s->mem_used == 0)) return oldest;
    return s->pending.end();
}

// Segment mode: builds the request's table with its first range, then
// launches one range of it on the job's slot (called without the lock).
void launch_seg_job(bp_server* s, Job* job) {
    bp_engine* le = s->slots[job->slot];
    Req* r = job->reqs[0];
    bp_status st = BP_OK;
    if (!r->query) st = bp_query_create(le, r->residues.data(), (int32_t)r->residues.size(), &s->o.params, &r->query);
    // the plain search over the range, behind the lane's previous job
    if (st == BP_OK && s->lane_used[job->lane] &&
        cudaStreamWaitEvent(le->stream, s->lane_tail[job->lane], 0) != cudaSuccess) {
        cudaGetLastError();
        st = BP_ERR_CUDA;
    }
    if (st == BP_OK)
        st = bp_search(le, s->db, r->query, s->seg_first[job->seg],
                       s->seg_first[job->seg + 1] - s->seg_first[job->seg], &job->result);
    if (st == BP_OK) {
        if (cudaEventRecord(s->lane_tail[job->lane], le->stream) == cudaSuccess) {
            s->lane_used[job->lane] = true;
        } else {
            cudaGetLastError();
            st = BP_ERR_CUDA;
        }
    }
    std::lock_guard<std::mutex> lock(s->mu);
    r->index = 0;
    if (st == BP_OK) {
        if (r->state == BP_REQ_ADMITTED) {
            r->state = BP_REQ_RUNNING;
            r->t_start = now_ms();
        }
        return;
    }
    job->done = true;
    if (r->state == BP_REQ_ADMITTED || r->state == BP_REQ_RUNNING) {
        fail_request(s, r, st);
        s->in_flight -= 1;
        s->active.erase(std::remove(s->active.begin(), s->active.end(), r), s->active.end());
    }
    s->cv_done.notify_all();
}

// Segment mode: every launched range of the request has finished.
bool segs_finished(const Req* r) {
    for (const Job* j : r->segs)
        if (!j->done) return false;
    return true;
}

// Segment mode: frees a released request whose launched ranges have all finished.
void retire_segmented(bp_server* s, Req* r) {
    for (Job* j : r->segs) {
        job_free(j);
        delete j;
    }
    r->segs.clear();
    bp_query_destroy(r->query);
    r->query = nullptr;
    s->mem_used -= r->bytes;
    s->reqs.erase(r->id);
    delete r;
}

// Segment mode: the request whose next range a free slot takes -- the
// earliest admitted, or (past max_wait_ms, the oldest waiting so long, else)
// the one with the least work left (ranges left x
// query length plus the per-letter-independent share of a scan, about 64
// letters' worth), earliest among equals.
Req* next_segment_request(bp_server* s) {
    if (s->active.empty()) return nullptr;
    const int n_seg = (int)s->seg_first.size() - 1;
    Req* best = s->active.front();
    if (s->o.admission != BP_ADMIT_SHORTEST) return best;
    if (s->o.max_wait_ms > 0) {
        // a request waiting past the limit goes first, the oldest of them
        Req* oldest = best;
        for (Req* r : s->active)
            if (r->t_arrive < oldest->t_arrive) oldest = r;
        if (now_ms() - oldest->t_arrive >= s->o.max_wait_ms) return oldest;
    }
    auto left = [n_seg](const Req* r) { return (double)(n_seg - r->seg_next) * ((double)r->residues.size() + 64.0); };
    for (Req* r : s->active)
        if (left(r) < left(best)) best = r;
    return best;
}

// Frees a job whose requests have all been released.
void retire_job(bp_server* s, Job* job) {
    job_free(job);
    for (Req* r : job->reqs) {
        bp_query_destroy(r->query);
        r->query = nullptr;
        s->reqs.erase(r->id);
        delete r;
    }
    s->mem_used -= job->bytes;
    delete job;
}

// Segment mode: a slot still holds one of the request's jobs.
bool seg_on_slot(const bp_server* s, const Req* r) {
    for (const Job* j : r->segs)
        if (std::find(s->slot_job.begin(), s->slot_job.end(), j) != s->slot_job.end()) return true;
    return false;
}

// Segment mode: one dispatcher round -- finished ranges, admissions (every
// queued request that fits the budget), and a range for every free slot.
bool dispatch_segments(bp_server* s, std::unique_lock<std::mutex>& lock) {
    bool worked = false;
    const int n_seg = (int)s->seg_first.size() - 1;
    for (size_t l = 0; l < s->slots.size(); ++l) {
        Job* job = s->slot_job[l];
        if (!job) continue;
        Req* r = job->reqs[0];
        if (!job->done) {
            if (cudaStreamQuery(s->slots[l]->stream) == cudaErrorNotReady) continue;
            cudaGetLastError();
            lock.unlock();
            const bp_status st = job_wait(job);   // re-runs on record overflow
            lock.lock();
            job->done = true;
            if (r->state == BP_REQ_RUNNING || r->state == BP_REQ_ADMITTED) {
                if (st != BP_OK) {
                    fail_request(s, r, st);
                    s->in_flight -= 1;
                    s->active.erase(std::remove(s->active.begin(), s->active.end(), r), s->active.end());
                } else if (++r->seg_done == n_seg) {
                    const double t = now_ms();
                    r->state = BP_REQ_DONE;
                    r->t_done = t;
                    s->latency_ms.push_back(r->t_done - r->t_arrive);
                    s->n_done += 1;
                    s->resq += (double)r->residues.size() * (double)s->db->nres;
                    s->t_last = std::max(s->t_last, t);
                    s->in_flight -= 1;
                }
            }
            s->cv_done.notify_all();
            worked = true;
        }
        s->slot_job[l] = nullptr;
        if (r->released && segs_finished(r) && !seg_on_slot(s, r)) retire_segmented(s, r);
    }
    while (!s->pending.empty()) {
        auto pick = pick_pending(s, 0);
        if (pick == s->pending.end()) break;
        Req* r = *pick;
        s->pending.erase(pick);
        r->state = BP_REQ_ADMITTED;
        s->mem_used += r->bytes;
        s->mem_peak = std::max(s->mem_peak, s->mem_used);
        s->in_flight += 1;
        s->max_in_flight = std::max(s->max_in_flight, s->in_flight);
        s->active.push_back(r);
        worked = true;
    }
    for (int pass = 0; pass < s->depth && !s->active.empty(); ++pass)
        for (size_t l = 0; l < (size_t)s->n_lanes && !s->active.empty(); ++l) {
            int slot = -1;
            for (int k = 0; k < s->depth && slot < 0; ++k)
                if (!s->slot_job[l * s->depth + k]) slot = (int)l * s->depth + k;
            if (slot < 0) continue;
            Req* r = next_segment_request(s);
            Job* job = new Job();
            job->lane = (int)l;
            job->slot = slot;
            job->reqs.push_back(r);
            job->live = 1;
            job->seg = r->seg_next++;
            r->segs.push_back(job);
            if (r->seg_next == n_seg) s->active.erase(std::find(s->active.begin(), s->active.end(), r));
            s->slot_job[slot] = job;
            s->n_batches += 1;
            s->batched_queries += 1;
            lock.unlock();
            launch_seg_job(s, job);
            lock.lock();
            if (job->done) {                 // failed to launch
                s->slot_job[slot] = nullptr;
                if (r->released && segs_finished(r) && !seg_on_slot(s, r)) retire_segmented(s, r);
            }
            worked = true;
        }
    return worked;
}

void dispatcher(bp_server* s) {
    std::unique_lock<std::mutex> lock(s->mu);
    while (!s->stop) {
        if (s->seg_first.size() > 2) {
            if (!dispatch_segments(s, lock))
                s->cv_work.wait_for(lock, std::chrono::microseconds(s->o.poll_us > 0 ? s->o.poll_us : 200));
            continue;
        }
        bool worked = false;
        // completions (a slot's stream holds its own batch only)
        for (size_t l = 0; l < s->slots.size(); ++l) {
            Job* job = s->slot_job[l];
            if (!job) continue;
            if (!job->done) {
                if (cudaStreamQuery(s->slots[l]->stream) == cudaErrorNotReady) continue;
                cudaGetLastError();
                lock.unlock();
                const bp_status st = job_wait(job);   // re-runs on record overflow
                lock.lock();
                const double t = now_ms();
                for (Req* r : job->reqs) {
                    if (r->state != BP_REQ_RUNNING) continue;
                    if (st != BP_OK) {
                        fail_request(s, r, st);
                        continue;
                    }
                    r->state = BP_REQ_DONE;
                    r->t_done = t;
                    s->latency_ms.push_back(r->t_done - r->t_arrive);
                    s->n_done += 1;
                    s->resq += (double)r->residues.size() * (double)s->db->nres;
                    s->t_last = std::max(s->t_last, t);
                }
                s->in_flight -= (int)job->reqs.size();
                job->done = true;
                s->cv_done.notify_all();
                worked = true;
            }
            s->slot_job[l] = nullptr;   // the slot is free; the job lives until released
            if (job->live == 0) retire_job(s, job);
        }
        // admissions: one batch per free slot, lanes in turn, in arrival order, within budget
        for (int pass = 0; pass < s->depth && !s->pending.empty(); ++pass)
        for (size_t l = 0; l < (size_t)s->n_lanes && !s->pending.empty(); ++l) {
            int slot = -1;
            for (int k = 0; k < s->depth && slot < 0; ++k)
                if (!s->slot_job[l * s->depth + k]) slot = (int)l * s->depth + k;
            if (slot < 0) continue;
            Job* job = new Job();
            job->lane = (int)l;
            job->slot = slot;
            while (!s->pending.empty() && (int)job->reqs.size() < s->o.max_batch_queries) {
                auto pick = pick_pending(s, job->bytes);
                if (pick == s->pending.end()) break;   // wait for memory
                Req* r = *pick;
                s->pending.erase(pick);
                r->state = BP_REQ_ADMITTED;
                r->job = job;
                job->reqs.push_back(r);
                job->bytes += r->bytes;
            }
            if (job->reqs.empty()) {
                delete job;
                break;
            }
            job->live = (int)job->reqs.size();
            s->mem_used += job->bytes;
            s->mem_peak = std::max(s->mem_peak, s->mem_used);
            s->slot_job[slot] = job;
            s->n_batches += 1;
            s->batched_queries += (int64_t)job->reqs.size();
            s->in_flight += (int)job->reqs.size();
            s->max_in_flight = std::max(s->max_in_flight, s->in_flight);
            lock.unlock();
            launch_job(s, job);
            lock.lock();
            if (job->done) {                 // failed to launch
                s->in_flight -= (int)job->reqs.size();
                s->slot_job[slot] = nullptr;
            }
            worked = true;
        }
        if (!worked) s->cv_work.wait_for(lock, std::chrono::microseconds(s->o.poll_us > 0 ? s->o.poll_us : 200));
    }
}

}  // namespace

extern "C" {

void bp_server_options_default(bp_server_options* o) {
    memset(o, 0, sizeof(*o));
    o->max_batch_queries = 32;
    o->device_memory_budget = (int64_t)16 << 30;
    o->chunk_residues = 1 << 20;
    o->schedule = BP_SCHED_DYNAMIC;
    o->lanes = 2;
    o->lane_depth = 1;
    o->admission = BP_ADMIT_ARRIVAL;
    o->segments = 1;
    o->max_wait_ms = 0;
    o->poll_us = 200;
    bp_params_default(&o->params);
}

bp_status bp_server_create(bp_engine* e, const bp_db* db, const bp_server_options* opt, bp_server** out) {
    if (!e || !db || !out) return bp_set_error(e, BP_ERR_INVALID, "bp_server_create: bad argument");
    *out = nullptr;
    bp_server* s = new bp_server();
    s->e = e;
    s->db = db;
    if (opt) s->o = *opt;
    else bp_server_options_default(&s->o);
    if (s->o.lanes < 1 || s->o.lanes > 16 || s->o.max_batch_queries < 1 || s->o.lane_depth < 1 ||
        s->o.lane_depth > 16 || (s->o.admission != BP_ADMIT_ARRIVAL && s->o.admission != BP_ADMIT_SHORTEST) ||
        s->o.segments < 1 || s->o.segments > 64 || s->o.max_wait_ms < 0) {
        delete s;
        return bp_set_error(e, BP_ERR_INVALID,
                            "bp_server_create: lanes and lane_depth must be 1..16, max_batch_queries >= 1, "
                            "segments 1..64, max_wait_ms >= 0");
    }
    if (s->o.segments > 1 && db->n > 0) {
        // consecutive subject ranges of about equal residues (empty ones dropped)
        s->seg_first.push_back(0);
        for (int k = 1; k <= s->o.segments; ++k) {
            const int64_t target = db->nres * k / s->o.segments;
            int32_t i = (int32_t)(std::lower_bound(db->h_off.begin(), db->h_off.end(), target) - db->h_off.begin());
            if (k == s->o.segments) i = db->n;
            i = std::min(std::max(i, s->seg_first.back()), db->n);
            if (i > s->seg_first.back()) s->seg_first.push_back(i);
        }
        if (s->seg_first.back() != db->n) s->seg_first.push_back(db->n);
    }
    s->n_lanes = s->o.lanes;
    s->depth = s->o.lane_depth;
    if (cudaSetDevice(e->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->readback, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        s->readback = nullptr;
        bp_server_destroy(s);
        return bp_set_error(e, BP_ERR_CUDA, "bp_server_create: read-back stream");
    }
    for (int l = 0; l < s->n_lanes; ++l) {
        cudaEvent_t ev = nullptr;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            bp_server_destroy(s);
            return bp_set_error(e, BP_ERR_CUDA, "bp_server_create: lane event");
        }
        s->lane_tail.push_back(ev);
        s->lane_used.push_back(false);
    }
    for (int k = 0; k < s->n_lanes * s->depth; ++k) {
        bp_engine* le = nullptr;
        const bp_status st = bp_engine_create(e->device, &le);
        if (st != BP_OK) {
            bp_server_destroy(s);
            return bp_set_error(e, st, "bp_server_create: slot engine");
        }
        s->slots.push_back(le);
        s->slot_job.push_back(nullptr);
        // scratch for plain searches over the whole database, sized now (a
        // later growth would synchronise the device under load): records for
        // two expected word hits per residue, a 1,000-letter query's worth
        const size_t recs = (size_t)std::min<double>(1 << 28, 2.5e-4 * 2.0 * (double)db->nres);
        const bp_status rs = bp_engine_reserve(le, db->n, recs);
        if (rs != BP_OK) {
            bp_server_destroy(s);
            return bp_set_error(e, rs, "bp_server_create: slot scratch");
        }
    }
    s->th = std::thread(dispatcher, s);
    *out = s;
    return BP_OK;
}

bp_status bp_server_submit(bp_server* s, const uint8_t* query, int32_t length, uint64_t* ticket) {
    if (!s || !ticket || length < 0 || (length > 0 && !query)) return BP_ERR_INVALID;
    if (length > BP_MAX_QUERY_LENGTH) return BP_ERR_TOO_LARGE;
    for (int32_t i = 0; i < length; ++i)
        if (query[i] == 0 || query[i] >= BP_ALPHABET) return BP_ERR_INVALID;
    Req* r = new Req();
    r->residues.assign(query, query + length);
    r->t_arrive = now_ms();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        r->id = s->next_id++;
        r->bytes = request_bytes(s, length);
        if (s->t_first < 0) s->t_first = r->t_arrive;
        s->reqs[r->id] = r;
        s->pending.push_back(r);
        *ticket = r->id;
    }
    s->cv_work.notify_one();
    return BP_OK;
}

int32_t bp_server_state(bp_server* s, uint64_t ticket) {
    if (!s) return BP_REQ_UNKNOWN;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->reqs.find(ticket);
    return it == s->reqs.end() ? BP_REQ_UNKNOWN : it->second->state;
}

bp_status bp_server_wait(bp_server* s, uint64_t ticket, int32_t timeout_ms) {
    if (!s) return BP_ERR_INVALID;
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return BP_ERR_INVALID;
    Req* r = it->second;
    const auto pred = [r] { return r->state == BP_REQ_DONE || r->state == BP_REQ_FAILED; };
    if (timeout_ms < 0) s->cv_done.wait(lock, pred);
    else if (!s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), pred)) return BP_ERR_NOT_READY;
    return r->state == BP_REQ_DONE ? BP_OK : r->status;
}

bp_status bp_server_result(bp_server* s, uint64_t ticket, int32_t* counters, int64_t* hsp_off, bp_hsp* hsps,
                           int64_t* n_hsps, double* latency_ms) {
    if (!s) return BP_ERR_INVALID;
    Job* job = nullptr;
    int index = -1;
    std::vector<Job*> pieces;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end()) return BP_ERR_INVALID;
        Req* r = it->second;
        if (r->state == BP_REQ_FAILED) return r->status;
        if (r->state != BP_REQ_DONE) return BP_ERR_NOT_READY;
        if (latency_ms) *latency_ms = r->t_done - r->t_arrive;
        job = r->job;
        index = r->index;
        pieces = r->segs;
    }
    // the jobs cannot be retired before this request is released
    if (pieces.empty()) return job_copy(job, index, counters, hsp_off, hsps, n_hsps);
    // segment mode: range k's piece goes to subjects [seg_first[k], seg_first[k + 1]), its
    // records after those of the ranges before it
    int64_t base = 0;
    for (size_t k = 0; k < pieces.size(); ++k) {
        const int32_t f = s->seg_first[k];
        int64_t nh = 0;
        const bp_status st = job_copy(pieces[k], 0, counters ? counters + 3 * (int64_t)f : nullptr,
                                      hsp_off ? hsp_off + f : nullptr, hsps ? hsps + base : nullptr, &nh);
        if (st != BP_OK) return st;
        if (hsp_off)
            for (int32_t i = f; i <= s->seg_first[k + 1]; ++i) hsp_off[i] += base;
        base += nh;
    }
    if (n_hsps) *n_hsps = base;
    return BP_OK;
}

bp_status bp_server_digest(bp_server* s, uint64_t ticket, uint64_t out[2]) {
    if (!s || !out) return BP_ERR_INVALID;
    Job* job = nullptr;
    int index = -1;
    std::vector<Job*> pieces;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end()) return BP_ERR_INVALID;
        Req* r = it->second;
        if (r->state == BP_REQ_FAILED) return r->status;
        if (r->state != BP_REQ_DONE) return BP_ERR_NOT_READY;
        job = r->job;
        index = r->index;
        pieces = r->segs;
    }
    // on the server's own read-back stream: a slot's stream may already run
    // the next batch, which a digest there would wait for
    std::lock_guard<std::mutex> rb(s->readback_mu);
    uint64_t sums[2] = {0, 0};
    if (pieces.empty()) {
        const bp_status st = job_digest_sums(s, job, index, 0, 0, true, sums);
        if (st != BP_OK) return st;
        bp_digest_finish(sums, s->db->n, out);
        return BP_OK;
    }
    // segment mode: the pieces' sums at their places in the whole result
    int64_t base = 0;
    for (size_t k = 0; k < pieces.size(); ++k) {
        int64_t nh = 0;
        bp_status st = job_copy(pieces[k], 0, nullptr, nullptr, nullptr, &nh);
        uint64_t part[2];
        if (st == BP_OK) st = job_digest_sums(s, pieces[k], 0, s->seg_first[k], base, k + 1 == pieces.size(), part);
        if (st != BP_OK) return st;
        sums[0] += part[0];
        sums[1] += part[1];
        base += nh;
    }
    bp_digest_finish(sums, s->db->n, out);
    return BP_OK;
}

bp_status bp_server_release(bp_server* s, uint64_t ticket) {
    if (!s) return BP_ERR_INVALID;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return BP_ERR_INVALID;
    Req* r = it->second;
    if (r->state != BP_REQ_DONE && r->state != BP_REQ_FAILED) return BP_ERR_NOT_READY;
    if (r->released) return BP_ERR_INVALID;
    r->released = true;
    if (!r->segs.empty()) {                      // segment mode
        if (segs_finished(r) && !seg_on_slot(s, r)) retire_segmented(s, r);
        s->cv_work.notify_one();
        return BP_OK;
    }
    Job* job = r->job;
    if (!job) {                                  // failed before admission
        s->reqs.erase(it);
        delete r;
        return BP_OK;
    }
    job->live -= 1;
    const bool on_lane = std::find(s->slot_job.begin(), s->slot_job.end(), job) != s->slot_job.end();
    if (job->live == 0 && job->done && !on_lane) retire_job(s, job);
    s->cv_work.notify_one();
    return BP_OK;
}

bp_status bp_server_stats(bp_server* s, bp_server_metrics* out) {
    if (!s || !out) return BP_ERR_INVALID;
    std::lock_guard<std::mutex> lock(s->mu);
    memset(out, 0, sizeof(*out));
    out->completed = s->n_done;
    out->failed = s->n_failed;
    out->batches = s->n_batches;
    out->mean_batch = s->n_batches ? (double)s->batched_queries / (double)s->n_batches : 0.0;
    out->pending = (int64_t)s->pending.size();
    out->max_in_flight = s->max_in_flight;
    out->mem_used = s->mem_used;
    out->mem_peak = s->mem_peak;
    if (!s->latency_ms.empty()) {
        std::vector<double> v = s->latency_ms;
        std::sort(v.begin(), v.end());
        auto pct = [&v](double p) {
            const size_t i = (size_t)std::min<double>((double)v.size() - 1, std::ceil(p * (double)v.size()) - 1);
            return v[i];
        };
        out->p50_ms = pct(0.50);
        out->p99_ms = pct(0.99);
        out->max_ms = v.back();
        const double span = (s->t_last - s->t_first) / 1e3;
        out->queries_per_s = span > 0 ? (double)s->n_done / span : 0.0;
        out->resq_per_s = span > 0 ? s->resq / span : 0.0;
    }
    return BP_OK;
}

void bp_server_destroy(bp_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->th.joinable()) s->th.join();
    // release everything still held, once nothing runs
    for (bp_engine* le : s->slots) {
        cudaSetDevice(le->device);
        cudaStreamSynchronize(le->stream);
    }
    cudaGetLastError();
    std::vector<Req*> segmented;
    for (auto& kv : s->reqs)
        if (!kv.second->segs.empty()) segmented.push_back(kv.second);
    for (Req* r : segmented) {
        for (Job* j : r->segs) {
            job_free(j);
            delete j;
        }
        r->segs.clear();
        bp_query_destroy(r->query);
        s->reqs.erase(r->id);
        delete r;
    }
    std::vector<Job*> jobs;
    for (auto& kv : s->reqs)
        if (kv.second->job && std::find(jobs.begin(), jobs.end(), kv.second->job) == jobs.end())
            jobs.push_back(kv.second->job);
    for (Job* j : jobs) {
        job_free(j);
        for (Req* r : j->reqs) {
            bp_query_destroy(r->query);
            s->reqs.erase(r->id);
            delete r;
        }
        delete j;
    }
    for (auto& kv : s->reqs) delete kv.second;
    for (bp_engine* le : s->slots) bp_engine_destroy(le);
    for (cudaEvent_t ev : s->lane_tail) cudaEventDestroy(ev);
    if (s->readback) cudaStreamDestroy(s->readback);
    delete s;
}

}  // extern "C"
