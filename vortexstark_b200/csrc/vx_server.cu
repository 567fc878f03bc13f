// Serving engine: continuous batching of Fibonacci proof requests of mixed
// sizes on one GPU (new; the reference proves one request at a time,
// prover.rs:2278-2319).
//
// Requests enter a FIFO.  A dispatcher thread admits any queued request for
// which a free proof slot of its size exists, or can be created inside the
// device-memory budget (slot buffers + the size's shared twiddle tables), up
// to `max_inflight` proofs on the device at once.  Each slot owns a stream,
// a pinned host buffer for its proof and a CUDA graph of one whole proof
// (captured once at slot creation), so admitting a request is: write (a, b)
// into the slot's pinned input words, launch the graph, record an event.
// Proofs of different requests therefore overlap on the device while each
// proof's own kernels stay in order; every proof is computed by the same
// kernels on its own buffers, so its bytes do not depend on what else runs.
//
// Scheduling policy (vx_server_set_policy).  A proof whose evaluation
// domain has at least 2^large_log_eval points (default 2^24) fills every SM
// by itself for most of its kernels, so two of them in flight only split the
// GPU and both finish later: at most `max_large` such proofs (default 1) are
// admitted at a time, others wait in the queue, oldest first.  Smaller
// proofs are chains of short kernels that leave most SMs idle.  Stream
// priorities decide whose blocks the hardware dispatches first when both
// wait: by default small proofs run on the highest-priority streams, so
// their blocks are dispatched ahead of a large proof's waiting blocks and
// fill the gaps it leaves; the reverse order keeps a large proof close to
// its solo time.  `small_cap` optionally bounds the small proofs in flight
// while a large one is.  With `split_large` (default) a large proof is two
// graphs: its head (LDE, the trace, quotient and FRI commitments of layers
// deeper than 16) counts against max_large; its tail (the small FRI layers,
// queries, decommitment) runs on a highest-priority stream and no longer
// does, so the next large proof's head overlaps it.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <mutex>
#include <thread>
#include <vector>

#include "vx_common.cuh"
#include "vx_prover.cuh"

namespace {

uint64_t now_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
    uint64_t tag;
    uint32_t log_n, a, b;
    uint64_t submit_ns;
};

// Default policy: evaluation domains of at least 2^24 points fill the GPU
// alone; one such proof in flight; small proofs on the highest-priority
// streams; no cap on small proofs.
constexpr uint32_t kLargeLogEval = 24;
constexpr uint32_t kMaxLargeInflight = 1;
constexpr int kPrioDefault = 0;
// A split large proof's tail: the line folds of layers of at most 2^16 values
// (one latency-bound reduce launch each), queries and decommitment.
constexpr uint32_t kTailStage = 6;

struct Slot {
    vx_prover *p = nullptr;
    uint32_t log_n = 0;
    bool large = false;
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    cudaGraphExec_t exec = nullptr;
    // split large proofs: exec is the head (inputs, LDE, trace / quotient / first FRI commitments) on st,
    // tail_exec the rest on tail_st (highest priority), after head_done
    cudaGraphExec_t tail_exec = nullptr;
    cudaStream_t tail_st = nullptr;
    cudaEvent_t head_done = nullptr;
    bool active = false;   // a large proof counted against max_large (in flight, or in its head if split)
    uint8_t *pinned_out = nullptr;
    uint32_t *pinned_ab = nullptr;
    uint32_t *dev_ab = nullptr;
    size_t bytes = 0;      // proof bytes
    size_t footprint = 0;  // device bytes held by the slot
    bool busy = false;
    Request req{};
    uint64_t start_ns = 0;
};

}  // namespace

struct vx_server {
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Request> pending;
    std::vector<Slot *> slots;
    std::map<uint32_t, size_t> table_bytes;  // per log_n, counted once
    std::map<uint64_t, std::vector<uint8_t>> results;
    std::vector<vx_completion> completed;
    std::thread worker;
    bool stop = false;
    size_t budget = 0, used = 0;
    // large_inflight: large proofs counted against max_large (see Slot::active)
    uint32_t max_inflight = 1, inflight = 0, large_inflight = 0, small_inflight = 0, blowup = 2, nq = 80;
    // policy (vx_server_set_policy)
    uint32_t large_log_eval = kLargeLogEval, max_large = kMaxLargeInflight, small_cap = 0;
    bool large_per_size = false;               // max_large counts per size instead of overall
    bool split_large = true;                   // large proofs as head + tail graphs (see slot_create)
    std::map<uint32_t, uint32_t> large_by_size;  // active large proofs per log_n
    int prio_mode = kPrioDefault;  // 0: small proofs highest, 1: all equal, 2: large proofs highest, 3: graded
    // order of waiting large proofs (vx_server_set_queue_order): oldest first,
    // or smallest first with the oldest going first once it has waited max_wait_ns
    bool smallest_first = false;
    uint64_t max_wait_ns = 0;
    int device = 0;
    bool use_graphs = true;
    int fatal = VX_OK;
    std::string fatal_msg;
};

using namespace vx;

namespace {

int slot_create(vx_server *s, uint32_t log_n, Slot **out) {
    auto *sl = new Slot();
    sl->log_n = log_n;
    int rc = vx_prover_create(log_n, s->blowup, s->nq, &sl->p);
    if (rc) { delete sl; return rc; }
    sl->bytes = prover_proof_bytes(sl->p);
    sl->footprint = vx_prover_slot_bytes(sl->p) + 256;
    auto fail = [&](const char *what, cudaError_t e) {
        set_last_error(VX_ERR_CUDA, "server slot: %s: %s", what, cudaGetErrorString(e));
        if (sl->st) cudaStreamDestroy(sl->st);
        if (sl->done) cudaEventDestroy(sl->done);
        if (sl->pinned_out) cudaFreeHost(sl->pinned_out);
        if (sl->pinned_ab) cudaFreeHost(sl->pinned_ab);
        if (sl->dev_ab) cudaFree(sl->dev_ab);
        vx_prover_destroy(sl->p);
        delete sl;
        return VX_ERR_CUDA;
    };
    cudaError_t e;
    sl->large = log_n + s->blowup >= s->large_log_eval;
    int prio_least = 0, prio_greatest = 0;
    if ((e = cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest)) != cudaSuccess) return fail("priorities", e);
    int prio = prio_least;
    if (s->prio_mode == 0) prio = sl->large ? prio_least : prio_greatest;
    if (s->prio_mode == 2) prio = sl->large ? prio_greatest : prio_least;
    if (s->prio_mode == 3) {  // graded: the two sizes below the large threshold in between
        const uint32_t le = log_n + s->blowup;
        prio = le >= s->large_log_eval ? prio_least
               : le + 2 >= s->large_log_eval ? (prio_least + prio_greatest) / 2 : prio_greatest;
    }
    if ((e = cudaStreamCreateWithPriority(&sl->st, cudaStreamNonBlocking, prio)) != cudaSuccess)
        return fail("stream", e);
    if ((e = cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming)) != cudaSuccess) return fail("event", e);
    // proof bytes, then the transcript status word
    if ((e = cudaMallocHost(&sl->pinned_out, sl->bytes + 16)) != cudaSuccess) return fail("pinned output", e);
    if ((e = cudaMallocHost(&sl->pinned_ab, 8)) != cudaSuccess) return fail("pinned input", e);
    if ((e = cudaMalloc(&sl->dev_ab, 256)) != cudaSuccess) return fail("device input", e);
    if (s->use_graphs && sl->large && s->split_large) {
        // A large proof's head fills the GPU; its tail (the small FRI layers,
        // queries, decommitment) is a chain of latency-bound launches.  The tail runs on a
        // highest-priority stream behind an event, and the next large proof
        // may start as soon as this head is done, so its head overlaps this
        // tail instead of the GPU idling through it.
        if ((e = cudaStreamCreateWithPriority(&sl->tail_st, cudaStreamNonBlocking, prio_greatest)) != cudaSuccess)
            return fail("tail stream", e);
        if ((e = cudaEventCreateWithFlags(&sl->head_done, cudaEventDisableTiming)) != cudaSuccess) {
            cudaStreamDestroy(sl->tail_st);
            return fail("head event", e);
        }
        rc = prover_capture_graph_split(sl->p, sl->st, sl->dev_ab, sl->pinned_ab, sl->pinned_out, kTailStage,
                                        &sl->exec, &sl->tail_exec);
    } else if (s->use_graphs) {
        rc = prover_capture_graph(sl->p, sl->st, sl->dev_ab, sl->pinned_ab, sl->pinned_out, &sl->exec);
    }
    if (rc) {
        if (sl->tail_st) cudaStreamDestroy(sl->tail_st);
        if (sl->head_done) cudaEventDestroy(sl->head_done);
        cudaStreamDestroy(sl->st); cudaEventDestroy(sl->done);
        cudaFreeHost(sl->pinned_out); cudaFreeHost(sl->pinned_ab); cudaFree(sl->dev_ab);
        vx_prover_destroy(sl->p);
        delete sl;
        return rc;
    }
    *out = sl;
    return VX_OK;
}

void slot_destroy(Slot *sl) {
    if (sl->exec) cudaGraphExecDestroy(sl->exec);
    if (sl->tail_exec) cudaGraphExecDestroy(sl->tail_exec);
    if (sl->tail_st) cudaStreamDestroy(sl->tail_st);
    if (sl->head_done) cudaEventDestroy(sl->head_done);
    cudaStreamDestroy(sl->st);
    cudaEventDestroy(sl->done);
    cudaFreeHost(sl->pinned_out);
    cudaFreeHost(sl->pinned_ab);
    cudaFree(sl->dev_ab);
    vx_prover_destroy(sl->p);
    delete sl;
}

// Device bytes a new slot of this size would take (tables counted once).
size_t slot_cost(vx_server *s, uint32_t log_n, size_t slot_bytes, size_t tab_bytes) {
    return slot_bytes + (s->table_bytes.count(log_n) ? 0 : tab_bytes);
}

int launch(vx_server *s, Slot *sl, const Request &r) {
    sl->busy = true;
    sl->req = r;
    sl->start_ns = now_ns();
    s->inflight++;
    if (sl->large) {
        s->large_inflight++;
        s->large_by_size[sl->log_n]++;
        sl->active = true;
    } else {
        s->small_inflight++;
    }
    if (sl->tail_exec) {
        sl->pinned_ab[0] = r.a;
        sl->pinned_ab[1] = r.b;
        VX_CUDA_TRY(cudaGraphLaunch(sl->exec, sl->st));
        VX_CUDA_TRY(cudaEventRecord(sl->head_done, sl->st));
        VX_CUDA_TRY(cudaStreamWaitEvent(sl->tail_st, sl->head_done, 0));
        VX_CUDA_TRY(cudaGraphLaunch(sl->tail_exec, sl->tail_st));
        VX_CUDA_TRY(cudaEventRecord(sl->done, sl->tail_st));
        return VX_OK;
    }
    if (sl->exec) {
        sl->pinned_ab[0] = r.a;
        sl->pinned_ab[1] = r.b;
        VX_CUDA_TRY(cudaGraphLaunch(sl->exec, sl->st));
    } else {
        int rc = vx_prover_prove_async(sl->p, r.a, r.b, sl->st);
        if (rc) return rc;
        rc = vx_prover_fetch_async(sl->p, sl->pinned_out, sl->st);
        if (rc) return rc;
        VX_CUDA_TRY(cudaMemcpyAsync(sl->pinned_out + sl->bytes, prover_chan_err(sl->p), 4, cudaMemcpyDeviceToHost,
                                    sl->st));
    }
    VX_CUDA_TRY(cudaEventRecord(sl->done, sl->st));
    return VX_OK;
}

// Device bytes a slot of this size takes, and its size's shared tables.
void size_estimate(vx_server *s, uint32_t log_n, size_t *slot_b, size_t *tab_b) {
    prover_footprint(log_n, s->blowup, s->nq, slot_b, tab_b);
    *slot_b += 256;  // the slot's device input words
}

// A large proof stops counting against max_large when its head is done
// (split) or when it completes.
void deactivate(vx_server *s, Slot *sl) {
    if (!sl->active) return;
    sl->active = false;
    s->large_inflight--;
    s->large_by_size[sl->log_n]--;
}

// Smallest-first order of the waiting large requests: the smallest log_n,
// oldest within a size; but once the oldest waiting large request has waited
// max_wait_ns it goes first.  `pending` is in arrival order.  False when no
// large request waits.
bool next_large(const vx_server *s, uint64_t now, uint64_t *tag) {
    const Request *oldest = nullptr, *best = nullptr;
    for (const Request &r : s->pending) {
        if (r.log_n + s->blowup < s->large_log_eval) continue;
        if (!oldest) oldest = &r;
        if (!best || r.log_n < best->log_n) best = &r;
    }
    if (!oldest) return false;
    *tag = (s->max_wait_ns && now - oldest->submit_ns >= s->max_wait_ns) ? oldest->tag : best->tag;
    return true;
}

void worker_loop(vx_server *s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        bool progress = false;
        // split large proofs whose head is done free their large-proof place
        for (Slot *sl : s->slots) {
            if (!sl->busy || !sl->active || !sl->tail_exec) continue;
            if (cudaEventQuery(sl->head_done) != cudaErrorNotReady) {
                deactivate(s, sl);
                progress = true;
            }
        }
        // complete finished proofs
        for (Slot *sl : s->slots) {
            if (!sl->busy) continue;
            cudaError_t q = cudaEventQuery(sl->done);
            if (q == cudaErrorNotReady) continue;
            vx_completion c{};
            c.tag = sl->req.tag;
            c.log_n = sl->req.log_n;
            c.submit_ns = sl->req.submit_ns;
            c.start_ns = sl->start_ns;
            c.done_ns = now_ns();
            c.proof_bytes = sl->bytes;
            c.status = q == cudaSuccess ? VX_OK : VX_ERR_CUDA;
            if (q == cudaSuccess) {
                uint32_t err = 0;
                memcpy(&err, sl->pinned_out + sl->bytes, 4);  // copied by the proof's own stream
                if (err) c.status = VX_ERR_DEVICE;
            }
            s->results[c.tag].assign(sl->pinned_out, sl->pinned_out + sl->bytes);
            s->completed.push_back(c);
            sl->busy = false;
            s->inflight--;
            if (sl->large) deactivate(s, sl);
            else s->small_inflight--;
            progress = true;
        }
        // the large request a free large place goes to
        uint64_t large_tag = 0;
        bool large_pick = s->smallest_first && !s->large_per_size && next_large(s, now_ns(), &large_tag);
        // admit queued requests, oldest first, skipping ones that cannot start
        // yet.  Requests are addressed by index: submitters append to
        // `pending` while the lock is released for a slot creation (which
        // invalidates deque iterators), and only this thread removes entries,
        // so an index keeps naming the same request.
        for (size_t qi = 0; qi < s->pending.size() && s->inflight < s->max_inflight;) {
            const uint32_t log_n = s->pending[qi].log_n;
            const bool large = log_n + s->blowup >= s->large_log_eval;
            if (large && (s->large_per_size ? s->large_by_size[log_n] : s->large_inflight) >= s->max_large) {
                ++qi;  // a large proof is running: this one waits, smaller ones behind it may start
                continue;
            }
            if (large && large_pick && s->pending[qi].tag != large_tag) {
                ++qi;  // another large request goes first
                continue;
            }
            if (!large && s->small_cap && s->large_inflight && s->small_inflight >= s->small_cap) {
                ++qi;  // small proofs at their cap beside a large one
                continue;
            }
            Slot *free_slot = nullptr;
            for (Slot *sl : s->slots)
                if (!sl->busy && sl->log_n == log_n) { free_slot = sl; break; }
            if (!free_slot) {
                size_t sb, tb;
                size_estimate(s, log_n, &sb, &tb);
                if (s->used + slot_cost(s, log_n, sb, tb) <= s->budget) {
                    Slot *sl = nullptr;
                    lk.unlock();
                    int rc = slot_create(s, log_n, &sl);
                    lk.lock();
                    if (rc) {
                        s->fatal = rc;
                        s->fatal_msg = vx_last_error();
                        s->stop = true;
                        break;
                    }
                    s->used += sl->footprint + (s->table_bytes.count(log_n) ? 0 : vx_prover_table_bytes(sl->p));
                    s->table_bytes[log_n] = vx_prover_table_bytes(sl->p);
                    s->slots.push_back(sl);
                    free_slot = sl;
                }
            }
            if (free_slot) {
                Request r = s->pending[qi];
                s->pending.erase(s->pending.begin() + (std::ptrdiff_t)qi);
                if (launch(s, free_slot, r) != VX_OK) {
                    s->fatal = VX_ERR_CUDA;
                    s->fatal_msg = vx_last_error();
                    s->stop = true;
                    break;
                }
                if (large && large_pick) large_pick = next_large(s, now_ns(), &large_tag);
                progress = true;
            } else {
                ++qi;
            }
        }
        if (!progress) {
            if (s->inflight == 0 && s->pending.empty()) {
                s->cv.wait_for(lk, std::chrono::milliseconds(50));
            } else {
                lk.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(20));
                lk.lock();
            }
        }
        s->cv.notify_all();
    }
}

}  // namespace

extern "C" int vx_server_create(size_t budget_bytes, uint32_t max_inflight, uint32_t blowup_bits, uint32_t n_queries,
                                int use_graphs, vx_server **out) {
    VX_CHECK_ARG(out != nullptr, "vx_server_create: out is null");
    VX_CHECK_ARG(max_inflight >= 1 && max_inflight <= 256, "vx_server_create: max_inflight must be in [1, 256]");
    VX_CHECK_ARG(blowup_bits >= 1 && blowup_bits <= 8, "vx_server_create: bad blowup_bits");
    VX_CHECK_ARG(n_queries >= 1 && n_queries <= 4096, "vx_server_create: bad n_queries");
    auto *s = new vx_server();
    cudaGetDevice(&s->device);
    s->budget = budget_bytes;
    s->max_inflight = max_inflight;
    s->blowup = blowup_bits;
    s->nq = n_queries;
    s->use_graphs = use_graphs != 0;
    s->worker = std::thread(worker_loop, s);
    *out = s;
    return VX_OK;
}

extern "C" int vx_server_set_policy(vx_server *s, uint32_t large_log_eval, uint32_t max_large, int priority,
                                    uint32_t small_cap, int large_per_size, int split_large) {
    VX_CHECK_ARG(s != nullptr, "vx_server_set_policy: null server");
    VX_CHECK_ARG(large_log_eval >= 1 && large_log_eval <= 32, "vx_server_set_policy: bad large_log_eval %u",
                 large_log_eval);
    VX_CHECK_ARG(max_large >= 1, "vx_server_set_policy: max_large must be at least 1");
    VX_CHECK_ARG(priority >= 0 && priority <= 3, "vx_server_set_policy: priority must be 0, 1, 2 or 3");
    std::lock_guard<std::mutex> lk(s->mu);
    VX_CHECK_ARG(s->slots.empty() && s->pending.empty(),
                 "vx_server_set_policy: call before the first prewarm or submit (slot streams keep their priority)");
    s->large_log_eval = large_log_eval;
    s->max_large = max_large;
    s->large_per_size = large_per_size != 0;
    s->split_large = split_large != 0;
    s->prio_mode = priority;
    s->small_cap = small_cap;
    return VX_OK;
}

extern "C" int vx_server_set_queue_order(vx_server *s, int smallest_first, uint32_t max_wait_us) {
    VX_CHECK_ARG(s != nullptr, "vx_server_set_queue_order: null server");
    std::lock_guard<std::mutex> lk(s->mu);
    s->smallest_first = smallest_first != 0;
    s->max_wait_ns = (uint64_t)max_wait_us * 1000ull;
    return VX_OK;
}

extern "C" int vx_server_submit(vx_server *s, uint64_t tag, uint32_t log_n, uint32_t a, uint32_t b) {
    VX_CHECK_ARG(s != nullptr, "vx_server_submit: null server");
    VX_CHECK_ARG(log_n >= 4 && log_n + s->blowup <= 31, "vx_server_submit: unsupported log_n %u", log_n);
    VX_CHECK_ARG(a < VX_P && b < VX_P, "vx_server_submit: public inputs must be canonical M31");
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->fatal) { set_last_error(s->fatal, "server stopped: %s", s->fatal_msg.c_str()); return s->fatal; }
    s->pending.push_back(Request{tag, log_n, a, b, now_ns()});
    s->cv.notify_all();
    return VX_OK;
}

extern "C" int vx_server_prewarm(vx_server *s, uint32_t log_n, uint32_t count) {
    VX_CHECK_ARG(s != nullptr, "vx_server_prewarm: null server");
    std::unique_lock<std::mutex> lk(s->mu);
    uint32_t have = 0;
    for (Slot *sl : s->slots) have += sl->log_n == log_n;
    while (have < count) {
        Slot *sl = nullptr;
        lk.unlock();
        int rc = slot_create(s, log_n, &sl);
        lk.lock();
        if (rc) return rc;
        s->used += sl->footprint + (s->table_bytes.count(log_n) ? 0 : vx_prover_table_bytes(sl->p));
        s->table_bytes[log_n] = vx_prover_table_bytes(sl->p);
        s->slots.push_back(sl);
        have++;
    }
    return VX_OK;
}

extern "C" int vx_server_poll(vx_server *s, vx_completion *out, uint32_t max, uint32_t *n_out, int wait_ms) {
    VX_CHECK_ARG(s != nullptr && n_out != nullptr && (out != nullptr || max == 0), "vx_server_poll: bad arguments");
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->completed.empty() && wait_ms > 0 && !s->fatal)
        s->cv.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->completed.empty() || s->fatal; });
    uint32_t n = 0;
    while (n < max && !s->completed.empty()) {
        out[n++] = s->completed.front();
        s->completed.erase(s->completed.begin());
    }
    *n_out = n;
    if (s->fatal && n == 0) { set_last_error(s->fatal, "server stopped: %s", s->fatal_msg.c_str()); return s->fatal; }
    return VX_OK;
}

extern "C" int vx_server_result(vx_server *s, uint64_t tag, uint8_t *out, size_t cap, size_t *len) {
    VX_CHECK_ARG(s != nullptr && len != nullptr, "vx_server_result: bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->results.find(tag);
    VX_CHECK_ARG(it != s->results.end(), "vx_server_result: no finished proof with tag %llu", (unsigned long long)tag);
    *len = it->second.size();
    if (out) {
        VX_CHECK_ARG(cap >= it->second.size(), "vx_server_result: capacity %zu < proof size %zu", cap,
                     it->second.size());
        memcpy(out, it->second.data(), it->second.size());
    }
    s->results.erase(it);
    return VX_OK;
}

extern "C" int vx_server_stats(vx_server *s, uint32_t *n_slots, uint32_t *inflight, uint32_t *pending,
                               size_t *bytes_used) {
    VX_CHECK_ARG(s != nullptr, "vx_server_stats: null server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (n_slots) *n_slots = (uint32_t)s->slots.size();
    if (inflight) *inflight = s->inflight;
    if (pending) *pending = (uint32_t)s->pending.size();
    if (bytes_used) *bytes_used = s->used;
    return VX_OK;
}

extern "C" void vx_server_destroy(vx_server *s) {
    if (!s) return;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        // let in-flight proofs finish before tearing down their buffers
        for (Slot *sl : s->slots)
            if (sl->busy) cudaEventSynchronize(sl->done);
        s->stop = true;
        s->cv.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    for (Slot *sl : s->slots) slot_destroy(sl);
    delete s;
}
