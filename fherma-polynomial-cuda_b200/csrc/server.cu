// Serving form: a request loop with continuous batching.
//
// New in this library (the reference has one synchronous product per call,
// src/main.cpp:164-204). A session fixes (W, L, q); its plans (one per ring
// size N, parameter tables resident on the device) are built when the session
// opens or on the first request of a new N. Requests are submitted from any
// thread and return at once.
//
// Requests flow through a three-stream pipeline:
//   copy-in   operands of request i+1 (host -> device, own buffers from a stream-ordered pool)
//   compute   request i: pad, product (one work arena shared by every request, since the
//             compute stream runs them one after another)
//   copy-out  result of request i-1 (device -> host), then the buffers are freed and a host
//             callback completes the request.
// One dispatcher thread admits queued requests in arrival order while fewer than `slots` are in
// the pipeline and the request's operand buffers (plus any growth of the shared arena) fit the
// HBM budget next to the resident plan tables. With max_queue set, a submit that finds that many
// requests already waiting is refused at once (NEGACYCLIC_EBUSY): under overload the queue, and
// with it the latency of what is admitted, stays bounded. A request that arrives while others are on the
// GPU joins the pipeline as soon as a place and memory free up, so its copies overlap their
// compute. With one compute stream the CTA-pair GEMM kernel is used; concurrent launches of
// that kernel from several streams stalled, so a process runs one server per device.
// Each request's product clears its plan's status word first and copies it to a page-locked
// slot right after (both on the compute stream, so requests of the same plan cannot mix up
// their words); the completion callback fails the request when the word is nonzero.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "plan_internal.h"

using namespace negacyclic;
using namespace negacyclic::detail;

namespace {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Session {
    uint32_t w = 0, limbs = 0;
    std::vector<uint32_t> q;
    std::map<uint32_t, std::unique_ptr<negacyclic_plan>> plans;  // by N
};

struct Request {
    uint64_t id = 0;
    uint32_t session = 0, n = 0;
    const uint32_t* a = nullptr;
    const uint32_t* b = nullptr;
    uint32_t* c = nullptr;
    double submitted = 0, admitted = 0, finished = 0;
    uint32_t status_slot = 0;  // index into the server's page-locked status words
    int status = NEGACYCLIC_OK;
    std::string error;
    bool done = false;
    size_t bytes = 0;  // operand/result buffers held while in flight
    cudaEvent_t copied_in = nullptr, computed = nullptr;
    struct negacyclic_server* server = nullptr;
};

}  // namespace

struct negacyclic_server {
    int device = 0;
    uint64_t budget = 0, resident = 0, in_flight = 0;
    uint32_t slots = 0, active = 0;  // pipeline depth, requests in it
    uint32_t max_queue = 0;          // 0 = unbounded admission queue
    uint64_t rejected = 0, max_queued = 0;
    std::vector<Session> sessions;
    std::deque<Request*> pending;
    std::map<uint64_t, std::unique_ptr<Request>> requests;
    uint64_t next_id = 1;
    cudaStream_t copy_in = nullptr, compute = nullptr, copy_out = nullptr;
    void* arena = nullptr;  // shared work space, stream-ordered on `compute`
    size_t arena_bytes = 0;
    // page-locked status words, one per request in flight: request id modulo kStatusSlots (at
    // most `slots` requests are in flight, admitted and completed in id order)
    static constexpr uint32_t kStatusSlots = 1024;
    uint32_t* status_host = nullptr;
    std::vector<cudaEvent_t> spare_events;  // completed events, reusable
    std::vector<cudaEvent_t> all_events;
    std::mutex mu;
    std::condition_variable wake, finished;
    std::thread dispatcher;
    bool stopping = false;
    std::vector<double> latencies;  // completed requests, ms
    uint64_t completed = 0, failed = 0;
    double first_submit = 0, last_finish = 0;

    void run();
    bool admit_one(std::unique_lock<std::mutex>& lock);
    cudaEvent_t take_event();
    void fail_head(Request* r, int status, const std::string& error);
    static void CUDART_CB on_done(void* data);
};

namespace {

size_t io_bytes(const negacyclic_plan& plan) {
    return 3 * ((size_t(plan.host.n) * plan.host.limbs * 4 + 255) / 256 * 256);
}

// Builds a session plan for ring size n. Must be called WITHOUT the server lock:
// plan creation can synchronise the device, and the completion callbacks of
// requests in flight need the lock to finish.
int build_session_plan(int device, uint32_t w, uint32_t limbs, const uint32_t* q, uint32_t n,
                       negacyclic_plan** out) {
    negacyclic_options o{};
    o.device = device;
    o.external_work = 1;
    return negacyclic_init(n, w, limbs, q, &o, out);
}

// Adds a built plan to a session under the budget. Caller holds the lock.
int install_plan(negacyclic_server& s, Session& session, uint32_t n, negacyclic_plan* plan, negacyclic_plan** out) {
    auto it = session.plans.find(n);
    if (it != session.plans.end()) {  // built twice: keep the first
        negacyclic_free(plan);
        *out = it->second.get();
        return NEGACYCLIC_OK;
    }
    if (s.resident + plan->table_bytes > s.budget) {
        negacyclic_free(plan);
        return fail(NEGACYCLIC_ENOMEM, "plan tables exceed the HBM budget");
    }
    s.resident += plan->table_bytes;
    session.plans.emplace(n, plan);
    *out = plan;
    return NEGACYCLIC_OK;
}

}  // namespace

// Caller holds the lock.
cudaEvent_t negacyclic_server::take_event() {
    if (!spare_events.empty()) {
        cudaEvent_t e = spare_events.back();
        spare_events.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    all_events.push_back(e);
    return e;
}

// Completes the queue head `r` (already popped) with an error. Caller holds the lock.
void negacyclic_server::fail_head(Request* r, int status, const std::string& error) {
    r->status = status;
    r->error = error;
    r->done = true;
    r->finished = now_ms();
    ++failed;
    finished.notify_all();
}

// Runs on the copy-out stream after the result landed: no CUDA calls allowed here.
void CUDART_CB negacyclic_server::on_done(void* data) {
    Request* r = static_cast<Request*>(data);
    negacyclic_server* s = r->server;
    std::lock_guard<std::mutex> lock(s->mu);
    r->finished = now_ms();
    r->done = true;
    s->in_flight -= r->bytes;
    --s->active;
    s->spare_events.push_back(r->copied_in);  // both completed before this callback
    s->spare_events.push_back(r->computed);
    // the status copy ran on the compute stream before `computed`, which this stream waited for
    const uint32_t flags = reinterpret_cast<volatile uint32_t*>(s->status_host)[r->status_slot];
    if (flags) {
        r->status = NEGACYCLIC_ECUDA;
        r->error = (flags & NEGACYCLIC_STATUS_GEMM_MASK) ? "tensor-core GEMM pipeline wait gave up"
                                                          : "reduction exceeded its proven correction bound";
        ++s->failed;
        s->finished.notify_all();
        s->wake.notify_one();
        return;
    }
    ++s->completed;
    s->latencies.push_back(r->finished - r->submitted);
    s->last_finish = std::max(s->last_finish, r->finished);
    s->finished.notify_all();
    s->wake.notify_one();
}

// Admits the head of the queue if the pipeline has room and its memory fits the budget.
bool negacyclic_server::admit_one(std::unique_lock<std::mutex>& lock) {
    if (pending.empty() || active >= slots) return false;
    Request* r = pending.front();
    negacyclic_plan* plan = nullptr;
    {
        Session& session = sessions[r->session];
        auto it = session.plans.find(r->n);
        if (it != session.plans.end()) {
            plan = it->second.get();
        } else {  // first request of this ring size: build its plan without the lock
            const uint32_t w = session.w, limbs = session.limbs;
            const std::vector<uint32_t> q = session.q;
            const uint32_t n = r->n, session_id = r->session;
            lock.unlock();
            negacyclic_plan* built = nullptr;
            int status = build_session_plan(device, w, limbs, q.data(), n, &built);
            std::string error = status == NEGACYCLIC_OK ? "" : negacyclic_last_error();
            lock.lock();
            if (status == NEGACYCLIC_OK) status = install_plan(*this, sessions[session_id], n, built, &plan);
            if (status != NEGACYCLIC_OK && error.empty()) error = negacyclic_last_error();
            if (status != NEGACYCLIC_OK) {
                r = pending.front();  // the queue head is unchanged: only this thread pops it
                pending.pop_front();
                fail_head(r, status, error);
            }
            return true;  // re-evaluate room and budget with the plan in place
        }
    }
    const size_t need = io_bytes(*plan);
    const size_t arena_need = std::max(arena_bytes, plan->work_bytes);
    if (resident + arena_need + in_flight + need > budget) {
        if (active == 0) {  // nothing in flight will free memory: it can never fit
            pending.pop_front();
            fail_head(r, NEGACYCLIC_ENOMEM, "request exceeds the HBM budget");
            return true;
        }
        return false;  // wait for memory to free up (arrival order is kept)
    }
    pending.pop_front();
    r->bytes = need;
    r->admitted = now_ms();
    in_flight += need;
    ++active;
    std::string error;
    bool locked = true;
    try {
        r->copied_in = take_event();
        r->computed = take_event();
        if (arena_need > arena_bytes) {  // grow the shared arena in compute-stream order
            void* grown = nullptr;
            check(cudaMallocAsync(&grown, arena_need, compute), "cudaMallocAsync");
            if (arena) check(cudaFreeAsync(arena, compute), "cudaFreeAsync");
            arena = grown;
            arena_bytes = arena_need;
        }
        void* work = arena;
        // enqueue without holding the lock (copies from pageable memory block the host)
        lock.unlock();
        locked = false;
        uint8_t* io = nullptr;
        check(cudaMallocAsync(reinterpret_cast<void**>(&io), need, copy_in), "cudaMallocAsync");
        const size_t words = size_t(r->n) * plan->host.limbs, slot = need / 3;
        uint32_t* d_a = reinterpret_cast<uint32_t*>(io);
        uint32_t* d_b = reinterpret_cast<uint32_t*>(io + slot);
        uint32_t* d_c = reinterpret_cast<uint32_t*>(io + 2 * slot);
        check(cudaMemcpyAsync(d_a, r->a, words * 4, cudaMemcpyHostToDevice, copy_in), "copy a");
        check(cudaMemcpyAsync(d_b, r->b, words * 4, cudaMemcpyHostToDevice, copy_in), "copy b");
        check(cudaEventRecord(r->copied_in, copy_in), "cudaEventRecord");
        check(cudaStreamWaitEvent(compute, r->copied_in, 0), "cudaStreamWaitEvent");
        // only this thread binds plans; kernel arguments are copied at launch
        const std::string why = bind_work(*plan, work);
        if (!why.empty()) throw CudaError{cudaErrorInvalidValue, "bind_work"};
        r->status_slot = uint32_t(r->id % kStatusSlots);
        check(cudaMemsetAsync(plan->status, 0, sizeof(uint32_t), compute), "cudaMemsetAsync");
        enqueue_device_product(*plan, d_a, d_b, d_c, compute);
        check(cudaMemcpyAsync(status_host + r->status_slot, plan->status, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                              compute),
              "status word");
        check(cudaEventRecord(r->computed, compute), "cudaEventRecord");
        check(cudaStreamWaitEvent(copy_out, r->computed, 0), "cudaStreamWaitEvent");
        check(cudaMemcpyAsync(r->c, d_c, words * 4, cudaMemcpyDeviceToHost, copy_out), "copy c");
        check(cudaFreeAsync(io, copy_out), "cudaFreeAsync");
        check(cudaLaunchHostFunc(copy_out, &negacyclic_server::on_done, r), "cudaLaunchHostFunc");
    } catch (const CudaError& e) {
        error = std::string(e.where) + ": " + cudaGetErrorString(e.code);
        cudaGetLastError();
    }
    if (!locked) lock.lock();
    if (!error.empty()) {  // nothing was left on the stream that calls back
        in_flight -= need;
        --active;
        fail_head(r, NEGACYCLIC_ECUDA, error);
    }
    return true;
}

void negacyclic_server::run() {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lock(mu);
    while (!stopping) {
        bool progress = false;
        while (admit_one(lock)) progress = true;
        if (!progress) wake.wait_for(lock, std::chrono::milliseconds(2));
    }
}

extern "C" {

int negacyclic_server_create(const negacyclic_server_options* opts, negacyclic_server** out) {
    if (!out) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    *out = nullptr;
    negacyclic_server_options o{};
    o.device = -1;
    if (opts) o = *opts;
    int device = o.device;
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) return fail(NEGACYCLIC_ENODEV, "no CUDA device");
    auto s = std::make_unique<negacyclic_server>();
    s->device = device;
    s->budget = o.hbm_budget ? o.hbm_budget : (uint64_t(60) << 30);
    s->slots = o.slots ? o.slots : 4;
    s->max_queue = o.max_queue;
    if (s->slots > negacyclic_server::kStatusSlots) return fail(NEGACYCLIC_EINVAL, "at most 1024 slots");
    DeviceGuard guard(device);
    try {
        for (cudaStream_t* st : {&s->copy_in, &s->compute, &s->copy_out})
            check(cudaStreamCreateWithFlags(st, cudaStreamNonBlocking), "cudaStreamCreate");
        check(cudaHostAlloc(reinterpret_cast<void**>(&s->status_host), negacyclic_server::kStatusSlots * sizeof(uint32_t),
                            cudaHostAllocDefault),
              "cudaHostAlloc");
        // keep freed request memory in the pool up to the budget instead of returning it
        cudaMemPool_t pool = nullptr;
        check(cudaDeviceGetDefaultMemPool(&pool, device), "cudaDeviceGetDefaultMemPool");
        uint64_t threshold = s->budget;
        check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold), "cudaMemPoolSetAttribute");
    } catch (const CudaError& e) {
        for (cudaStream_t st : {s->copy_in, s->compute, s->copy_out})
            if (st) cudaStreamDestroy(st);
        if (s->status_host) cudaFreeHost(s->status_host);
        return cuda_failure(e);
    }
    negacyclic_server* raw = s.release();
    raw->dispatcher = std::thread([raw] { raw->run(); });
    *out = raw;
    return NEGACYCLIC_OK;
}

int negacyclic_server_open_session(negacyclic_server* s, uint32_t w, uint32_t limbs, const uint32_t* q,
                                   const uint32_t* ns, uint32_t count, uint32_t* session) {
    if (!s || !q || !session) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    if (limbs != (w + 31) / 32) return fail(NEGACYCLIC_EINVAL, "invalid point: L must equal (W + 31) / 32");
    DeviceGuard guard(s->device);
    uint32_t id = 0;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        Session sess;
        sess.w = w;
        sess.limbs = limbs;
        sess.q.assign(q, q + limbs);
        s->sessions.push_back(std::move(sess));
        id = uint32_t(s->sessions.size() - 1);
    }
    for (uint32_t i = 0; ns && i < count; ++i) {  // resident plans for the announced ring sizes
        negacyclic_plan* plan = nullptr;
        int status = build_session_plan(s->device, w, limbs, q, ns[i], &plan);
        if (status != NEGACYCLIC_OK) return status;
        std::lock_guard<std::mutex> lock(s->mu);
        negacyclic_plan* installed = nullptr;
        status = install_plan(*s, s->sessions[id], ns[i], plan, &installed);
        if (status != NEGACYCLIC_OK) return status;
    }
    *session = id;
    return NEGACYCLIC_OK;
}

int negacyclic_server_submit(negacyclic_server* s, uint32_t session, uint32_t n, const uint32_t* a,
                             const uint32_t* b, uint32_t* c, uint64_t* request) {
    if (!s || !a || !b || !c || !request) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    if (session >= s->sessions.size()) return fail(NEGACYCLIC_EINVAL, "unknown session");
    if (s->max_queue && s->pending.size() >= s->max_queue) {
        ++s->rejected;
        return fail(NEGACYCLIC_EBUSY, "request queue full");
    }
    auto r = std::make_unique<Request>();
    r->id = s->next_id++;
    r->session = session;
    r->n = n;
    r->a = a;
    r->b = b;
    r->c = c;
    r->server = s;
    r->submitted = now_ms();
    if (s->first_submit == 0) s->first_submit = r->submitted;
    *request = r->id;
    s->pending.push_back(r.get());
    s->max_queued = std::max<uint64_t>(s->max_queued, s->pending.size());
    s->requests.emplace(r->id, std::move(r));
    s->wake.notify_one();
    return NEGACYCLIC_OK;
}

int negacyclic_server_wait(negacyclic_server* s, uint64_t request, double timeout_ms, double* latency_ms) {
    if (!s) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->requests.find(request);
    if (it == s->requests.end()) return fail(NEGACYCLIC_EINVAL, "unknown request");
    Request* r = it->second.get();
    const auto deadline = std::chrono::steady_clock::now() +
                          std::chrono::microseconds(int64_t((timeout_ms > 0 ? timeout_ms : 1e9) * 1000));
    while (!r->done)
        if (s->finished.wait_until(lock, deadline) == std::cv_status::timeout && !r->done)
            return fail(NEGACYCLIC_ECUDA, "request did not finish in time");
    if (latency_ms) *latency_ms = r->finished - r->submitted;
    const int status = r->status;
    const std::string error = r->error;
    s->requests.erase(it);
    if (status != NEGACYCLIC_OK) return fail(status, error);
    return NEGACYCLIC_OK;
}

int negacyclic_server_get_stats(negacyclic_server* s, negacyclic_server_stats* out) {
    if (!s || !out) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    *out = negacyclic_server_stats{};
    out->completed = s->completed;
    out->failed = s->failed;
    out->queued = s->pending.size();
    out->resident_bytes = s->resident + s->arena_bytes;
    out->in_flight_bytes = s->in_flight;
    out->rejected = s->rejected;
    out->max_queued = s->max_queued;
    std::vector<double> lat = s->latencies;
    if (!lat.empty()) {
        std::sort(lat.begin(), lat.end());
        auto at = [&](double f) { return lat[std::min(lat.size() - 1, size_t(f * (lat.size() - 1) + 0.5))]; };
        out->p50_ms = at(0.50);
        out->p99_ms = at(0.99);
        double sum = 0;
        for (double x : lat) sum += x;
        out->mean_ms = sum / lat.size();
        const double span = s->last_finish - s->first_submit;
        out->products_per_s = span > 0 ? 1000.0 * lat.size() / span : 0;
    }
    return NEGACYCLIC_OK;
}

void negacyclic_server_free(negacyclic_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stopping = true;
        s->wake.notify_all();
    }
    if (s->dispatcher.joinable()) s->dispatcher.join();
    {
        int previous = 0;
        cudaGetDevice(&previous);
        cudaSetDevice(s->device);
        for (cudaStream_t st : {s->copy_in, s->compute, s->copy_out})
            if (st) cudaStreamSynchronize(st);
        if (s->arena) cudaFree(s->arena);
        if (s->status_host) cudaFreeHost(s->status_host);
        for (cudaEvent_t e : s->all_events) cudaEventDestroy(e);
        for (cudaStream_t st : {s->copy_in, s->compute, s->copy_out})
            if (st) cudaStreamDestroy(st);
        cudaSetDevice(previous);
    }
    delete s;
}

}  // extern "C"
