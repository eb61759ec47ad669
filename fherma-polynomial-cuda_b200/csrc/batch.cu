// Batched form: many products of uneven (N, L, q) in one graph-captured launch.
//
// The reference runs one product per harness call (src/main.cpp:164-204) and has
// no batched form; this is new work on top of the same per-product pipeline.
//
//   * one plan per instance (parameter tables resident), work space external;
//   * an autotuner picks, per shape (N, L), the ring split s (which sets the NTT
//     length N' = N/s and the prime set) and the GEMM kernel (CTA-pair 256x256
//     tiles, single-CTA 128x256 tiles, or the SIMT kernel) by timing each
//     candidate on the device; results are cached in a text file;
//   * by default the batch runs in two phases. Small instances (a tuned or estimated
//     device time under kSmallMs) run first, concurrently, assigned longest-first to
//     kSmallLanes compute streams with single-CTA tensor GEMMs: a small product
//     leaves most of the GPU idle between its short kernels, and other instances'
//     kernels fill those gaps. The large instances then run one after another on
//     lane 0 with the CTA-pair GEMM, which fills the GPU by itself and never shares
//     it with another kernel (several cluster kernels resident at once stalled);
//   * `lanes` > 0 instead assigns every instance longest-first to that many lanes
//     (single-CTA GEMMs when more than one);
//   * each lane owns one work arena (sized for its largest instance, lane 0's for the
//     large phase too) that its instances use one after another;
//   * the whole batch — every lane's chain of products — is captured once into a
//     CUDA graph, so a batch run is a single cudaGraphLaunch;
//   * with host arrays, operand copies run on a copy-in stream and result copies
//     on a copy-out stream, so instance i's compute overlaps the copy-in of the
//     instances after it and the copy-out of those before it;
//   * each instance has a device status word (NEGACYCLIC_STATUS_*) in one array, cleared at
//     the start of every run: the blocking host form checks it before returning, and
//     negacyclic_batch_status reads it after a device run.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "plan_internal.h"

using namespace negacyclic;
using namespace negacyclic::detail;

namespace {

struct TuneChoice {
    uint32_t split = 0;  // 0 = automatic
    uint32_t gemm = NEGACYCLIC_GEMM_AUTO;
    double ms = 0;  // measured device time of one product (0 = not measured)
};

using ShapeKey = std::pair<uint32_t, uint32_t>;  // (N, L)

std::mutex g_cache_mutex;

std::map<ShapeKey, TuneChoice> load_cache(const std::string& path) {
    std::map<ShapeKey, TuneChoice> cache;
    if (path.empty()) return cache;
    std::ifstream in(path);
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream fields(line);
        uint32_t n = 0, limbs = 0;
        TuneChoice c;
        if (fields >> n >> limbs >> c.split >> c.gemm >> c.ms) cache[{n, limbs}] = c;
    }
    return cache;
}

void save_cache(const std::string& path, const std::map<ShapeKey, TuneChoice>& cache) {
    if (path.empty()) return;
    std::ofstream out(path, std::ios::trunc);
    out.precision(17);
    out << "# N L split gemm ms  (negacyclic batch autotuner)\n";
    for (const auto& [key, c] : cache)
        out << key.first << ' ' << key.second << ' ' << c.split << ' ' << c.gemm << ' ' << c.ms << '\n';
}

// Device time of one product for a plan (operands uninitialised: the arithmetic
// is data-independent apart from the rare final corrections).
double time_plan(negacyclic_plan& plan, int repeats) {
    const HostPlan& h = plan.host;
    const size_t words = size_t(h.n) * h.limbs;
    uint32_t* io = nullptr;
    check(cudaMalloc(&io, 3 * words * sizeof(uint32_t)), "cudaMalloc");
    check(cudaMemset(io, 0x5a, 3 * words * sizeof(uint32_t)), "cudaMemset");
    cudaEvent_t start = nullptr, stop = nullptr;
    check(cudaEventCreate(&start), "cudaEventCreate");
    check(cudaEventCreate(&stop), "cudaEventCreate");
    cudaStream_t st = plan.stream;
    enqueue_device_product(plan, io, io + words, io + 2 * words, st);  // warm-up
    check(cudaEventRecord(start, st), "cudaEventRecord");
    for (int i = 0; i < repeats; ++i) enqueue_device_product(plan, io, io + words, io + 2 * words, st);
    check(cudaEventRecord(stop, st), "cudaEventRecord");
    check(cudaEventSynchronize(stop), "tuning products");
    float ms = 0;
    check(cudaEventElapsedTime(&ms, start, stop), "cudaEventElapsedTime");
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
    cudaFree(io);
    return double(ms) / repeats;
}

// Candidate (split, gemm) pairs for a shape, timed with the instance's own q.
TuneChoice tune_shape(const negacyclic_point& point, int device) {
    std::vector<uint32_t> splits;
    {
        HostPlan probe;
        std::string error;
        int status = 0;
        if (!build_host_plan(point.n, point.limbs, point.q, 0, probe, error, status)) return TuneChoice{};
        splits.push_back(probe.split);
        const uint32_t wider = probe.split * 2;
        if (wider <= kMaxSplit && point.n / wider >= 256) splits.push_back(wider);
    }
    TuneChoice best;
    for (uint32_t split : splits) {
        for (uint32_t gemm : {uint32_t(NEGACYCLIC_GEMM_AUTO), uint32_t(NEGACYCLIC_GEMM_TENSOR_SINGLE),
                              uint32_t(NEGACYCLIC_GEMM_SIMT)}) {
            // the SIMT GEMM only competes on small shapes: skip it where tensor cores apply
            if (gemm == NEGACYCLIC_GEMM_SIMT && best.ms > 0 && uint64_t(point.n) * point.limbs > (1u << 16)) continue;
            negacyclic_options o{};
            o.split = split;
            o.gemm = gemm;
            o.device = device;
            negacyclic_plan* plan = nullptr;
            if (negacyclic_init(point.n, point.w, point.limbs, point.q, &o, &plan) != NEGACYCLIC_OK) continue;
            std::unique_ptr<negacyclic_plan> owner(plan);
            double ms = 0;
            try {
                ms = time_plan(*plan, 3);
            } catch (const CudaError&) {
                cudaGetLastError();
                continue;
            }
            if (best.ms == 0 || ms < best.ms) best = TuneChoice{split, gemm, ms};
        }
    }
    return best;
}

// Rough device time of one product, for balancing lanes when nothing was measured.
double estimate_ms(const negacyclic_plan& plan) {
    const HostPlan& h = plan.host;
    const double ops = 2.0 * (2.0 * h.n) * (4.0 * h.limbs) * (4.0 * plan.r) + 2.0 * h.n * (4.0 * plan.r) * (4.0 * h.words);
    const double bytes = 16.0 * plan.r * double(h.n) * 4;
    return ops / 2.0e15 * 1e3 + bytes / 4.0e12 * 1e3 + 0.05;
}

}  // namespace

// Automatic lanes: instances under kSmallMs of device time share the GPU on kSmallLanes streams.
constexpr double kSmallMs = 1.0;
constexpr uint32_t kSmallLanes = 4;

struct negacyclic_batch {
    int device = 0;
    std::vector<std::unique_ptr<negacyclic_plan>> plans;
    std::vector<TuneChoice> choices;
    std::vector<uint32_t> lane_of;
    std::vector<std::vector<uint32_t>> lane_order;  // the concurrent phase, per lane
    std::vector<uint32_t> large;                    // the sequential phase (lane 0), in order
    std::vector<cudaStream_t> lanes;
    std::vector<void*> arenas;
    void* io = nullptr;
    uint32_t* status = nullptr;     // [count] status words, one per instance
    std::vector<size_t> io_offset;  // a, then b, then c per instance
    cudaStream_t capture = nullptr, copy_in = nullptr, copy_out = nullptr;
    std::vector<cudaEvent_t> copied_in, computed;  // per instance, host-array runs
    cudaEvent_t fork = nullptr, phase = nullptr;
    std::vector<cudaEvent_t> joins;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;

    ~negacyclic_batch() {
        int previous = 0;
        cudaGetDevice(&previous);
        cudaSetDevice(device);
        cudaDeviceSynchronize();
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (cudaEvent_t e : joins) cudaEventDestroy(e);
        for (cudaEvent_t e : copied_in) cudaEventDestroy(e);
        for (cudaEvent_t e : computed) cudaEventDestroy(e);
        if (copy_in) cudaStreamDestroy(copy_in);
        if (copy_out) cudaStreamDestroy(copy_out);
        if (fork) cudaEventDestroy(fork);
        if (phase) cudaEventDestroy(phase);
        for (cudaStream_t s : lanes) cudaStreamDestroy(s);
        if (capture) cudaStreamDestroy(capture);
        for (void* a : arenas) cudaFree(a);
        if (io) cudaFree(io);
        if (status) cudaFree(status);
        plans.clear();
        cudaSetDevice(previous);
    }

    size_t words(uint32_t i) const { return size_t(plans[i]->host.n) * plans[i]->host.limbs; }
    uint32_t* slot(uint32_t i, uint32_t which) const {
        return reinterpret_cast<uint32_t*>(static_cast<uint8_t*>(io) + io_offset[3 * i + which]);
    }
};

extern "C" {

int negacyclic_batch_create(const negacyclic_point* points, uint32_t count, const negacyclic_batch_options* opts,
                            negacyclic_batch** out) {
    if (!points || !count || !out) return fail(NEGACYCLIC_EINVAL, "NULL or empty batch");
    *out = nullptr;
    negacyclic_batch_options o{};
    o.device = -1;
    if (opts) o = *opts;
    int device = o.device;
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) return fail(NEGACYCLIC_ENODEV, "no CUDA device");
    auto b = std::make_unique<negacyclic_batch>();
    b->device = device;
    DeviceGuard guard(device);
    const std::string cache_path = o.tune_cache ? o.tune_cache : (getenv("NEGACYCLIC_TUNE_CACHE") ? getenv("NEGACYCLIC_TUNE_CACHE") : "");
    try {
        // 1. choices per shape (tuned or cached), then one plan per instance
        std::map<ShapeKey, TuneChoice> cache;
        {
            std::lock_guard<std::mutex> lock(g_cache_mutex);
            cache = load_cache(cache_path);
        }
        bool cache_dirty = false;
        b->choices.resize(count);
        for (uint32_t i = 0; i < count; ++i) {
            const ShapeKey key{points[i].n, points[i].limbs};
            auto it = cache.find(key);
            if (it == cache.end() && o.tune) {
                TuneChoice c = tune_shape(points[i], device);
                it = cache.emplace(key, c).first;
                cache_dirty = true;
            }
            b->choices[i] = it == cache.end() ? TuneChoice{} : it->second;
            negacyclic_options po{};
            po.split = b->choices[i].split;
            po.gemm = b->choices[i].gemm;
            po.device = device;
            po.external_work = 1;
            negacyclic_plan* plan = nullptr;
            int status = negacyclic_init(points[i].n, points[i].w, points[i].limbs, points[i].q, &po, &plan);
            if (status != NEGACYCLIC_OK && (po.split || po.gemm)) {  // a stale cache entry: fall back to defaults
                po.split = 0;
                po.gemm = NEGACYCLIC_GEMM_AUTO;
                b->choices[i] = TuneChoice{};
                status = negacyclic_init(points[i].n, points[i].w, points[i].limbs, points[i].q, &po, &plan);
            }
            if (status != NEGACYCLIC_OK)
                return fail(status, "batch instance " + std::to_string(i) + ": " + negacyclic_last_error());
            b->plans.emplace_back(plan);
        }
        if (cache_dirty) {
            std::lock_guard<std::mutex> lock(g_cache_mutex);
            save_cache(cache_path, cache);
        }

        // 2. lanes: longest-first assignment of the concurrent phase's instances
        std::vector<double> cost(count);
        for (uint32_t i = 0; i < count; ++i)
            cost[i] = b->choices[i].ms > 0 ? b->choices[i].ms : estimate_ms(*b->plans[i]);
        std::vector<uint32_t> order(count);
        std::iota(order.begin(), order.end(), 0u);
        std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return cost[x] > cost[y]; });
        std::vector<uint32_t> concurrent;
        if (o.lanes) {
            concurrent = order;  // every instance shares the lanes the caller asked for
        } else {
            for (uint32_t i : order) (cost[i] < kSmallMs ? concurrent : b->large).push_back(i);
        }
        const uint32_t lanes = o.lanes ? std::min(o.lanes, count)
                                       : std::max(1u, std::min<uint32_t>(kSmallLanes, uint32_t(concurrent.size())));
        // Products on several lanes run concurrently: they use the single-CTA tensor-core kernel,
        // because concurrent launches of the CTA-pair (cluster) kernel from several streams stalled.
        if (lanes > 1)
            for (uint32_t i : concurrent) b->plans[i]->gemm_pairs_allowed = false;
        std::vector<double> load(lanes, 0.0);
        b->lane_of.assign(count, 0);
        b->lane_order.assign(lanes, {});
        for (uint32_t i : concurrent) {
            const uint32_t lane = uint32_t(std::min_element(load.begin(), load.end()) - load.begin());
            load[lane] += cost[i];
            b->lane_of[i] = lane;
            b->lane_order[lane].push_back(i);
        }

        // 3. device memory: one work arena per lane (lane 0's also serves the sequential phase),
        // one I/O arena for every instance
        b->lanes.resize(lanes);
        b->arenas.assign(lanes, nullptr);
        for (uint32_t lane = 0; lane < lanes; ++lane) {
            check(cudaStreamCreateWithFlags(&b->lanes[lane], cudaStreamNonBlocking), "cudaStreamCreate");
            std::vector<uint32_t> users = b->lane_order[lane];
            if (lane == 0) users.insert(users.end(), b->large.begin(), b->large.end());
            size_t need = 256;
            for (uint32_t i : users) need = std::max(need, b->plans[i]->work_bytes);
            check(cudaMalloc(&b->arenas[lane], need), "cudaMalloc");
            for (uint32_t i : users) {
                const std::string why = bind_work(*b->plans[i], b->arenas[lane]);
                if (!why.empty()) return fail(NEGACYCLIC_EINVAL, why);
            }
        }
        size_t io_bytes = 0;
        b->io_offset.resize(3 * size_t(count));
        for (uint32_t i = 0; i < count; ++i)
            for (uint32_t which = 0; which < 3; ++which) {
                b->io_offset[3 * i + which] = io_bytes;
                io_bytes += (b->words(i) * 4 + 255) / 256 * 256;
            }
        check(cudaMalloc(&b->io, io_bytes), "cudaMalloc");
        check(cudaMemset(b->io, 0, io_bytes), "cudaMemset");
        check(cudaMalloc(&b->status, size_t(count) * sizeof(uint32_t)), "cudaMalloc");
        check(cudaMemset(b->status, 0, size_t(count) * sizeof(uint32_t)), "cudaMemset");
        for (uint32_t i = 0; i < count; ++i) b->plans[i]->status = b->status + i;
        check(cudaStreamCreateWithFlags(&b->copy_in, cudaStreamNonBlocking), "cudaStreamCreate");
        check(cudaStreamCreateWithFlags(&b->copy_out, cudaStreamNonBlocking), "cudaStreamCreate");
        b->copied_in.resize(count);
        b->computed.resize(count);
        for (uint32_t i = 0; i < count; ++i) {
            check(cudaEventCreateWithFlags(&b->copied_in[i], cudaEventDisableTiming), "cudaEventCreate");
            check(cudaEventCreateWithFlags(&b->computed[i], cudaEventDisableTiming), "cudaEventCreate");
        }

        // 4. capture every lane's chain of products into one graph
        check(cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking), "cudaStreamCreate");
        check(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "cudaEventCreate");
        check(cudaEventCreateWithFlags(&b->phase, cudaEventDisableTiming), "cudaEventCreate");
        b->joins.resize(lanes);
        for (auto& e : b->joins) check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
        check(cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        try {
            check(cudaMemsetAsync(b->status, 0, b->plans.size() * sizeof(uint32_t), b->capture), "cudaMemsetAsync");
            check(cudaEventRecord(b->fork, b->capture), "cudaEventRecord");
            for (uint32_t lane = 0; lane < lanes; ++lane) {
                check(cudaStreamWaitEvent(b->lanes[lane], b->fork, 0), "cudaStreamWaitEvent");
                for (uint32_t i : b->lane_order[lane])
                    enqueue_device_product(*b->plans[i], b->slot(i, 0), b->slot(i, 1), b->slot(i, 2), b->lanes[lane]);
                check(cudaEventRecord(b->joins[lane], b->lanes[lane]), "cudaEventRecord");
                check(cudaStreamWaitEvent(b->capture, b->joins[lane], 0), "cudaStreamWaitEvent");
            }
            // the sequential phase, on lane 0 once every lane has finished
            if (!b->large.empty()) {
                check(cudaEventRecord(b->phase, b->capture), "cudaEventRecord");
                check(cudaStreamWaitEvent(b->lanes[0], b->phase, 0), "cudaStreamWaitEvent");
                for (uint32_t i : b->large)
                    enqueue_device_product(*b->plans[i], b->slot(i, 0), b->slot(i, 1), b->slot(i, 2), b->lanes[0]);
                check(cudaEventRecord(b->joins[0], b->lanes[0]), "cudaEventRecord");
                check(cudaStreamWaitEvent(b->capture, b->joins[0], 0), "cudaStreamWaitEvent");
            }
        } catch (...) {
            cudaGraph_t abandoned = nullptr;
            cudaStreamEndCapture(b->capture, &abandoned);
            if (abandoned) cudaGraphDestroy(abandoned);
            throw;
        }
        check(cudaStreamEndCapture(b->capture, &b->graph), "cudaStreamEndCapture");
        check(cudaGraphInstantiate(&b->exec, b->graph, 0), "cudaGraphInstantiate");
        check(cudaGraphUpload(b->exec, b->capture), "cudaGraphUpload");
        check(cudaStreamSynchronize(b->capture), "cudaGraphUpload");
    } catch (const CudaError& e) {
        cudaGetLastError();
        return e.code == cudaErrorMemoryAllocation ? fail(NEGACYCLIC_ENOMEM, "device allocation failed")
                                                   : cuda_failure(e);
    }
    *out = b.release();
    return NEGACYCLIC_OK;
}

int negacyclic_batch_io(negacyclic_batch* b, uint32_t index, uint32_t** d_a, uint32_t** d_b, uint32_t** d_c) {
    if (!b || index >= b->plans.size()) return fail(NEGACYCLIC_EINVAL, "bad batch index");
    if (d_a) *d_a = b->slot(index, 0);
    if (d_b) *d_b = b->slot(index, 1);
    if (d_c) *d_c = b->slot(index, 2);
    return NEGACYCLIC_OK;
}

int negacyclic_batch_get_info(const negacyclic_batch* b, uint32_t index, negacyclic_batch_instance* info) {
    if (!b || !info || index >= b->plans.size()) return fail(NEGACYCLIC_EINVAL, "bad batch index");
    *info = negacyclic_batch_instance{};
    negacyclic_get_info(b->plans[index].get(), &info->plan);
    info->lane = b->lane_of[index];
    info->phase = std::find(b->large.begin(), b->large.end(), index) != b->large.end() ? 1u : 0u;
    info->tuned_ms = b->choices[index].ms;
    info->requested_gemm = b->choices[index].gemm;
    return NEGACYCLIC_OK;
}

int negacyclic_batch_run_device(negacyclic_batch* b, void* stream) {
    if (!b) return fail(NEGACYCLIC_EINVAL, "NULL batch");
    DeviceGuard guard(b->device);
    const cudaError_t e = cudaGraphLaunch(b->exec, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(NEGACYCLIC_ECUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
    return NEGACYCLIC_OK;
}

int negacyclic_batch_run_one(negacyclic_batch* b, uint32_t index, void* stream) {
    if (!b || index >= b->plans.size()) return fail(NEGACYCLIC_EINVAL, "bad batch index");
    DeviceGuard guard(b->device);
    try {
        enqueue_device_product(*b->plans[index], b->slot(index, 0), b->slot(index, 1), b->slot(index, 2),
                               static_cast<cudaStream_t>(stream));
    } catch (const CudaError& e) {
        return cuda_failure(e);
    }
    return NEGACYCLIC_OK;
}

int negacyclic_batch_run(negacyclic_batch* b, const uint32_t* const* a, const uint32_t* const* bb, uint32_t* const* c) {
    if (!b || !a || !bb || !c) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    DeviceGuard guard(b->device);
    try {
        // issue order: round-robin over the concurrent lanes' sequences, so every lane gets work
        // early, then the sequential phase
        std::vector<uint32_t> order;
        std::vector<size_t> next(b->lanes.size(), 0);
        size_t concurrent = 0;
        for (const auto& lane : b->lane_order) concurrent += lane.size();
        while (order.size() < concurrent)
            for (uint32_t lane = 0; lane < b->lanes.size(); ++lane)
                if (next[lane] < b->lane_order[lane].size()) order.push_back(b->lane_order[lane][next[lane]++]);
        order.insert(order.end(), b->large.begin(), b->large.end());
        // copy-in -> compute (the instance's lane) -> copy-out, linked by events; every lane's first
        // product waits for a copy-in event recorded after the status words are cleared; the first
        // product of the sequential phase also waits for every lane's last concurrent product
        check(cudaMemsetAsync(b->status, 0, b->plans.size() * sizeof(uint32_t), b->copy_in), "cudaMemsetAsync");
        for (size_t at = 0; at < order.size(); ++at) {
            const uint32_t i = order[at];
            const size_t bytes = b->words(i) * 4;
            check(cudaMemcpyAsync(b->slot(i, 0), a[i], bytes, cudaMemcpyHostToDevice, b->copy_in), "copy a");
            check(cudaMemcpyAsync(b->slot(i, 1), bb[i], bytes, cudaMemcpyHostToDevice, b->copy_in), "copy b");
            check(cudaEventRecord(b->copied_in[i], b->copy_in), "cudaEventRecord");
            cudaStream_t lane = b->lanes[b->lane_of[i]];
            if (at == concurrent && concurrent > 0)
                for (uint32_t other = 1; other < b->lanes.size(); ++other) {
                    check(cudaEventRecord(b->joins[other], b->lanes[other]), "cudaEventRecord");
                    check(cudaStreamWaitEvent(lane, b->joins[other], 0), "cudaStreamWaitEvent");
                }
            check(cudaStreamWaitEvent(lane, b->copied_in[i], 0), "cudaStreamWaitEvent");
            enqueue_device_product(*b->plans[i], b->slot(i, 0), b->slot(i, 1), b->slot(i, 2), lane);
            check(cudaEventRecord(b->computed[i], lane), "cudaEventRecord");
            check(cudaStreamWaitEvent(b->copy_out, b->computed[i], 0), "cudaStreamWaitEvent");
            check(cudaMemcpyAsync(c[i], b->slot(i, 2), bytes, cudaMemcpyDeviceToHost, b->copy_out), "copy c");
        }
        check(cudaStreamSynchronize(b->copy_out), "batch");
        for (cudaStream_t st : b->lanes) check(cudaStreamSynchronize(st), "batch");
        std::vector<uint32_t> flags(b->plans.size());
        check(cudaMemcpy(flags.data(), b->status, flags.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost),
              "status words");
        for (uint32_t i = 0; i < flags.size(); ++i)
            if (flags[i]) return status_failure(flags[i], "batch instance " + std::to_string(i));
    } catch (const CudaError& e) {
        return cuda_failure(e);
    }
    return NEGACYCLIC_OK;
}

int negacyclic_batch_status(negacyclic_batch* b, uint32_t* flags) {
    if (!b || !flags) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    DeviceGuard guard(b->device);
    const size_t bytes = b->plans.size() * sizeof(uint32_t);
    if (cudaDeviceSynchronize() != cudaSuccess || cudaMemcpy(flags, b->status, bytes, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemset(b->status, 0, bytes) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
        return fail(NEGACYCLIC_ECUDA, cudaGetErrorString(cudaGetLastError()));
    return NEGACYCLIC_OK;
}

int negacyclic_batch_run_plain(negacyclic_batch* b, const uint32_t* const* a, const uint32_t* const* bb,
                               uint32_t* const* c) {
    if (!b || !a || !bb || !c) return fail(NEGACYCLIC_EINVAL, "NULL argument");
    for (uint32_t i = 0; i < b->plans.size(); ++i) {
        const int status = negacyclic_run(b->plans[i].get(), a[i], bb[i], c[i]);
        if (status != NEGACYCLIC_OK) return status;
    }
    return NEGACYCLIC_OK;
}

void negacyclic_batch_free(negacyclic_batch* b) { delete b; }

}  // extern "C"
