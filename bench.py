"""Benchmark: exact negacyclic products per second at N=65536, L=1747 limbs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One step = one product c = a*b mod (X^65536+1, q), q a 55904-bit random odd
modulus (1747 limbs), a and b uniform in [0, q) (seeded synthetic inputs, 458 MB
per operand: every step reads inputs larger than the 126 MB L2).

  value     products/s, device-resident: operands already in HBM, K products
            through negacyclic_run_device, CUDA events on the launching stream
  e2e       products/s through negacyclic_run (the host-facing C ABI) with pinned
            host buffers: H2D of a and b and D2H of c inside the timed region
  batched_e2e  products/s through negacyclic_batch_run: K products (at most 32 GB) of the same
            workload from page-locked host arrays, copies of one product overlapping
            the compute of the next (plain_value = e2e, one product per call)
  e2e_fherma_run  the same metric through fherma_run exactly as the platform harness
            calls it: pageable std::vectors in and a freshly allocated output vector
            (fherma-polynomial-cuda_b200/fherma_timer, steady_clock around each call)
  config2   N=32768, L=868 (q from seed 1): 20 seeded instances, device-resident and
            end to end (page-locked host buffers)
  roofline  the conversion GEMM (the largest kernel): algorithmic int8 ops per
            launch / its CUDA-event time, against the int8 tensor peak (2 x the
            measured burst bf16 figure; the sustained figure beside it)
  refpoints the reference's own points (N=65536, W=1747 bits; N=32768, W=868 bits;
            the checker's prime q and its 20 stress seeds): per-case fherma_run medians
            of the reference's best entries (candidates/ordered-streaming,
            candidates/caller-fused-strips, built for sm_100a) and of this library
            behind the same unmodified harness, all outputs checked against the
            reference checker's hashes
  cpu_baseline  the GMP Kronecker oracle (the reference checker's algorithm) on a
            bounded sample (N/16 coefficients, same q width), scaled to one product by
            the full-size/sample time ratio measured once on the GPU box's host
            (--mode cpu-calibrate)

Multi-GPU: one independent product stream per GPU (replicas, weak scaling),
barrier + synchronize around the timed region, max time over ranks. Under
torchrun the ranks come from its environment; `--gpus N` without it relaunches
this script under torch.distributed.run with N ranks.
--impl reference times the reference's CPU path (the oracle port, all host
cores, one independent sample per core) on the same workload.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
PACKAGE_DIR = os.path.join(REPO, "fherma-polynomial-cuda_b200")

N, LIMBS, SEED = 65536, 1747, 2
METRIC = "products/s at N=65536,W=1747 (limbs)"
WORKLOAD = "negacyclic product N=65536, L=1747 limbs (55904-bit random odd q, seed 2), a,b uniform in [0,q)"
CPU_SAMPLE_N = N // 16  # bounded CPU sample: 4096 coefficients of the same width
# GMP's product is superlinear: one full N=65536, L=1747 Kronecker product against the N=4096
# sample, timed back to back on one core of the GPU box's host (bench.py --mode cpu-calibrate;
# profiles/cpu_baseline_gmp_N65536_L1747.md); without it the linear factor N / CPU_SAMPLE_N is used
CPU_FULL_OVER_SAMPLE = 19.35  # 77.74 s against 4.01 s (median of 3), 16-core Xeon host of a B200 box
# DRAM bytes (read + write) of one conversion-GEMM launch on this workload, from a one-pass ncu
# capture (dram__bytes_read.sum 4.32 GB + dram__bytes_write.sum 1.90 GB) of
#   python bench.py --workload 65536,1747 --steps 1 --warmup 1 --device-only
CONVERT_DRAM_BYTES = 6.22e9
# sm__pipe_tensor_cycles_active of the conversion GEMM alone, from the single-kernel capture
#   ncu --set full --clock-control none -k regex:gemm_tc -c 2 \
#       python bench.py --workload 16384,1747 --steps 1 --warmup 1 --device-only
# (profiles/gemm_tc_N16384_L1747.md): the clock-free fraction of the int8 tensor pipe's peak
CONVERT_TENSOR_PIPE_ACTIVE = 0.836


def _load(name, path, package_dir=None):
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, path,
                                                  submodule_search_locations=[package_dir] if package_dir else None)
    module = importlib.util.module_from_spec(spec)
    sys.modules[name] = module
    spec.loader.exec_module(module)
    return module


def load_inputs():
    return _load("fpc_b200_inputs", os.path.join(PACKAGE_DIR, "inputs.py"))


def peaks():
    """(HBM GB/s, bf16 dense TF/s burst, bf16 dense TF/s sustained, source). The timed loop of
    products lasts well under a second, so the burst GEMM figure is the roofline's peak; the
    sustained one (seconds at the 1 kW power cap) is reported beside it."""
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
        return (data["hbm_gbs"], data["bf16_tflops"], data.get("bf16_tflops_sustained", data["bf16_tflops"]),
                "measured")
    return 6650.0, 1590.0, 1400.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 100 ms while running."""

    FIELDS = ["index", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, gpu: int):
        self.gpu, self.rows, self.proc = gpu, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={','.join(self.FIELDS)}",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            deadline = time.time() + 3.0  # start timing only once samples are flowing
            while not self.rows and time.time() < deadline:
                time.sleep(0.02)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == len(self.FIELDS):
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(self.rows[0][2]) if self.rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(self.rows)}


def cpu_scale():
    """(factor from one sample's time to one full product's, how it was obtained)."""
    if CPU_FULL_OVER_SAMPLE:
        return CPU_FULL_OVER_SAMPLE, f"x{CPU_FULL_OVER_SAMPLE:.2f} (full-size/sample time ratio measured on the GPU box)"
    linear = N / CPU_SAMPLE_N
    return linear, f"x{linear:g} (linear in N; GMP's superlinear product makes this an underestimate)"


def cpu_sample_seconds(sample_n: int, index: int = 0) -> float:
    """One oracle product on the bounded sample (same q width, sample_n coefficients)."""
    oracle = _load("negacyclic_oracle", os.path.join(REPO, "oracle", "oracle.py"))
    inputs = load_inputs()
    q, a, b = inputs.instance(sample_n, LIMBS, SEED, 1000 + index)
    start = time.perf_counter()
    oracle.kronecker(q, a, b)
    return time.perf_counter() - start


def _cpu_worker(args):
    sample_n, index = args
    return cpu_sample_seconds(sample_n, index)


def distributed():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(x: float, world: int, device: str = "cpu") -> float:
    """The slowest rank's time: every rank takes part, every rank gets the maximum."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, steps: int, seconds: float) -> float:
    """Whole-job products/s of `world` replicas that each ran `steps` products, timed by the slowest."""
    return world * steps / seconds


def run_reference(args):
    """The reference's CPU path (GMP Kronecker, restated) on all host cores."""
    world, rank, _ = distributed()
    if rank != 0:
        return
    import multiprocessing as mp

    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    scale, how = cpu_scale()
    with ctx.Pool(cores) as pool:
        for w in range(args.warmup):
            pool.map(_cpu_worker, [(CPU_SAMPLE_N, w * cores + i) for i in range(cores)])
        start = time.perf_counter()
        per_step = []
        for k in range(args.steps):
            t0 = time.perf_counter()
            pool.map(_cpu_worker, [(CPU_SAMPLE_N, 100 + k * cores + i) for i in range(cores)])
            per_step.append(time.perf_counter() - t0)
        total = time.perf_counter() - start
    # each step: `cores` samples of 1/scale of a product each
    value = args.steps * cores / scale / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "products/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "mpz (GMP integers)",
        "data": "synthetic", "config": {"workload": WORKLOAD, "sample": f"N={CPU_SAMPLE_N} of {N} coefficients"},
        "cpu_baseline": {"value": value, "unit": "products/s", "cores": cores, "kind": "port",
                         "sample": f"{cores} concurrent GMP Kronecker products of N={CPU_SAMPLE_N}, L={LIMBS} per step,"
                                   f" each scaled {how} to one N={N} product", "same_config": False},
        "e2e": {"value": value, "unit": "products/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def path_roofline(n: int, limbs: int, info: dict, stage_ms: dict, product_ms: float, int8_tops: float,
                  hbm_gbs: float) -> dict:
    """Roofline of the whole plain device path: the sum over stages of ops / int8 peak (the two
    GEMMs) or algorithmic bytes / HBM peak (the rest), against the measured time per product."""
    r, padded_r, words = info["primes"], info["padded_primes"], info["words"]
    padded_limbs = (limbs + 31) // 32 * 32
    dots_stride = (words + 7) // 8 * 8
    ops = {"convert": 2.0 * (2 * n) * (4 * limbs) * (4 * r), "crt": 2.0 * n * (4 * r) * (4 * words)}
    hbm_bytes = {
        "pad": 4.0 * 2 * n * (limbs + padded_limbs),      # read a, b; write padded operand rows
        "forward": 4.0 * 2 * 2 * r * n,                   # both operands' residues, in place
        "pointwise": 4.0 * 3 * r * n,                     # read two transform sets, write one
        "inverse": 4.0 * 2 * r * n,                       # in place
        "transpose": 4.0 * (r + padded_r) * n,            # prime-major -> coefficient-major
        "reduce": 8.0 * dots_stride * n + 4.0 * n * limbs,  # word sums in, c out
    }
    stages, roof_total = {}, 0.0
    for name, ms in stage_ms.items():
        if name in ops:
            roof, bound, work = ops[name] / (int8_tops * 1e12) * 1e3, "int8 tensor", ops[name]
        else:
            roof, bound, work = hbm_bytes[name] / (hbm_gbs * 1e9) * 1e3, "hbm", hbm_bytes[name]
        roof_total += roof
        stages[name] = {"ms": round(ms, 4), "roof_ms": round(roof, 4), "bound": bound, "work": work,
                        "frac": round(roof / ms, 3) if ms > 0 else None}
    return {"stages": stages, "roof_ms": round(roof_total, 3), "measured_ms": round(product_ms, 3),
            "measured_over_roof": round(product_ms / roof_total, 3),
            "peaks": {"int8_tops": int8_tops, "hbm_gbs": hbm_gbs}}


def fherma_run_leg(args) -> dict:
    """The headline workload through fherma_run as the platform harness calls it (pageable vectors
    in, a fresh output vector out): fherma-polynomial-cuda_b200/fherma_timer, a separate process."""
    binary = os.path.join(PACKAGE_DIR, "fherma_timer")
    steps = min(args.steps, 5)
    done = subprocess.run([binary, str(N), str(LIMBS), str(SEED), str(steps), "1"], capture_output=True, text=True,
                          timeout=900)
    if done.returncode != 0:
        return {"error": (done.stderr or done.stdout).strip()[-300:]}
    result = json.loads(done.stdout.strip().splitlines()[-1])
    return {"value": 1000.0 / result["median_ms"], "unit": "products/s", "median_ms": result["median_ms"],
            "mean_ms": result["mean_ms"], "min_ms": result["min_ms"], "max_ms": result["max_ms"],
            "calls": result["steps"], "init_s": result["init_s"], "commutes": result["commutes"],
            "api": "fherma_run (include/fherma_b200.h), pageable std::vector operands, fresh output vector per call",
            "h2d_bytes_per_step": 2 * N * LIMBS * 4, "d2h_bytes_per_step": N * LIMBS * 4}


CONFIG2 = (32768, 868, 1, 20)  # N, L, seed of q, instances (operand indices 0..19)


def config2_leg(fpc, torch, args) -> dict:
    """Config 2: N=32768, L=868, q from seed 1, 20 seeded instances: device-resident products/s
    (every product reads another instance's operands) and end to end through negacyclic_run with
    page-locked host buffers (each instance's operands copied into them before its timed call)."""
    n, limbs, seed, count = CONFIG2
    inputs = load_inputs()
    t0 = time.perf_counter()
    instances = [inputs.instance(n, limbs, seed, i) for i in range(count)]
    gen_s = time.perf_counter() - t0
    q = instances[0][0]
    plan = fpc.Plan(n, 32 * limbs, limbs, q)
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    dev = [(torch.from_numpy(a.view(np.int32)).cuda(), torch.from_numpy(b.view(np.int32)).cuda())
           for _, a, b in instances]
    dc = torch.empty_like(dev[0][0])
    for da, db in dev[:3]:  # warm-up
        plan.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), sptr)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    for da, db in dev:
        plan.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), sptr)
    stop.record(stream)
    stop.synchronize()
    device_ms = start.elapsed_time(stop) / count
    status = plan.status()
    del dev
    pa = torch.empty((n, limbs), dtype=torch.int32).pin_memory()
    pb, pc = torch.empty_like(pa).pin_memory(), torch.empty_like(pa).pin_memory()
    ha, hb, hc = (t.numpy().view(np.uint32) for t in (pa, pb, pc))
    ha[:], hb[:] = instances[0][1], instances[0][2]
    plan.run(ha, hb, out=hc)  # warm-up
    calls = []
    for _, a, b in instances:
        ha[:], hb[:] = a, b
        t1 = time.perf_counter()
        plan.run(ha, hb, out=hc)
        calls.append(time.perf_counter() - t1)
    plan.close()
    e2e_ms = 1000 * statistics.median(calls)
    return {"workload": f"N={n}, L={limbs} limbs (27776-bit random odd q, seed {seed}), {count} seeded instances",
            "device": {"value": 1000.0 / device_ms, "unit": "products/s", "ms_per_product": round(device_ms, 4)},
            "e2e": {"value": 1000.0 / e2e_ms, "unit": "products/s", "median_ms": round(e2e_ms, 4),
                    "mean_ms": round(1000 * statistics.mean(calls), 4), "api": "negacyclic_run, page-locked buffers",
                    "h2d_bytes_per_step": 2 * n * limbs * 4, "d2h_bytes_per_step": n * limbs * 4},
            "status_word": status, "generation_s": round(gen_s, 1)}


# The reference's two ranked points (README.md:9-11): N, W bits; the checker's prime q and stress seeds
REF_POINTS = [(65536, 1747), (32768, 868)]
REF_SEEDS = list(range(10001, 10021))  # tools/stress_local.py:16-20: 20 seeds at each ranked point
REF_BINARIES = [("ordered_streaming", "candidates/ordered-streaming (best ranked entry)"),
                ("caller_fused_strips", "candidates/caller-fused-strips (fastest measured entry)"),
                ("harness_b200", "this library: fherma_init/run/free behind the reference's unmodified src/main.cpp")]


def refpoints_leg() -> dict:
    """Per-case fherma_run times of the reference's best entries and of this library, behind the
    same unmodified harness, at the reference's own points; every output checked against the
    reference checker's hashes (tests/golden/reference_points.json)."""
    import hashlib
    import shutil
    import tempfile

    ref_dir = os.path.join(REPO, "oracle", "_ref")
    missing = [name for name, _ in REF_BINARIES if not os.path.exists(os.path.join(ref_dir, name))]
    if missing:
        return {"unavailable": f"not built: {', '.join(missing)} (oracle/build_ref.sh needs the reference sources)"}
    cases = _load("fherma_golden_cases", os.path.join(REPO, "tests", "golden", "cases.py"))
    with open(os.path.join(REPO, "tests", "golden", "reference_points.json")) as f:
        golden = json.load(f)["points"]
    harness = _load("fpc_b200_harness", os.path.join(PACKAGE_DIR, "harness.py"))
    out = {"seeds": f"{REF_SEEDS[0]}..{REF_SEEDS[-1]}", "timing": "steady_clock around fherma_run (src/main.cpp:181-186)",
           "points": []}
    for n, width in REF_POINTS:
        point = next(p for p in golden if p["N"] == n and p["W"] == width and p["kind"] == "stress_pairs")
        q, limbs = int(point["q_hex"], 16), point["L"]
        want = [c["c_sha256"] for c in point["cases"][: len(REF_SEEDS)]]
        pairs = cases.reference_pairs(n, q, REF_SEEDS, False)
        arrays = [(np.frombuffer(cases.pack(a, limbs), "<u4").reshape(n, limbs),
                   np.frombuffer(cases.pack(b, limbs), "<u4").reshape(n, limbs)) for a, b in pairs]
        root = harness.write_point(tempfile.mkdtemp(prefix="refpoint_"), n, width, limbs,
                                   np.frombuffer(q.to_bytes(4 * limbs, "little"), "<u4"), arrays)
        entry = {"N": n, "W_bits": width, "L": limbs}
        try:
            for name, what in REF_BINARIES:
                shutil.rmtree(root / "out", ignore_errors=True)
                done = subprocess.run([os.path.join(ref_dir, name), str(root)], capture_output=True, text=True,
                                      timeout=600)
                result = {"what": what, "rc": done.returncode}
                if done.returncode == 0:
                    results = harness.read_results(root)
                    ms = [1000 * c["seconds"] for c in results["cases"] if c["status"] == "ok"]
                    hashes = [hashlib.sha256((root / "out" / f"{i:06d}" / "c.bin").read_bytes()).hexdigest()
                              for i in range(len(pairs))]
                    result.update(median_ms=round(statistics.median(ms), 4), first_ms=round(ms[0], 4),
                                  median_after_first_ms=round(statistics.median(ms[1:]), 4),
                                  min_ms=round(min(ms), 4), init_s=round(results["init_s"], 3),
                                  cases=len(ms), exact=hashes == want)
                else:
                    result["stderr"] = (done.stderr or done.stdout).strip()[-300:]
                entry[name] = result
        finally:
            shutil.rmtree(root, ignore_errors=True)
        ours, best = entry["harness_b200"], entry["ordered_streaming"]
        if "median_ms" in ours and "median_ms" in best:
            entry["ordered_streaming_over_b200"] = round(best["median_ms"] / ours["median_ms"], 3)
        out["points"].append(entry)
    out["published_ms"] = {"ordered_streaming": {"65536": 1.0712435, "32768": 0.3752785},
                           "source": "candidates/ordered-streaming/official-results.json:29,45 (RTX PRO 6000 Blackwell)"}
    return out


def run_cpu_calibrate(args):
    """One full-size GMP Kronecker product (N=65536, L=1747) and the bounded sample, on one core,
    back to back: the ratio that scales the sample to a product."""
    full = cpu_sample_seconds(N, 0)
    samples = [cpu_sample_seconds(CPU_SAMPLE_N, i) for i in range(3)]
    sample = statistics.median(samples)
    print(json.dumps({"mode": "cpu-calibrate", "full_s": round(full, 3), "sample_n": CPU_SAMPLE_N,
                      "sample_s": [round(x, 3) for x in samples], "full_over_sample": round(full / sample, 3),
                      "cores": 1, "cpu": _cpu_name()}), flush=True)


def _cpu_name() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_b200(args):
    import torch
    import torch.distributed as dist

    world, rank, local = distributed()
    n_coeff, limbs = args.n, args.limbs
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=600))
    fpc = _load("fpc_b200", os.path.join(PACKAGE_DIR, "__init__.py"), PACKAGE_DIR)
    inputs = load_inputs()
    q, a, b = inputs.instance(n_coeff, limbs, SEED, rank)
    plan = fpc.Plan(n_coeff, 32 * limbs, limbs, q, device=local)
    info = plan.info()
    stream = torch.cuda.Stream()
    da = torch.from_numpy(a.view(np.int32)).cuda()
    db = torch.from_numpy(b.view(np.int32)).cuda()
    dc = torch.empty_like(da)
    sptr = stream.cuda_stream

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    # --- device-resident products (clocks sampled from the warm-up through the timed region)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        for _ in range(args.warmup):
            plan.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), sptr)
        barrier()
        start.record(stream)
        for _ in range(args.steps):
            plan.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), sptr)
        stop.record(stream)
        stop.synchronize()
    device_ms = max_over_ranks(start.elapsed_time(stop), world, "cuda")
    barrier()
    value = replica_throughput(world, args.steps, device_ms / 1000)

    # --- per-stage CUDA-event times over the same number of products (roofline)
    stage_ms = {name: 0.0 for name in fpc.STAGES}
    for _ in range(args.steps):
        for name, ms in plan.run_device_timed(da.data_ptr(), db.data_ptr(), dc.data_ptr(), sptr).items():
            stage_ms[name] += ms / args.steps

    # --- end to end through the host-facing C ABI, pinned host buffers
    if args.device_only:
        plan.close()
        if rank == 0:
            print(json.dumps({"workload": f"N={n_coeff} L={limbs}", "value": value, "unit": "products/s",
                              "ms_per_step": device_ms / args.steps,
                              "stages_ms": {k: round(v, 4) for k, v in stage_ms.items()}}), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return
    pa = torch.from_numpy(a.view(np.int32)).pin_memory()
    pb = torch.from_numpy(b.view(np.int32)).pin_memory()
    pc = torch.empty_like(pa).pin_memory()
    ha, hb, hc = (t.numpy().view(np.uint32) for t in (pa, pb, pc))
    for _ in range(max(1, args.warmup)):
        plan.run(ha, hb, out=hc)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        plan.run(ha, hb, out=hc)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, "cuda")
    barrier()
    e2e_value = replica_throughput(world, args.steps, e2e_s)
    # the device product must equal the host-path product (both through the C ABI)
    if not np.array_equal(dc.cpu().numpy().view(np.uint32), hc):
        raise RuntimeError("device-resident and host products differ")

    # --- batched form on the same workload: K products from the same page-locked host arrays
    # through negacyclic_batch_run (copy-in, compute and copy-out streams overlap across products)
    batched = None
    if not args.no_batched:
        count = max(4, min(args.steps, int(32e9 // (3 * a.nbytes))))  # device slots: at most 32 GB
        t1 = time.perf_counter()
        batch = fpc.Batch([(n_coeff, 32 * limbs, limbs, q)] * count, device=local)
        setup_s = time.perf_counter() - t1
        pcb = torch.empty_like(pa).pin_memory()
        hcb = pcb.numpy().view(np.uint32)
        batch.run([ha] * count, [hb] * count, [hcb] * count)  # warm-up
        batch_s = []
        for _ in range(2):
            barrier()
            t1 = time.perf_counter()
            batch.run([ha] * count, [hb] * count, [hcb] * count)
            batch_s.append(max_over_ranks(time.perf_counter() - t1, world, "cuda"))
        batch.close()
        if not np.array_equal(hcb, hc):
            raise RuntimeError("batched and per-call products differ")
        batched = {"value": replica_throughput(world, count, min(batch_s)), "unit": "products/s",
                   "products_per_call": count, "api": "negacyclic_batch_run, page-locked host arrays",
                   "h2d_bytes_per_product": int(a.nbytes + b.nbytes), "d2h_bytes_per_product": int(a.nbytes),
                   "plain_value": e2e_value, "setup_s": round(setup_s, 2)}

    # --- roofline of the conversion GEMM: 2 ops per byte MAC, M=2N rows, K=4L bytes, 4r weight columns
    hbm_gbs, bf16_tflops, bf16_sustained, source = peaks()
    int8_peak = 2 * bf16_tflops  # dense int8 = 2x dense bf16 on B200 (4.5 vs 2.25 PFLOP/s nominal)
    conv_ops = 2.0 * (2 * n_coeff) * (4 * limbs) * (4 * info["primes"])
    crt_ops = 2.0 * n_coeff * (4 * info["primes"]) * (4 * info["words"])
    conv_tops = conv_ops / (stage_ms["convert"] / 1000) / 1e12
    padded_limbs = (limbs + 31) // 32 * 32
    roofline = {
        "bound": "tensor", "kernel": "gemm_tc_kernel (conversion, tcgen05 kind::i8)",
        "achieved": round(conv_tops, 1), "peak": round(int8_peak, 1), "unit": "TOPS (int8)",
        "frac": round(conv_tops / int8_peak, 4),
        "frac_of_sustained": round(conv_tops / (2 * bf16_sustained), 4),
        # ncu sm__pipe_tensor_cycles_active of the conversion GEMM alone (N=16384, L=1747): the
        # tensor pipe's busy share of cycles, free of the clock under the power cap
        "tensor_pipe_active_per_cycle": CONVERT_TENSOR_PIPE_ACTIVE,
        "traffic": CONVERT_DRAM_BYTES if (n_coeff, limbs) == (N, LIMBS) else None,
        "traffic_unit": "bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)",
        # operand rows (padded to 32 limbs), conversion weights, residues written
        "algorithmic_bytes_per_launch": float(2 * n_coeff * 4 * padded_limbs + 4 * info["padded_primes"] * 4 * padded_limbs
                                              + 2 * info["primes"] * n_coeff * 4),
        "peak_source": f"2 x bf16 dense, {source} burst: {bf16_tflops} TF/s (sustained {bf16_sustained})",
        "algorithmic_ops_per_launch": conv_ops,
        "stages_ms": {k: round(v, 4) for k, v in stage_ms.items()},
        "crt_gemm_tops": round(crt_ops / (stage_ms["crt"] / 1000) / 1e12, 1),
        "whole_path": path_roofline(n_coeff, limbs, info, stage_ms, device_ms / args.steps, int8_peak, hbm_gbs),
        "whole_path_at_sustained": path_roofline(n_coeff, limbs, info, stage_ms, device_ms / args.steps,
                                                 2 * bf16_sustained, hbm_gbs)["measured_over_roof"],
    }

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        scale, how = cpu_scale()
        seconds = cpu_sample_seconds(CPU_SAMPLE_N)
        cpu = {"value": 1.0 / (seconds * scale), "unit": "products/s", "cores": 1, "kind": "port",
               "sample": f"one GMP Kronecker product (the reference checker's algorithm) of N={CPU_SAMPLE_N}, "
                         f"L={LIMBS}, {seconds:.2f} s, scaled {how} to N={N}", "same_config": False}

    extra = {}
    if rank == 0 and world == 1 and (n_coeff, limbs) == (N, LIMBS):
        if not args.no_fherma_run:
            extra["e2e_fherma_run"] = fherma_run_leg(args)
        if not args.no_config2:
            extra["config2"] = config2_leg(fpc, torch, args)
        if not args.no_refpoints:
            extra["refpoints"] = refpoints_leg()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "products/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": device_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 (int8 tensor GEMMs, exact)", "data": "synthetic",
            "config": {"workload": WORKLOAD, "primes": info["primes"], "split": info["split"],
                       "ntt_length": info["n_sub"], "tensor_gemms": info["gemm"],
                       "l2": "inputs larger than L2 (458 MB per operand), no flush needed",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_value, "unit": "products/s", "h2d_bytes_per_step": int(a.nbytes + b.nbytes),
                    "d2h_bytes_per_step": int(a.nbytes)},
            "batched_e2e": batched,
            "roofline": roofline,
            "cpu_baseline": cpu,
            **extra,
            "clocks": clocks.summary(),
            "gpu_launches": args.steps * info["kernels_per_product"],
        }
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.destroy_process_group()


SIZES = (4096, 8192, 16384, 32768, 65536)


def uneven_instances(count: int, seed: int):
    """Instances of the batched configuration: N uniform over SIZES, L log-uniform in [32, 1747],
    a distinct random odd q per instance (top limb nonzero), a and b uniform in [0, q)."""
    inputs = load_inputs()
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(count):
        n = int(rng.choice(SIZES))
        limbs = int(np.floor(np.exp(rng.uniform(np.log(32), np.log(1748)))))
        q, a, b = inputs.instance(n, min(limbs, 1747), seed * 1000 + i, 0)
        out.append((n, q.shape[0], q, a, b))
    return out


def log(msg):
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def run_batch(args):
    """64 uneven products: one graph launch (batched) against one call per product (plain)."""
    import ctypes

    import torch

    torch.cuda.set_device(0)
    fpc = _load("fpc_b200", os.path.join(PACKAGE_DIR, "__init__.py"), PACKAGE_DIR)
    t0 = time.perf_counter()
    instances = uneven_instances(args.count, 100)
    log(f"generated {len(instances)} instances in {time.perf_counter() - t0:.1f} s")
    cudart = ctypes.CDLL("libcudart.so.12")
    cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    batch = fpc.Batch([(n, 32 * l, l, q) for n, l, q, _, _ in instances], lanes=args.lanes, tune=args.tune,
                      tune_cache=args.tune_cache)
    setup_s = time.perf_counter() - t0
    log(f"batch created ({setup_s:.1f} s since start)")
    for i, (n, l, q, a, b) in enumerate(instances):
        da, db, _ = batch.io(i)
        cudart.cudaMemcpy(da, a.ctypes.data, a.nbytes, 1)
        cudart.cudaMemcpy(db, b.ctypes.data, b.nbytes, 1)
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t1 = time.perf_counter()
    batch.run_device(sptr)
    torch.cuda.synchronize()
    log(f"first batch run {time.perf_counter() - t1:.2f} s, pipeline status {fpc.pipeline_status()}")
    for _ in range(args.warmup):
        batch.run_device(sptr)
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(args.steps):
        batch.run_device(sptr)
    stop.record(stream)
    stop.synchronize()
    batched_ms = start.elapsed_time(stop) / args.steps
    log(f"batched {batched_ms:.1f} ms per batch, pipeline status {fpc.pipeline_status()}")
    # plain per-call path: one product per call, each call completing before the next
    plain_ms = 0.0
    for _ in range(max(1, args.steps // 2)):
        start.record(stream)
        for i in range(len(instances)):
            batch.run_one(i, sptr)
            stream.synchronize()
        stop.record(stream)
        stop.synchronize()
        plain_ms += start.elapsed_time(stop) / max(1, args.steps // 2)
    log(f"plain {plain_ms:.1f} ms per batch, pipeline status {fpc.pipeline_status()}")
    # host arrays (page-locked): batched (copy-in, compute and copy-out streams overlap) vs one call each
    pinned = lambda x: torch.from_numpy(x.view(np.int32)).pin_memory().numpy().view(np.uint32)  # noqa: E731
    ha = [pinned(a) for _, _, _, a, _ in instances]
    hb = [pinned(b) for _, _, _, _, b in instances]
    hc = [pinned(np.empty_like(a)) for _, _, _, a, _ in instances]
    batch.run(ha, hb, hc)
    t1 = time.perf_counter()
    batch.run(ha, hb, hc)
    host_batched_ms = (time.perf_counter() - t1) * 1000
    batch.run(ha, hb, hc, plain=True)
    t1 = time.perf_counter()
    batch.run(ha, hb, hc, plain=True)
    host_plain_ms = (time.perf_counter() - t1) * 1000
    log(f"host arrays: batched {host_batched_ms:.1f} ms, plain {host_plain_ms:.1f} ms")
    ops = sum(2.0 * (2 * n) * (4 * l) * (4 * batch.info(i)["primes"]) + 2.0 * n * (4 * batch.info(i)["primes"]) *
              (4 * (l + 5)) for i, (n, l, *_r) in enumerate(instances))
    infos = [batch.info(i) for i in range(len(instances))]
    batch.close()
    small = small_half(fpc, torch, instances, infos, args, cudart)
    line = {"metric": f"products/s, {len(instances)} uneven products (N in 4096..65536, L log-uniform 32..1747)",
            "value": len(instances) / (batched_ms / 1000), "unit": "products/s", "mode": "batched graph",
            "plain_value": len(instances) / (plain_ms / 1000), "batched_over_plain": plain_ms / batched_ms,
            "ms_per_batch": batched_ms, "plain_ms_per_batch": plain_ms, "int8_tops": ops / (batched_ms / 1000) / 1e12,
            "host_e2e": {"batched_products_per_s": len(instances) / (host_batched_ms / 1000),
                         "plain_products_per_s": len(instances) / (host_plain_ms / 1000),
                         "batched_over_plain": host_plain_ms / host_batched_ms,
                         "bytes_per_batch": int(sum(3 * a.nbytes for _, _, _, a, _ in instances))},
            "lanes": args.lanes or "two phases (concurrent small instances on up to 4 lanes, then large ones alone)",
            "concurrent_phase": small,
            "tuned": bool(args.tune), "setup_s": setup_s,
            "steps": args.steps, "warmup": args.warmup, "data": "synthetic (seed 100)"}
    print(json.dumps(line), flush=True)


def small_half(fpc, torch, instances, infos, args, cudart) -> dict:
    """The batch's concurrent phase alone (the instances under about 1 ms of device time): one
    graph launch of just those instances against the plain per-call loop over the same ones."""
    chosen = [i for i, info in enumerate(infos) if info["phase"] == 0]
    if not chosen:
        return {"instances": 0}
    subset = [instances[i] for i in chosen]
    batch = fpc.Batch([(n, 32 * l, l, q) for n, l, q, _, _ in subset], lanes=args.lanes, tune=args.tune,
                      tune_cache=args.tune_cache)
    for j, (n, l, q, a, b) in enumerate(subset):
        da, db, _ = batch.io(j)
        cudart.cudaMemcpy(da, a.ctypes.data, a.nbytes, 1)
        cudart.cudaMemcpy(db, b.ctypes.data, b.nbytes, 1)
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(max(3, args.warmup)):
        batch.run_device(sptr)
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(args.steps):
        batch.run_device(sptr)
    stop.record(stream)
    stop.synchronize()
    batched_ms = start.elapsed_time(stop) / args.steps
    if batch.status().any():
        raise RuntimeError("concurrent phase: a status word is set")
    plain_ms = 0.0
    for _ in range(max(1, args.steps // 2)):
        start.record(stream)
        for j in range(len(subset)):
            batch.run_one(j, sptr)
            stream.synchronize()
        stop.record(stream)
        stop.synchronize()
        plain_ms += start.elapsed_time(stop) / max(1, args.steps // 2)
    lanes = sorted({batch.info(j)["lane"] for j in range(len(subset))})
    batch.close()
    return {"instances": len(subset), "shapes": [[n, l] for n, l, *_r in subset], "lanes": len(lanes),
            "batched_ms": batched_ms, "plain_ms": plain_ms, "batched_products_per_s": len(subset) / (batched_ms / 1000),
            "plain_products_per_s": len(subset) / (plain_ms / 1000), "batched_over_plain": plain_ms / batched_ms}


def run_serve(args):
    """Poisson arrivals over 8 sessions (fixed L and q each, N per request) at each offered rate;
    p50/p99 latency and products/s, then the same request mix through the plain per-call path."""
    import torch

    torch.cuda.set_device(0)
    fpc = _load("fpc_b200", os.path.join(PACKAGE_DIR, "__init__.py"), PACKAGE_DIR)
    inputs = load_inputs()
    rng = np.random.Generator(np.random.PCG64(200))
    max_limbs = args.serve_max_limbs
    sessions = []
    server = fpc.Server(hbm_budget=int(args.budget_gb * (1 << 30)), slots=args.slots, max_queue=args.max_queue)
    for sidx in range(8):
        limbs = int(np.floor(np.exp(rng.uniform(np.log(32), np.log(max_limbs + 1)))))
        q = inputs.random_modulus(limbs, 200 + sidx)
        sid = server.open_session(32 * limbs, limbs, q, ns=SIZES)
        pool = {}
        log(f"session {sidx}: L={limbs}")
        for n in SIZES:  # page-locked operand pairs per ring size
            pairs = []
            for k in range(args.serve_pairs):
                a = torch.from_numpy(inputs.random_operand(rng, n, q).view(np.int32)).pin_memory()
                b = torch.from_numpy(inputs.random_operand(rng, n, q).view(np.int32)).pin_memory()
                pairs.append((a.numpy().view(np.uint32), b.numpy().view(np.uint32)))
            pool[n] = pairs
        sessions.append((sid, limbs, q, pool))
    outputs = {}
    for sid, limbs, _, pool in sessions:
        for n in SIZES:
            outputs[(sid, n)] = [torch.empty((n, limbs), dtype=torch.int32).pin_memory().numpy().view(np.uint32)
                                 for _ in range(args.slots + 1)]
    log("sessions and buffers ready")
    # warm-up: one request per (session, N) before the timed runs, so that first-use costs (the
    # first launch of each kernel instance loads its module) stay out of the latency figures
    t0 = time.perf_counter()
    warm = [server.submit(sid, *pool[n][0], out=outputs[(sid, n)][0]) for sid, _, _, pool in sessions for n in SIZES]
    for rid in warm:
        server.wait(rid)
    warm_s = time.perf_counter() - t0
    log(f"warm-up: {len(warm)} requests in {warm_s:.2f} s")

    def schedule_for(rate, duration):
        t, out = 0.0, []
        while t < duration:
            t += rng.exponential(1.0 / rate)
            out.append((t, int(rng.integers(len(sessions))), int(rng.choice(SIZES)), int(rng.integers(args.serve_pairs))))
        return out

    runs = []
    for rate in [float(x) for x in args.rates.split(",")]:
        duration = args.duration  # the same arrival window at every rate; overload is shed at submit
        schedule = schedule_for(rate, duration)
        ids, out_counter, refused = [], {}, 0
        before = server.stats()
        start = time.perf_counter()
        for when, s_index, n, k in schedule:
            delay = when - (time.perf_counter() - start)
            if delay > 0:
                time.sleep(delay)
            sid, limbs, _, pool = sessions[s_index]
            ring = outputs[(sid, n)]
            slot = out_counter.get((sid, n), 0)
            out_counter[(sid, n)] = slot + 1
            a, b = pool[n][k]
            rid = server.submit(sid, a, b, out=ring[slot % len(ring)])
            if rid is None:
                refused += 1
            else:
                ids.append(rid)
        latencies = np.array([server.wait(rid)[1] for rid in ids])
        elapsed = time.perf_counter() - start
        after = server.stats()
        runs.append({"offered_rate": rate, "arrival_window_s": round(duration, 3), "offered": len(schedule),
                     "completed": len(ids), "rejected": refused,
                     "rejected_by_server": int(after["rejected"] - before["rejected"]),
                     "max_queue_depth": int(after["max_queued"]), "products_per_s": len(ids) / elapsed,
                     "p50_ms": float(np.percentile(latencies, 50)), "p99_ms": float(np.percentile(latencies, 99)),
                     "mean_ms": float(latencies.mean()), "elapsed_s": round(elapsed, 3)})
        log(f"rate {rate:g}: {runs[-1]}")
    stats = server.stats()
    server.close()

    # the same request mix through the plain per-call path (negacyclic_run, page-locked buffers),
    # one (session, N) plan at a time
    mix = schedule_for(1.0, float(args.plain_requests))[: args.plain_requests]
    groups = {}
    for _, s_index, n, k in mix:
        groups.setdefault((s_index, n), []).append(k)
    plain_s = 0.0
    for (s_index, n), ks in groups.items():
        sid, limbs, q, pool = sessions[s_index]
        plan = fpc.Plan(n, 32 * limbs, limbs, q)
        out = outputs[(sid, n)][0]
        plan.run(*pool[n][ks[0]], out=out)  # warm-up
        for k in ks:
            t0 = time.perf_counter()
            plan.run(*pool[n][k], out=out)
            plain_s += time.perf_counter() - t0
        plan.close()
    plain_value = len(mix) / plain_s
    best = max(r["products_per_s"] for r in runs)
    line = {"metric": "served products/s, Poisson arrivals, 8 sessions (fixed q, L each), N in 4096..65536",
            "value": best, "unit": "products/s", "mode": "serving (continuous batching)", "runs": runs,
            "plain_per_call_products_per_s": plain_value, "plain_requests": len(mix),
            "served_over_plain": best / plain_value, "slots": args.slots, "hbm_budget_gb": args.budget_gb,
            "max_queue": args.max_queue,
            "session_limbs": [limbs for _, limbs, _, _ in sessions], "failed": stats["failed"],
            "warmup": {"requests": len(warm), "seconds": round(warm_s, 3)},
            "data": "synthetic (seed 200)"}
    print(json.dumps(line), flush=True)


def relaunch_under_torchrun(gpus: int) -> int:
    """`--gpus N` without torchrun: run this same command as N ranks under torch.distributed.run
    (one process per GPU, rendezvous on 127.0.0.1); returns its exit code."""
    import socket

    with socket.socket() as probe:
        probe.bind(("127.0.0.1", 0))
        port = probe.getsockname()[1]
    command = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
               "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.run(command).returncode


def main():
    parser = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=20)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=("b200", "reference"), default="b200")
    parser.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    parser.add_argument("--no-batched", action="store_true", help="skip the batched host-array measurement")
    parser.add_argument("--no-fherma-run", action="store_true", help="skip the fherma_run (pageable) leg")
    parser.add_argument("--no-config2", action="store_true", help="skip the N=32768, L=868 leg")
    parser.add_argument("--no-refpoints", action="store_true", help="skip the reference-points comparison")
    parser.add_argument("--workload", default=f"{N},{LIMBS}",
                        help="N,L of a smaller case for profiling (the benchmark line is N=65536,L=1747)")
    parser.add_argument("--device-only", action="store_true",
                        help="device-resident products and stage times only (profiling runs)")
    parser.add_argument("--mode", choices=("plain", "batch", "serve", "cpu-calibrate"), default="plain",
                        help="plain: the benchmark line; batch / serve: the batched and serving forms; "
                             "cpu-calibrate: one full-size CPU product against the bounded sample")
    parser.add_argument("--count", type=int, default=64, help="batch: number of uneven products")
    parser.add_argument("--lanes", type=int, default=0,
                        help="batch: compute lanes (0 = two phases: small instances concurrently, then large ones)")
    parser.add_argument("--tune", action="store_true", help="batch: run the autotuner for uncached shapes")
    parser.add_argument("--tune-cache", default=None, help="batch: autotuner cache file")
    parser.add_argument("--rates", default="200,1000,5000", help="serve: Poisson arrival rates (requests/s)")
    parser.add_argument("--duration", type=float, default=60.0, help="serve: seconds of arrivals at each rate")
    parser.add_argument("--max-queue", type=int, default=64,
                        help="serve: requests waiting for admission beyond which submits are refused")
    parser.add_argument("--plain-requests", type=int, default=200, help="serve: requests of the plain comparison")
    parser.add_argument("--slots", type=int, default=4, help="serve: concurrent requests")
    parser.add_argument("--budget-gb", type=float, default=60.0, help="serve: HBM budget (GiB)")
    parser.add_argument("--serve-max-limbs", type=int, default=1747, help="serve: largest session L")
    parser.add_argument("--serve-pairs", type=int, default=1, help="serve: operand pairs per (session, N)")
    args = parser.parse_args()
    args.n, args.limbs = (int(x) for x in args.workload.split(","))
    world = int(os.environ.get("WORLD_SIZE", "0"))
    if world and world != args.gpus:
        parser.error(f"--gpus {args.gpus} but torchrun started {world} ranks")
    if not world and args.gpus > 1:
        sys.exit(relaunch_under_torchrun(args.gpus))
    if args.mode == "cpu-calibrate":
        run_cpu_calibrate(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.mode == "batch":
        run_batch(args)
    elif args.mode == "serve":
        run_serve(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
