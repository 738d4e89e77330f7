"""Benchmark: batched RNS NTT round trip + polymul on B200.

Workload (the batched configuration of the lattice-arithmetic path):
N = 2^16, L = 24 primes (descending below 2^50, q = 1 mod 2^17), 64
ciphertexts x 2 polynomials = 128 DCRT polys with uniform residues from a seed,
one 24-limb plaintext (uniform, kept in the NTT domain in HBM).  One step =
forward NTT, pointwise product with the plaintext, inverse NTT of all 128
polys -- one fused cluster launch (`pg_dcrt_polymul_ntt_plain`).  The metric
counts "2^16 x 24-prime NTTs" (one forward or inverse transform of one 24-limb
poly): 256 per step.  Inputs are 1.61 GB, larger than the 126 MB L2, so no L2
flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line.  `--impl reference` times the CPU restatement of the
reference's own algorithm (the oracle port of its Rust code) on the host's
cores over a bounded sample of the same workload.  The line also carries the
end-to-end rate through the C ABI with host buffers (beside the host link's
own rate), the roofline of the fused kernel, the CPU baseline and the check of
the timed output against the oracle.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LOG_N, L, POLYS = 16, 24, 128
N = 1 << LOG_N
SEED = 0x5EED0001
NTT_PER_STEP = 2 * POLYS
METRIC = "2^16x24-prime NTT/s (batched fwd -> x plain -> inv, bit-exact)"
UNIT = "NTT/s"
WORKLOAD = {
    "workload": "batched RNS NTT round trip + polymul: N=2^16, L=24 primes < 2^50 (q = 1 mod 2^17), "
                "64 ciphertexts x 2 polys, NTT-domain plaintext resident",
    "N": N, "L": L, "polys": POLYS,
    "l2": "inputs 1.61 GB per step > 126 MB L2 (no flush needed)",
}
# algorithmic bytes of one step: read + write every residue once, read the plaintext once
ALGO_BYTES = 2 * POLYS * L * N * 8 + L * N * 8


def set_polys(p: int):
    global POLYS, NTT_PER_STEP, ALGO_BYTES
    if p != POLYS:
        POLYS = p
        NTT_PER_STEP = 2 * p
        ALGO_BYTES = 2 * p * L * N * 8 + L * N * 8
        WORKLOAD["polys"] = p
        WORKLOAD["workload"] += f" [reduced to {p} polys for a profiler capture]"


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p)).get("polymul_round_trip_bytes_per_launch")
        except Exception:
            return None
    return None


class ClockSampler:
    """nvidia-smi sampling during the timed region (SM clock, throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus, backend="nccl"):
    """One process per GPU under torchrun; returns (rank, world, local_rank, dist-or-None).
    The path runs as replicas: the process group carries only the barriers and the
    max-over-ranks of the timings (gloo for the CPU tests of that logic)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
        return rank, world, local, dist
    return rank, world, local, None


def dist_max(dist, value: float, local: int) -> float:
    if dist is None:
        return value
    import torch
    device = f"cuda:{local}" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(dist):
    if dist is not None:
        dist.barrier()


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def host_description():
    """The host the CPU legs ran on: CPU model, usable threads, AVX-512 IFMA."""
    model, flags = "unknown", ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name") and model == "unknown":
                    model = line.split(":", 1)[1].strip()
                elif line.startswith("flags") and not flags:
                    flags = line
    except OSError:
        pass
    return {"cpu_model": model, "threads": cpu_threads(), "nproc": os.cpu_count(),
            "avx512ifma": " avx512ifma" in flags}


def cpu_reference(moduli, seconds_target=12.0, threads=None, path=None):
    """Time the reference's CPU path for this workload on the host cores over a bounded
    sample; returns (NTT/s, sample text, threads).  The path is the one the reference
    dispatches to (primus_ntt/src/ntt/hexl/mod.rs:473-540): the HEXL-style AVX-512
    IFMA52 transforms when the host has avx512ifma and q < 2^50 (oracle/hexl_ifma.c),
    else the scalar UintNttTable restatement.  OpenMP over rows."""
    import oracle as O
    threads = threads or cpu_threads()
    ref = O.DcrtTable(LOG_N, moduli)
    plain = O.uniform_rns(SEED + 7, 0, moduli, N)
    plain = ref.forward(plain)
    use_hexl = (path or ("hexl" if O.hexl_available() else "scalar")) == "hexl"
    if use_hexl:
        hx = O.HexlDcrt(ref)
        plain_p = hx.prepare(plain)
        run = lambda x: hx.polymul_roundtrip(x, plain, plain_p, threads=threads)  # noqa: E731
        label = "HEXL-style AVX-512 IFMA52 restatement of the reference's fastest CPU path"
    else:
        run = lambda x: ref.polymul_roundtrip(x, plain, threads=threads)  # noqa: E731
        label = "C restatement of UintNttTable/DcrtPolynomial (scalar)"
    one = O.uniform_rns(SEED, 0, moduli, N).ravel().copy()
    t0 = time.perf_counter()
    run(one)
    per_poly = max(time.perf_counter() - t0, 1e-4)
    # at least one poly per thread so every core works; bounded to ~seconds_target
    polys = int(max(threads, min(POLYS, seconds_target / per_poly)))
    polys = max(1, min(POLYS, polys))
    x = np.concatenate([O.uniform_rns(SEED, p * L, moduli, N).ravel() for p in range(polys)])
    # repeat the sample until about seconds_target of CPU time has passed (bounded)
    reps, t0 = 0, time.perf_counter()
    while True:
        run(x)
        reps += 1
        dt = time.perf_counter() - t0
        if dt >= seconds_target or reps >= 1000:
            break
    par = f"OpenMP over rows on {threads} threads" if threads > 1 else "one thread"
    return 2 * polys * reps / dt, f"{label}, {par}; {polys} of {POLYS} polys (24 limbs, N=2^16) round " \
                                  f"trip x {reps}, {dt:.2f} s", threads


class RowCheck:
    """Checks the bench's own outputs against the oracle after the timed region.

    Every leg of the bench applies the same map to the batch in place (forward
    NTT, product with the NTT-domain plaintext, inverse NTT), so after R round
    trips row r holds RT^R(x_r).  Four rows (one limb each of four polys) are
    regenerated from the seed on the host and carried forward by the oracle
    (UintNttTable transforms, primus_ntt/src/ntt/primitive.rs:211-296, and the
    pointwise product); `check` compares the device's rows with them after any
    number of round trips.  It runs outside every timed region."""

    def __init__(self, moduli, seed, threads):
        import oracle as O
        self.O = O
        self.polys = sorted({0, POLYS // 3, (2 * POLYS) // 3, POLYS - 1})
        self.limbs = [(7 * i + 3) % L for i in range(len(self.polys))]
        self.moduli = [moduli[l] for l in self.limbs]
        self.ref = O.DcrtTable(LOG_N, self.moduli)
        plain = O.DcrtTable(LOG_N, moduli).forward(O.uniform_rns(SEED + 7, 0, moduli, N), threads=threads)
        self.plain = np.stack([plain.reshape(L, N)[l] for l in self.limbs])
        # the rows after k round trips, for every k a check has asked for: legs run on
        # copies of the batch (the end-to-end leg on a host slice), so a later check
        # may ask for fewer round trips than an earlier one
        self.states = {0: np.stack([O.uniform(seed, p * L + l, moduli[l], N)
                                    for p, l in zip(self.polys, self.limbs)])}
        self.threads = threads
        self.results = []

    def state_at(self, rounds):
        k = max(r for r in self.states if r <= rounds)
        st = self.states[k]
        while k < rounds:
            st = self.ref.polymul_roundtrip(st, self.plain, threads=self.threads).reshape(st.shape)
            k += 1
        self.states[k] = st
        return st

    def rows_of(self, read_row):
        return np.stack([read_row(p * L + l) for p, l in zip(self.polys, self.limbs)])

    def check(self, name, rounds, read_row):
        ok = bool(np.array_equal(self.rows_of(read_row), self.state_at(rounds)))
        self.results.append({"leg": name, "round_trips": rounds, "ok": ok})
        return ok

    def summary(self):
        return {"verified": all(r["ok"] for r in self.results) and bool(self.results),
                "rows": [f"poly {p} limb {l}" for p, l in zip(self.polys, self.limbs)],
                "checks": self.results,
                "oracle": "UintNttTable restatement (oracle/primus_oracle.c), rows regenerated from the seed"}


def device_row(nat, buf, stream):
    def read(row):
        out = np.empty(N, dtype=np.uint64)
        nat.call("pg_memcpy_d2h", out.ctypes.data, buf.ptr + row * N * 8, N * 8, stream.h)
        nat.call("pg_stream_synchronize", stream.h)
        return out
    return read


def run_reference(args):
    # a CPU arm: under torchrun rank 0 alone times it and prints; the other ranks
    # exit without work (no process group, so nothing waits on them)
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle as O
    moduli = O.ntt_primes(1 << 50, 2 * N, L)
    vals = []
    sample = ""
    thr = cpu_threads()
    for _ in range(args.warmup):
        cpu_reference(moduli, seconds_target=2.0, threads=thr)
    for _ in range(max(1, args.steps)):
        v, sample, thr = cpu_reference(moduli, seconds_target=max(2.0, 60.0 / max(1, args.steps)), threads=thr)
        vals.append(v)
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": NTT_PER_STEP / value * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded uniform residues)", "config": WORKLOAD,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": thr, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_gpu(args):
    rank, world, local, dist = dist_setup(args.gpus)
    import primus_b200 as P
    from primus_b200 import _native as nat
    nat.call("pg_set_device", local)
    moduli = P.ntt_primes(1 << 50, 2 * N, L)
    tab = P.DcrtTable(LOG_N, moduli)
    stream = P.Stream()
    data = P.DeviceBuffer(POLYS * L * N)
    plain = P.DeviceBuffer(L * N)
    plain_q = P.DeviceBuffer(L * N)
    tab.fill_uniform(data, POLYS, seed=SEED + rank, stream=stream)
    tab.fill_uniform(plain, 1, seed=SEED + 7, stream=stream)
    tab.forward(plain, 1, stream=stream)
    tab.shoup_prepare(plain, plain_q, 1, stream=stream)
    stream.synchronize()
    # kernel shape per (N, L): the autotuner times every shape of N = 2^16 on this
    # table before the warm-up and keeps the fastest in the table
    if args.no_tune:  # profiler captures: the default shapes, no tuning launches
        tuning = {k: {"variant": 0, "name": "default", "us": 0.0, "default_us": 0.0}
                  for k in ("forward", "inverse", "round_trip")}
    else:
        tuning = tab.autotune(POLYS)
    rt_shape = tuning["round_trip"]
    # built-in ceilings (streaming copy, register-only butterfly rates), measured before the warm-up
    cal = P.calibrate()
    # template arguments <LOG_N, LOG_M (block), LOG_E, MODE (2 = round trip), schedule>;
    # schedule 3 = FP64 butterflies (every q < 2^50, the default there), 2 = fast integer
    kernel_name = {"default": "ntt_cluster_kernel<16, 12, 4, 2, 3>",
                   "fp64 cluster of 16 x 4096": "ntt_cluster_kernel<16, 12, 4, 2, 3>",
                   "fp64 cluster of 8 x 8192": "ntt_cluster_kernel<16, 13, 4, 2, 3>",
                   "cluster of 8 x 8192": "ntt_cluster_kernel<16, 13, 4, 2, 2>"}.get(rt_shape["name"], rt_shape["name"])

    def step():
        tab.polymul_ntt_plain(data, plain, plain_q, POLYS, stream=stream)

    for _ in range(args.warmup):
        step()
    stream.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    e0, e1 = P.Event(), P.Event()
    dist_barrier(dist)
    stream.synchronize()
    launches0 = P.launch_count()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    stream.synchronize()
    launches = P.launch_count() - launches0
    ms = e0.elapsed_ms(e1)
    dist_barrier(dist)
    clocks = sampler.stop()
    ms_max = dist_max(dist, ms, local)
    per_step = ms_max / args.steps
    value = NTT_PER_STEP * world / (per_step / 1e3)
    # every fused launch so far (warm-up and timed) is one round trip of the batch
    rounds = args.warmup + args.steps
    check = RowCheck(moduli, SEED + rank, cpu_threads())
    check.check("timed fused launches", rounds, device_row(nat, data, stream))

    # ---- plain one-call-per-op GPU form (fwd, mul, inv as separate launches), same data
    for _ in range(2):
        tab.forward(data, POLYS, stream=stream)
        tab.mul(data, plain, POLYS, rhs_polys=1, stream=stream)
        tab.inverse(data, POLYS, stream=stream)
    e0.record(stream)
    plain_steps = max(3, args.steps // 2)
    for _ in range(plain_steps):
        tab.forward(data, POLYS, stream=stream)
        tab.mul(data, plain, POLYS, rhs_polys=1, stream=stream)
        tab.inverse(data, POLYS, stream=stream)
    e1.record(stream)
    stream.synchronize()
    plain_ms = e0.elapsed_ms(e1) / plain_steps
    rounds += 2 + plain_steps
    check.check("plain three-launch form", rounds, device_row(nat, data, stream))

    # ---- end to end through the public C ABI with pinned host buffers
    import ctypes as C
    nbytes = POLYS * L * N * 8
    hp = C.c_void_p()
    nat.call("pg_host_alloc", C.byref(hp), nbytes)
    host = np.ctypeslib.as_array((C.c_uint64 * (POLYS * L * N)).from_address(hp.value))
    host[:] = data.numpy()

    def e2e_step():
        # the reference-facing call on a host slice: copies in, fused launches and
        # copies out pipelined over chunks inside the library (synchronous)
        nat.call("pg_dcrt_polymul_ntt_plain_host", tab.h, hp.value, plain.ptr, plain_q.ptr, POLYS, stream.h)

    for _ in range(2):
        e2e_step()
    stream.synchronize()
    e2e_steps = max(3, min(args.steps, 10))
    dist_barrier(dist)
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    stream.synchronize()
    e2e_ms = dist_max(dist, e0.elapsed_ms(e1) / e2e_steps, local)
    check.check("end to end through the host-slice call", rounds + 2 + e2e_steps,
                lambda row: host[row * N:(row + 1) * N].copy())
    # the host link of the machine: the step's H2D and D2H bytes as two concurrent copies
    # on two streams with no kernels (one cudaMemcpyAsync each); the end-to-end leg
    # cannot run faster than this
    hp2 = C.c_void_p()
    nat.call("pg_host_alloc", C.byref(hp2), nbytes)
    dev2 = P.DeviceBuffer(POLYS * L * N)
    s2, ea, eb = P.Stream(), P.Event(), P.Event()
    link_runs = []
    for _ in range(3):
        stream.synchronize()
        s2.synchronize()
        e0.record(stream)
        nat.call("pg_memcpy_h2d", dev2.ptr, hp.value, nbytes, stream.h)
        nat.call("pg_memcpy_d2h", hp2.value, data.ptr, nbytes, s2.h)
        ea.record(stream)
        eb.record(s2)
        stream.synchronize()
        s2.synchronize()
        link_runs.append(max(e0.elapsed_ms(ea), e0.elapsed_ms(eb)))
    link_ms = min(link_runs)
    nat.call("pg_host_free", hp2.value)
    del dev2
    s2.close()
    nat.call("pg_host_free", hp.value)
    e2e_value = NTT_PER_STEP * world / (e2e_ms / 1e3)

    # ---- the same fused step on the integer schedules only (FP64 schedule off):
    # identical residues, the butterflies on the integer multiply pipe
    integer_only = None
    if tab.fp64:
        tab.set_fp64(False)
        int_tuning = tab.autotune(POLYS) if not args.no_tune else {"round_trip": {"name": "default"}}
        for _ in range(3):
            step()
        stream.synchronize()
        int_steps = max(3, args.steps // 2)
        e0.record(stream)
        for _ in range(int_steps):
            step()
        e1.record(stream)
        stream.synchronize()
        int_ms = e0.elapsed_ms(e1) / int_steps
        rounds += 3 + int_steps
        check.check("integer schedules only", rounds, device_row(nat, data, stream))
        tab.set_fp64(True)
        int_gbfly = NTT_PER_STEP * L * (N // 2) * LOG_N / (int_ms / 1e3) / 1e9
        integer_only = {"value": NTT_PER_STEP / (int_ms / 1e3), "unit": UNIT, "ms_per_step": int_ms,
                        "g_butterflies_per_s": int_gbfly,
                        "frac_of_int_ceiling": int_gbfly / cal["int_butterflies_gps"],
                        "kernel_shape": int_tuning["round_trip"]["name"],
                        "note": "pg_ntt_set_fp64(table, 0): the same fused step with integer butterflies "
                                "(Shoup products on the integer multiply pipe); same outputs"}

    peak, peak_kind = load_peaks()
    achieved = ALGO_BYTES / (per_step / 1e3) / 1e9
    out = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            import oracle as O  # the CPU oracle, timed here as the CPU baseline only
            moduli = O.ntt_primes(1 << 50, 2 * N, L)
            v, sample, thr = cpu_reference(moduli, seconds_target=args.cpu_seconds)
            cpu = {"value": v, "unit": UNIT, "cores": thr, "kind": "port", "sample": sample}
            if O.hexl_available():  # the scalar restatement beside it, on a short sample
                sv, ssample, _ = cpu_reference(moduli, seconds_target=3.0, threads=thr, path="scalar")
                cpu["scalar_port"] = {"value": sv, "sample": ssample}
            sv1, ssample1, _ = cpu_reference(moduli, seconds_target=2.0, threads=1, path="scalar")
            cpu["scalar_port_1_thread"] = {"value": sv1, "sample": ssample1}
            cpu["host"] = host_description()
        workloads = None
        if world == 1 and not args.no_extra:
            workloads = {"polymul_n1024": bench_polymul_1024(P, stream),
                         "uneven_batch": bench_uneven(P, stream),
                         "ext_product": bench_ext_product(P, stream, cpu=not args.no_cpu),
                         "hybrid_ks": bench_hybrid_ks(P, stream),
                         "widened": bench_widened(P, stream),
                         "pointwise": bench_pointwise(P, stream),
                         "expand": bench_expand(P, stream),
                         "served_mixed": bench_served(P, stream),
                         "autotune_L24": bench_autotune(P)}
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded uniform residues, device generator)",
            "config": dict(WORKLOAD, parallelism=f"replicas x{world}" if world > 1 else "single GPU",
                           kernel_shape=f"{rt_shape['name']} (autotuned: "
                                        + ", ".join(f"{k} {tuning[k]['name']} {tuning[k]['us']:.0f} us"
                                                    for k in ('forward', 'inverse', 'round_trip')) + ")"),
            "clocks": clocks,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                    "ms_per_step": e2e_ms, "path": "pg_dcrt_polymul_ntt_plain_host (pinned host slice; chunked H2D / fused launch / D2H on 3 streams)",
                    "host_link_ms_per_step": link_ms, "frac_of_host_link": link_ms / e2e_ms,
                    "host_link_note": "the same H2D and D2H bytes as two concurrent copies, no kernels (this machine)"},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": load_traffic(), "peak_source": peak_kind,
                         "kernel": kernel_name + " (fused fwd -> x plain -> inv)",
                         "algorithmic_bytes_per_launch": ALGO_BYTES,
                         # the bound that binds: arithmetic issue (FP64 pipe on the FP64 schedule)
                         "butterflies_per_launch": NTT_PER_STEP * L * (N // 2) * LOG_N,
                         "g_butterflies_per_s": NTT_PER_STEP * L * (N // 2) * LOG_N / (per_step / 1e3) / 1e9,
                         "compute_ceiling": {
                             "pipe": "fp64" if tab.fp64 else "integer",
                             "g_butterflies_per_s": cal["fp64_butterflies_gps" if tab.fp64 else "int_butterflies_gps"],
                             "frac": (NTT_PER_STEP * L * (N // 2) * LOG_N / (per_step / 1e3) / 1e9)
                                     / cal["fp64_butterflies_gps" if tab.fp64 else "int_butterflies_gps"],
                             "source": "pg_calibrate: register-only forward butterflies of the same schedule"},
                         "builtin_copy_gbs": cal["hbm_copy_gbs"]},
            "verified": check.summary()["verified"],
            "verification": check.summary(),
            "integer_only": integer_only,
            "plain_gpu": {"value": NTT_PER_STEP / (plain_ms / 1e3), "unit": UNIT, "ms_per_step": plain_ms,
                          "form": "pg_ntt_forward + pg_dcrt_mul + pg_ntt_inverse (3 launches)"},
            "cpu_baseline": cpu,
            "workloads": workloads,
        }
        print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()
    return 0


# --------------------------------------------------------------------------
# Secondary workloads of the same path, reported beside the headline number.
# --------------------------------------------------------------------------
def _time_stream(P, stream, fn, reps):
    e0, e1 = P.Event(), P.Event()
    fn()
    stream.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    stream.synchronize()
    return e0.elapsed_ms(e1) / reps


def bench_polymul_1024(P, stream):
    """64 pairs of N = 1024 polys, q = largest prime < 2^50 with q = 1 mod 2048:
    forward both, pointwise product, inverse (one graph-replayed submission)."""
    q = P.prev_prime_congruent(1 << 50, 2048)
    tab = P.DcrtTable(10, [q])
    batch = P.PolymulBatch([tab])
    a = P.DeviceBuffer(64 * 1024)
    b = P.DeviceBuffer(64 * 1024)
    tab.fill_uniform(a, 64, seed=0x5EED0000, stream=stream)
    tab.fill_uniform(b, 64, seed=0x5EED0100, stream=stream)
    # the job arrays are built once, as a C or Rust caller holds them
    jobs = batch.prepare([(_Slice(a, i * 1024), _Slice(b, i * 1024), 10, 1) for i in range(64)])
    ms = _time_stream(P, stream, lambda: batch.run(jobs, use_graph=True, stream=stream), 50)
    one = batch.prepare([(_Slice(a, 0), _Slice(b, 0), 10, 1)])
    ms_one = _time_stream(P, stream, lambda: batch.run(one, use_graph=False, stream=stream), 50)
    return {"workload": "64 products of N=1024 polys (q < 2^50, q = 1 mod 2048): fwd x2, mul, inv",
            "batch_latency_us": ms * 1e3, "pairs_per_s": 64 / (ms / 1e3),
            "single_pair_latency_us": ms_one * 1e3}


class _Slice:
    """a view into a DeviceBuffer at an element offset (for job descriptors)"""

    def __init__(self, buf, off):
        self.buf, self.ptr = buf, buf.ptr + 8 * off


def bench_uneven(P, stream, jobs_n=512):
    """512 products with N uniform in {2^10..2^16} and L uniform in 1..32
    (primes < 2^50, q = 1 mod 2N, descending), one graph-replayed submission
    vs one call per job."""
    rng = np.random.default_rng(0x5EED0002)
    log_ns = list(range(10, 17))
    shape = [(int(rng.choice(log_ns)), int(rng.integers(1, 33))) for _ in range(jobs_n)]
    tables = {ln: P.DcrtTable(ln, P.ntt_primes(1 << 50, 2 << ln, 32)) for ln in log_ns}
    batch = P.PolymulBatch(list(tables.values()))
    jobs, total_bytes = [], 0
    for j, (ln, L) in enumerate(shape):
        n = 1 << ln
        t = tables[ln]
        # buffers hold all 32 limbs so the device generator fills them in one call;
        # the job uses the first L
        a, b = P.DeviceBuffer(t.L * n), P.DeviceBuffer(t.L * n)
        t.fill_uniform(a, 1, seed=0x5EED0003, stream0=64 * j, stream=stream)
        t.fill_uniform(b, 1, seed=0x5EED0004, stream0=64 * j, stream=stream)
        jobs.append((a, b, ln, L))
        total_bytes += 24 * n * L
    stream.synchronize()
    prepared = batch.prepare(jobs)
    singles = [batch.prepare([j]) for j in jobs]
    ms_graph = _time_stream(P, stream, lambda: batch.run(prepared, use_graph=True, stream=stream), 10)
    ms_plain = _time_stream(P, stream, lambda: [batch.run(j, use_graph=False, stream=stream) for j in singles], 3)
    # tails: each degree class alone (its own launches, its own tail) against the
    # whole set in one graph; and the butterfly rate against the fused
    # round-trip kernel's (3 transforms of L rows per job: fwd a, fwd b, inv a)
    per_class = {}
    for ln in log_ns:
        cls = batch.prepare([j for j in jobs if j[2] == ln])
        per_class[f"N=2^{ln}"] = _time_stream(P, stream, lambda: batch.run(cls, use_graph=False, stream=stream), 5)
    bfly = sum(3 * L * (1 << (ln - 1)) * ln for ln, L in shape)
    return {"workload": "512 products, N uniform in 2^10..2^16, L uniform in 1..32, one graph launch",
            "jobs": jobs_n, "ms_per_batch": ms_graph, "jobs_per_s": jobs_n / (ms_graph / 1e3),
            "algorithmic_gb": total_bytes / 1e9, "achieved_gbs": total_bytes / (ms_graph / 1e3) / 1e9,
            "g_butterflies_per_s": bfly / (ms_graph / 1e3) / 1e9,
            "per_class_alone_ms": per_class, "sum_of_classes_alone_ms": sum(per_class.values()),
            "plain_per_job_ms": ms_plain, "plain_jobs_per_s": jobs_n / (ms_plain / 1e3)}


def bench_ext_product(P, stream, batch=4096, cpu=False):
    """GLWE x GGSW external products: N = 2048, q = largest prime < 2^54 with
    q = 1 mod 4096, log_basis 7 (7 digits), k = 1, L = 1, one GGSW, 4096 ciphertexts."""
    q = P.prev_prime_congruent(1 << 54, 4096)
    tab = P.DcrtTable(11, [q])
    g = P.GadgetBasis(P.RnsBase([q]), 7)
    k, n = 1, 2048
    ggsw = P.DeviceBuffer((k + 1) * g.d * (k + 1) * n)
    glwe = P.DeviceBuffer(batch * (k + 1) * n)
    out = P.DeviceBuffer(batch * (k + 1) * n)
    tab.fill_uniform(ggsw, (k + 1) * g.d * (k + 1), seed=0x5EED0004, stream=stream)
    tab.fill_uniform(glwe, batch * (k + 1), seed=0x5EED0005, stream=stream)
    ws = P.DeviceBuffer(P.ext_product_workspace_size(tab, g, k, batch) // 8 + 1)
    ms = _time_stream(P, stream, lambda: P.external_product(tab, g, k, glwe, ggsw, out, batch, workspace=ws,
                                                            stream=stream), 10)
    ms_coeff = _time_stream(P, stream, lambda: P.external_product_coeff(tab, g, k, glwe, ggsw, out, batch,
                                                                        workspace=ws, stream=stream), 10)
    # butterflies per ciphertext: (k+1)*d forward + (k+1) inverse NTTs of N/2 * log2 N
    bfly_fwd = (k + 1) * g.d * (n // 2) * 11
    bfly_all = bfly_fwd + (k + 1) * (n // 2) * 11
    io_bytes = batch * (k + 1) * n * 8 * 2 + ggsw.count * 8
    res = {"workload": "GLWE x GGSW external product, N=2048, q < 2^54, B = 2^7, d = 7, k = 1, 4096 ciphertexts",
           "kernel": "ext_fused_kernel (decompose -> NTT -> MAC [-> INTT] in one launch, one CTA per ciphertext)",
           "ms_per_batch": ms, "ext_products_per_s": batch / (ms / 1e3),
           "ntt_domain_out": {"ms_per_batch": ms, "ext_products_per_s": batch / (ms / 1e3),
                              "g_butterflies_per_s": batch * bfly_fwd / (ms / 1e3) / 1e9,
                              "hbm_gbs": io_bytes / (ms / 1e3) / 1e9},
           "coeff_out_with_intt": {"ms_per_batch": ms_coeff, "ext_products_per_s": batch / (ms_coeff / 1e3),
                                   "g_butterflies_per_s": batch * bfly_all / (ms_coeff / 1e3) / 1e9,
                                   "hbm_gbs": io_bytes / (ms_coeff / 1e3) / 1e9}}
    if cpu:
        import oracle as O
        t0 = time.perf_counter()
        ot = O.DcrtTable(11, [q])
        ob = O.RnsBase([q])
        og = O.GadgetBasis(ob, 7)
        lat = O.Lattice(ot, ob, og)
        sample = 2048
        gg = O.uniform(1, 1, q, (k + 1) * og.d * (k + 1) * n)
        ct = O.uniform(2, 2, q, sample * (k + 1) * n)
        t0 = time.perf_counter()
        lat.external_product(k, ct, gg, batch=sample, threads=cpu_threads())
        dt = time.perf_counter() - t0
        res["cpu_port_ext_products_per_s"] = sample / dt
        res["cpu_port_sample"] = f"{sample} ciphertexts on {cpu_threads()} threads, {dt:.2f} s"
    return res


def bench_hybrid_ks(P, stream, batches=(1, 8, 32)):
    """Hybrid RNS key switch (N = 2^15, L = 16 primes + K = 4 special primes,
    4-limb digit groups, k = 1): time per key switch at several batch sizes."""
    moduli = P.ntt_primes(1 << 50, 1 << 16, 20)
    kt = P.DcrtTable(15, moduli)
    kt.autotune(8)
    kq = P.DcrtTable(15, moduli[:16])
    hks = P.HybridKeySwitch(kt, 16, 4, 4)
    key = P.DeviceBuffer(hks.dnum * 2 * 20 * 32768)
    kt.fill_uniform(key, hks.dnum * 2, seed=0x5EED0006, stream=stream)
    res = {"workload": "hybrid key switch, N=2^15, L=16 + K=4 special primes, alpha=4 (dnum=4), k=1",
           "rows_transformed_per_key_switch": 4 * 20 + 4 * 2 + 16 * 2}
    for B in batches:
        di, do = P.DeviceBuffer(B * 2 * 16 * 32768), P.DeviceBuffer(B * 2 * 16 * 32768)
        kq.fill_uniform(di, 2 * B, seed=0x5EED0007, stream=stream)
        ws = P.DeviceBuffer(hks.workspace_size(1, 1, B) // 8 + 1)
        ms = _time_stream(P, stream, lambda: hks.key_switch(1, 1, key, di, do, B, workspace=ws, stream=stream), 5)
        res[f"batch_{B}"] = {"ms_per_batch": ms, "us_per_key_switch": ms * 1e3 / B,
                             "key_switches_per_s": B / (ms / 1e3)}
        del di, do, ws
    return res


def bench_widened(P, stream, batch=64):
    """The rows built beside the hot path, on the key-switch shape (N = 2^15,
    L = 16 primes < 2^50, k = 1): GLWE encryption, BFV decryption and the
    NTT-domain automorphism (BigUint gadget, log_basis 50 -> 16 digits), per
    ciphertext, with the HBM bytes each one must move."""
    import numpy as np
    log_n, L, k, n = 15, 16, 1, 1 << 15
    moduli = P.ntt_primes(1 << 50, 2 * n, L)
    tab = P.DcrtTable(log_n, moduli)
    tab.autotune(16)
    ct_words = (k + 1) * L * n
    sk = P.DeviceBuffer(k * L * n)
    tab.fill_uniform(sk, k, seed=0x51, stream=stream)
    msg = P.DeviceBuffer(batch * L * n)
    tab.fill_uniform(msg, batch, seed=0x52, stream=stream)
    ct = P.DeviceBuffer(batch * ct_words)
    out = P.DeviceBuffer(batch * ct_words)
    enc = P.GlweEncryptor(tab)
    scale = [1] * L
    res = {"shape": "N=2^15, L=16 primes < 2^50, k=1, batch %d" % batch}
    ms = _time_stream(P, stream, lambda: enc.encrypt(k, sk, msg, scale, 7, 0, ct, batch, stream=stream), 5)
    nbytes = batch * (ct_words + L * n) * 8
    res["encrypt"] = {"us_per_ciphertext": ms * 1e3 / batch, "hbm_gbs": nbytes / (ms / 1e3) / 1e9}
    dec = P.BfvDecryptor(tab, 65537, 2199023190017)
    m = P.DeviceBuffer(batch * n)
    ms = _time_stream(P, stream, lambda: dec.decrypt(k, sk, ct, m, batch, stream=stream), 5)
    nbytes = batch * (ct_words + n) * 8
    res["decrypt"] = {"us_per_ciphertext": ms * 1e3 / batch, "hbm_gbs": nbytes / (ms / 1e3) / 1e9}
    g = P.GadgetBasis(P.RnsBase(moduli), 50)
    key = P.DeviceBuffer(k * g.d * (k + 1) * L * n)
    tab.fill_uniform(key, k * g.d * (k + 1), seed=0x53, stream=stream)
    ws = P.DeviceBuffer(P.lattice.nat.lib().pg_glwe_automorphism_workspace_size(tab.h, g.h, k, batch) // 8 + 1)
    ms = _time_stream(P, stream, lambda: P.glwe_automorphism(tab, g, k, 5, key, ct, out, batch, workspace=ws,
                                                             stream=stream), 3)
    res["automorphism"] = {"us_per_ciphertext": ms * 1e3 / batch, "digits": g.d,
                           "rows_transformed_per_ciphertext": L + g.d * L}
    # the reference-form key switch (CrtGlweKeySwitchingKey::key_swithching_inplace,
    # BigUint gadget over all 16 limbs, 16 digits): coefficient-form input,
    # NTT-domain output, k_in = k_out = 1
    c_in = P.DeviceBuffer(batch * ct_words)
    tab.fill_uniform(c_in, batch * (k + 1), seed=0x54, stream=stream)
    kws = P.DeviceBuffer(P.key_switch_workspace_size(tab, g, k, k, batch) // 8 + 1)
    ms = _time_stream(P, stream, lambda: P.key_switch(tab, g, k, k, key, c_in, out, batch, workspace=kws,
                                                      stream=stream), 3)
    res["key_switch_biguint_gadget"] = {"us_per_ciphertext": ms * 1e3 / batch, "digits": g.d,
                                        "rows_transformed_per_ciphertext": L + g.d * L,
                                        "path": "pg_key_switch: compose -> digits -> forward NTT lifting the "
                                                "digits on load -> MAC"}
    return res


def bench_expand(P, stream, cpu=False):
    """Coefficient expansion and field trace on the reference benchmark's shapes
    (primus_fhe_core/benches/expand_coeff.rs: k = 2, two primes < 2^50,
    log_basis 20, N = 2^10, 2^11, 2^12, full expansion count = N): device time of
    one expansion (N-1 automorphisms in log2 N levels) and of a trace."""
    import time
    res = {"shape": "k=2, L=2 primes < 2^50, log_basis 20, count = N"}
    k = 2
    for log_n in (10, 11, 12):
        n = 1 << log_n
        moduli = P.ntt_primes(1 << 50, 2 << 12, 2)
        tab = P.DcrtTable(log_n, moduli)
        g = P.GadgetBasis(P.RnsBase(moduli), 20)
        glwe = (k + 1) * 2 * n
        keys = P.DeviceBuffer(log_n * k * g.d * glwe)
        tab.fill_uniform(keys, log_n * k * g.d * (k + 1), seed=0x90 + log_n, stream=stream)
        ct = P.DeviceBuffer(glwe)
        tab.fill_uniform(ct, k + 1, seed=0xA0 + log_n, stream=stream)
        out = P.DeviceBuffer(n * glwe)
        ws = P.DeviceBuffer(P.lattice.nat.lib().pg_glwe_expand_workspace_size(tab.h, g.h, k, n) // 8 + 1)
        ms = _time_stream(P, stream, lambda: P.glwe_expand_coefficients(tab, g, k, keys, n, ct, out, workspace=ws,
                                                                        stream=stream), 3)
        tb = 64
        cts = P.DeviceBuffer(tb * glwe)
        tab.fill_uniform(cts, tb * (k + 1), seed=0xB0 + log_n, stream=stream)
        tout = P.DeviceBuffer(tb * glwe)
        tws = P.DeviceBuffer(P.lattice.nat.lib().pg_glwe_trace_workspace_size(tab.h, g.h, k, tb) // 8 + 1)
        ms_tr = _time_stream(P, stream, lambda: P.glwe_trace(tab, g, k, keys, cts, tout, tb, workspace=tws,
                                                             stream=stream), 3)
        res[f"N=2^{log_n}"] = {"expand_ms": ms, "automorphisms": n - 1, "digits": g.d,
                               "us_per_automorphism": ms * 1e3 / (n - 1),
                               "trace_batch64_us_per_ciphertext": ms_tr * 1e3 / tb}
        if cpu and log_n == 10:
            import numpy as np
            import oracle as O
            lat = O.Lattice(O.DcrtTable(log_n, moduli), O.RnsBase(moduli), O.GadgetBasis(O.RnsBase(moduli), 20))
            hk = keys.numpy()[: k * g.d * glwe * log_n].astype(np.uint64)
            t0 = time.perf_counter()
            lat.expand(k, hk, n, ct.numpy())
            dt = time.perf_counter() - t0
            res[f"N=2^{log_n}"]["cpu_port_expand_ms"] = dt * 1e3
            res[f"N=2^{log_n}"]["cpu_port_sample"] = "one full expansion, oracle restatement, 1 thread"
    return res


def bench_pointwise(P, stream, polys=64):
    """Pointwise DCRT ops (DcrtPolynomial::mul_assign / add_mul_assign / add_assign /
    mul_scalar_assign) on 64 polys of N = 2^16, L = 24 (0.8 GB per operand, beyond
    L2): HBM GB/s of each against the measured copy peak."""
    L_, N_ = 24, 1 << 16
    tab = P.DcrtTable(16, P.ntt_primes(1 << 50, 2 * N_, L_))
    x, y, z = (P.DeviceBuffer(polys * L_ * N_) for _ in range(3))
    for i, b in enumerate((x, y, z)):
        tab.fill_uniform(b, polys, seed=0x70 + i, stream=stream)
    peak, kind = load_peaks()
    words = polys * L_ * N_
    ops = {"mul": (lambda: tab.mul(x, y, polys, stream=stream), 3),
           "add_mul": (lambda: tab.add_mul(x, y, z, polys, stream=stream), 4),
           "add": (lambda: tab.add(x, y, polys, stream=stream), 3),
           "mul_scalar": (lambda: tab.mul_scalar(x, [3] * L_, polys, stream=stream), 2)}
    res = {"shape": f"{polys} polys x 24 limbs x 2^16", "peak_gbs": peak, "peak_source": kind}
    for name, (fn, streams) in ops.items():
        ms = _time_stream(P, stream, fn, 10)
        gbs = streams * words * 8 / (ms / 1e3) / 1e9
        res[name] = {"ms": ms, "hbm_gbs": gbs, "frac_of_peak": gbs / peak}
    return res


def run_workload(args):
    """One secondary workload alone (for profiler captures and focused runs)."""
    import primus_b200 as P
    stream = P.Stream()
    fn = {"polymul_n1024": lambda: bench_polymul_1024(P, stream),
          "uneven_batch": lambda: bench_uneven(P, stream),
          "ext_product": lambda: bench_ext_product(P, stream, cpu=not args.no_cpu),
          "hybrid_ks": lambda: bench_hybrid_ks(P, stream, batches=tuple(args.ks_batches)),
          "widened": lambda: bench_widened(P, stream),
          "pointwise": lambda: bench_pointwise(P, stream),
          "expand": lambda: bench_expand(P, stream, cpu=not args.no_cpu),
          "served_mixed": lambda: bench_served(P, stream),
          "autotune_L24": lambda: bench_autotune(P)}[args.workload]
    print(json.dumps({"workload_name": args.workload, **fn()}))
    return 0


def bench_autotune(P):
    """Kernel shape chosen by the autotuner for each ring degree (L = 24 primes,
    about 2^24 residues per launch), with the default shape's time beside it."""
    out = {}
    for ln in range(10, 17):
        n = 1 << ln
        t = P.DcrtTable(ln, P.ntt_primes(1 << 50, 2 * n, 24))
        polys = max(1, (1 << 24) // (n * 24))
        r = t.autotune(polys)
        out[f"N=2^{ln}"] = {k: {"shape": r[k]["name"], "us": round(r[k]["us"], 1),
                                "default_us": round(r[k]["default_us"], 1)}
                            for k in ("forward", "inverse", "round_trip")}
        out[f"N=2^{ln}"]["polys"] = polys
    return out


def bench_served(P, stream, count=2000, seed=0x5EED0005, slots=4):
    """Mixed request stream: 50% RNS polymul (N = 2^12..2^16, L = 4..24), 30%
    external product (the N = 2048 shape above), 20% hybrid RNS key switch
    (N = 2^15, L = 16 plus K = 4 special primes, 4-limb digit groups, k = 1).  The plain form runs
    each request as its own synchronous call; the served form replays the same
    trace into the continuous-batching server at Poisson arrival rates."""
    rng = np.random.default_rng(seed)
    pm_lns = list(range(12, 17))
    pm_tables = {ln: P.DcrtTable(ln, P.ntt_primes(1 << 50, 2 << ln, 24)) for ln in pm_lns}
    for t in pm_tables.values():  # kernel shapes per degree, as a serving process would at start-up
        t.autotune(max(1, (1 << 22) // (t.n * 24)))
    pm_batch = P.PolymulBatch(list(pm_tables.values()))
    xq = P.prev_prime_congruent(1 << 54, 4096)
    xt = P.DcrtTable(11, [xq])
    xg = P.GadgetBasis(P.RnsBase([xq]), 7)
    xkey = P.DeviceBuffer(2 * xg.d * 2 * 2048)
    xt.fill_uniform(xkey, 2 * xg.d * 2, seed=seed + 1, stream=stream)
    # hybrid key switch: Q = 16 primes, P = 4 special primes, 4-limb digit groups
    ks_moduli = P.ntt_primes(1 << 50, 1 << 16, 20)
    kt = P.DcrtTable(15, ks_moduli)
    kt.autotune(8)
    kq = P.DcrtTable(15, ks_moduli[:16])  # Q limbs only, for the input generator
    hks = P.HybridKeySwitch(kt, 16, 4, 4)
    kkey = P.DeviceBuffer(hks.dnum * 2 * 20 * 32768)
    kt.fill_uniform(kkey, hks.dnum * 2, seed=seed + 2, stream=stream)
    kinds = rng.choice(3, size=count, p=[0.5, 0.3, 0.2])
    trace = []  # (kind, buffers...)
    for i, kd in enumerate(kinds):
        if kd == 0:
            ln, L = int(rng.choice(pm_lns)), int(rng.integers(4, 25))
            t = pm_tables[ln]
            a, b = P.DeviceBuffer(t.L << ln), P.DeviceBuffer(t.L << ln)
            t.fill_uniform(a, 1, seed=seed + 3, stream0=64 * i, stream=stream)
            t.fill_uniform(b, 1, seed=seed + 4, stream0=64 * i, stream=stream)
            # the job array is built once, as the served request is
            trace.append(("pm", a, b, ln, L, pm_batch.prepare([(a, b, ln, L)])))
        elif kd == 1:
            di, do = P.DeviceBuffer(2 * 2048), P.DeviceBuffer(2 * 2048)
            xt.fill_uniform(di, 2, seed=seed + 5, stream0=2 * i, stream=stream)
            trace.append(("xp", di, do))
        else:
            di, do = P.DeviceBuffer(2 * 16 * 32768), P.DeviceBuffer(2 * 16 * 32768)
            kq.fill_uniform(di, 2, seed=seed + 6, stream0=32 * i, stream=stream)
            trace.append(("ks", di, do))
    stream.synchronize()

    # ---- plain: one synchronous call per request, in arrival order
    def plain_call(it):
        if it[0] == "pm":
            pm_batch.run(it[5], use_graph=False, stream=stream)
        elif it[0] == "xp":
            P.external_product(xt, xg, 1, it[1], xkey, it[2], 1, stream=stream)
        else:
            hks.key_switch(1, 1, kkey, it[1], it[2], 1, stream=stream)

    for it in trace[:50]:
        plain_call(it)
    stream.synchronize()
    e0, e1 = P.Event(), P.Event()
    service = np.zeros(count)
    t_all = time.perf_counter()
    for i, it in enumerate(trace):
        e0.record(stream)
        plain_call(it)
        e1.record(stream)
        stream.synchronize()
        service[i] = e0.elapsed_ms(e1) * 1e3
    plain_wall = time.perf_counter() - t_all
    plain_rps = count / plain_wall
    kind_names = {"pm": "polymul", "xp": "ext_product", "ks": "key_switch"}
    per_kind = {}
    for key, name in kind_names.items():
        sel = np.array([it[0] == key for it in trace])
        per_kind[name] = {"count": int(sel.sum()), "gpu_service_p50_us": float(np.percentile(service[sel], 50))}

    def plain_replay(arrivals):
        # a single FIFO worker running each request as its own synchronous call
        lat = np.zeros(count)
        t0 = time.perf_counter()
        for i, it in enumerate(trace):
            target = t0 + arrivals[i] * 1e-6
            while time.perf_counter() < target:
                pass
            plain_call(it)
            stream.synchronize()
            lat[i] = (time.perf_counter() - target) * 1e6
        return lat, time.perf_counter() - t0

    # ---- served
    srv = P.Server(memory_budget_bytes=2 * slots << 30, slots=slots, max_batch=512,
                   polymul_tables=list(pm_tables.values()))
    xid = srv.register_key(2, xt, xg, 1, 1, xkey)
    kid = srv.register_hybrid_key(hks, 1, 1, kkey)
    reqs = []
    for it in trace:
        if it[0] == "pm":
            reqs.append(P.polymul_request(it[1], it[2], it[3], it[4]))
        elif it[0] == "xp":
            reqs.append(P.ext_product_request(xid, it[1], it[2]))
        else:
            reqs.append(P.key_switch_request(kid, it[1], it[2]))
    # warm-up: the whole trace at once, then at twice the plain rate
    srv.replay(reqs, np.zeros(count))
    srv.replay(reqs, np.cumsum(rng.exponential(1e6 / (2 * plain_rps), count)))
    srv.stats(reset=True)

    kind_of = np.array([kind_names[it[0]] for it in trace])

    def summary(lat, wall, offered):
        ok = lat[lat >= 0]
        # per kind: which requests make up the tail
        p99_kind = {name: float(np.percentile(lat[(kind_of == name) & (lat >= 0)], 99))
                    for name in kind_names.values() if ((kind_of == name) & (lat >= 0)).any()}
        return {"offered_rps": offered, "throughput_rps": len(ok) / wall, "p50_us": float(np.percentile(ok, 50)),
                "p99_us": float(np.percentile(ok, 99)), "p99_us_by_kind": p99_kind,
                "rejected": int((lat < 0).sum())}

    plain_runs, served_runs = [], []
    for mult in (0.5, 0.9, 2.0, 2.25, 2.5, 2.75, 3.0, 3.25, 3.5, 3.75, 4.0, 8.0, None):
        offered = None if mult is None else plain_rps * mult
        arrivals = np.zeros(count) if mult is None else np.cumsum(rng.exponential(1e6 / offered, count))
        if mult is not None and mult < 1:
            lat, wall = plain_replay(arrivals)
            plain_runs.append(summary(lat, wall, offered))
        t0 = time.perf_counter()
        lat = srv.replay(reqs, arrivals)
        served_runs.append(summary(lat, time.perf_counter() - t0, offered))
        st = srv.stats(reset=True)
        served_runs[-1].update({k: st[k] for k in ("mean_batch", "enqueue_mean_us", "enqueue_max_us")})
    srv.close()
    best = max(r["throughput_rps"] for r in served_runs)
    # the served figure at no worse tail latency: the highest served throughput
    # whose p99 is within the plain path's p99 at 0.9x its own capacity
    plain_p99 = max(r["p99_us"] for r in plain_runs)
    within = [r["throughput_rps"] for r in served_runs if r["p99_us"] <= plain_p99]
    at_p99 = max(within) if within else None
    return {"workload": "served mixed stream: 50% polymul N=2^12..2^16 L=4..24, 30% ext product (N=2048, k=1, "
                        "7-bit gadget), 20% hybrid key switch (N=2^15, L=16 + K=4 special primes, 4-limb digit "
                        "groups); Poisson arrivals",
            "requests": count, "slots": slots, "plain_capacity_rps": plain_rps, "per_kind": per_kind,
            "plain": plain_runs, "served": served_runs, "served_max_rps": best,
            "served_over_plain_capacity": best / plain_rps,
            "plain_p99_us_at_0_9x": plain_p99, "served_rps_at_plain_p99": at_p99,
            "served_over_plain_at_plain_p99": (at_p99 / plain_rps) if at_p99 else None}

def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="primus_b200", choices=["primus_b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-extra", action="store_true", help="skip the secondary workloads")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default kernel shapes (no autotuner launches), for profiler captures")
    ap.add_argument("--polys", type=int, default=POLYS,
                    help="polys per step (default 128 = the workload; smaller only for profiler captures)")
    ap.add_argument("--workload", default=None,
                    choices=["polymul_n1024", "uneven_batch", "ext_product", "hybrid_ks", "widened",
                             "pointwise", "expand", "served_mixed", "autotune_L24"],
                    help="run only this secondary workload and print its result")
    ap.add_argument("--ks-batches", type=int, nargs="+", default=[1, 8, 32],
                    help="key switches per call timed by --workload hybrid_ks")
    args = ap.parse_args(argv)
    set_polys(args.polys)
    if args.workload:
        return run_workload(args)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
