"""Benchmark: LULESH sedov Lagrange step, zone-cycles/s on B200.

Workload (the headline metric, zone-cycles/s at -s 100 on one B200): one domain of
-s 100 (1,000,000 hex elements, 1,030,301 nodes), FP64, 11 regions, balance 1,
cost 1.  A step is one cycle (TimeIncrement + LagrangeLeapFrog) over the
whole mesh.  State (~0.57 GB) is far larger than the 126 MB L2, so no flush
is needed between cycles.

  value   zone-cycles/s over exactly K device-timed cycles (CUDA events on the
          library's stream), graph-captured, no host sync inside
  e2e     the same metric through the host-driven C-ABI call
          (lulesh_host_cycle): per cycle the host copies the time state in
          (H2D) and reads time/dt/status back (D2H) and waits, as the
          reference's loop does (TimeIncrement + checkErrors on the host)
  energy_check
          Final Origin Energy read right after the K timed cycles (cycle
          W + K), against the reference CUDA build's energy at that cycle:
          the golden table tests/golden/cuda_reference.json (written by
          tests/golden/make_golden_cuda.py) and the live gpu_reference run

With --gpus N (torchrun), the ranks run the decomposed problem: 2x2x2
subdomains of one global sedov mesh split over the ranks (distributed.py),
with the halos and the dt minimum exchanged between GPUs every cycle; each
GPU holds about 1,000,000 elements (weak scaling).  value is the total over
ranks using the max time over ranks.

--impl reference times the reference's own OpenMP CPU build
(oracle/_ref/lulesh_omp, compiled from LULESH/omp_4.0) on this host's cores.

At one GPU the line also carries:
  gpu_reference  the reference's own CUDA single-domain build
                 (oracle/_ref/lulesh_ref_cuda) on the same GPU: its timed
                 region (lulesh.cu:4851-4886) over 500 cycles, and its energy
                 after W + K cycles
  mixed          config 4: -s 120, 1000 cycles, FP64 against the mixed-precision
                 path (device time, energy and symmetry error)
  subdomains     config 2's two forms: -s 100 as one domain against 2x2x2
                 subdomains of -s 50 (fused and staged halo exchange), device
                 time per cycle and the energies after the same cycles
  serving        the seeded Poisson stream of sedov jobs (lambda 50/s, edge
                 log-uniform in [8,64], regions U[5,20], iterations
                 U[100,2000]; all 2,000 jobs by default) served with continuous
                 batching vs the same stream run job by job through the plain
                 path: zone-cycles/s over the makespan, p50/p99 job latency
                 (completion - arrival, wall clock), capacity (all queued; the
                 plain path's as the median of 3 repeats over a 1-in-10
                 sample), energies compared per job
  batch          the 64-job batch (rng seed 0) in one graph launch with
                 autotuned launch shapes vs each job's own plain run
  cpu_baseline   the reference omp build on this host (thread count from a
                 sweep at -s 100 -i 3, 2 repeats per count, shared with
                 --impl reference)
"""
import argparse
import json
import os
import socket
import statistics
import subprocess
import tempfile
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "cuda-ipc-benchmarks_b200")
ORACLE = os.path.join(REPO, "oracle")
GOLDEN_CUDA = os.path.join(REPO, "tests", "golden", "cuda_reference.json")
for _p in (PKG, ORACLE):
    if _p not in sys.path:
        sys.path.insert(0, _p)

NX = 100
ZONES = NX ** 3
METRIC = "zone-cycles/s at -s 100 on 1 B200"
UNIT = "zone-cycles/s"
ENERGY_RTOL = 1e-9  # the parity bar against the reference CUDA build
# Algorithmic bytes per zone-cycle of each phase (compulsory traffic at the
# four dependency boundaries of the step, enumerated array by array in
# bytes_model.py): force 152, nodal update 128, kinematics + monoQ gradient
# 176, monoQ region + EOS + volume + dt 196; 652 per cycle.  This build's own
# traffic (corner forces written and read back) is 896.
import bytes_model  # noqa: E402

ALG_BYTES = {k: float(v) for k, v in bytes_model.phase_bytes().items()}
ALG_BYTES_STEP = bytes_model.step_bytes()
BUILD_BYTES = {k: float(v) for k, v in bytes_model.phase_bytes(bytes_model.THIS_BUILD).items()}
BUILD_BYTES_STEP = bytes_model.step_bytes(bytes_model.THIS_BUILD)
LAUNCHES_PER_CYCLE = 5  # time_increment, force, nodal, kinematics, eos
# FP64 flops per element of each phase (an FMA counts 2), measured with
# ncu's smsp__sass_thread_inst_executed_op_{dfma,dadd,dmul}_pred_on counters
# at -s 64 (profiles/cycle_kernels_s64_full.md; the EOS after its
# unit-density form, profiles/eos_unit_density_s64.md); nodal is per node.
FP64_FLOPS = {"force": 1427.0, "nodal": 50.2, "kinematics": 814.0, "eos": 359.9}


def fp64_peak_tflops(dev):
    """Nominal FP64 (non-tensor) peak of the device: SMs x 64 FMA lanes x 2
    flops x max SM clock.  No measured FP64 figure exists for this pool."""
    import torch

    props = torch.cuda.get_device_properties(dev)
    mhz = 1965.0
    try:
        out = subprocess.run(["nvidia-smi", "-i", str(dev), "--query-gpu=clocks.max.sm",
                              "--format=csv,noheader,nounits"], capture_output=True, text=True,
                             timeout=20).stdout.strip()
        mhz = float(out.splitlines()[0])
    except Exception:
        pass
    return props.multi_processor_count * 64 * 2 * mhz * 1e6 / 1e12


def measured_peak_gbs():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def lscpu_summary() -> dict:
    """CPU model and core counts as lscpu reports them."""
    keys = {"Model name": "model", "CPU(s)": "cpus", "Core(s) per socket": "cores_per_socket",
            "Socket(s)": "sockets", "Thread(s) per core": "threads_per_core"}
    out = {"affinity_cpus": host_cores()}
    try:
        text = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=20).stdout
    except Exception:
        return out
    for line in text.splitlines():
        if ":" not in line:
            continue
        k, v = (t.strip() for t in line.split(":", 1))
        if k in keys:
            out[keys[k]] = int(v) if v.isdigit() else v
    if isinstance(out.get("cores_per_socket"), int) and isinstance(out.get("sockets"), int):
        out["physical_cores"] = out["cores_per_socket"] * out["sockets"]
    return out


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, period_ms: int = 100):
        self.gpu = gpu_index
        self.period = period_ms
        self.proc = None
        self.path = None

    def start(self):
        # the samples go to BENCH_CLOCKS_DIR (default: the system temp dir)
        out_dir = os.environ.get("BENCH_CLOCKS_DIR") or tempfile.gettempdir()
        os.makedirs(out_dir, exist_ok=True)
        self.path = os.path.join(out_dir, f"clocks_gpu{self.gpu}_{os.getpid()}.csv")
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", str(self.period)],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                t = [x.strip() for x in line.split(",")]
                if len(t) < 9:
                    continue
                try:
                    sm.append(float(t[1]))
                    smax.append(float(t[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, t[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# the reference's own builds (CPU baseline and GPU reference legs)

def omp_run(args, threads):
    import oracle

    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close")
    out = subprocess.run([oracle.REF_OMP, *args], env=env, capture_output=True, text=True,
                         timeout=900)
    if out.returncode != 0:
        raise RuntimeError(f"lulesh_omp {' '.join(args)} failed: {out.stderr[-300:]}")
    return oracle.parse_report(out.stdout)


def omp_sweep(cores, its=3, repeats=2):
    """Thread count of the omp build: each candidate runs -s 100 -i 3 twice
    and the best median rate wins.  The omp build needs >= 2 threads (1
    segfaults at lulesh.cc:585) and degrades badly when over-subscribed.
    The result is kept in a file in the temp dir (per host and core count),
    so the reference arm and this arm, run one after the other on the same
    machine, use the same thread count."""
    cache = os.path.join(tempfile.gettempdir(),
                         f"lulesh_omp_sweep_{socket.gethostname()}_{cores}.json")
    try:
        with open(cache) as f:
            d = json.load(f)
        if d.get("cores") == cores and d.get("threads"):
            return dict(d, cached=True)
    except Exception:
        pass
    cand = sorted({t for t in (2, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256)
                   if t <= cores} | ({cores} if cores >= 2 else set()))
    table = []
    for t in cand:
        rates = []
        for _ in range(repeats):
            r = omp_run(["-s", str(NX), "-i", str(its)], t)
            rates.append(1e6 / r["grind"] if r.get("grind") else 0.0)
        table.append({"threads": t, "zone_cycles_per_s": rates,
                      "median": statistics.median(rates)})
    best = max(table, key=lambda e: e["median"])
    d = {"cores": cores, "threads": best["threads"], "rate": best["median"],
         "sweep": f"-s {NX} -i {its}, {repeats} runs per thread count", "table": table,
         "lscpu": lscpu_summary()}
    try:
        with open(cache, "w") as f:
            json.dump(d, f)
    except Exception:
        pass
    return dict(d, cached=False)


def cpu_baseline_sample(target_s=12.0):
    """Reference omp_4.0 build on this host, bounded sample of -s 100."""
    import oracle

    if not os.path.exists(oracle.REF_OMP):
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "oracle/_ref/lulesh_omp missing (built from the reference tree)"}
    cores = host_cores()
    sw = omp_sweep(cores)
    threads, rate = sw["threads"], sw["rate"]
    its = int(max(2, min(60, target_s * rate / ZONES))) if rate > 0 else 3
    r = omp_run(["-s", str(NX), "-i", str(its)], threads)
    value = 1e6 / r["grind"]
    return {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"lulesh_omp -s {NX} -i {its} (reference LULESH/omp_4.0), "
                      f"OMP_NUM_THREADS={threads} of {cores} host CPUs, elapsed "
                      f"{r['elapsed']:.2f} s",
            "thread_sweep": sw}


def golden_energy(nx, cycles):
    """The reference CUDA build's Final Origin Energy after `cycles` cycles
    of -s nx, from the committed golden table (None if not tabulated)."""
    try:
        with open(GOLDEN_CUDA) as f:
            runs = json.load(f)["runs"]
    except Exception:
        return None
    r = runs.get(f"-s {nx} -i {cycles}")
    if r and r.get("cycles") == cycles:
        return r["energy"]
    return None


def gpu_reference_leg(energy_cycles, timing_cycles=500):
    """The reference CUDA single-domain build (oracle/_ref/lulesh_ref_cuda,
    compiled from LULESH/cuda/src for sm_100a) on this GPU: its own timed
    region (lulesh.cu:4851-4886, host loop with a dt readback per cycle)
    over `timing_cycles` cycles, and its energy after `energy_cycles`."""
    import oracle

    if not os.path.exists(oracle.REF_CUDA):
        return {"unavailable": "oracle/_ref/lulesh_ref_cuda was not built"}
    out = {"binary": "oracle/_ref/lulesh_ref_cuda (reference LULESH/cuda/src, sm_100a)"}
    with tempfile.TemporaryDirectory() as d:  # it writes xyz.asc in its cwd
        for key, its in (("timing", timing_cycles), ("energy", energy_cycles)):
            r = subprocess.run([oracle.REF_CUDA, "-s", str(NX), "x", str(its)], cwd=d,
                               capture_output=True, text=True, timeout=600)
            if r.returncode != 0:
                return {"unavailable": f"lulesh_ref_cuda exited {r.returncode}: "
                                       f"{r.stderr[-200:]}"}
            rep = oracle.parse_report(r.stdout)
            out[key] = {"cycles": rep.get("cycles"), "energy": rep.get("energy"),
                        "elapsed_s": rep.get("elapsed"), "grind_us": rep.get("grind")}
    t = out["timing"]
    out["zone_cycles_per_s"] = 1e6 / t["grind_us"] if t.get("grind_us") else None
    out["ms_per_cycle"] = t["grind_us"] * ZONES / 1e3 if t.get("grind_us") else None
    return out


# ---------------------------------------------------------------------------
# multi-rank helpers

def max_over_ranks(x: float, dist=None, device="cpu") -> float:
    """Max of a per-rank timing over all ranks (any torch.distributed backend)."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: int, seconds_max: float, world: int) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    return world * units_per_rank / seconds_max


def traffic_per_launch(kernel):
    p = os.path.join(REPO, "profiles", "traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return d["kernels"][kernel]["dram_bytes_per_launch_scaled"]
    except Exception:
        return None


def timed_cycles(s, stream, n):
    """Device time (ms) of n cycles on `stream` (CUDA events on that stream)."""
    import torch

    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    s.step(n)
    t1.record(stream)
    torch.cuda.synchronize()
    return t0.elapsed_time(t1)


# ---------------------------------------------------------------------------
# the side legs (one GPU)

def mixed_leg(nx=120, cycles=1000):
    """Config 4: -s nx for `cycles` cycles from the start, FP64 and mixed
    precision, device-timed; the mixed run's energy and symmetry error
    against the FP64 run, and the FP64 energy against the reference CUDA
    golden of the same run."""
    import torch
    import lulesh_b200 as L

    stream = torch.cuda.Stream()
    out = {"nx": nx, "zones": nx ** 3, "cycles": cycles}
    for name, flags in (("fp64", 0), ("mixed", L.FLAG_MIXED)):
        with L.LuleshSet(nx=nx, its=-1, flags=flags) as s:
            s.set_stream(stream.cuda_stream)
            s.step(0)  # build the graphs before the timed region
            ms = timed_cycles(s, stream, cycles)
            st = s.state()
            out[name] = {"ms_per_cycle": ms / cycles,
                         "zone_cycles_per_s": nx ** 3 * cycles / (ms / 1e3),
                         "energy": s.origin_energy(), "symmetry": s.symmetry(),
                         "cycle": st["cycle"], "status": st["status"]}
    e64, e32 = out["fp64"]["energy"], out["mixed"]["energy"]
    out["speedup"] = out["fp64"]["ms_per_cycle"] / out["mixed"]["ms_per_cycle"]
    out["energy_rel_error"] = abs(e32 - e64) / abs(e64)
    out["symmetry_max_abs"] = {"fp64": out["fp64"]["symmetry"][0],
                               "mixed": out["mixed"]["symmetry"][0]}
    g = golden_energy(nx, cycles)
    out["fp64_vs_reference_cuda"] = (None if g is None else
                                     {"golden": g, "rel": abs(e64 - g) / abs(g)})
    return out


def subdomain_leg(warmup=5, cycles=100):
    """Config 2's forms at -s 100 (1e6 elements): one domain, and 2x2x2
    subdomains of -s 50 with the fused and with the staged (reference
    Comm* sequence) halo exchange; device time per cycle after the same
    warm-up, and the energies after warm-up + cycles."""
    import torch
    import lulesh_b200 as L

    stream = torch.cuda.Stream()
    out = {"warmup": warmup, "cycles": cycles}
    forms = (("single_s100", dict(nx=100, tp=1, flags=0)),
             ("subdomains_2x2x2_s50_fused", dict(nx=50, tp=2, flags=0)),
             ("subdomains_2x2x2_s50_staged", dict(nx=50, tp=2, flags=L.FLAG_COMM_STAGED)))
    for name, kw in forms:
        with L.LuleshSet(its=-1, **kw) as s:
            s.set_stream(stream.cuda_stream)
            s.step(warmup)
            ms = timed_cycles(s, stream, cycles)
            out[name] = {"us_per_cycle": 1e3 * ms / cycles,
                         "zone_cycles_per_s": 1e6 * cycles / (ms / 1e3),
                         "energy": s.origin_energy(), "cycle": s.state()["cycle"]}
    e0 = out["single_s100"]["energy"]
    out["fused_equals_single_bitwise"] = out["subdomains_2x2x2_s50_fused"]["energy"] == e0
    out["staged_rel_vs_single"] = abs(out["subdomains_2x2x2_s50_staged"]["energy"] - e0) / abs(e0)
    return out


def unstructured_vs_structured(nx, steps, warmup):
    """The -s nx cube written as an lmesh file and run through the
    unstructured kernels (mesh tables read from HBM) against the -s nx run
    (tables computed from the element index): device time per cycle."""
    import torch
    import lmesh
    import lulesh_b200 as L

    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    out = {"nx": nx, "zones": nx ** 3, "steps": steps, "warmup": warmup}
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, f"box{nx}.lmesh")
        lmesh.write(path, lmesh.box(nx))
        for kind in ("structured", "unstructured"):
            s = (L.LuleshSet(nx=nx, its=-1) if kind == "structured"
                 else L.LuleshSet.from_mesh(path, its=-1))
            s.set_stream(stream.cuda_stream)
            s.step(warmup)
            ms = timed_cycles(s, stream, steps)
            out[kind] = {"ms_per_cycle": ms / steps,
                         "zone_cycles_per_s": nx ** 3 * steps / (ms / 1e3),
                         "phases_ms": s.profile_phases(5)}
            s.close()
    # (energies agree only at nx = 45, where the -s deposit equals the
    # lmesh one; the bit-for-bit comparison is a GPU test)
    out["ratio"] = out["unstructured"]["zone_cycles_per_s"] / out["structured"]["zone_cycles_per_s"]
    return out


# ---------------------------------------------------------------------------
# the arms

def run_ours(a, rank, world, local_rank):
    if world > 1:
        return run_distributed(a, rank, world, local_rank)
    import torch
    import lulesh_b200 as L

    torch.cuda.set_device(local_rank)
    dev = torch.cuda.current_device()
    # a real (non-legacy) stream: the library captures its cycle graph on it
    # and the timing events below are recorded on the same stream
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    total = a.warmup + a.steps
    s = L.LuleshSet(nx=NX, its=-1, device=dev)
    s.set_stream(stream.cuda_stream)
    tuning = None
    if a.tune:
        # the library's autotuner picks the launch shape (it restores the
        # state it started from); the tuned graphs are then built on a copy
        # of the state, so the cycle count below stays warm-up + steps
        tuning = s.autotune(trial_cycles=20, rounds=2)["best"]
        snap = s.checkpoint()
        s.step(max(1, tuning["graph_cycles"]))
        s.sync()
        s.restore(snap)
    s.step(a.warmup)
    s.sync()
    st0 = s.state()
    if st0["done"]:
        raise RuntimeError("problem finished during warm-up")

    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.3)  # let the sampler start before the timed region
    ms = timed_cycles(s, stream, a.steps)
    ck = clocks.stop()
    # the state at the end of the timed region: cycle W + K and its energy
    st = s.state()
    energy = s.origin_energy()
    if st["status"] != 0 or st["cycle"] != total or st["done"]:
        raise RuntimeError(f"run did not complete {total} cycles cleanly: {st}")
    value = aggregate_rate(ZONES * a.steps, ms / 1e3, 1)

    # per-phase device times (events around each phase, same stream); the
    # state goes on from here, so these and the e2e cycles run after the
    # energy above was read
    phases = s.profile_phases(a.profile_cycles)
    dom = max((k for k in ALG_BYTES), key=lambda k: phases.get(k, 0.0))
    peak, peak_kind = measured_peak_gbs()
    ach = ALG_BYTES[dom] * ZONES / (phases[dom] / 1e3) / 1e9
    step_ms_sum = sum(phases.values())
    fp64_nominal = fp64_peak_tflops(dev)
    # measured: independent FMA chains on every SM (lulesh_measure_fp64_peak)
    fp64_peak = 2.0 * L.measure_fp64_peak(dev) / 1e12
    fp64 = {k: FP64_FLOPS[k] * ZONES / (phases[k] / 1e3) / 1e12 for k in FP64_FLOPS}
    ach_step = ALG_BYTES_STEP * ZONES / (ms / a.steps / 1e3) / 1e9
    ach_build = BUILD_BYTES_STEP * ZONES / (ms / a.steps / 1e3) / 1e9

    # end-to-end through the host-driven C-ABI call
    # at least e2e_cycles host-driven cycles (a few tens of ms), so the
    # figure does not rest on a handful of host round trips
    e2e_n = max(a.steps, a.e2e_cycles)
    _, cur = s.host_cycle(None)
    tw = time.perf_counter()
    for _ in range(e2e_n):
        stc, cur = s.host_cycle(cur)
        if stc != 0:
            raise RuntimeError(f"host cycle failed: {stc}")
    e2e_s = time.perf_counter() - tw
    e2e_val = aggregate_rate(ZONES * e2e_n, e2e_s, 1)
    cycles_total = s.state()["cycle"]
    s.close()
    torch.cuda.synchronize()

    golden = golden_energy(NX, total)
    gpu_ref = gpu_reference_leg(total) if a.gpu_reference else None
    live = None
    if gpu_ref and "energy" in gpu_ref and gpu_ref["energy"].get("cycles") == total:
        live = gpu_ref["energy"]["energy"]
    energy_check = {
        "cycle": total, "energy": energy, "rtol": ENERGY_RTOL,
        "reference_cuda_golden": golden,
        "rel_vs_golden": None if golden is None else abs(energy - golden) / abs(golden),
        "reference_cuda_live": live,
        "rel_vs_live": None if live is None else abs(energy - live) / abs(live),
    }
    rels = [r for r in (energy_check["rel_vs_golden"], energy_check["rel_vs_live"])
            if r is not None]
    energy_check["ok"] = (all(r <= ENERGY_RTOL for r in rels) if rels else None)

    mixed_res = mixed_leg() if a.mixed else None
    sub_res = subdomain_leg() if a.subdomains else None
    serving_res = batch_res = None
    if a.serve_jobs > 0:
        import serving

        stream_jobs = serving.make_stream(n_jobs=2000)[:a.serve_jobs]
        cmp = serving.compare(stream_jobs, plain_repeats=a.plain_repeats)
        serving_res = dict(cmp, jobs=a.serve_jobs, of=2000, lambda_per_s=50.0)
    if a.batch_jobs > 0:
        import batching

        batch_res = batching.run_batch_vs_plain(batching.config3_jobs(n=a.batch_jobs))
    unstructured_res = None
    if a.unstructured > 0:
        unstructured_res = unstructured_vs_structured(a.unstructured, 200, 5)
    cpu = cpu_baseline_sample() if a.cpu_baseline else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: sedov blast generated in code (reference problem setup)",
        "config": {"workload": "LULESH sedov single domain -s 100 (1,000,000 elements), "
                               "FP64, -r 11 -b 1 -c 1, one cycle per step",
                   "nx": NX, "zones": ZONES, "regions": 11, "balance": 1, "cost": 1,
                   "parallelism": "single GPU",
                   "l2": "state ~0.57 GB > 126 MB L2: no flush needed",
                   "launch_shape": tuning or "defaults (--no-tune)"},
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": 16,
                "d2h_bytes_per_step": 80, "cycles": e2e_n,
                "how": "lulesh_host_cycle: H2D time/dt, one graph-launched cycle, "
                       "D2H time-control record, host waits each cycle"},
        "gpu_launches": LAUNCHES_PER_CYCLE * a.steps,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak,
                     "unit": "GB/s", "frac": ach / peak, "peak_kind": peak_kind,
                     "alg_bytes_per_zone": ALG_BYTES[dom],
                     "traffic": traffic_per_launch(dom),
                     "traffic_kind": "ncu dram bytes per launch (profiles/traffic.json), a "
                                     "lower bound: ncu writes L2 back between captured "
                                     "launches, so late write-backs fall outside the window",
                     "traffic_model": BUILD_BYTES[dom] * ZONES,
                     "traffic_model_kind": f"bytes_model.THIS_BUILD: {BUILD_BYTES[dom]:.0f} B "
                                           f"per element moved by this build's {dom} kernel"},
        "roofline_fp64": {"bound": "fp64", "unit": "TFLOP/s", "peak": fp64_peak,
                          "peak_kind": "measured (lulesh_measure_fp64_peak: independent "
                                       "register FMA chains on every SM, FMA = 2 flops)",
                          "nominal_peak": fp64_nominal,
                          "nominal_kind": "SMs x 64 FMA x 2 x max SM clock",
                          "kernels": {k: {"achieved": v, "frac": v / fp64_peak}
                                      for k, v in fp64.items()},
                          "flops_per_element": FP64_FLOPS},
        "roofline_step": {"achieved": ach_step, "frac": ach_step / peak,
                          "alg_bytes_per_zone_cycle": ALG_BYTES_STEP,
                          "build_bytes_per_zone_cycle": BUILD_BYTES_STEP,
                          "build_achieved": ach_build, "build_frac": ach_build / peak},
        "phases_ms": phases, "phases_sum_ms": step_ms_sum,
        "clocks": ck,
        "origin_energy": energy, "origin_energy_cycle": total,
        "energy_check": energy_check,
        "cycles_timed": a.steps, "cycles_total": cycles_total,
        "cycles_note": "the energy is read at the end of the timed region (warm-up + steps); "
                       "profile_phases and the e2e leg run on from there",
        "gpu_reference": gpu_ref,
        "cpu_baseline": cpu,
        "mixed": mixed_res, "subdomains": sub_res,
        "serving": serving_res, "batch": batch_res,
    }
    if unstructured_res is not None:
        line["unstructured"] = unstructured_res
    print(json.dumps(line), flush=True)


def run_distributed(a, rank, world, local_rank):
    """N > 1: the decomposed problem over the ranks (distributed.py)."""
    import datetime

    import torch
    import torch.distributed as dist
    import distributed as D

    # one GPU per rank; with fewer GPUs than ranks (a test of the host
    # transport on one GPU) ranks share devices round-robin
    torch.cuda.set_device(local_rank % max(1, torch.cuda.device_count()))
    backend = "gloo" if a.transport == "host" else "nccl"
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    clock = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    try:
        res = D.bench_decomposed(a.warmup, a.steps, dist, transport=a.transport, clock=clock)
    finally:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    ms = res["ms_max_over_ranks"]
    value = res["zones_total"] * a.steps / (ms / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: sedov blast generated in code (reference problem setup)",
        "config": {"workload": f"LULESH sedov -s {res['global_nx']} as 2x2x2 subdomains of "
                               f"-s {res['sub_nx']} over {world} GPUs "
                               f"({res['zones_total'] // world} elements per GPU), FP64",
                   "nx": res["sub_nx"], "tp": 2, "zones": res["zones_total"],
                   "parallelism": f"domain decomposition x{world}",
                   "transport": res["transport"],
                   "l2": "state per GPU > 126 MB L2: no flush needed"},
        "e2e": {"value": res["zones_total"] * a.steps / res["e2e_s_max_over_ranks"],
                "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": res["e2e_d2h_bytes_per_step"], "cycles": a.steps,
                "how": "the same cycles driven from the host through the exchange layer, each "
                       "cycle's reduced dt record read back to the host; host clock, max over "
                       "ranks"},
        "gpu_launches": res["launches_per_cycle"] * a.steps,
        "clocks": res["clocks"],
        "origin_energy": res["energy"], "origin_energy_cycle": a.warmup + a.steps,
        "halo_bytes_per_cycle": res["halo_bytes_per_cycle"],
    }
    print(json.dumps(line), flush=True)


def run_reference(a, rank, world):
    if rank != 0:
        return
    import oracle

    if not os.path.exists(oracle.REF_OMP):
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/lulesh_omp was not built"}))
        return
    cores = host_cores()
    sw = omp_sweep(cores)
    threads, rate = sw["threads"], sw["rate"]
    # warm-up run, then K cycles of the reference's own timed loop, bounded
    # to about two minutes of CPU time
    omp_run(["-s", str(NX), "-i", str(max(1, min(a.warmup, 3)))], threads)
    its = a.steps
    if rate > 0 and its * ZONES / rate > 120.0:
        its = max(2, int(120.0 * rate / ZONES))
    r = omp_run(["-s", str(NX), "-i", str(its)], threads)
    value = 1e6 / r["grind"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": r["elapsed"] * 1e3 / its,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: sedov blast generated in code",
        "config": {"workload": "LULESH sedov single domain -s 100 (1,000,000 elements), "
                               "FP64, -r 11 -b 1 -c 1, one cycle per step", "nx": NX,
                   "regions": 11, "balance": 1, "cost": 1},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"lulesh_omp -s {NX} -i {its} (LULESH/omp_4.0), "
                                   f"OMP_NUM_THREADS={threads} of {cores} host CPUs",
                         "thread_sweep": sw},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "origin_energy": r.get("energy"), "origin_energy_cycle": its,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--profile-cycles", dest="profile_cycles", type=int, default=5)
    ap.add_argument("--e2e-cycles", dest="e2e_cycles", type=int, default=200)
    ap.add_argument("--serve-jobs", dest="serve_jobs", type=int, default=2000,
                    help="jobs of the serving stream (2000 = the full stream; 0 skips)")
    ap.add_argument("--plain-repeats", dest="plain_repeats", type=int, default=3,
                    help="repeats of the plain path's capacity run (1-in-10 sample)")
    ap.add_argument("--batch-jobs", dest="batch_jobs", type=int, default=64,
                    help="jobs of the batch comparison (0 skips)")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="keep the default launch shape instead of autotuning it")
    ap.add_argument("--unstructured", type=int, default=0,
                    help="also time the -s N cube read as an lmesh file (0 skips)")
    ap.add_argument("--no-gpu-reference", dest="gpu_reference", action="store_false",
                    help="skip the reference CUDA build leg")
    ap.add_argument("--no-mixed", dest="mixed", action="store_false",
                    help="skip the config-4 mixed-precision leg")
    ap.add_argument("--no-subdomains", dest="subdomains", action="store_false",
                    help="skip the config-2 subdomain leg")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false",
                    help="skip the reference omp CPU baseline")
    ap.add_argument("--transport", default="nccl", choices=["nccl", "host", "direct"],
                    help="halo transport between GPUs when N > 1 (direct: peer stores into "
                         "the neighbours' mailboxes, dt over NCCL)")
    a = ap.parse_args()
    if a.warmup < 3:
        ap.error("--warmup must be >= 3")
    if a.warmup + a.steps > 3000:
        ap.error("-s 100 reaches t = 0.01 after ~3500 cycles: keep warmup + steps <= 3000")
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(a.gpus)))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        run_reference(a, rank, world)
    else:
        run_ours(a, rank, world, local_rank)


if __name__ == "__main__":
    main()
