"""Near-field direct-force benchmark (one JSON line on stdout, rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload clustered512|clustered256|uniform64|...]

A step is one full near-field sweep of a synthetic box (every sink of every
x-slab against its 5x5x5 cell neighbourhood), the box's positions already
resident in HBM.  The default workload is the clustered box the target is set
on: 512^3 particles, cpd 125, 40% uniform + 60% in 2000 seeded NFW clumps,
single-spline softening at 1/40 of the mean spacing, float32, compensated
accumulation.

metric: pair interactions/s (unpadded pairs, PencilOnPencil.cc:412 counting),
plus p50/p99 slab latency.  Beside the sweep the line carries, for the same
box: the end-to-end rate through the C ABI from pinned host buffers, the
plain drop-in (NearFieldDriver -> SICs, wall clock and summed kernel time),
the reference's own GPU kernel on one SIC per slab, the compensated-vs-plain
precision study against the FP64 oracle on 0.1% of the sinks, per-component
parity against the reference CPU direct on a fixed seeded sample of rows,
and the five-box serving workload.

Multi-GPU (torchrun): one box split over the ranks by x-slab ranges with a
2-slab halo exchanged over NCCL (strong scaling); --replicas runs one
independent box per rank instead (weak scaling).  The timed region is
bracketed by a barrier and the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FLOPS_PER_PAIR = {0: 23, 1: 24, 2: 24, 3: 24}  # counted flops (FFMA=2, rsqrt=1, Newton incl.)


def _pkg():
    import importlib.util
    if "abacus_public_b200" not in sys.modules:
        spec = importlib.util.spec_from_file_location(
            "abacus_public_b200", ROOT / "abacus-public_b200" / "__init__.py",
            submodule_search_locations=[str(ROOT / "abacus-public_b200")])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["abacus_public_b200"] = mod
        spec.loader.exec_module(mod)
    return sys.modules["abacus_public_b200"]


WORKLOADS = {
    "clustered256": dict(n_side=256, cpd=65, softening=1, kind="clustered", seed=2,
                         desc="256^3 particles, cpd 65, 40% uniform + 60% in 2000 NFW clumps "
                              "(c=10, r_t=0.6 cell), single spline eps_pl=spacing/40"),
    "uniform64": dict(n_side=64, cpd=17, softening=0, kind="uniform", seed=1,
                      desc="64^3 uniform particles, cpd 17, Plummer eps=spacing/40"),
    "clustered512": dict(n_side=512, cpd=125, softening=1, kind="clustered", seed=3,
                         desc="512^3 particles, cpd 125, clustered mixture as clustered256"),
    "clustered128": dict(n_side=128, cpd=33, softening=1, kind="clustered", seed=4,
                         desc="128^3 particles, cpd 33, clustered mixture as clustered256 "
                              "(the profiling case)"),
    "uniform256": dict(n_side=256, cpd=65, softening=0, kind="uniform", seed=5,
                       desc="256^3 uniform particles, cpd 65, Plummer eps=spacing/40"),
    "clustered1024": dict(n_side=1024, cpd=255, softening=1, kind="clustered_device", seed=6,
                          desc="1024^3 particles, cpd 255, clustered mixture as clustered256, "
                               "generated on the GPU; a step sweeps a bounded range of slabs"),
}


def make_box(w, seed_offset=0):
    _pkg()
    from abacus_public_b200 import synth
    n = w["n_side"] ** 3
    if w["kind"] == "uniform":
        return synth.uniform_box(n, w["cpd"], w["seed"] + seed_offset)
    return synth.clustered_box(n, w["cpd"], w["seed"] + seed_offset)


def box_nc(w):
    """Partial components per sink: x, y, z (+ density when b2 > 0)."""
    return 4 if w.get("b2", 0.0) > 0 else 3


def staging_hbm(n, nc, kernel_ms, traffic, R=2):
    """HBM side of the pencil kernel: algorithmic bytes per launch (one
    16-byte position record per particle read, (2R+1) x nc double partials per
    particle written), the rate they imply over the launch, and the same for
    the ncu-measured DRAM bytes when a capture is on file."""
    alg = n * (16 + (2 * R + 1) * nc * 8)
    secs = kernel_ms / 1e3
    out = {"algorithmic_bytes": int(alg), "algorithmic_gbs": alg / secs / 1e9,
           "measured_bytes": traffic,
           "measured_gbs": None if traffic is None else traffic / secs / 1e9}
    peaks = ROOT / "MEASURED_PEAKS.json"
    try:
        hbm = float(json.loads(peaks.read_text())["hbm_gbs"])
        out["hbm_peak_gbs"] = hbm
        out["frac_of_hbm_peak"] = out["algorithmic_gbs"] / hbm
    except (OSError, ValueError, KeyError):
        pass
    return out


def kernel_eps(w):
    from abacus_public_b200 import synth
    return synth.kernel_eps(w["softening"], synth.plummer_eps(w["n_side"]))


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_init(n_gpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return rank, world, local


def _reduce_device():
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def barrier_max(value: float, world: int) -> float:
    """Max over ranks (the timed region's duration is the slowest rank's)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def all_sum(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def rank_seed_offset(rank: int) -> int:
    """Each rank sweeps its own independent box: seed + rank."""
    return rank


def aggregate(pairs_per_rank: float, ms_per_rank: float, world: int) -> tuple[float, float]:
    """Whole-job pairs/s: all ranks' pairs over the slowest rank's time."""
    total = all_sum(pairs_per_rank, world)
    ms = barrier_max(ms_per_rank, world)
    return total / (ms / 1e3), ms


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own kernel compiled from its sources
# (oracle/_ref, -Ofast), driven by the ExecuteSlabCPU cell loop
# ---------------------------------------------------------------------------
CPU_SAMPLE_SEED = 123


def cell_pairs(box, R=2):
    """Pairs of every sink cell (its count times the count of its (2R+1)^3
    neighbourhood, periodic), shape (cpd, cpd, cpd); sums to DirectTotal."""
    cpd = box.cpd
    c3 = box.counts.reshape(cpd, cpd, cpd).astype(np.int64)
    nb = c3
    for axis in range(3):
        nb = sum(np.roll(nb, d, axis=axis) for d in range(-R, R + 1))
    return c3 * nb


def cpu_sample(box, target_pairs, seed=CPU_SAMPLE_SEED):
    """A fixed seeded sample for the CPU reference: sink cells (the unit of
    ExecuteSlabCPU's work, extras_directdriver.cpp:59-122) taken in a seeded
    order of the non-empty cells until target_pairs is reached (the whole
    box if it holds fewer), exact pair counts.  Cells and not whole rows or
    slabs: on the clustered boxes one row through a clump holds ~3e10 pairs,
    half a minute of the host's work.  Both bench arms take the same cells.
    Returns (cells, sinks, pairs, description)."""
    cp = cell_pairs(box).ravel()
    nz = np.nonzero(box.counts)[0]
    order = np.random.default_rng(seed).permutation(nz)
    cum = np.cumsum(cp[order])
    k = min(int(np.searchsorted(cum, target_pairs)) + 1, order.size)
    cells = np.sort(order[:k])
    cs = box.cell_start
    n = (cs[cells + 1] - cs[cells]).astype(np.int64)
    sinks = np.repeat(cs[cells] - np.cumsum(n) + n, n) + np.arange(int(n.sum()))
    pairs = int(cp[cells].sum())
    desc = (f"{k} seeded non-empty sink cells (seed {seed}; {sinks.size} sinks, "
            f"{pairs:.4e} pairs)")
    return cells, sinks, pairs, desc


def host_cpu():
    """The host CPU the baseline ran on: model name, logical CPUs of the host
    and the ones this process may use (the threads the baseline takes)."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        usable = os.cpu_count()
    return {"model": model, "host_logical_cpus": os.cpu_count(), "usable_cpus": usable}


def cpu_reference_run(box, w, cells, threads):
    """The reference CPU direct on the sample's cells: (float32[N, 3] with the
    sample's rows written, seconds, kind)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    soft, eps = w["softening"], kernel_eps(w)
    acc = np.zeros((box.n, 3), np.float32)
    t0 = time.perf_counter()
    if oracle.have_ref(soft, "fast"):
        oracle.ref_cells(box, soft, eps, cells, flavour="fast", threads=threads, acc=acc)
        kind = "reference"
    else:
        oracle.ref32_cells(box, soft, eps, cells, acc=acc)
        kind = "port"
    return acc, time.perf_counter() - t0, kind


def parity_vs_reference(a_gpu, a_ref, sinks, tol=1e-4):
    """Per sink and component |a - a_ref| <= tol |a_ref| (vector norm of the
    reference's acceleration), on the sample's sinks."""
    ref = a_ref[sinks].astype(np.float64)
    got = np.asarray(a_gpu[sinks, :3], np.float64)
    norm = np.linalg.norm(ref, axis=1)
    dev = np.abs(got - ref).max(axis=1)
    ok = norm > 0
    rel = dev[ok] / norm[ok]
    vrel = np.linalg.norm(got - ref, axis=1)[ok] / norm[ok]
    return {"sinks": int(sinks.size), "tolerance": f"|a - a_ref|_c <= {tol:g} |a_ref|",
            "max_comp_rel": float(rel.max()) if rel.size else 0.0,
            "rms_rel": float(np.sqrt(np.mean(vrel ** 2))) if vrel.size else 0.0,
            "pass": bool(np.all(dev <= tol * norm))}


def workload_config(args, w, box, pairs, world=1):
    """The `config` of the bench line: the workload alone, identical in both
    arms at N = 1."""
    l2_bytes = 126 * 2 ** 20
    big = 136 * int(box.n) > l2_bytes  # 16 B positions + 120 B partials per particle
    return {"workload": args.workload, "desc": w["desc"], "particles_per_gpu": int(box.n),
            "cpd": int(box.cpd), "pairs_per_step_per_gpu": int(pairs),
            "l2": ("inputs larger than L2 (positions 16 B x N + 120 B x N partials)" if big
                   else "inputs fit in L2 and are not flushed between steps (a small box)"),
            "parallelism": f"independent boxes x{world}"}


def reference_arm(args, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if w["kind"] == "clustered_device":
        print(json.dumps({"impl": "reference", "unavailable": "the 1024^3 box is generated on "
                          "the GPU and does not fit the host-side sample of the CPU direct"}))
        return 0
    box = make_box(w)
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    threads = oracle.host_threads()
    # per step: the fixed seeded sample of rows the other arm reports
    cells, sinks, pairs, desc = cpu_sample(box, args.cpu_pairs)
    times, kind = [], "port"
    for i in range(args.warmup + args.steps):
        _, dt, kind = cpu_reference_run(box, w, cells, threads)
        if i >= args.warmup:
            times.append(dt)
    ms = 1e3 * sum(times) / len(times)
    value = pairs / (ms / 1e3)
    line = {
        "impl": "reference", "metric": "pair_interactions_per_s", "value": value,
        "unit": "pairs/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": workload_config(args, w, box, int(cell_pairs(box).sum())),
        "step": "the reference CPU direct on a fixed seeded sample of sink cells of the box "
                "(a whole sweep takes hours on the host)",
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads, "kind": kind,
                         "sample": desc, "cpu": host_cpu()},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json_line(line), flush=True)
    return 0


def json_line(obj):
    """One strict-JSON line: NaN and infinities (a ratio with an empty
    denominator, say) become null."""
    def clean(v):
        if isinstance(v, float) and not math.isfinite(v):
            return None
        if isinstance(v, dict):
            return {k: clean(x) for k, x in v.items()}
        if isinstance(v, (list, tuple)):
            return [clean(x) for x in v]
        return v
    return json.dumps(clean(obj), allow_nan=False)


def percentile(xs, q):
    return float(np.percentile(np.asarray(xs), q)) if xs else None


def plain_dropin(capi, box, w, device, a_batched=None, steps=2, fp64=None):
    """The plain drop-in: the NearFieldDriver mirror (SIC planning, y-splits,
    one launch per SIC, host slabs staged per SIC, AccSlab written back) over
    every slab of the box.  Wall clock per full sweep with DirectBPD 3, then
    one sweep with DirectBPD 1 (SICs one after another) for the summed
    pencil-kernel time of its SICs.  a_batched: the batched sweep's result, to
    compare the drop-in's output with (over every sink; the sink where they
    differ most is checked against the FP64 oracle too).  fp64 = (sinks,
    FP64 accelerations): the drop-in's own error on those sinks."""
    from abacus_public_b200 import synth
    length = synth.plummer_eps(w["n_side"])
    drv = capi.Driver(box, softening=w["softening"], softening_length=length, device=device,
                      direct_bpd=3)
    try:
        drv.run_all()  # warm-up: buffers, pinned staging
        times = []
        for _ in range(steps):
            t0 = time.perf_counter()
            acc = drv.run_all()
            times.append(time.perf_counter() - t0)
        st = drv.stats()
        pairs = st.direct_interactions // (steps + 1)
        sec = float(np.mean(times))
        res = {"value": pairs / sec, "unit": "pairs/s", "ms_per_step": 1e3 * sec,
               "splits_per_slab": st.mean_splits_per_slab, "buffers": st.nbuffers,
               "gb_to_device_per_step": st.total_gb_to / (steps + 1),
               "what": "host slabs -> NearFieldDriver -> SIC -> AccSlab, wall clock"}
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle
        if a_batched is not None:
            ref = np.asarray(a_batched[:, :3], np.float64)
            norm = np.maximum(np.linalg.norm(ref, axis=1), 1e-300)
            rel = np.abs(acc[:, :3] - ref).max(axis=1) / norm
            k = int(np.argmax(rel))
            res["max_comp_rel_vs_batched"] = float(rel[k])
            a64 = oracle.fp64_sinks(box, w["softening"], kernel_eps(w), np.array([k]))
            m64 = float(np.linalg.norm(a64))
            med = float(np.median(norm[::max(1, box.n // 100000)]))
            res["worst_sink"] = {
                "sink": k, "abs_a_over_median": m64 / med,
                "plain_frac_err_vs_fp64": float(np.linalg.norm(acc[k, :3] - a64[0]) / m64),
                "batched_frac_err_vs_fp64": float(np.linalg.norm(ref[k] - a64[0]) / m64)}
        if fp64 is not None:
            rms, mx, _ = oracle.frac_errors(acc[fp64[0], :3], fp64[1])
            res["vs_fp64"] = {"rms_frac": rms, "max_frac": mx, "sinks": int(fp64[0].size)}
        del acc
    finally:
        drv.close()
    drv = capi.Driver(box, softening=w["softening"], softening_length=length, device=device,
                      direct_bpd=1)
    try:
        drv.run_all()
        drv.sic_timing(reset=True)
        drv.run_all()
        kms, nsic, kpairs = drv.sic_timing()
    finally:
        drv.close()
    res["kernel"] = {"pairs_per_s": kpairs / (kms / 1e3), "kernel_ms": kms, "sics": nsic,
                     "pairs": kpairs,
                     "what": "summed pencil-kernel time of the drop-in's SICs (DirectBPD 1, "
                             "CUDA events around each SIC's launch)"}
    return res


def ref_gpu_leg(box, w, a_batched, fp64=None):
    """The reference's own GPU kernel (ComputeDirects, PencilKernel.cu:97-188,
    compiled from its sources for sm_100a) on every x-slab of the box as one
    SIC, each laid out on the host as PencilOnPencil.cc / PencilPlan.cc do
    while the previous slab runs: pairs / summed launch time, and the largest
    per-component deviation of its forces from the batched sweep's.  fp64 =
    (sinks, FP64 accelerations): the kernel's own error against the FP64
    oracle on those sinks, beside the batched sweep's."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    from concurrent.futures import ThreadPoolExecutor
    soft, eps = w["softening"], kernel_eps(w)
    if not oracle.have_ref_gpu(soft):
        return {"unavailable": "the reference GPU kernel is not built for this softening"}
    tot_ms, pairs, worst = 0.0, 0, 0.0
    mine = None if fp64 is None else np.zeros((fp64[0].size, 3), np.float32)
    with ThreadPoolExecutor(1) as ex:
        fut = ex.submit(oracle.sic_arrays, box, 0)
        for s in range(box.cpd):
            arr = fut.result()
            if s + 1 < box.cpd:
                fut = ex.submit(oracle.sic_arrays, box, s + 1)
            acc, ms, p = oracle.ref_gpu_run(box, soft, eps, s, arr, repeats=1)
            del arr
            tot_ms += ms
            pairs += p
            p0, p1 = box.slab_range(s)
            if mine is not None:
                sel = (fp64[0] >= p0) & (fp64[0] < p1)
                mine[sel] = acc[fp64[0][sel] - p0]
            ref = acc.astype(np.float64)
            norm = np.linalg.norm(ref, axis=1)
            ok = norm > 0
            if ok.any():
                dev = np.abs(np.asarray(a_batched[p0:p1, :3], np.float64) - ref).max(axis=1)
                worst = max(worst, float((dev[ok] / norm[ok]).max()))
    out = {}
    if mine is not None:
        rms, mx, _ = oracle.frac_errors(mine, fp64[1])
        out = {"vs_fp64": {"rms_frac": rms, "max_frac": mx, "sinks": int(fp64[0].size),
                           "what": "its own error on the precision study's FP64 sinks"}}
    return {"value": pairs / (tot_ms / 1e3), "unit": "pairs/s", "kernel_ms": tot_ms,
            "pairs": pairs, "sics": box.cpd, "max_comp_rel_vs_batched": worst, **out,
            "what": "reference ComputeDirects (PencilKernel.cu) built for sm_100a with its "
                    "default GPU flags, one SIC per x-slab, summed CUDA-event launch time"}


def serving_phase(capi, ctx, w, args, rank, seed=7):
    """Seeded Poisson slab requests over several clustered boxes resident on
    the same GPU, at fractions of the measured closed-loop capacity; p50/p99
    latency from submission to the result in the caller's device buffer,
    split into queue and run time.  Boxes: N = 64*cpd^3 for each cpd of
    --serve-boxes (default 45, 65, 85, 105, 125), generated on the device,
    each with its own softening at 1/40 of its mean spacing."""
    import torch
    from abacus_public_b200 import synth
    soft = w["softening"]
    cpds = [int(c) for c in args.serve_boxes.split(",")]
    dbs, names = [], []
    hosts, epss = [], []
    for k, c in enumerate(cpds):
        x, y, z, cs = synth.clustered_box_device(64 * c ** 3, c, seed=100 + 17 * k + rank)
        d = ctx.box(synth.Box(c, x, y, z, cs, f"serve cpd {c}"))
        # a host copy for the FP64 check of the served results
        hosts.append(synth.Box(c, x.cpu().numpy(), y.cpu().numpy(), z.cpu().numpy(), cs,
                               f"serve cpd {c}"))
        del x, y, z
        epss.append(synth.kernel_eps(soft, synth.plummer_eps(4 * c)))  # 64 per cell: spacing h/4
        d.set_eps(epss[-1])
        dbs.append(d)
        names.append(f"64*{c}^3 cpd {c} clustered")
    torch.cuda.empty_cache()
    slabs = [(i, s) for i, d in enumerate(dbs) for s in range(d.cpd)]
    outs = {}
    for i, s in slabs:
        p0, p1 = dbs[i].slab_particles(s, s + 1)
        outs[(i, s)] = torch.empty((max(p1 - p0, 1), 4), dtype=torch.float32, device="cuda")
    rng = np.random.default_rng(seed)
    n_req = args.serve_requests
    levels = []
    with capi.Server(ctx, max_inflight=args.serve_slots) as srv:
        for _ in range(2):  # warm-up (plans, tuning); the second pass gives capacity
            t0 = time.perf_counter()
            tk = [srv.submit(dbs[i], s, outs[(i, s)].data_ptr(), True) for i, s in slabs]
            for t in tk:
                srv.wait(t, timeout_s=600.0)
            cap = len(slabs) / (time.perf_counter() - t0)
        # each slab alone on the GPU once: the service times the workload
        # itself sets (a floor under any request's latency)
        solo = []
        for i, s in slabs:
            t = srv.submit(dbs[i], s, outs[(i, s)].data_ptr(), True)
            srv.wait(t, timeout_s=600.0)
            solo.append(srv.info(t).run_ms)
        # overload (1.5x) only grows the queue: a shorter stream shows it
        for load, per_level in ((0.5, n_req), (1.0, n_req), (1.5, min(n_req, 2000))):
            rate = load * cap
            arr = np.cumsum(rng.exponential(1.0 / rate, per_level))
            pick = rng.integers(0, len(slabs), per_level)
            srv.reset_stats()
            tk = []
            t_start = time.perf_counter()
            for k in range(per_level):
                target = t_start + arr[k]
                while True:
                    now = time.perf_counter()
                    if now >= target:
                        break
                    time.sleep(min(target - now, 2e-4))
                i, s = slabs[pick[k]]
                tk.append(srv.submit(dbs[i], s, outs[(i, s)].data_ptr(), True))
            for t in tk:
                srv.wait(t, timeout_s=600.0)
            elapsed = time.perf_counter() - t_start
            st = srv.stats()
            runs = [srv.info(t).run_ms for t in tk]
            levels.append({"load": load, "rate_per_s": rate, "requests": per_level,
                           "p50_ms": st.p50_ms, "p99_ms": st.p99_ms, "mean_ms": st.mean_ms,
                           "queue_p50_ms": st.queue_p50_ms, "queue_p99_ms": st.queue_p99_ms,
                           "run_p50_ms": percentile(runs, 50), "run_p99_ms": percentile(runs, 99),
                           "pairs_per_s": st.pairs / elapsed,
                           "max_concurrent": st.max_concurrent})
    # accuracy of the served results (the last request of each slab wrote
    # its buffer): 3 seeded slabs of every box, up to 200 seeded sinks each,
    # against the FP64 oracle
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    acc = {}
    for i, d in enumerate(dbs):
        r = np.random.default_rng(300 + i)
        got, a64 = [], []
        for s in r.choice(d.cpd, 3, replace=False):
            p0, p1 = d.slab_particles(int(s), int(s) + 1)
            if p1 - p0 == 0:
                continue
            loc = np.sort(r.choice(p1 - p0, min(200, p1 - p0), replace=False))
            got.append(outs[(i, int(s))][torch.from_numpy(loc).cuda(), :3].cpu().numpy())
            a64.append(oracle.fp64_sinks(hosts[i], soft, epss[i], loc + p0))
        rms, mx, _ = oracle.frac_errors(np.concatenate(got), np.concatenate(a64))
        acc[names[i]] = {"rms_frac": rms, "max_frac": mx, "sinks": int(sum(len(g) for g in got))}
    for d in dbs:
        d.close()
    p50, p99 = percentile(solo, 50), percentile(solo, 99)
    return {"boxes": names, "slots": args.serve_slots, "capacity_slabs_per_s": cap,
            "solo_service_ms": {"p50": p50, "p99": p99, "p99_over_p50": p99 / p50,
                                "what": "each slab alone on the GPU, admission to result "
                                        "(uniform over the boxes' slabs, as the requests)"},
            "accuracy_vs_fp64": acc,
            "levels": levels}


def precision_study(capi, box, w, device, stream, steps, comp_out, variant, frac=1e-3, seed=11):
    """Compensated vs plain FP32 accumulation on the same box: the plain
    form's sweep rate (device time, positions resident, the compensated
    sweep's kernel shape) and both results' RMS / max fractional error against
    the FP64 oracle on a seeded subsample of `frac` of the sinks.  `comp_out`
    is the compensated sweep's result."""
    import torch
    soft, eps = w["softening"], kernel_eps(w)
    ctx = capi.Context(softening=soft, eps=eps, device=device, accumulation=capi.ACC_PLAIN,
                       kernel_variant=variant)
    ctx.set_stream(stream.cuda_stream)
    db = ctx.box(box)
    out = torch.empty((box.n, 4), dtype=torch.float32, device=f"cuda:{device}")
    db.forces_device(0, box.cpd, out.data_ptr())
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        db.forces_device(0, box.cpd, out.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    pairs = db.pair_count()
    plain_out = out.cpu().numpy()
    del out
    db.close()
    ctx.close()
    torch.cuda.empty_cache()
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    k = max(2000, int(frac * box.n))
    sinks = np.sort(np.random.default_rng(seed).choice(box.n, k, replace=False))
    t0 = time.perf_counter()
    ref = oracle.fp64_sinks(box, soft, eps, sinks)
    t_ref = time.perf_counter() - t0
    res = {"sinks": k, "fraction": k / box.n, "seed": seed, "fp64_oracle_s": t_ref,
           "plain_pairs_per_s": pairs / (ms / 1e3), "plain_ms_per_step": ms, "plain_steps": steps}
    mag = np.linalg.norm(ref, axis=1)
    res["small_force_sinks"] = int((mag < 1e-3 * np.median(mag)).sum())  # |a64| < 1e-3 median
    for name, a in (("compensated", comp_out), ("plain", plain_out)):
        rms, mx, _ = oracle.frac_errors(a[sinks, :3], ref)
        res[name] = {"rms_frac": rms, "max_frac": mx}
    return res, (sinks, ref)


class Phases:
    """Wall time of each bench phase (stderr as they end; kept for the line)."""

    def __init__(self, rank):
        self.rank = rank
        self.t = {}

    def run(self, name, fn, *a, **kw):
        t0 = time.perf_counter()
        r = fn(*a, **kw)
        dt = time.perf_counter() - t0
        self.t[name] = round(dt, 2)
        if self.rank == 0:
            print(f"[bench] {name}: {dt:.1f} s", file=sys.stderr, flush=True)
        return r


def peak_from(sust, clocks, sms):
    """max(probe, clock-derived) for an already measured probe value; the
    clock-derived peak is None when no clock sample fell in the timed region
    (a timed region shorter than the sampling period)."""
    mhz = clocks.get("sm_mhz") if isinstance(clocks, dict) else None
    derived = sms * 128 * 2 * mhz * 1e6 / 1e12 if mhz else None
    return (max(sust, derived) if mhz else sust), derived


def fp32_peaks(ctx, clocks, sms):
    """The FP32 roofline denominator: the paired-FMA probe (sustained) and the
    clock-derived peak sms x 128 lanes x 2 flops x the median SM clock sampled
    in the timed region; the larger of the two is used."""
    burst, sust = ctx.fp32_peak(1.0)
    mhz = clocks.get("sm_mhz") if isinstance(clocks, dict) else None
    derived = sms * 128 * 2 * mhz * 1e6 / 1e12 if mhz else None
    peak = max(sust, derived) if mhz else sust
    src = ("clock-derived: %d SMs x 128 FP32 lanes x 2 flops x %.0f MHz (median SM clock "
           "sampled in the timed region)" % (sms, mhz)) if mhz and derived >= sust else \
        "paired-FMA probe on this GPU in this run, sustained over ~1 s"
    return {"peak": peak, "peak_source": src, "peak_probe_sustained": sust,
            "peak_probe_burst": burst, "peak_clock_derived": derived}


def our_arm(args, w):
    import torch
    rank, world, local = dist_init(args.gpus)
    _pkg()
    from abacus_public_b200 import capi
    ph = Phases(rank)
    box = ph.run("generate_box", make_box, w, seed_offset=rank_seed_offset(rank))
    eps = kernel_eps(w)
    soft = w["softening"]
    ctx = capi.Context(softening=soft, eps=eps, device=local)
    torch.cuda.set_device(local)
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)  # the library launches on the stream the events time
    db = ph.run("upload", ctx.box, box)
    pairs = db.pair_count()
    n = box.n
    out_dev = torch.empty((n, 4), dtype=torch.float32, device=f"cuda:{local}")

    def warm():
        # the first call tunes the kernel shape and captures the graph
        for _ in range(args.warmup):
            db.forces_device(0, box.cpd, out_dev.data_ptr())
        torch.cuda.synchronize()
    ph.run("tune_and_warmup", warm)
    kernel_ms, step_ms_dev = [], []

    def timed():
        clk = ClockSampler(local)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with clk:
            barrier(world)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(args.steps):
                db.forces_device(0, box.cpd, out_dev.data_ptr())
                t = ctx.last_timing()
                kernel_ms.append(t.kernel_ms)
                step_ms_dev.append(t.total_ms)
            e1.record(stream)
            torch.cuda.synchronize()
            barrier(world)
        return e0.elapsed_time(e1), clk.summary(), t
    elapsed, clocks, t = ph.run("timed_sweeps", timed)
    elapsed = barrier_max(elapsed, world)
    ms_per_step = elapsed / args.steps
    total_pairs = all_sum(float(pairs), world)
    value = total_pairs / (ms_per_step / 1e3)
    launches = args.steps * t.launches

    if args.profile:
        if rank == 0:
            print(json.dumps({"profile_run": args.workload, "ms_per_step": ms_per_step,
                              "kernel_ms": float(np.mean(kernel_ms)), "pairs": pairs,
                              "pairs_per_s": value}), flush=True)
        db.close()
        ctx.close()
        return 0
    peaks = ph.run("fp32_peak", fp32_peaks, ctx, clocks, sms)
    # end to end through the C ABI with pinned host buffers: H2D positions,
    # sweep, D2H accelerations, every step
    hx = torch.from_numpy(box.x).pin_memory()
    hy = torch.from_numpy(box.y).pin_memory()
    hz = torch.from_numpy(box.z).pin_memory()
    hout = torch.empty((n, 4), dtype=torch.float32).pin_memory()
    xa, ya, za, oa = hx.numpy(), hy.numpy(), hz.numpy(), hout.numpy()
    e2e_steps = args.e2e_steps or args.steps

    def e2e():
        # one call per step: copies in, sweeps and copies out overlap over 8
        # slab chunks (nf_box_step); the first call builds the chunk plans
        db.step(xa, ya, za, oa)
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            db.step(xa, ya, za, oa)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / e2e_steps
    e2e_ms = barrier_max(ph.run("e2e", e2e), world)
    e2e_value = total_pairs / (e2e_ms / 1e3)
    tv, tms = db.tuning()
    db.close()
    del out_dev
    torch.cuda.empty_cache()

    precision = plain = refk = fp64 = None
    if rank == 0 and not args.no_precision:
        precision, fp64 = ph.run("precision_study", precision_study, capi, box, w, local,
                                 stream, args.precision_steps, oa, tv)
    if rank == 0 and not args.no_plain:
        plain = ph.run("plain_dropin", plain_dropin, capi, box, w, local, a_batched=oa,
                       fp64=fp64)
        plain["batched_over_plain"] = e2e_value / plain["value"]
        plain["batched_over_plain_what"] = "e2e (nf_box_step from pinned host buffers) over " \
                                           "the drop-in's wall clock, same box"
    if rank == 0 and not args.no_ref_kernel:
        refk = ph.run("reference_gpu_kernel", ref_gpu_leg, box, w, oa, fp64)
    serving = None if args.no_serving else ph.run("serving", serving_phase, capi, ctx, w, args,
                                                  rank)
    # slab latency at half the measured closed-loop capacity (at 1.0x the
    # queue, not the device, sets the latency; every level is in "serving")
    lvl1 = None if serving is None else [v for v in serving["levels"] if v["load"] == 0.5][0]

    lib = capi.lib()
    tune_info = {"variant": tv, "shape": lib.nf_kernel_variant_name(tv).decode(),
                 "candidates_ms": {lib.nf_kernel_variant_name(i).decode(): round(m, 3)
                                   for i, m in enumerate(tms) if m > 0}}
    flops = FLOPS_PER_PAIR[soft]
    k_ms = float(np.mean(kernel_ms))
    achieved = pairs * flops / (k_ms / 1e3) / 1e12
    traffic = None
    prof = ROOT / "profiles" / f"pencil_kernel_{args.workload}.json"
    if prof.exists():
        try:
            traffic = json.loads(prof.read_text()).get("dram_bytes_per_launch")
        except (ValueError, OSError):
            traffic = None
    result = {
        "metric": "pair_interactions_per_s", "value": value, "unit": "pairs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": workload_config(args, w, box, pairs, world),
        "padded_pairs_per_step_per_gpu": int(t.padded_pairs),
        "accumulation": "compensated",
        "slab_latency_ms": None if lvl1 is None else {
            "p50": lvl1["p50_ms"], "p99": lvl1["p99_ms"], "n": lvl1["requests"],
            "queue_p99": lvl1["queue_p99_ms"], "run_p99": lvl1["run_p99_ms"],
            "solo_p50": serving["solo_service_ms"]["p50"],
            "solo_p99": serving["solo_service_ms"]["p99"],
            "what": "serving at 0.5x measured capacity: Poisson slab requests over the "
                    "resident boxes, submit to result in the caller's device buffer"},
        "serving": serving,
        "precision": precision,
        "plain_dropin": plain,
        "ref_gpu_kernel": refk,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peaks["peak"],
                     "unit": "TFLOP/s", "frac": achieved / peaks["peak"], "traffic": traffic,
                     "kernel": "pencil_kernel", "kernel_ms": k_ms,
                     "flops_per_pair": flops, "peak_source": peaks["peak_source"],
                     "peak_probe_sustained": peaks["peak_probe_sustained"],
                     "peak_probe_burst": peaks["peak_probe_burst"],
                     "peak_clock_derived": peaks["peak_clock_derived"],
                     "staging_hbm": staging_hbm(n, box_nc(w), k_ms, traffic)},
        "e2e": {"value": e2e_value, "unit": "pairs/s", "ms_per_step": e2e_ms,
                "steps": e2e_steps,
                "h2d_bytes_per_step": int(12 * n), "d2h_bytes_per_step": int(16 * n)},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "autotune": tune_info,
    }
    if precision is not None:
        result["accuracy_vs_fp64"] = {"rms_frac": precision["compensated"]["rms_frac"],
                                      "max_frac": precision["compensated"]["max_frac"],
                                      "sinks": precision["sinks"]}
    if rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle
        threads = oracle.host_threads()
        cells, sinks, spairs, desc = cpu_sample(box, args.cpu_pairs)
        a_ref, dt, kind = ph.run("cpu_baseline", cpu_reference_run, box, w, cells, threads)
        result["cpu_baseline"] = {"value": spairs / dt, "unit": "pairs/s", "cores": threads,
                                  "kind": kind, "sample": f"{desc}, {dt:.1f} s",
                                  "cpu": host_cpu()}
        result["parity_vs_reference"] = dict(
            parity_vs_reference(oa, a_ref, sinks),
            reference="the reference CPU direct (Direct::Execute, -Ofast build) on the "
                      "cpu_baseline sample",
            ours="the last end-to-end sweep's output (nf_box_step)")
    result["phase_s"] = ph.t
    ctx.close()
    if rank == 0:
        print(json_line(result), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def big_arm(args, w):
    """The largest box (1024^3, generated on the GPU: it does not fit the
    host-side generator).  A full sweep is ~5e14 pairs (minutes), so a step
    sweeps the slab range [0, --slabs) as one persistent launch; value =
    that range's pairs / device time.  The kernel shape is fixed (shape 0,
    the one the autotuner picks on the 256^3 and 512^3 boxes): tuning would
    cost five launches of the range.  Accuracy: the FP64 oracle on 2000
    seeded sinks of the range; no CPU baseline (its sample would take
    hours)."""
    import torch
    _pkg()
    from abacus_public_b200 import capi, synth
    torch.cuda.set_device(0)
    n = w["n_side"] ** 3
    x, y, z, cs = synth.clustered_box_device(n, w["cpd"], w["seed"], device="cuda")
    hbox = synth.Box(w["cpd"], x.cpu().numpy(), y.cpu().numpy(), z.cpu().numpy(), cs, "clustered1024")
    dbox = synth.Box(w["cpd"], x, y, z, cs, "clustered1024")
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    eps = kernel_eps(w)
    ctx = capi.Context(softening=w["softening"], eps=eps, kernel_variant=0)
    ctx.set_stream(stream.cuda_stream)
    peak_b, peak_s = ctx.fp32_peak(1.0)
    db = ctx.box(dbox)
    del x, y, z, dbox
    torch.cuda.empty_cache()
    if args.full:
        return big_full_sweep(args, w, capi, ctx, db, hbox, eps, peak_s, stream)
    lo, hi = 0, min(args.slabs, w["cpd"])
    p0, p1 = db.slab_particles(lo, hi)
    out = torch.empty((p1 - p0, 4), dtype=torch.float32, device="cuda")
    pairs = db.pair_count(lo, hi)
    for _ in range(args.warmup):
        db.forces_device(lo, hi, out.data_ptr())
    torch.cuda.synchronize()
    kms = []
    with ClockSampler(0) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            db.forces_device(lo, hi, out.data_ptr())
            kms.append(ctx.last_timing().kernel_ms)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    t = ctx.last_timing()
    k_ms = float(np.mean(kms))
    clocks = clk.summary()
    peak, derived = peak_from(peak_s, clocks, torch.cuda.get_device_properties(0).multi_processor_count)
    flops = FLOPS_PER_PAIR[w["softening"]]
    achieved = pairs * flops / (k_ms / 1e3) / 1e12
    res = out.cpu().numpy()
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    sinks = np.sort(np.random.default_rng(5).choice(np.arange(p0, p1), 2000, replace=False))
    rms, mx, _ = oracle.frac_errors(res[sinks - p0, :3], oracle.fp64_sinks(hbox, w["softening"], eps, sinks))
    counts = np.diff(cs)
    result = {
        "metric": "pair_interactions_per_s", "value": pairs / (ms / 1e3), "unit": "pairs/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (generated on the GPU)",
        "config": {"workload": args.workload, "desc": w["desc"], "particles": n, "cpd": w["cpd"],
                   "slabs": [lo, hi], "particles_in_slabs": p1 - p0, "pairs_per_step": pairs,
                   "padded_pairs_per_step": int(t.padded_pairs),
                   "max_particles_per_cell": int(counts.max()), "kernel_shape": 0},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None, "kernel": "pencil_kernel",
                     "kernel_ms": k_ms, "flops_per_pair": flops,
                     "peak_probe_sustained": peak_s, "peak_clock_derived": derived,
                     "staging_hbm": staging_hbm(p1 - p0, box_nc(w), k_ms, None)},
        "accuracy_vs_fp64": {"rms_frac": rms, "max_frac": mx, "sinks": 2000},
        "gpu_launches": int(args.steps * t.launches),
        "clocks": clocks,
        "device_bytes": db.device_bytes() if hasattr(db, "device_bytes") else None,
    }
    db.close()
    ctx.close()
    print(json_line(result), flush=True)
    return 0


def big_full_sweep(args, w, capi, ctx, db, hbox, eps, peak_s, stream):
    """The whole 1024^3 box, compensated and then plain FP32 accumulation:
    one persistent launch per range of --slabs slabs (the partials of the
    whole box would not fit beside the positions), device time summed over
    the ranges; FP64 oracle on 2000 seeded sinks for each mode."""
    import torch
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    cpd, soft = w["cpd"], w["softening"]
    ranges = [(lo, min(cpd, lo + args.slabs)) for lo in range(0, cpd, args.slabs)]
    sinks = np.sort(np.random.default_rng(5).choice(hbox.n, 2000, replace=False))
    a64 = oracle.fp64_sinks(hbox, soft, eps, sinks)
    flops = FLOPS_PER_PAIR[soft]
    modes = {}
    for name, acc in (("compensated", capi.ACC_COMPENSATED), ("plain", capi.ACC_PLAIN)):
        if db is None:
            ctx = capi.Context(softening=soft, eps=eps, kernel_variant=0, accumulation=acc)
            ctx.set_stream(stream.cuda_stream)
            db = ctx.box(hbox)
        got = np.zeros((sinks.size, 3), np.float32)
        tot_ms = k_ms = 0.0
        pairs = 0
        with ClockSampler(0) as clk:
            for lo, hi in ranges:
                p0, p1 = db.slab_particles(lo, hi)
                out = torch.empty((max(p1 - p0, 1), 4), dtype=torch.float32, device="cuda")
                db.forces_device(lo, hi, out.data_ptr())
                t = ctx.last_timing()
                tot_ms += t.total_ms
                k_ms += t.kernel_ms
                pairs += int(t.pairs)
                sel = (sinks >= p0) & (sinks < p1)
                if sel.any():
                    got[sel] = out[torch.from_numpy(sinks[sel] - p0).cuda(), :3].cpu().numpy()
                del out
        rms, mx, _ = oracle.frac_errors(got, a64)
        achieved = pairs * flops / (k_ms / 1e3) / 1e12
        clocks = clk.summary()
        peak, derived = peak_from(peak_s, clocks,
                                  torch.cuda.get_device_properties(0).multi_processor_count)
        modes[name] = {"pairs": pairs, "device_ms": tot_ms, "kernel_ms": k_ms,
                       "pairs_per_s": pairs / (tot_ms / 1e3), "frac_of_fp32_peak": achieved / peak,
                       "peak": peak, "peak_clock_derived": derived, "peak_probe_sustained": peak_s,
                       "rms_frac": rms, "max_frac": mx, "clocks": clocks}
        db.close()
        ctx.close()
        db = None
        torch.cuda.empty_cache()
    c = modes["compensated"]
    result = {
        "metric": "pair_interactions_per_s", "value": c["pairs_per_s"], "unit": "pairs/s",
        "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": c["device_ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (generated on the GPU)",
        "config": {"workload": args.workload, "desc": w["desc"], "particles": hbox.n, "cpd": cpd,
                   "full_sweep": True, "slabs_per_launch": args.slabs, "launches": len(ranges),
                   "kernel_shape": 0,
                   "max_particles_per_cell": int(np.diff(hbox.cell_start).max())},
        "roofline": {"bound": "fp32", "achieved": c["pairs"] * flops / (c["kernel_ms"] / 1e3) / 1e12,
                     "peak": c["peak"], "unit": "TFLOP/s", "frac": c["frac_of_fp32_peak"],
                     "traffic": None, "kernel": "pencil_kernel", "kernel_ms": c["kernel_ms"],
                     "flops_per_pair": flops,
                     "staging_hbm": staging_hbm(hbox.n, box_nc(w), c["kernel_ms"], None)},
        "modes": modes,
        "accuracy_vs_fp64": {"rms_frac": c["rms_frac"], "max_frac": c["max_frac"], "sinks": 2000},
        "gpu_launches": 2 * len(ranges) * 2,
    }
    print(json_line(result), flush=True)
    return 0


def shard_arm(args, w):
    """One box split over the ranks (strong scaling): contiguous x-slab
    ranges balanced by pair count, a 2-slab position halo exchanged per step
    over NCCL point-to-point messages, each rank sweeping its own slabs from
    a window box (owned + halo slabs).  A step = halo exchange + upload of
    the window's positions (device to device) + the owned slabs' sweep."""
    import torch
    rank, world, local = dist_init(args.gpus)
    _pkg()
    from abacus_public_b200 import capi, shard
    torch.cuda.set_device(local)
    box = make_box(w)  # the same box on every rank; each keeps only its slabs
    parts = shard.partition(box.cpd, world, weights=shard.slab_pairs(box),
                            min_slabs=2 if world > 1 else 1)
    lo, hi = parts[rank]
    owned_h = shard.extract(box, range(lo, hi))
    dev = torch.device(f"cuda:{local}")
    owned = {s: (d.counts, torch.from_numpy(np.stack([d.x, d.y, d.z])).to(dev))
             for s, d in owned_h.items()}
    halo = shard.exchange_device(owned, rank, world, box.cpd, parts=parts)
    wslabs = shard.window_slabs(lo, hi, box.cpd)
    wbox = shard.window_box(box.cpd, shard.extract(box, wslabs))
    del box
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    ctx = capi.Context(softening=w["softening"], eps=kernel_eps(w), device=local)
    ctx.set_stream(stream.cuda_stream)
    db = ctx.box(wbox)
    p0, p1 = db.slab_particles(lo, hi)
    out = torch.empty((max(p1 - p0, 1), 4), dtype=torch.float32, device=dev)
    pairs = db.pair_count(lo, hi)

    def step():
        hl = shard.exchange_device(owned, rank, world, box_cpd, parts=parts)
        allp = {**hl, **owned}
        xyz = torch.cat([allp[s][1] for s in wslabs], dim=1).contiguous()
        db.update_device(xyz[0].data_ptr(), xyz[1].data_ptr(), xyz[2].data_ptr())
        db.forces_device(lo, hi, out.data_ptr())
        return xyz

    box_cpd = wbox.cpd
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    kms = []
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
            kms.append(ctx.last_timing().kernel_ms)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
    ms = barrier_max(e0.elapsed_time(e1) / args.steps, world)
    total_pairs = all_sum(float(pairs), world)
    k_ms = barrier_max(float(np.mean(kms)), world)
    # end to end: owned positions from pinned host memory, owned results back
    host = {s: v[1].cpu().pin_memory() for s, v in owned.items()}
    hout = torch.empty(tuple(out.shape), dtype=torch.float32).pin_memory()
    barrier(world)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        for s in owned:
            owned[s][1].copy_(host[s], non_blocking=True)
        step()
        hout.copy_(out, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = barrier_max(e0.elapsed_time(e1) / args.steps, world)
    nbytes = all_sum(float(sum(v.numel() * 4 for v in host.values())), world)
    flops = FLOPS_PER_PAIR[w["softening"]]
    clocks = clk.summary()
    peaks = fp32_peaks(ctx, clocks, torch.cuda.get_device_properties(local).multi_processor_count)
    peak_s = peaks["peak"]
    achieved = pairs * flops / (k_ms / 1e3) / 1e12
    result = {
        "metric": "pair_interactions_per_s", "value": total_pairs / (ms / 1e3), "unit": "pairs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": args.workload, "desc": w["desc"], "pairs_per_step": total_pairs,
                   "parallelism": f"slab-sharded x{world} (2-slab halo over NCCL)",
                   "slabs": parts, "l2": "inputs larger than L2"},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak_s, "unit": "TFLOP/s",
                     "frac": achieved / peak_s, "traffic": None, "kernel": "pencil_kernel",
                     "kernel_ms": k_ms, "note": "slowest rank's kernel time, its own pairs",
                     "peak_source": peaks["peak_source"]},
        "e2e": {"value": total_pairs / (e2e_ms / 1e3), "unit": "pairs/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(nbytes), "d2h_bytes_per_step": int(16 * (p1 - p0) * world)},
        # per step: the sweep's launches, plus order_keys and pack_ordered of the upload
        "gpu_launches": int(args.steps * (ctx.last_timing().launches + 2)),
        "clocks": clocks,
    }
    db.close()
    ctx.close()
    if rank == 0:
        print(json_line(result), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="clustered512")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-pairs", type=float, default=1.2e10,
                    help="pairs in the fixed seeded row sample of the CPU reference (both arms)")
    ap.add_argument("--e2e-steps", type=int, default=0,
                    help="timed end-to-end steps (0: --steps)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain drop-in phase")
    ap.add_argument("--no-ref-kernel", action="store_true",
                    help="skip the reference GPU kernel leg")
    ap.add_argument("--no-precision", action="store_true",
                    help="skip the compensated-vs-plain precision study")
    ap.add_argument("--precision-steps", type=int, default=3,
                    help="timed sweeps of the plain-accumulation form")
    ap.add_argument("--serve-requests", type=int, default=10000,
                    help="slab requests per serving load level (at most 2000 at 1.5x)")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving phase")
    ap.add_argument("--serve-boxes", default="45,65,85,105,125",
                    help="serve clustered boxes of N=64*cpd^3 for these cpds (comma list)")
    ap.add_argument("--serve-slots", type=int, default=2, help="serving slots (max_inflight)")
    ap.add_argument("--slabs", type=int, default=32,
                    help="clustered1024: the slab range [0, SLABS) a step sweeps (with "
                         "--full: slabs per launch)")
    ap.add_argument("--full", action="store_true",
                    help="clustered1024: one full sweep of the box, compensated and plain")
    ap.add_argument("--replicas", action="store_true",
                    help="with N > 1: one independent box per rank (weak scaling) instead of "
                         "one box split over the ranks")
    ap.add_argument("--shard", action="store_true",
                    help="split one box over the ranks even at N = 1")
    ap.add_argument("--profile", action="store_true",
                    help="timed sweeps only (no peak probe, CPU baseline, e2e or latency "
                         "phases): the command profiled under ncu")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    w = WORKLOADS[args.workload]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        return reference_arm(args, w)
    if args.shard or (world > 1 and not args.replicas):
        return shard_arm(args, w)
    if w["kind"] == "clustered_device":
        return big_arm(args, w)
    return our_arm(args, w)


if __name__ == "__main__":
    sys.exit(main())
