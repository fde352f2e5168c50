"""Benchmark: Wilson-flow link-updates/s at 32^4, mixed (FP32 links, FP64 reductions)
vs FP64, on B200.

One "step" is one Luscher RK3 flow step over a whole 32^4 configuration:
4 * 32^4 = 4,194,304 link-updates; the mixed forms reunitarise in FP64 after
every 10th step inside the timed region (the 32^4 configuration's schedule).
The stage form (fused kernel, two kernels through a stored plaquette field,
or one kernel with a tile's plaquette field in shared memory) is the
project's autotuner's choice for the lattice and precision; on B200 it picks
the two-kernel stage at 32^4 in every precision.  The default
precision is the 12-real FP32 form.  Inputs are seeded
synthetic fields U = e^{i a H} (a = 0.35, H Gaussian traceless Hermitian per
link), generated on the device; 32^4 links plus the generator field are larger
than the 126 MB L2 (no flush needed).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp32_12|fp32_18|fp64]
                  [--no-autotune | --stage-form 0|1|2 [--tile ty,tz,lpt,lean]]
  python bench.py --impl reference     # the reference's own CPU code on the host cores

Multi-GPU (torchrun, one rank per GPU): every rank flows its own configuration
(replicas; the flow of independent configurations has no data-path exchange),
timing is the max over ranks, `value` the sum of all ranks' link-updates.

  python bench.py --decompose [--gpus N]   # ONE 32^4 configuration split along t

--decompose times one configuration split into N time slabs, one per rank,
with halos exchanged by NCCL after every stage (strong scaling).  At N = 1
the single slab exchanges with itself, which prices the exchange on one GPU.

  python bench.py --workload 8 | 16x32 | 64   # the other configurations, every precision against FP64
  python bench.py --profile [--profile-kernel obs] --precision P   # only the timed kernels, for ncu

The JSON line carries, besides the contract's keys: `roofline` (HBM: the
compulsory bytes of a stage, 6 s_U + 4 s_Z per link-update over three
launches, over the stage kernel's time in the graph-replayed steps, `frac`;
the whole step's fraction, `step_frac_8d`; the DRAM bytes the ncu captures in
profiles/ count, over the compulsory ones; `field_kernel` the plaquette-field
kernel of the two-kernel stage on its own bytes),
`alu_roofline` (the reference algorithm's flops over the step's kernel time,
against the measured FP32 or FP64 FMA peak),
`accuracy_vs_fp64` (t^2 E and Q at t = 4), `ensemble` (64 configurations of
four sizes) and `cpu_baseline` (the reference's own code on one host core).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Wilson-flow link-updates/s at 32^4: mixed vs FP64 on GPU at dE/E<1e-6; %HBM"
UNIT = "link-updates/s"
DIMS = (32, 32, 32, 32)
EPS = 0.01
A = 0.35
SEED = 20260
T_CHECK = 400  # accuracy check: flow to t = 4.0 (config: eps 0.01, 400 steps)
REUNIT_EVERY = 10  # the mixed forms' FP64 reunitarisation period (the 32^4 configuration's)
LINK_BYTES = {"fp64": 144, "fp32_18": 72, "fp32_12": 48}
FORCE_BYTES = {"fp64": 64, "fp32_18": 32, "fp32_12": 32}


def bytes_per_link_update(prec: str) -> int:
    """Compulsory HBM bytes of one link through the three fused stages with
    ping-pong link buffers: read + write the link per stage (6 s_U) and the
    8-real generator written in stage 0, read + written in stage 1, read in
    stage 2 (4 s_Z)."""
    return 6 * LINK_BYTES[prec] + 4 * FORCE_BYTES[prec]


def split_bytes_per_link(prec: str):
    """Compulsory HBM bytes per link of one launch of each kernel of the
    two-kernel stage, averaged over the three stages: the plaquette-field
    kernel reads the link (s_U) and writes the site's six plane generators
    (6 s_Z per site = 1.5 s_Z per link); the stage kernel reads the link and
    the plane generators, writes the link, and moves the RK generator (4 s_Z
    over three stages)."""
    su, sz = LINK_BYTES[prec], FORCE_BYTES[prec]
    return su + 1.5 * sz, 2 * su + 1.5 * sz + 4 * sz / 3.0


# Algorithmic flops of one link through one RK3 stage, as the reference's
# algorithm counts them: 12 staple products + U Omega + Q^2 + e^{iQ} U, 198 flops
# per 3x3 complex product, plus about 300 scalar flops (projection, RK combine,
# tr Q^3, Cayley-Hamilton coefficients, f0 + f1 Q + f2 Q^2).
FLOPS_PER_LINK_STAGE = 15 * 198 + 300


STAGE_KERNELS = {
    0: ("rk_stage", "rk_stage_kernel (fused RK3 stage, staples per link)"),
    1: ("rk_split_stage", "rk_split_stage_kernel (RK3 stage from the stored plaquette field)"),
    2: ("rk_tile_stage", "rk_tile_stage_kernel (one-kernel RK3 stage, a tile's plaquette field in shared memory)"),
}


def roofline_8d(prec: str, links: int, lups: float, stage_launch_s: float, peak_gbs: float) -> dict:
    """The HBM roofline on the compulsory bytes of the three stages
    (6 s_U + 4 s_Z per link-update, whatever the kernels move): `frac` for one
    stage launch (a third of them over its duration) and `step_frac` for the
    whole step at `lups` link-updates/s."""
    per_launch = bytes_per_link_update(prec) * links / 3.0
    achieved = per_launch / stage_launch_s / 1e9
    step = lups * bytes_per_link_update(prec) / 1e9
    return {"algorithmic_bytes_per_launch": per_launch, "achieved": achieved, "frac": achieved / peak_gbs,
            "step_achieved": step, "step_frac": step / peak_gbs}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(prec: str, dims, alg_bytes_avg: float, kernel: str = "rk_stage"):
    """DRAM bytes of an average launch of `kernel` from the committed ncu
    summary (profiles/<kernel>_<dims>_<prec>.md), or None.  The summary holds
    one captured launch with its own algorithmic bytes; its
    traffic/algorithmic ratio is applied to the average launch."""
    name = "%s_%s_%s.md" % (kernel, "x".join(str(d) for d in dims), prec)
    p = ROOT / "profiles" / name
    if not p.exists():
        return None
    vals = {}
    for line in p.read_text().splitlines():
        for key in ("traffic_bytes_per_launch:", "algorithmic_bytes_per_launch:"):
            if line.startswith(key):
                vals[key] = float(line.split(":")[1])
    if len(vals) != 2:
        return None
    return vals["traffic_bytes_per_launch:"] / vals["algorithmic_bytes_per_launch:"] * alg_bytes_avg


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 8:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)

    def summary(self):
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in self.rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in self.rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[4 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ----------------------------------------------------------------------------------------------
# distributed plumbing (torchrun); single GPU needs none
# ----------------------------------------------------------------------------------------------
class Dist:
    def __init__(self, n_gpus: int):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.torch = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            self.torch = torch
            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.dist = dist
            self.dev = torch.device("cuda", self.local) if backend == "nccl" else torch.device("cpu")

    def barrier(self):
        if self.torch:
            self.dist.barrier()
            if self.dev.type == "cuda":
                self.torch.cuda.synchronize()

    def max(self, v: float) -> float:
        if not self.torch:
            return v
        t = self.torch.tensor([v], dtype=self.torch.float64, device=self.dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.torch:
            self.dist.barrier()
            self.dist.destroy_process_group()


# ----------------------------------------------------------------------------------------------
# CPU side: the reference's own code (oracle/_ref/ref_flow) on the host cores
# ----------------------------------------------------------------------------------------------
def write_reference_input(path: Path, dims, seed: int) -> None:
    from oracle import ymoracle as yo

    yo.write_bin(yo.gen_expiah(dims, A, seed), path)


def host_processes(per_proc_gb: float) -> int:
    cores = os.cpu_count() or 1
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        pass
    avail_gb = None
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                avail_gb = int(line.split()[1]) / 1e6
    except OSError:
        pass
    n = cores
    if avail_gb:
        n = min(n, max(1, int(0.5 * avail_gb / per_proc_gb)))
    return max(1, min(n, 64))


def host_cpu() -> dict:
    """The host's CPU model and usable cores (for the CPU baseline's record)."""
    model = None
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count()
    return {"cpu_model": model, "nproc": cores}


def run_reference(dims, nproc: int, steps: int):
    """nproc concurrent single-rank reference processes, each flowing its own copy of
    the seeded configuration `steps` RK3 steps.  Returns (link-updates/s, detail)."""
    from oracle import ymoracle as yo

    if not yo.ref_available():
        return None, "oracle/_ref/ref_flow is not built"
    with tempfile.TemporaryDirectory() as d:
        conf = Path(d) / "conf.bin"
        write_reference_input(conf, dims, SEED)
        args = [str(yo.REF_BIN), "time", str(conf)] + [str(v) for v in dims] + [repr(EPS), str(steps)]
        procs = [subprocess.Popen(args, stdout=subprocess.PIPE, text=True) for _ in range(nproc)]
        outs = []
        for p in procs:
            out, _ = p.communicate()
            if p.returncode != 0:
                return None, "ref_flow failed"
            outs.append(json.loads(out.strip().splitlines()[-1]))
    t = max(o["flow_seconds"] for o in outs)
    links = 4 * dims[0] * dims[1] * dims[2] * dims[3]
    return nproc * links * steps / t, {"flow_seconds_max": t, "obs_seconds": outs[0]["obs_seconds"]}


def reference_arm(args):
    per_proc_gb = 3.6 * (DIMS[0] * DIMS[1] * DIMS[2] * DIMS[3]) / 32 ** 4
    nproc = host_processes(per_proc_gb)
    steps = 1
    value, detail = run_reference(DIMS, nproc, steps)
    if value is None:
        print(json.dumps({"impl": "reference", "unavailable": detail}))
        return
    sample = ("%d concurrent single-rank reference processes (src/ compiled against a one-rank MPI "
              "stand-in), each one RK3 step of its own 32^4 configuration" % nproc)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": 0, "ms_per_step": detail["flow_seconds_max"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded e^{iaH}, a=0.35)",
        "config": {"workload": "32^4 Wilson flow, RK3 eps=0.01, reference CPU code", "lattice": list(DIMS),
                   "parallelism": "%d host processes" % nproc},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": "reference", "sample": sample,
                         "host": host_cpu()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ----------------------------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------------------------
def ensemble_sizes():
    """The batched workload: 64 configurations, 16 each of 8^4, 12^4, 16^4 and 16^3 x 32."""
    return [(8,) * 4] * 16 + [(12,) * 4] * 16 + [(16,) * 4] * 16 + [(16, 16, 16, 32)] * 16


def ensemble_measure(prec: str, steps: int, dev: int):
    """Aggregate link-updates/s of the batched ensemble (one persistent launch per
    stage for all 64 configurations) against flowing them one by one."""
    import numpy as np

    from latticeyangmills_b200 import Ensemble, GluonField

    sizes = ensemble_sizes()
    rng = np.random.default_rng(4)
    a_list = rng.uniform(0.25, 0.45, size=len(sizes))
    links = sum(4 * s[0] * s[1] * s[2] * s[3] for s in sizes)
    ens = Ensemble(sizes, prec, device=dev)
    for c in range(len(sizes)):
        ens.init_links(c, "expiah", float(a_list[c]), SEED + c, c)
    block, grid = ens.autotune(EPS)
    form = ens.tuning()[0]
    ens.time_steps(EPS, 3)
    ms = ens.time_steps(EPS, steps)
    ens.close()
    one_ms = 0.0
    for c, n in enumerate(sizes):
        f = GluonField(n, prec, device=dev)
        f.init_links("expiah", float(a_list[c]), SEED + c, c)
        f.time_steps(EPS, 3)
        el, _ = f.time_steps(EPS, steps)
        one_ms += el
        f.close()
    return {"configs": len(sizes), "sizes": "16x8^4 + 16x12^4 + 16x16^4 + 16x16^3x32", "precision": prec,
            "steps": steps, "link_updates_per_s": links * steps / (ms / 1e3),
            "one_by_one_link_updates_per_s": links * steps / (one_ms / 1e3),
            "speedup_vs_one_by_one": one_ms / ms,
            "autotuned": {"stage_form": form, "block": block, "grid": grid}}


def workload_run(args, dev: int):
    """The other configurations of the benchmark set, each flowed in every precision
    from the same seeded field, with each observable's error against FP64:
      16x32: 16^3 x 32, a = 0.35, eps 0.01 to t = 2, observables every 10 steps
      64:    64^4, a = 0.35 plus 5 % Haar-random links, eps 0.02 to t = 6,
             observables every 5 steps (about 24 GB in FP64)
      8:     8^4 Metropolis field (beta 6, 200 sweeps of 30 hits from cold, made by the
             device generator in FP64), eps 0.01, 100 steps, observables every step."""
    import time

    import numpy as np

    from latticeyangmills_b200 import GluonField

    field = None
    if args.workload == "16x32":
        dims, a, haar, eps, nsteps, every = (16, 16, 16, 32), A, 0.0, 0.01, 200, 10
    elif args.workload == "8":
        dims, a, haar, eps, nsteps, every = (8, 8, 8, 8), 0.0, 0.0, 0.01, 100, 1
        with GluonField(dims, "fp64", device=dev) as g:
            acceptance = g.generate_metropolis(6.0, 0.24, 200, 30, SEED, "cold")
            field = g.download()
    else:
        dims, a, haar, eps, nsteps, every = (64, 64, 64, 64), A, 0.05, 0.02, 300, 5
    links = 4 * dims[0] * dims[1] * dims[2] * dims[3]

    def load(f):
        if field is None:
            f.init_links("expiah", a, SEED, 0, haar)
        else:
            f.upload(field)

    res = {}
    for p in ["fp64", "fp32_18", "fp32_12"]:
        f = GluonField(dims, p, device=dev)
        load(f)
        t0 = time.perf_counter()
        rows = f.flow(eps, nsteps, every, reunit_every=10 if p != "fp64" else 0)
        wall = time.perf_counter() - t0
        load(f)
        f.time_steps(eps, 3)
        ms, _ = f.time_steps(eps, 20)
        f.close()
        res[p] = (rows, links * 20 / (ms / 1e3), wall)
    r64 = res["fp64"][0]
    out = {"workload": args.workload, "lattice": list(dims), "eps": eps, "steps": nsteps, "measure_every": every,
           "haar_fraction": haar, "t_final": float(r64[-1, 1]), "t2E_fp64_final": float(r64[-1, 5]),
           "Q_fp64_final": float(r64[-1, 3])}
    if field is not None:
        out.update({"field": "Metropolis beta 6, 200 sweeps x 30 hits, su3eps 0.24, from cold",
                    "metropolis_acceptance": acceptance, "plaq_t0": float(r64[0, 2])})
    for p in ["fp64", "fp32_18", "fp32_12"]:
        rows, lups, wall = res[p]
        d = {"link_updates_per_s": lups, "flow_wall_s_with_measurements": wall}
        if p != "fp64":
            rel = np.abs(rows[1:, 5] - r64[1:, 5]) / np.abs(r64[1:, 5])
            d.update({"max_rel_err_t2E": float(rel.max()), "rel_err_t2E_final": float(rel[-1]),
                      "max_abs_err_Q": float(np.abs(rows[:, 3] - r64[:, 3]).max()),
                      "max_abs_err_plaq": float(np.abs(rows[:, 2] - r64[:, 2]).max())})
        out[p] = d
    print(json.dumps(out))


def our_arm(args, dist: Dist):
    import ctypes

    import numpy as np

    from latticeyangmills_b200 import GluonField, _native as N

    V = DIMS[0] * DIMS[1] * DIMS[2] * DIMS[3]
    links = 4 * V
    prec = args.precision
    dev = dist.local
    seed = SEED + 1000 * dist.rank
    reunit = 0 if prec == "fp64" else REUNIT_EVERY

    f = GluonField(DIMS, prec, device=dev)
    f.init_links("expiah", A, seed)
    if args.profile and args.profile_kernel == "obs":
        # observables only (plaquette, clover energy and charge), for ncu captures
        for _ in range(args.warmup + args.steps):
            f.observables()
        f.close()
        if dist.rank == 0:
            print(json.dumps({"profile": True, "kernel": "observables", "precision": prec, "lattice": list(DIMS)}))
        return
    # the stage form and tile: the project's autotuner (cached per lattice and
    # precision), or the one given on the command line
    if args.stage_form is not None:
        if args.stage_form == 2 and args.tile:
            f.set_tile(*[int(v) for v in args.tile.split(",")])
        f.set_option(N.OPT_STAGE_FORM, args.stage_form)
    tuned = None if (args.no_autotune or args.stage_form is not None) else f.autotune(EPS)
    form = f.get_option(N.OPT_STAGE_FORM)
    tile = f.get_option(N.OPT_TILE)
    f.set_option(N.OPT_TIMED_REUNIT, reunit)  # the FP64 reunitarisation of the mixed forms, every 10 steps
    f.time_steps(EPS, args.warmup)  # untimed warm-up

    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.5)
    f.time_steps(EPS, max(args.warmup, 3))  # brings clocks up before the sampled window
    dist.barrier()
    elapsed_ms, _ = f.time_steps(EPS, args.steps)
    dist.barrier()
    if args.profile:
        clocks.stop()
        f.close()
        if dist.rank == 0:
            print(json.dumps({"profile": True, "precision": prec, "lattice": list(DIMS), "stage_form": form,
                              "ms_per_step": elapsed_ms / args.steps}))
        return
    # The stage kernels alone, in the same graph-replayed execution without the
    # reunitarisation (per launch: a third of a step), and with events around
    # every launch of a third pass (instrumented: no graph).
    f.set_option(N.OPT_TIMED_REUNIT, 0)
    graph_ms, _ = f.time_steps(EPS, args.steps)
    _, field_ms, stage_ms = f.time_kernels(EPS, args.steps)
    f.set_option(N.OPT_TIMED_REUNIT, reunit)
    clocks.stop()
    t_max = dist.max(elapsed_ms / 1e3)
    value = dist.world * links * args.steps / t_max
    n_reunit = args.steps // reunit if reunit else 0

    # FP64 path on the same workload (the "vs FP64" of the metric), autotuned the same way
    fp64_value = fp64_form = None
    if prec != "fp64":
        g = GluonField(DIMS, "fp64", device=dev)
        g.init_links("expiah", A, seed)
        if not args.no_autotune:
            g.autotune(EPS)
        fp64_form = g.get_option(N.OPT_STAGE_FORM)
        g.time_steps(EPS, args.warmup)
        dist.barrier()
        ms64, _ = g.time_steps(EPS, args.steps)
        fp64_value = dist.world * links * args.steps / dist.max(ms64 / 1e3)
        g.close()

    # roofline of the dominant kernel, on the compulsory bytes of the three stages
    peak, peak_kind = measured_peaks()
    kprefix, kname = STAGE_KERNELS[form]
    split = form == 1
    kernels_per_stage = 2 if split else 1
    if split:  # the stage kernel's share of the graph-timed stage, from the instrumented pass
        stage_launch_s = graph_ms / 1e3 / (3 * args.steps) * stage_ms / (field_ms + stage_ms)
    else:
        stage_launch_s = graph_ms / 1e3 / (3 * args.steps)
    roof = roofline_8d(prec, links, value / dist.world, stage_launch_s, peak)
    alg = roof["algorithmic_bytes_per_launch"]
    traffic = profiled_traffic(prec, DIMS, alg, kprefix)
    # DRAM bytes of all of a stage's kernels (the plaquette field's too) over its compulsory bytes
    stage_traffic = traffic
    if split and traffic is not None:
        ft = profiled_traffic(prec, DIMS, split_bytes_per_link(prec)[0] * links, "plaq_field")
        stage_traffic = traffic + ft if ft is not None else None
    field_roof = None
    if split:
        field_b, stage_b = split_bytes_per_link(prec)
        field_s = field_ms / 1e3 / (3 * args.steps)
        field_roof = {"kernel": "plaq_field_kernel (six plane generators per site)",
                      "design_bytes_per_launch": field_b * links, "avg_launch_ms_events": field_s * 1e3,
                      "design_frac": field_b * links / field_s / 1e9 / peak,
                      "share_of_kernel_time": field_ms / (field_ms + stage_ms)}
    # arithmetic roofline: the reference algorithm's flops over the step's kernel
    # time, against the measured CUDA-core FMA peak
    fma_tf = ctypes.c_double(0.0)
    N.check(N.load().ymflow_fma_peak(dev, N.FP64 if prec == "fp64" else N.FP32_18, ctypes.byref(fma_tf)))
    alu_achieved = links * FLOPS_PER_LINK_STAGE / (graph_ms / 1e3 / (3 * args.steps)) / 1e12

    # accuracy of the mixed form against FP64 at t = 4 (400 steps), same seeded field
    accuracy = None
    if not args.skip_accuracy and dist.rank == 0:
        res = {}
        for p in sorted({prec, "fp64"}):
            h = GluonField(DIMS, p, device=dev)
            h.init_links("expiah", A, SEED)
            if not args.no_autotune:
                h.autotune(EPS)  # the cached choice of the timed contexts
            rows = h.flow(EPS, T_CHECK, 0, reunit_every=REUNIT_EVERY if p != "fp64" else 0)
            res[p] = rows[-1]
            h.close()
        r64, rm = res["fp64"], res[prec]
        accuracy = {"t": float(rm[1]), "t2E_fp64": float(r64[5]), "t2E": float(rm[5]),
                    "rel_err_t2E": abs(float(rm[5]) - float(r64[5])) / abs(float(r64[5])),
                    "Q_fp64": float(r64[3]), "abs_err_Q": abs(float(rm[3]) - float(r64[3])),
                    "abs_err_plaq": abs(float(rm[2]) - float(r64[2])), "reunit_every": REUNIT_EVERY}

    # end to end through the C ABI with host buffers: upload the .bin-layout FP64
    # configuration from pinned memory, flow K steps, read the observables back
    host = ctypes.c_void_p()
    nbytes = links * 18 * 8
    N.check(N.load().ymflow_host_alloc(nbytes, ctypes.byref(host)))
    hbuf = np.ctypeslib.as_array(ctypes.cast(host, ctypes.POINTER(ctypes.c_double)), shape=(links * 18,))
    hbuf[:] = f.download().reshape(-1)
    e2e_iters = 3
    f.upload(hbuf)
    f.flow(EPS, 2, 0)  # warm path
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_iters):
        f.upload(hbuf)
        rows = f.flow(EPS, args.steps, 0, reunit_every=reunit)
    t_e2e = dist.max(time.perf_counter() - t0)
    e2e_value = dist.world * links * args.steps * e2e_iters / t_e2e
    N.load().ymflow_host_free(host)
    rows_bytes = 2 * 48  # two measurement rows (before / after) come back per job

    ensemble = None
    if not args.skip_ensemble and dist.rank == 0:
        ensemble = ensemble_measure(prec if prec != "fp64" else "fp32_18", args.steps, dev)

    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.skip_cpu:
        val, detail = run_reference(DIMS, 1, 1)
        if val is not None:
            cpu = {"value": val, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": "one RK3 step of the 32^4 configuration by the reference's own code "
                             "(oracle/_ref/ref_flow), one core", "host": host_cpu()}
    f.close()

    if dist.rank == 0:
        launches = 3 * args.steps * kernels_per_stage + n_reunit
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if prec != "fp64" else "f64",
            "data": "synthetic (seeded U = e^{iaH}, a = 0.35, generated on the device)",
            "config": {"workload": "32^4 Wilson flow, Luscher RK3, eps = 0.01",
                       "lattice": list(DIMS), "precision": prec,
                       "reductions": "f64", "l2": "inputs larger than L2 (links + generator > 126 MB)",
                       "reunit_every": reunit or None,
                       "timed_region": "K RK3 steps%s, graph-replayed" % (
                           ", with the FP64 reunitarisation after every %d-th (%d launches)" % (reunit, n_reunit)
                           if reunit else ""),
                       "parallelism": "replicas x%d" % dist.world,
                       "stage_form": form, "tile": [tile >> 16, tile & 0xFFFF] if form == 2 else None,
                       "autotuned": tuned is not None,
                       "fp64_link_updates_per_s": fp64_value, "fp64_stage_form": fp64_form,
                       "mixed_over_fp64": (value / fp64_value) if fp64_value else None},
            "roofline": {"bound": "hbm", "achieved": roof["achieved"], "peak": peak, "unit": "GB/s",
                         "frac": roof["frac"], "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": kname,
                         "bytes": "compulsory bytes of the three stages, 6 s_U + 4 s_Z per link-update "
                                  "(%d B), a third per stage launch" % bytes_per_link_update(prec),
                         "algorithmic_bytes_per_launch": alg,
                         "avg_launch_ms": stage_launch_s * 1e3,
                         "avg_launch_ms_events": stage_ms / (3 * args.steps),
                         "launch_time_from": "graph-replayed steps without the reunitarisation, a third of a "
                                             "step per stage launch%s" % (
                                                 " times the stage kernel's share of the instrumented pass"
                                                 if split else ""),
                         "frac_8d": roof["frac"],
                         "step_achieved": roof["step_achieved"], "step_frac_8d": roof["step_frac"],
                         "dram_over_compulsory": stage_traffic / alg if stage_traffic else None,
                         "dram_over_compulsory_what": "DRAM bytes of a stage's kernels (ncu captures in profiles/, "
                                                      "scaled to an average stage) over its compulsory bytes",
                         "field_kernel": field_roof},
            "alu_roofline": {"bound": "fp64 fma" if prec == "fp64" else "fp32 fma", "achieved": alu_achieved,
                             "peak": fma_tf.value, "unit": "TFLOP/s", "frac": alu_achieved / fma_tf.value,
                             "peak_kind": "measured (ymflow_fma_peak, 8 independent FMA chains per thread)",
                             "flops_per_link_update": 3 * FLOPS_PER_LINK_STAGE},
            "accuracy_vs_fp64": accuracy,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": nbytes / args.steps,
                    "d2h_bytes_per_step": rows_bytes / args.steps,
                    "what": "per job: ymflow_upload of the .bin-layout FP64 field from pinned host memory, "
                            "ymflow_flow of K steps (reunitarisation every %s), observables rows back to the host"
                            % (reunit or "never")},
            "ensemble": ensemble,
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))


def decomposed_run(args, dist: Dist):
    """One configuration split along t over the ranks; NCCL halo exchange."""
    import ctypes

    import numpy as np

    from latticeyangmills_b200 import GluonField, _native as N, nccl_unique_id, slab_partition

    prec = args.precision
    V = DIMS[0] * DIMS[1] * DIMS[2] * DIMS[3]
    t0, nt, lo, hi = slab_partition(DIMS[3], dist.world, dist.rank)
    f = GluonField.slab(DIMS, t0, nt, prec, device=dist.local)
    f.init_links("expiah", A, SEED)
    if dist.world > 1:
        box = [nccl_unique_id() if dist.rank == 0 else None]
        dist.dist.broadcast_object_list(box, src=0)
        nid = box[0]
    else:
        nid = nccl_unique_id()
    f.connect(nid, dist.rank, dist.world, lo, hi)
    f.time_steps(EPS, args.warmup)
    clocks = ClockSampler(dist.local)
    clocks.start()
    time.sleep(0.5)
    f.time_steps(EPS, max(args.warmup, 3))
    dist.barrier()
    elapsed_ms, _ = f.time_steps(EPS, args.steps)
    dist.barrier()
    split = f.get_option(N.OPT_STAGE_FORM) == 1
    _, field_ms, stage_ms = f.time_kernels(EPS, args.steps)
    kernel_ms = field_ms + stage_ms
    clocks.stop()
    t_max = dist.max(elapsed_ms / 1e3)
    value = 4 * V * args.steps / t_max
    peak, peak_kind = measured_peaks()
    links_local = 4 * DIMS[0] * DIMS[1] * DIMS[2] * nt
    if split:
        bpl = split_bytes_per_link(prec)[1] * links_local
        kname = "rk_split_stage_kernel on rank 0's slab"
    else:
        bpl = bytes_per_link_update(prec) * links_local / 3.0
        kname = "rk_stage_kernel on rank 0's slab"
    avg_launch_s = stage_ms / 1e3 / (3 * args.steps)
    # end to end: every rank uploads its slab from pinned host memory, flows, reads the rows
    host = np.ascontiguousarray(f.download())
    t0w = time.perf_counter()
    f.upload(host)
    rows = f.flow(EPS, args.steps, 0)
    t_e2e = dist.max(time.perf_counter() - t0w)
    f.close()
    if dist.rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32" if prec != "fp64" else "f64",
            "data": "synthetic (seeded U = e^{iaH}, a = 0.35, generated on the device)",
            "config": {"workload": "one 32^4 configuration split along t, Luscher RK3, eps = 0.01",
                       "lattice": list(DIMS), "precision": prec, "parallelism": "t-slabs x%d" % dist.world,
                       "slices_per_rank": nt, "halo": "one time slice per side, NCCL send/recv after each stage",
                       "kernel_share_of_step": kernel_ms / elapsed_ms,
                       "l2": "inputs larger than L2 (links + generator > 126 MB per rank at N <= 2)"},
            "roofline": {"bound": "hbm", "achieved": bpl / avg_launch_s / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": bpl / avg_launch_s / 1e9 / peak, "traffic": None, "peak_kind": peak_kind,
                         "kernel": kname, "avg_launch_ms": avg_launch_s * 1e3,
                         "field_kernel_ms_per_launch": field_ms / (3 * args.steps) if split else None},
            "e2e": {"value": 4 * V * args.steps / t_e2e, "unit": UNIT,
                    "h2d_bytes_per_step": host.nbytes * dist.world / args.steps,
                    "d2h_bytes_per_step": 2 * 48 / args.steps,
                    "what": "per rank: upload of its slab from host memory, a K-step collective flow, rows back",
                    "t_end": float(rows[-1, 1])},
            "gpu_launches": 3 * args.steps * (2 if split else 1), "clocks": clocks.summary(), "cpu_baseline": None,
        }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32_12", choices=["fp64", "fp32_18", "fp32_12"])
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-accuracy", action="store_true")
    ap.add_argument("--skip-ensemble", action="store_true")
    ap.add_argument("--lattice", type=int, default=32, help="L of the L^4 lattice (profiling of smaller cases)")
    ap.add_argument("--workload", default="32", choices=["32", "16x32", "64", "8"],
                    help="32: the headline 32^4 benchmark; 8 / 16x32 / 64: accuracy and throughput of the "
                         "other configurations against FP64")
    ap.add_argument("--profile-kernel", default="stage", choices=["stage", "obs"],
                    help="with --profile: the RK stage kernels or the observables kernel")
    ap.add_argument("--decompose", action="store_true",
                    help="one 32^4 configuration split along t over the ranks (NCCL halo exchange)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default stage form instead of the autotuner's choice")
    ap.add_argument("--stage-form", type=int, choices=[0, 1, 2], default=None,
                    help="run this stage form (0 fused, 1 two kernels, 2 shared-memory tile) instead of the "
                         "autotuner's choice")
    ap.add_argument("--tile", default=None, help="with --stage-form 2: ty,tz[,links per thread[,lean]]")
    ap.add_argument("--profile", action="store_true",
                    help="only the warm-up and timed steps of one precision (for ncu captures)")
    args = ap.parse_args()
    global DIMS
    DIMS = (args.lattice,) * 4
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        # CPU-only: under torchrun rank 0 runs and prints, the other ranks exit at once
        if int(os.environ.get("RANK", "0")) == 0:
            reference_arm(args)
        return
    if args.workload != "32":
        workload_run(args, int(os.environ.get("LOCAL_RANK", "0")))
        return
    dist = Dist(args.gpus)
    try:
        if args.decompose:
            decomposed_run(args, dist)
        else:
            our_arm(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
