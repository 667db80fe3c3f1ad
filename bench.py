"""Element-cycle benchmark: element-updates/s of the split-FP32 path vs plain FP64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload shell_plate|hex_block|mixed_mesh|batched_parts]
                    [--sub-workloads mixed_mesh,batched_parts] [--eager-cycles N --mesh-n M --tile T]

One step = one complete run of the workload (all its cycles) from the uploaded
initial state; the state is reset between steps outside the timed region and
L2 is flushed (a 256 MB write) before every timed step.  Under torchrun a deck
of several independent parts (batched_parts) is sharded: each rank runs its
share of the parts (largest-first on element count, openradioss_b200/shard.py),
strong scaling over the fixed deck; a single-mesh deck is replicated, one copy
per rank (weak scaling).  Neither needs a data-path collective.  Timing is the
max over ranks of device time.  Prints one JSON line on rank 0.

The line also states the split form's error against the FP64 run per output
(nodal D, V, VR, stresses, plastic strains, internal / kinetic / hourglass
energy, plastic work), beside the FP64 run's own sensitivity floor (the same
FP64 run from coordinates perturbed by 1e-12) at the same cycle count, and
both again after 1000 cycles; on one GPU it adds a record of the 2.08 M-element
mixed mesh (split and FP64 rates, per-kernel roofline, split error).

--eager-cycles N runs N cycles of a workload without a CUDA graph (one launch
per kernel per cycle) and prints per-phase device times: the command that the
ncu captures under profiles/ run.
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

WORKLOADS = {
    # name: (deck factory, cycles, description)
    "shell_plate": ("c2_shell_plate", 2000,
                    "200x200 BT shells, 5 IP, LAW2 Johnson-Cook Al, 2 MPa pressure, 2000 cycles"),
    "hex_block": ("c1_hex_block", 1000, "10x10x40 hexas, LAW1 steel, -10 m/s, clamped base, 1000 cycles"),
    "mixed_mesh": ("c4_mixed_mesh", 5000,
                   "100x100x200 LAW2 steel hexas + 80,000-shell skin, -20 m/s, 5000 cycles"),
    "batched_parts": ("c3_batched_parts", 500, "64 uneven hex/shell parts, own dt each, 500 cycles"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="shell_plate", choices=sorted(WORKLOADS))
    ap.add_argument("--cycles", type=int, default=0, help="override cycles per step")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sub-workloads", default="mixed_mesh,batched_parts",
                    help="comma-separated workloads recorded beside the headline on one GPU ('' = none)")
    ap.add_argument("--sub-steps", type=int, default=3)
    ap.add_argument("--sub-tile", type=int, default=128)
    ap.add_argument("--eager-cycles", type=int, default=0,
                    help="profiling mode: run this many eager cycles and print per-phase times")
    ap.add_argument("--persistent-cycles", type=int, default=0,
                    help="profiling mode: three step() calls of this many cycles through the persistent shell "
                         "cycle, timed with events")
    ap.add_argument("--adjoint-cycles", type=int, default=0,
                    help="profiling mode: one or_ecycle_adjoint over this many cycles of the C5 plate (FP64)")
    ap.add_argument("--mesh-n", type=int, default=0, help="profiling mode: mesh size parameter (0 = workload's)")
    ap.add_argument("--tile", type=int, default=0, help="profiling mode: elements per patch (0 = library default)")
    ap.add_argument("--precision", default="split", choices=["split", "fp64"], help="profiling mode")
    return ap.parse_args()


def make_deck(name, n=0):
    """The workload's deck; n > 0 scales the mesh (profiling of smaller cases)."""
    from openradioss_b200 import decks
    if not n:
        return getattr(decks, WORKLOADS[name][0])()
    return {"shell_plate": lambda: decks.c2_shell_plate(n=n, size=n * 1e-3),
            "hex_block": lambda: decks.c1_hex_block(nx=n, ny=n, nz=4 * n),
            "mixed_mesh": lambda: decks.c4_mixed_mesh(nx=n, ny=n, nz=2 * n),
            "batched_parts": lambda: decks.c3_batched_parts()}[name]()


def workload_config(name, deck, cycles, world, sharded):
    """The `config` of the JSON line: the workload as both arms run it."""
    from openradioss_b200 import decks
    nel = decks.num_elements(deck)
    return {"workload": name, "description": WORKLOADS[name][2], "elements_per_gpu": nel,
            "nodes_per_gpu": decks.num_nodes(deck), "cycles_per_step": cycles,
            "elements_per_step_all_ranks": nel if sharded else world * nel,
            "parallelism": (f"parts sharded over {world} ranks" if sharded else f"{world} independent replica(s)"),
            "l2": "256 MB buffer written before every timed step"}


def outputs(h):
    """Per-output arrays of a handle's state (the quantities the split error is stated on)."""
    import numpy as np
    out = {}
    nodes = [h.get_nodes(p) for p in range(h.nparts)]
    for k, name in (("d", "D"), ("v", "V"), ("vr", "VR")):
        out[name] = np.concatenate([n[k].ravel() for n in nodes])
    if h.shell_groups:
        st = [h.shell_state(g) for g in range(len(h.shell_groups))]
        out["sigma_shell"] = np.concatenate([s["sig"].ravel() for s in st])
        out["pla_shell"] = np.concatenate([s["pla"].ravel() for s in st])
    if h.hex_groups:
        st = [h.hex_state(g) for g in range(len(h.hex_groups))]
        out["sigma_hex"] = np.concatenate([s["sig"].ravel() for s in st])
        out["pla_hex"] = np.concatenate([s["pla"].ravel() for s in st])
    en = [h.energies(p) for p in range(h.nparts)]
    for k in ("internal", "kinetic", "hourglass", "plastic_work"):
        out["E_" + k] = np.array([sum(e[k] for e in en)])
    return out


def output_errors(a, b):
    """max|a - b| / max|b| per output (0 where b is zero everywhere and a too)."""
    import numpy as np
    err = {}
    for k in b:
        den = float(np.abs(b[k]).max()) if b[k].size else 0.0
        num = float(np.abs(a[k] - b[k]).max()) if b[k].size else 0.0
        err[k] = num / den if den > 0 else (0.0 if num == 0 else float("inf"))
    return err


def perturbed_run(h, deck, cycles, eps=1e-12, seed=7):
    """The handle's run from its uploaded state with every coordinate moved by a
    relative eps (seeded signs): the run's own sensitivity to rounding-level input."""
    import numpy as np
    rng = np.random.default_rng(seed)
    h.reset()
    for p, part in enumerate(deck["parts"]):
        x = part["x"] * (1.0 + eps * rng.choice([-1.0, 1.0], size=part["x"].shape))
        h.set_nodes(p, x=x)
    h.step(cycles)
    return outputs(h)


def persistent_profile(args):
    """--persistent-cycles: the persistent shell cycle alone (one launch per step() call)."""
    import torch
    from openradioss_b200 import abi, build, decks
    from openradioss_b200.ecycle import ECycle
    build.build()
    d = make_deck(args.workload, args.mesh_n)
    prec = abi.OR_PREC_SPLIT if args.precision == "split" else abi.OR_PREC_FP64
    tiles = dict(block_shell=args.tile) if args.tile else {}
    h = ECycle(d, precision=prec, graph=1, **tiles)
    on, ctas, threads = h.persistent_info()
    if not on:
        raise SystemExit("this deck does not run the persistent shell cycle")
    s = torch.cuda.ExternalStream(h.stream())
    ms = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(s)
        h.step(args.persistent_cycles)
        e1.record(s)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    print(json.dumps({"workload": args.workload, "elements": decks.num_elements(d), "ctas": ctas, "threads": threads,
                      "cycles_per_launch": args.persistent_cycles,
                      "us_per_cycle": [m * 1e3 / args.persistent_cycles for m in ms]}))


def eager_profile(args):
    """--eager-cycles: per-phase device times of eager cycles (no graph)."""
    from openradioss_b200 import abi, build, decks
    from openradioss_b200.ecycle import ECycle
    build.build()
    d = make_deck(args.workload, args.mesh_n)
    prec = abi.OR_PREC_SPLIT if args.precision == "split" else abi.OR_PREC_FP64
    tiles = dict(block_hex=args.tile, block_shell=args.tile) if args.tile else {}
    h = ECycle(d, precision=prec, graph=0, **tiles)
    h.step(args.eager_cycles)
    print(json.dumps({"workload": args.workload, "elements": decks.num_elements(d), "cycles": args.eager_cycles,
                      "phase_ms": h.phase_times(), "launches": h.launch_count(), "time": h.time()}))


# ---------------------------------------------------------------------------
class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
            return
        # nvidia-smi takes a few hundred ms to start: wait for its first row, so that
        # a timed region of a few hundred ms is sampled from its start, then drop the
        # rows taken before it
        t0 = time.time()
        while not self.rows and self.proc.poll() is None and time.time() - t0 < 10.0:
            time.sleep(0.01)
        self.rows.clear()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
                for k, n in enumerate(names):
                    if r[4 + k].lower().startswith("active"):
                        reasons.add(n)
            except (ValueError, IndexError):
                pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
def cpu_baseline(deck, cycles, budget_s, fast=True):
    """Times the CPU oracle (C++ restatement of the reference path, OpenMP on
    all host threads) on a bounded sample of the workload's cycles."""
    from oracle.oracle import Oracle
    from openradioss_b200 import abi, decks
    nthreads = os.cpu_count() or 1
    nel = decks.num_elements(deck)
    o = Oracle(deck, precision=abi.OR_PREC_FP64, nthreads=nthreads, fast=fast)
    t0 = time.perf_counter()
    o.step(2)
    t1 = (time.perf_counter() - t0) / 2
    n = int(max(3, min(cycles, budget_s / max(t1, 1e-9))))
    t0 = time.perf_counter()
    o.step(n)
    dt = time.perf_counter() - t0
    return {"value": nel * n / dt, "unit": "element-updates/s", "cores": nthreads, "kind": "port",
            "sample": f"{n} timed cycles (after 2 untimed) of the {cycles}-cycle deck, FP64, "
                      f"C++ restatement of the reference CPU path, OpenMP {nthreads} threads"}


def reference_arm(args, rank, world):
    deck = make_deck(args.workload)
    from openradioss_b200 import decks
    from oracle.oracle import Oracle
    from openradioss_b200 import abi
    cycles = args.cycles or WORKLOADS[args.workload][1]
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    nel = decks.num_elements(deck)
    o = Oracle(deck, precision=abi.OR_PREC_FP64, nthreads=nthreads, fast=True)
    t0 = time.perf_counter()
    o.step(1)
    t1 = time.perf_counter() - t0
    per_step = int(max(2, min(cycles, (150.0 / max(1, args.steps + args.warmup)) / max(t1, 1e-9))))
    for _ in range(args.warmup):
        o.step(per_step)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.step(per_step)
        ts.append(time.perf_counter() - t0)
    tot = sum(ts)
    value = nel * per_step * args.steps / tot
    sample = (f"{per_step} cycles per step of the {args.workload} deck (of {cycles}), FP64, "
              f"C++ restatement of the reference CPU path, OpenMP {nthreads} threads")
    sharded = world > 1 and len(deck["parts"]) > 1
    line = {"metric": "element-updates/s", "value": value, "unit": "element-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
            "higher_is_better": True, "scaling": "strong" if sharded else "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded numpy decks with the workload's shapes)",
            "impl": "reference",
            "config": workload_config(args.workload, deck, cycles, world, sharded),
            "sample": {"cycles_per_step": per_step, "of_cycles": cycles, "ranks_running": 1},
            "cpu_baseline": {"value": value, "unit": "element-updates/s", "cores": nthreads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "element-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def adjoint_timing(device, ncycles=500, checkpoint=50, reps=3):
    """Wall time of or_ecycle_adjoint (forward sweep, recompute, reverse) on the
    C5 plate, and of the same cycles forward only, both FP64 and synchronous."""
    from openradioss_b200 import abi, adjoint, decks
    from openradioss_b200.ecycle import ECycle
    deck = decks.c5_adjoint_plate(ncycles=ncycles)
    deck["dtmx"] = 1.4e-7                     # dt below every element's: the dt sequence is fixed
    node = adjoint.centre_node(deck)
    h = ECycle(deck, precision=abi.OR_PREC_FP64, device=device, graph=1)
    h.adjoint(ncycles, node=node, w_disp=1.0, w_plastic=1.0, checkpoint=checkpoint)   # allocation, warm-up
    ta, tf = [], []
    for _ in range(reps):
        h.reset()
        t0 = time.perf_counter()
        h.adjoint(ncycles, node=node, w_disp=1.0, w_plastic=1.0, checkpoint=checkpoint)
        ta.append(time.perf_counter() - t0)
        h.reset()
        t0 = time.perf_counter()
        h.step(ncycles)
        tf.append(time.perf_counter() - t0)
    nel = decks.num_elements(deck)
    a, f = min(ta), min(tf)
    return {"workload": f"C5 plate 200x200, per-element A and thickness, {ncycles} cycles, FP64, "
                        f"checkpoint every {checkpoint} cycles, responses w(T) + plastic work",
            "adjoint_ms": a * 1e3, "forward_ms": f * 1e3, "adjoint_over_forward": a / f,
            "element_cycles_per_s_adjoint": nel * ncycles / a}


# ---------------------------------------------------------------------------
def kernel_roofline(h, deck, cycles, workload, s=4, step_ms=None):
    """Per-kernel device times (each phase kernel launched back to back from a graph
    on the state a full run leaves, CUDA events on the handle's stream) and the
    roofline of the dominant one.  When the handle steps with the persistent shell
    cycle, that kernel is the dominant one: one launch per step of ``cycles``
    cycles, timed live (``step_ms``), and its algorithmic bytes are those of the
    work it does, the per-cycle element and node bytes times the cycles (the
    state it keeps on chip is not re-read, so its DRAM traffic is far below
    them).  Resets the handle."""
    from openradioss_b200 import roofline
    h.reset()
    h.step(cycles)
    kt = h.kernel_times(reps=64)            # microseconds per launch; resets the handle
    eb_hex = sum(g["ixs"].shape[0] * roofline.hex_bytes(s, g["mat"]["law"]) for p in deck["parts"] for g in p["hex"])
    eb_shell = sum(g["ixc"].shape[0] * roofline.shell_bytes(s, g["prop"]["npt"])
                   for p in deck["parts"] for g in p["shell"])
    eb, nb, _ = roofline.deck_bytes(deck, s)
    peak, peak_src = roofline.measured_peak()
    kern = {"hex": (kt["hex"] * 1e-3, eb_hex), "shell": (kt["shell"] * 1e-3, eb_shell), "node": (kt["node"] * 1e-3, nb)}
    dom = max(kern, key=lambda k: kern[k][0])
    dom_ms, dom_bytes = kern[dom]
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(workload, {}).get(f"{dom}_split")
        except (OSError, ValueError):
            traffic = None
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9 if dom_ms > 0 else 0.0
    per_kernel = {k: {"us_per_launch": v[0] * 1e3, "algorithmic_bytes": v[1],
                      "frac": (v[1] / (v[0] * 1e-3) / 1e9 / peak) if v[0] > 0 else None}
                  for k, v in kern.items()}
    roof = {"bound": "hbm", "kernel": f"{dom}_patch_kernel" if dom != "node" else "node_kernel",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "algorithmic_bytes_per_launch": dom_bytes,
            "avg_launch_ms": dom_ms, "peak_source": peak_src}
    if h.persistent_info()[0] and step_ms:
        pb = (eb + nb) * cycles
        ptraffic = None
        if os.path.exists(tpath):     # staged once per launch: the DRAM bytes do not grow with its cycles
            try:
                ptraffic = json.load(open(tpath)).get(workload, {}).get("persistent_split_per_launch")
            except (OSError, ValueError):
                ptraffic = None
        pa = pb / (step_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": "shell_persistent_kernel", "achieved": pa, "peak": peak, "unit": "GB/s",
                "frac": pa / peak, "traffic": ptraffic, "algorithmic_bytes_per_launch": pb, "avg_launch_ms": step_ms,
                "cycles_per_launch": cycles, "peak_source": peak_src,
                "note": "per-phase kernels below are timed alone for comparison; the timed steps ran this kernel"}
    return roof, per_kernel, eb + nb, peak


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return reference_arm(args, rank, world)
    if args.eager_cycles:
        return eager_profile(args)
    if args.persistent_cycles:
        return persistent_profile(args)
    if args.adjoint_cycles:
        import torch
        from openradioss_b200 import build
        build.build()
        torch.cuda.set_device(0)
        print(json.dumps(adjoint_timing(0, ncycles=args.adjoint_cycles, reps=1)))
        return None

    import torch
    import torch.distributed as dist
    from datetime import timedelta
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    from openradioss_b200 import abi, build, decks, shard
    from openradioss_b200.ecycle import ECycle
    build.build()
    full = make_deck(args.workload)
    sharded = world > 1 and len(full["parts"]) > 1
    deck = shard.rank_deck(full, rank, world) if sharded else full
    cycles = args.cycles or WORKLOADS[args.workload][1]
    nel = decks.num_elements(deck)
    # element-updates of one step over all ranks
    nel_job = decks.num_elements(full) if sharded else world * nel

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(*vals):
        tt = torch.tensor(list(vals), dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return [float(v) for v in tt]

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed_runs(h, ncyc, nsteps, nwarm):
        s = torch.cuda.ExternalStream(h.stream())
        ms, launches = [], 0
        for k in range(nwarm + nsteps):
            h.reset()
            flush.fill_(float(k))
            torch.cuda.synchronize()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            h.step(ncyc)
            e1.record(s)
            torch.cuda.synchronize()
            if k >= nwarm:
                ms.append(e0.elapsed_time(e1))
                launches += h.launch_count()
        return ms, launches

    # ---- tile shapes from the autotuner (timed on this GPU, cached) ----
    from openradioss_b200 import autotune
    bh_s, bs_s, pe_s, tune_s = autotune.tune(deck, abi.OR_PREC_SPLIT, device=local)
    bh_d, bs_d, pe_d, tune_d = autotune.tune(deck, abi.OR_PREC_FP64, device=local)

    # ---- split form (the headline) ----
    hs = ECycle(deck, precision=abi.OR_PREC_SPLIT, device=local, graph=1, block_hex=bh_s, block_shell=bs_s,
                persistent=pe_s)
    persistent_on = bool(hs.persistent_info()[0])
    timed_runs(hs, cycles, 0, 1)              # graph capture + first-touch outside timing
    sampler = ClockSampler(local)
    sampler.start()
    ms_split, launches = timed_runs(hs, cycles, args.steps, args.warmup)
    clocks = sampler.stop()
    out_split = outputs(hs)

    # ---- plain FP64 form ----
    hd = ECycle(deck, precision=abi.OR_PREC_FP64, device=local, graph=1, block_hex=bh_d, block_shell=bs_d,
                persistent=pe_d)
    timed_runs(hd, cycles, 0, 1)
    ms_fp64, _ = timed_runs(hd, cycles, max(2, args.steps // 2), 1)
    out_fp64 = outputs(hd)

    t_split, t_fp64 = max_over_ranks(sum(ms_split) / len(ms_split), sum(ms_fp64) / len(ms_fp64))
    value = nel_job * cycles / (t_split * 1e-3)
    value_fp64 = nel_job * cycles / (t_fp64 * 1e-3)

    # ---- split error per output, against the FP64 run's own floor (1e-12 perturbed
    # coordinates), at the full cycle count and after 1000 cycles ----
    accuracy = {"cycles": cycles, "split_vs_fp64": output_errors(out_split, out_fp64),
                "fp64_floor": output_errors(perturbed_run(hd, deck, cycles), out_fp64),
                "floor_input_perturbation": 1e-12}
    if cycles > 1000:
        hd.reset()
        hd.step(1000)
        f1000 = outputs(hd)
        hs.reset()
        hs.step(1000)
        accuracy["at_1000_cycles"] = {"split_vs_fp64": output_errors(outputs(hs), f1000),
                                      "fp64_floor": output_errors(perturbed_run(hd, deck, 1000), f1000)}
    hd.close()
    split_err = accuracy["split_vs_fp64"]["D"]

    roof, per_kernel, cyc_bytes, peak = kernel_roofline(hs, deck, cycles, args.workload, step_ms=t_split)
    cyc_achieved = cyc_bytes * cycles / (t_split * 1e-3) / 1e9

    # ---- end to end through the C-ABI with host buffers ----
    e2e_value, h2d, d2h, e2e_same = e2e_rate(hs, deck, cycles, args.warmup, max(2, args.steps // 2), flush, barrier,
                                             max_over_ranks, out_split["D"], nel_job)
    hs.close()

    # ---- C5: the adjoint on the sensitivity plate (FP64), next to its forward ----
    adj = None
    if world == 1 and args.workload == "shell_plate":
        adj = adjoint_timing(local)

    # ---- further workloads recorded beside the headline (one GPU) ----
    subs = {}
    if world == 1:
        for name in [w for w in args.sub_workloads.split(",") if w and w != args.workload]:
            subs[name] = sub_record(name, local, args.sub_steps, args.sub_tile, timed_runs, flush, barrier,
                                    max_over_ranks)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(deck, cycles, args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": "element-updates/s", "value": value, "unit": "element-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_split, "higher_is_better": True,
            "scaling": "strong" if sharded else "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded numpy decks with the workload's shapes)",
            "config": workload_config(args.workload, full, cycles, world, sharded),
            "precision": "split: FP32 element/material math, FP64 X/D/volumes/energies",
            "tuning": {"cuda_graph_cycles": 32, "tile_hex": bh_s, "tile_shell": bs_s,
                       "persistent_cycle": persistent_on,
                       "autotune_ms_per_cycle": {"split": tune_s, "fp64": tune_d},
                       "autotune_keys": "tile (hAsB: hexa tile A, shell tile B), p = persistent shell cycle"},
            "fp64": {"value": value_fp64, "ms_per_step": t_fp64, "dtype": "f64", "tile_hex": bh_d, "tile_shell": bs_d,
                     "persistent_cycle": pe_d == 0},
            "split_over_fp64": value / value_fp64,
            "split_rel_disp_error_vs_fp64": split_err,
            "accuracy": accuracy,
            "roofline": roof,
            "cycle_roofline": {"algorithmic_bytes_per_cycle": cyc_bytes,
                               "bytes_per_element_update": cyc_bytes / nel,
                               "achieved": cyc_achieved, "frac": cyc_achieved / peak,
                               "kernels": per_kernel},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "element-updates/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "same_result_as_device_run": e2e_same},
            "clocks": clocks,
            "gpu_launches": launches,
        }
        if adj is not None:
            line["adjoint"] = adj
        if subs:
            line["workloads"] = subs
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def e2e_rate(hs, deck, cycles, nwarm, nsteps, flush, barrier, max_over_ranks, d_ref, nel_job):
    """The metric end to end through the C-ABI with host buffers: per step, upload
    the initial X, D, V, VR from pinned host buffers, run all cycles, download X, D,
    V, VR into separate pinned host buffers.  Returns (rate, h2d bytes, d2h bytes,
    whether the downloaded D equals the device run's)."""
    import ctypes as C
    import torch
    dptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    pinned = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float64)).pin_memory().numpy()
    host_in, host_out = [], []
    for p in deck["parts"]:
        n = p["x"].shape[0]
        host_in.append({"x": pinned(p["x"]), "d": pinned(np.zeros((n, 3))), "v": pinned(p["v"]),
                        "vr": pinned(p["vr"])})
        host_out.append({k: pinned(np.zeros((n, 3))) for k in ("x", "d", "v", "vr")})
    h2d = sum(sum(a.nbytes for a in hb.values()) for hb in host_in)
    d2h = sum(sum(a.nbytes for a in hb.values()) for hb in host_out)
    e2e_t = []
    for k in range(nwarm + nsteps):
        hs.reset()
        flush.fill_(float(k))
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        for pi, hb in enumerate(host_in):
            hs._call("set_nodes", pi, *(dptr(hb[q]) for q in ("x", "d", "v", "vr")))
        hs.step(cycles)
        for pi, hb in enumerate(host_out):
            hs._call("get_nodes", pi, *(dptr(hb[q]) for q in ("x", "d", "v", "vr")))
        t1 = time.perf_counter()
        if k >= nwarm:
            e2e_t.append(t1 - t0)
    d_e2e = np.concatenate([hb["d"].ravel() for hb in host_out])
    same = bool(np.array_equal(d_e2e, d_ref))
    (te,) = max_over_ranks(sum(e2e_t) / len(e2e_t))
    return nel_job * cycles / te, h2d, d2h, same


def sub_record(name, local, steps, tile, timed_runs, flush, barrier, max_over_ranks):
    """Split and FP64 rates, per-kernel roofline and split error per output of a
    further workload on this GPU (fixed tile, a few steps, L2 flushed between)."""
    from openradioss_b200 import abi, decks
    from openradioss_b200.ecycle import ECycle
    deck = make_deck(name)
    cycles = WORKLOADS[name][1]
    nel = decks.num_elements(deck)
    hs = ECycle(deck, precision=abi.OR_PREC_SPLIT, device=local, graph=1, block_hex=tile, block_shell=tile)
    sampler = ClockSampler(local)
    sampler.start()
    ms_s, launches = timed_runs(hs, cycles, steps, 3)
    clocks = sampler.stop()
    out_s = outputs(hs)
    hd = ECycle(deck, precision=abi.OR_PREC_FP64, device=local, graph=1, block_hex=tile, block_shell=tile)
    ms_d, _ = timed_runs(hd, cycles, max(2, steps - 1), 1)
    out_d = outputs(hd)
    hd.close()
    t_s, t_d = sum(ms_s) / len(ms_s), sum(ms_d) / len(ms_d)
    e2e_value, h2d, d2h, same = e2e_rate(hs, deck, cycles, 1, 2, flush, barrier, max_over_ranks, out_s["D"], nel)
    roof, per_kernel, cyc_bytes, peak = kernel_roofline(hs, deck, cycles, name)
    hs.close()
    return {"config": workload_config(name, deck, cycles, 1, False), "steps": steps, "warmup": 3,
            "value": nel * cycles / (t_s * 1e-3), "ms_per_step": t_s,
            "fp64": {"value": nel * cycles / (t_d * 1e-3), "ms_per_step": t_d},
            "split_over_fp64": t_d / t_s, "tile": tile,
            "split_vs_fp64": output_errors(out_s, out_d),
            "roofline": roof,
            "cycle_roofline": {"algorithmic_bytes_per_cycle": cyc_bytes, "bytes_per_element_update": cyc_bytes / nel,
                               "achieved": cyc_bytes * cycles / (t_s * 1e-3) / 1e9,
                               "frac": cyc_bytes * cycles / (t_s * 1e-3) / 1e9 / peak, "kernels": per_kernel},
            "e2e": {"value": e2e_value, "unit": "element-updates/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "same_result_as_device_run": same},
            "clocks": clocks, "gpu_launches": launches}


if __name__ == "__main__":
    main()
