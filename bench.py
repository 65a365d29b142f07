#!/usr/bin/env python
"""Benchmark of the split-operator propagation step on B200: 6D grid-point-steps/s, mixed vs FP64.

Workload: config 3 = the config-2 grid (nZ 128, nR 48, nX = nY 16, ntheta 16, nphi 32, n_rot 256,
nZSpecular 512, dt 2, 5 time steps per analysis step; 8.05e8 6D points) in the mixed form, with the
same workload in the FP64 form beside it. Seeded synthetic tables with the configuration's shapes
(spo_b200.workload); the step does the same work whatever the values.

One bench step = one analysis step (PropagationBackend::propagate_analysis_step: 5 time steps, i.e.
6 kinetic sub-steps and 5 potential steps). value = 6D points * time steps / device time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

--impl reference times the reference's own CPU implementation of the step (oracle/_ref, the
reference compiled from its sources) on the host cores, on a bounded sample of the same workload.
Multi-GPU runs (torchrun) are independent replicas (one wave packet per GPU, as the reference's
ensembles are run): no data-path collective, a barrier and a max-over-ranks of the device time.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cpp-spo-dvr_b200"))

METRIC = "6D SPO grid-point-steps/s on 1 B200, mixed vs FP64 at |ΔP_react|≤1e-6"
UNIT = "grid-point-steps/s"
CONFIG2_INPUT = os.path.join(ROOT, "tests", "golden", "inputs", "config2_dz.json")
REF_TOOL = os.path.join(ROOT, "oracle", "_ref", "spo_ref_tool")
FALLBACK_HBM_GBS = 6650.0


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        self.proc.wait()
        rows = [r.split(", ") for r in open(self.path).read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        for r in rows:
            for name, val in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"], r[5:9]):
                if val.strip() == "Active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(rows[0][2]),
                "reasons": sorted(reasons), "samples": len(rows)}


def step_bytes(case, s: int) -> float:
    """Algorithmic bytes of one time step: s (4 N_fbr + N_tab + 4 N_spec), N_fbr = nZ nR nX nY n_rot,
    N_tab = nzpot nR n_rep ntheta nphi, N_spec = nZsp nR (psi read and written once for T and once for
    V, the exp(-iV dt) table read once, chi likewise)."""
    n_fbr = case.nz * case.nr * case.nx * case.ny * case.n_rot
    n_tab = case.nz_potential * case.nr * case.n_rep * case.n_theta * case.n_phi
    n_spec = case.nz_specular * case.nr
    return s * (4.0 * n_fbr + n_tab + 4.0 * n_spec)


def measure(case, precision, steps, warmup, device, world):
    import numpy as np
    import torch

    from spo_b200 import B200Backend

    be = B200Backend(case, precision=precision, device=device)
    stream = torch.cuda.Stream(device=device)
    be.set_stream(stream.cuda_stream)
    # The initial wave packet: an empty scattering grid and the incoming packet on the specular grid.
    psi0 = torch.zeros(case.psi_shape + (2,), dtype=torch.float64, pin_memory=True).numpy().view(np.complex128)[..., 0]
    chi0 = np.ascontiguousarray(case.a["chi_initial"].reshape(case.chi_shape))
    be.read_wave_packet(psi0, chi0)
    for _ in range(warmup):
        be.propagate_analysis_step()

    def barrier():
        torch.cuda.synchronize(device)
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(device)

    # Device throughput: K analysis steps with the state resident in HBM.
    barrier()
    clocks = ClockSampler(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        be.propagate_analysis_step()
    e1.record(stream)
    torch.cuda.synchronize(device)
    clock = clocks.stop()
    ms = e0.elapsed_time(e1)
    launches = be.last_launch_count() * steps
    barrier()

    # Per-kernel CUDA-event times over the same K steps (a second pass, events around every launch).
    be.profile(True)
    for _ in range(steps):
        be.propagate_analysis_step()
    records = be.profile_records()
    be.profile(False)
    barrier()

    # End to end through the C ABI with host buffers: the state uploaded from pinned host memory, then
    # per analysis step the readbacks the reference's time loop makes (specular wave and the BK plane,
    # src/propagation/propagation.cpp:81-84).
    chi = torch.empty(case.chi_shape + (2,), dtype=torch.float64, pin_memory=True).numpy().view(np.complex128)[..., 0]
    plane = torch.empty((case.nr, case.nx, case.ny, case.n_rot, 2), dtype=torch.float64,
                        pin_memory=True).numpy().view(np.complex128)[..., 0]
    iz_a = int(case.m.get("iz_analysis", case.nz // 2))
    e0.record(stream)
    be.read_wave_packet(psi0, chi0)
    for _ in range(steps):
        be.propagate_analysis_step()
        be.specular(out=chi)
        be.z_plane(iz_a, out=plane)
    e1.record(stream)
    torch.cuda.synchronize(device)
    e2e_ms = e0.elapsed_time(e1)
    h2d = (psi0.nbytes + chi0.nbytes) / steps
    d2h = chi.nbytes + plane.nbytes
    kernels = be.describe()
    be.close()
    return {"ms": ms, "launches": launches, "records": records, "clocks": clock, "e2e_ms": e2e_ms,
            "h2d": h2d, "d2h": d2h, "kernels": kernels}


def reduce_max(x, world, device):
    """The maximum of x over the ranks (every rank takes part; NCCL on the GPUs, any other backend on
    the host)."""
    if world == 1:
        return x
    import torch
    on_gpu = torch.distributed.get_backend() == "nccl"
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{device}" if on_gpu else "cpu")
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_rate(points, time_steps, ms_max, world):
    """Whole-job grid-point-steps/s of `world` replicas, each advancing `points` grid points by
    `time_steps`, timed by the slowest rank (ms_max)."""
    return world * points * time_steps / (ms_max / 1000.0)


def cpu_sample_input(nx: int):
    """The config-2 reference input with nX = nY = nx (a bounded sample for the CPU timings)."""
    cfg = json.load(open(CONFIG2_INPUT))
    cfg.update({"nX": nx, "nY": nx, "Title": f"config 2 sample, nX = nY = {nx}"})
    path = tempfile.mktemp(suffix=".json")
    json.dump(cfg, open(path, "w"))
    return path


def host_cpu():
    """The host's CPU model, logical CPUs and physical cores (from /proc/cpuinfo)."""
    model, cores = None, set()
    phys = core = None
    try:
        for line in open("/proc/cpuinfo"):
            key, _, val = line.partition(":")
            key, val = key.strip(), val.strip()
            if key == "model name" and model is None:
                model = val
            elif key == "physical id":
                phys = val
            elif key == "core id":
                core = val
            elif not key and phys is not None and core is not None:
                cores.add((phys, core))
                phys = core = None
        if phys is not None and core is not None:
            cores.add((phys, core))
    except OSError:
        pass
    logical = os.cpu_count() or 1
    return {"model": model, "logical_cpus": logical, "physical_cores": len(cores) or logical}


def reference_timing(analysis_steps: int, warmup: int, nx: int = 4):
    """The reference CPU path (oracle/_ref) on one thread per physical core: JSON of spo_ref_tool time."""
    if not os.path.exists(REF_TOOL):
        return None, f"{REF_TOOL} is not built"
    path = cpu_sample_input(nx)
    env = dict(os.environ)
    cpu = host_cpu()
    env.setdefault("OMP_NUM_THREADS", str(cpu["physical_cores"]))
    try:
        r = subprocess.run([REF_TOOL, "time", path, "--analysis-steps", str(analysis_steps), "--warmup", str(warmup)],
                           capture_output=True, text=True, env=env, timeout=1800)
    finally:
        os.unlink(path)
    if r.returncode != 0:
        return None, r.stderr.strip()[-300:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    grid = "the full grid" if nx == 16 else f"nX = nY = {nx} ({nx * nx}/256 of the points)"
    out["sample"] = (f"config-2 reference input (Dai-Light PES, HD, JMax = MJMax = 15) on {grid}: "
                     f"{int(out['n_points'])} 6D points, {analysis_steps} analysis steps of 5 time steps after "
                     f"{warmup} warm-up; reference CpuBackend compiled from its sources (FFT: the project's FP64 "
                     f"substitute, FFTW being absent); {out['threads']} OpenMP threads on "
                     f"{cpu['physical_cores']} physical cores ({cpu['logical_cpus']} logical) of {cpu['model']}")
    out["cpu"] = cpu
    return out, None


PRECISION_RECORD = os.path.join(ROOT, "tests", "golden", "precision_config3.json")


def precision_record():
    """The committed record of the precision form's error on this workload (tests/golden/precision_config3.py:
    configuration 2 and 3 through the reference program with the B200 backend, 20000 steps, 81 energies)."""
    try:
        with open(PRECISION_RECORD) as f:
            r = json.load(f)
    except (OSError, ValueError):
        return None
    return {"dP_reaction": r["dp_reaction_max"], "dP_state_max": r["dp_state_max"],
            "bar": 1e-6, "time_steps": r["time_steps"], "energies": r["energies"],
            "open_channels": r["open_channels"],
            "source": "tests/golden/precision_config3.json: configuration 2 (FP64) and 3 (mixed) through the "
                      "reference program with the B200 backend (oracle/_ref/spodvr_b200), 20000 time steps"}


def run_reference(args, rank):
    if rank != 0:
        return
    out, err = reference_timing(args.steps, args.warmup)
    if out is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return
    v = out["grid_point_steps_per_s"]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * out["seconds"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "the reference's own set-up of the config-2 input (Dai-Light PES), bounded sample",
            "config": {"workload": out["sample"], "step": "one analysis step = 5 time steps"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": out["threads"], "kind": "reference",
                             "sample": out["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# Shapes of the ensemble workload, from the configuration-4 ranges: Z 96-128, r 40-48, x = y 12-16,
# theta 12-16 and phi 24-32 (heteronuclear JMax = MJMax 11-15), specular Z grid 512.
ENSEMBLE_SHAPES = [
    {"nz": 96, "nr": 40, "nx": 12, "ny": 12, "j_max": 11, "mj_max": 11, "nz_potential": 63},
    {"nz": 112, "nr": 48, "nx": 12, "ny": 12, "j_max": 13, "mj_max": 13, "nz_potential": 74},
    {"nz": 128, "nr": 40, "nx": 16, "ny": 16, "j_max": 11, "mj_max": 11, "nz_potential": 84},
    {"nz": 128, "nr": 48, "nx": 16, "ny": 16, "j_max": 15, "mj_max": 15, "nz_potential": 84},
]


# DRAM bytes per algorithmic byte of the mixed-form potential kernel (potential5), from one ncu capture of
# the small case (nX = nY = 8; profiles/potential5_small_nx8.md): dram__bytes_read.sum + dram__bytes_write.sum
# = 1.852 + 0.507 GB against 2.378 GB algorithmic (interaction-region psi read and written once, the exp(i A)
# table read once with its 2-byte modulus corrections). The traffic grows with the columns processed, so the
# ratio carries over to configuration 3.
POTENTIAL_DRAM_PER_ALGORITHMIC = (1.852132e9 + 0.506512e9) / 2.378170368e9


def run_ensemble(args):
    """32 mixed-form wave packets of uneven grids (8 of each shape), one CUDA graph launch per analysis
    step (spo_ensemble_*), against the same members stepped one after another."""
    import numpy as np
    import torch

    from spo_b200 import B200Backend, Ensemble, workload

    torch.cuda.set_device(0)
    members, points = [], 0
    for shape in ENSEMBLE_SHAPES:
        case = workload.config_case(shape)
        chi0 = np.ascontiguousarray(case.a["chi_initial"].reshape(case.chi_shape))
        for _ in range(8):
            be = B200Backend(case, precision="mixed")
            be.read_wave_packet(None, chi0)
            members.append(be)
            points += case.n_points
        case.a.clear()  # the descriptor's host tables are only read by spo_create
    steps_per_analysis = members[0].case.steps_per_analysis
    stream = torch.cuda.current_stream()

    def timed(fn, k):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    with Ensemble(members) as ens:
        for _ in range(args.warmup):
            ens.propagate_analysis_step()
        # the ensemble step synchronises its own stream, so wall-clock events on the current stream bracket it
        ms_graph = timed(ens.propagate_analysis_step, args.steps)
        launches = ens.launch_count()
    ms_seq = timed(lambda: [m.propagate_analysis_step() for m in members], args.steps)
    for m in members:
        m.close()
    rate = points * steps_per_analysis * args.steps / (ms_graph / 1000.0)
    print(json.dumps({
        "metric": METRIC + " (ensemble)", "value": rate, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_graph / args.steps, "higher_is_better": True, "dtype": "c64",
        "data": "synthetic", "config": {"workload": "32 mixed-form packets of the configuration-4 size ranges (8 each "
                                                    "of 4 shapes), one graph launch per analysis step",
                                        "shapes": ENSEMBLE_SHAPES, "points": points},
        "one_after_another": {"value": points * steps_per_analysis * args.steps / (ms_seq / 1000.0),
                              "ms_per_step": ms_seq / args.steps},
        "gpu_launches": launches * args.steps,
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="config3", choices=["config3", "small", "ensemble"],
                    help="small: the config-2 tables on nX = nY = 8 (psi 0.8 GB mixed, above L2), for profiler captures")
    args = ap.parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload == "ensemble":
        if rank == 0:
            run_ensemble(args)
        return

    import torch

    from spo_b200 import workload

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                             device_id=torch.device(f"cuda:{local}"))
    case = workload.config_case({"nx": 8, "ny": 8} if args.workload == "small" else None)
    res = {}
    for precision in ("mixed", "fp64"):
        res[precision] = measure(case, precision, args.steps, args.warmup, local, world)
    time_steps = args.steps * case.steps_per_analysis
    points = float(case.n_points)
    out = {}
    for precision, r in res.items():
        ms = reduce_max(r["ms"], world, local)
        e2e_ms = reduce_max(r["e2e_ms"], world, local)
        out[precision] = {"ms": ms, "value": job_rate(points, time_steps, ms, world),
                          "e2e": job_rate(points, time_steps, e2e_ms, world)}
    if world > 1:
        torch.distributed.barrier()
    if rank == 0:
        peak, peak_kind = hbm_peak()
        m = res["mixed"]
        top = max(m["records"], key=lambda r: r["ms"])
        avg_ms = top["ms"] / top["launches"]
        achieved = top["bytes_per_launch"] / (avg_ms / 1000.0) / 1e9
        b_step = step_bytes(case, 8)
        step_gbs = b_step * time_steps / (out["mixed"]["ms"] / 1000.0) / 1e9 / world
        total_kernel_ms = sum(r["ms"] for r in m["records"])
        cpu = None
        if world == 1 and not args.no_cpu_baseline and args.workload == "config3":
            ref, err = reference_timing(1, 1)
            if ref is not None:
                cpu = {"value": ref["grid_point_steps_per_s"], "unit": UNIT, "cores": ref["threads"],
                       "kind": "reference", "sample": ref["sample"]}
            else:
                cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference", "sample": err}
        line = {
            "metric": METRIC, "value": out["mixed"]["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": out["mixed"]["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": {"workload": ("config 3: config-2 grid nZ 128, nR 48, nX = nY 16, ntheta 16, nphi 32 "
                                    "(JMax = MJMax = 15, n_rot 256), nZSpecular 512, nzpot 84, dt 2, mixed form "
                                    "(complex64 psi, FP32 FFTs and factors, exp(-iV dt) formed in FP64)")
                       if args.workload == "config3" else "small: config-2 tables on nX = nY = 8 (profiling)",
                       "points": int(points), "step": "one analysis step = 5 time steps",
                       "time_steps_per_step": case.steps_per_analysis,
                       "l2": "inputs larger than L2 (psi 3.2 GB mixed / 6.4 GB FP64, table 2.6 / 5.3 GB)",
                       "parallelism": f"replicas x{world}",
                       "kernels_mixed": m["kernels"], "kernels_fp64": res["fp64"]["kernels"]},
            "fp64": {"value": out["fp64"]["value"], "ms_per_step": out["fp64"]["ms"] / args.steps,
                     "e2e": out["fp64"]["e2e"],
                     "kernels": [{"name": r["name"], "launches": r["launches"],
                                  "avg_ms": round(r["ms"] / r["launches"], 5)} for r in res["fp64"]["records"]]},
            "mixed_over_fp64": out["mixed"]["value"] / out["fp64"]["value"],
            "roofline": {"bound": "hbm", "kernel": top["name"], "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": top["bytes_per_launch"] * POTENTIAL_DRAM_PER_ALGORITHMIC
                         if top["name"] == "potential" else None,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one potential5 launch "
                                           "on the small case (nX = nY = 8: 2.359 GB for 2.378 GB algorithmic), "
                                           "scaled to this launch by the columns processed",
                         "bytes_per_launch": top["bytes_per_launch"], "avg_launch_ms": avg_ms,
                         "share_of_kernel_time": top["ms"] / total_kernel_ms},
            "step_roofline": {"bytes_per_time_step": b_step, "achieved": step_gbs, "peak": peak, "unit": "GB/s",
                              "frac": step_gbs / peak, "peak_kind": peak_kind},
            "kernels": [{"name": r["name"], "launches": r["launches"], "ms": round(r["ms"], 4),
                         "avg_ms": round(r["ms"] / r["launches"], 5),
                         "gbs": round(r["bytes_per_launch"] / (r["ms"] / r["launches"] / 1000.0) / 1e9, 1)}
                        for r in m["records"]],
            "cpu_baseline": cpu,
            "e2e": {"value": out["mixed"]["e2e"], "unit": UNIT, "h2d_bytes_per_step": int(m["h2d"]),
                    "d2h_bytes_per_step": int(m["d2h"])},
            "gpu_launches": m["launches"],
            "clocks": m["clocks"],
        }
        prec = precision_record()
        if prec is not None and args.workload == "config3":
            line["dP_reaction"] = prec["dP_reaction"]
            line["dP_state_max"] = prec["dP_state_max"]
            line["precision"] = prec
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
