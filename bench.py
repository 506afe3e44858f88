"""Benchmark: steps/s of the stable-fluids step at 256^3 on B200.

Workload (one "step" = one stable_fluids_step_cuda call = one step-graph
launch): the seeded 256^3 buoyant plume -- dt 0.1, viscosity 1e-4, density
diffusion 1e-5, 20 diffusion and 80 pressure iterations, Stam walls, two
Gaussian sources (radius 8) with upward forces U[1, 10] (seed 1) -- run with
the reference-compatible red-black Gauss-Seidel scheme, whose results match
the reference backend's. The working set (~1.2 GB) is far larger than L2, so
no flush is needed between steps.

  value : whole-job steps/s with inputs resident on the device, CUDA events on
          the simulation stream, max over ranks.
  e2e   : the same steps through the public C ABI with host buffers: every
          step uploads the force field from pinned host memory
          (stable_fluids_update_vector_field_cuda with host pointers) and
          reads the density field back to pinned host memory.
  roofline : the dominant kernel family (the pressure solve), timed with
          CUDA events on the context stream through the stage hook.
  cpu_baseline : the reference step sequence transcribed to C++/OpenMP
          (oracle/, FP32), on a bounded sample of the same workload.

--impl reference runs the reference's own implementation of the path -- its
CUDA backend compiled unmodified from backend-cuda.cu (oracle/_ref) -- on the
same scene through the same C ABI. The reference has no CPU implementation.

Multi-GPU (torchrun, N>1): the step does not shard; each rank runs its own
replica of the workload ("scaling": "weak").
"""

from __future__ import annotations

import argparse
import importlib
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "steps/s at 256³: learned-warm-start vs plain Jacobi at equal ‖∇·u‖ residual"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", choices=("b200", "reference"), default="b200")
    p.add_argument("--size", type=int, default=256)
    p.add_argument("--scheme", choices=("rbgs", "jacobi"), default="rbgs")
    p.add_argument("--iterations-per-pass", type=int, default=0)
    p.add_argument("--e2e-steps", type=int, default=30)
    p.add_argument("--cpu-steps", type=int, default=1)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-clocks", action="store_true")
    p.add_argument("--equal-residual", default="rbgs-zero,rbgs-previous,jacobi-previous", help="solver variants timed at equal rel_res (empty: skip)")
    p.add_argument("--residual-tolerance", type=float, default=1e-3)
    p.add_argument("--residual-steps", type=int, default=3)
    p.add_argument("--residual-cap", type=int, default=20000)
    a = p.parse_args()
    a.warmup = max(a.warmup, 3)
    return a


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device_index: int, enabled: bool):
        self.enabled = enabled
        self.device_index = device_index
        self.proc = None

    def __enter__(self):
        if self.enabled:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            try:
                self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
            except OSError:
                self.proc = None
            time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None:
            return None
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
                except ValueError:
                    continue
        os.unlink(self.file.name)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for _, _, r in rows for k in range(4) if r[k].lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def time_steps(sim, steps, world):
    import torch

    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    start.record(sim.stream)
    sim.step(steps)
    end.record(sim.stream)
    torch.cuda.synchronize()
    barrier(world)
    return start.elapsed_time(end) / 1000.0


def time_stage(sim, stage, repeats):
    """Average duration of one kernel of a stage, CUDA events on the context
    stream (the stage is enqueued directly on it)."""
    import torch

    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    sim.enqueue_stage(stage)  # warm
    torch.cuda.synchronize()
    launches = 0
    start.record(sim.stream)
    for _ in range(repeats):
        launches += sim.enqueue_stage(stage)
    end.record(sim.stream)
    torch.cuda.synchronize()
    return start.elapsed_time(end) / 1000.0, launches


def e2e_run(sf, sim, scene, steps):
    """Steps through the public ABI with host buffers: per step the force
    field goes up from pinned host memory and the density comes back."""
    import numpy as np
    import torch

    n = sim.cells
    host_force = [torch.from_numpy(np.ascontiguousarray(f, dtype=np.float32)).pin_memory() for f in scene.force]
    host_rho = torch.empty(n, dtype=torch.float32).pin_memory()
    h = sim.scalar_handles[0]
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(sim.stream)
    for _ in range(steps):
        rc = sim.lib.stable_fluids_update_vector_field_cuda(sim.ctx, 1, host_force[0].data_ptr(), host_force[1].data_ptr(), host_force[2].data_ptr())
        if rc != 0:
            raise RuntimeError(f"update_vector_field with host pointers failed ({rc})")
        sim.step(1)
        rho = sim.view(sf.VIEW_SCALAR_FIELD_DATA, h)
        with torch.cuda.stream(sim.stream):
            host_rho.copy_(rho.reshape(-1), non_blocking=True)
    end.record(sim.stream)
    torch.cuda.synchronize()
    t = start.elapsed_time(end) / 1000.0
    return t, 3 * n * 4, n * 4


def equal_residual(sf, scene, variants, tol, steps, cap, warmup):
    """Steps/s of the plume when the pressure is iterated until the FP64
    relative Poisson residual is <= tol (inside the step graph), for solver
    variants scheme-warmstart; reports the iterations each step needed."""
    import torch

    out = {}
    for v in variants:
        scheme, warm = v.split("-")
        opts = sf.default_options()
        opts.scheme = sf.SCHEME_JACOBI if scheme == "jacobi" else sf.SCHEME_RBGS
        opts.warm_start = {"zero": sf.WARM_START_ZERO, "previous": sf.WARM_START_PREVIOUS}[warm]
        opts.residual_tolerance = tol
        opts.residual_check_interval = 16
        opts.max_pressure_iterations = cap
        sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, options=opts)
        sf.scenes.apply_inputs(sim, scene, 0)
        sim.step(warmup)
        torch.cuda.synchronize()
        its, res, total = [], [], 0.0
        for _ in range(steps):
            start = torch.cuda.Event(enable_timing=True)
            end = torch.cuda.Event(enable_timing=True)
            start.record(sim.stream)
            sim.step(1)
            end.record(sim.stream)
            st = sim.stats()
            total += start.elapsed_time(end) / 1000.0
            its.append(st.pressure_iterations)
            res.append(st.rel_residual)
        sim.close()
        out[v] = {"steps_per_s": steps / total, "pressure_iterations": its, "rel_residual": res, "hit_cap": any(r > tol for r in res)}
    return out


def cpu_baseline(sf, scene, steps):
    from oracle import oracle as orc

    threads = orc.set_threads(os.cpu_count() or 1)
    o = orc.Oracle(scene.config, scene.scalars, scene.vectors, precision=32)
    sf.scenes.apply_inputs(o, scene, 0)
    t0 = time.perf_counter()
    o.step(steps)
    t = time.perf_counter() - t0
    o.close()
    n = scene.config.nx
    return {"value": steps / t, "unit": "steps/s", "cores": threads, "kind": "port", "sample": f"{steps} step(s) of the {n}^3 workload, FP32 C++/OpenMP transcription of backend-cuda.cu's step sequence"}


def main():
    args = parse()
    import torch

    world, rank, local = dist_setup(args)
    sf = importlib.import_module("stable-fluids_b200")
    scene = sf.scenes.config1(n=args.size)
    n = args.size
    config = {"workload": f"plume {n}^3 FP32, 20 diffusion + 80 pressure iterations, 1 scalar + 1 force field, Stam walls",
              "grid": [n, n, n], "scheme": args.scheme, "l2": "working set > L2 (no flush needed)", "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}

    if args.impl == "reference":
        from oracle import oracle as orc

        if world > 1 and rank != 0:
            return
        lib = sf.load_library(orc.REF_LIB_PATH)
        sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=lib)
        sf.scenes.apply_inputs(sim, scene, 0)
        sim.step(args.warmup)
        torch.cuda.synchronize()
        with Clocks(local, not args.no_clocks) as clk:
            t = time_steps(sim, args.steps, 1)
        value = args.steps / t
        line = {"metric": METRIC, "value": value, "unit": "steps/s", "impl": "reference", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1000.0 * t / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded plume)",
                "config": config, "cell_updates_per_s": value * n ** 3,
                "cpu_baseline": {"value": value, "unit": "steps/s", "cores": 1, "kind": "reference", "sample": f"{args.steps} steps; the reference has no CPU implementation, so its own CUDA backend (backend-cuda.cu built unmodified for sm_100a) runs on the GPU"},
                "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        c = clk.summary()
        if c:
            line["clocks"] = c
        print(json.dumps(line))
        sim.close()
        return

    opts = sf.default_options()
    opts.scheme = sf.SCHEME_JACOBI if args.scheme == "jacobi" else sf.SCHEME_RBGS
    opts.iterations_per_pass = args.iterations_per_pass
    sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, options=opts, device=local)
    sf.scenes.apply_inputs(sim, scene, 0)
    sim.step(args.warmup)
    torch.cuda.synchronize()
    info = sim.info()

    with Clocks(local, not args.no_clocks and rank == 0) as clk:
        t = time_steps(sim, args.steps, world)
    t = max_over_ranks(t, world)
    value = world * args.steps / t

    # roofline of the dominant kernel family: the pressure solve
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    t_stage, launches = time_stage(sim, sf.STAGE_PRESSURE, 3)
    per_launch = t_stage / max(launches, 1)
    cells = n ** 3
    if args.scheme == "jacobi" or not info.blocked:
        bytes_per_launch = (12 if args.scheme == "jacobi" else 6) * cells
        unit_note = "one Jacobi sweep: read x + rhs, write x = 12 B/cell" if args.scheme == "jacobi" else "one red-black colour sweep: read n/2 other colour + n/2 rhs, write n/2 = 6 B/cell"
    else:
        bytes_per_launch = 12 * cells
        unit_note = "one temporally blocked pass: read p + rhs, write p = 12 B/cell"
    achieved = bytes_per_launch / per_launch / 1e9
    roofline = {"bound": "hbm", "kernel": "pressure stencil", "achieved": achieved, "peak": hbm_peak, "peak_source": peak_src, "unit": "GB/s", "frac": achieved / hbm_peak,
                "traffic": None, "bytes_per_launch": bytes_per_launch, "launch_us": per_launch * 1e6, "unit_of_work": unit_note}

    e2e = None
    if args.e2e_steps > 0:
        te, h2d, d2h = e2e_run(sf, sim, scene, args.e2e_steps)
        te = max_over_ranks(te, world)
        e2e = {"value": world * args.e2e_steps / te, "unit": "steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": args.e2e_steps}

    line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded plume)", "config": config,
            "cell_updates_per_s": value * cells, "gpu_launches": info.kernels_per_step * args.steps, "kernels_per_step": info.kernels_per_step,
            "roofline": roofline, "e2e": e2e}
    c = clk.summary() if rank == 0 else None
    if c:
        line["clocks"] = c
    if rank == 0 and world == 1 and args.equal_residual:
        variants = [v for v in args.equal_residual.split(",") if v]
        line["equal_residual"] = {"tolerance": args.residual_tolerance, "steps": args.residual_steps, "warmup": 2, "variants": equal_residual(sf, scene, variants, args.residual_tolerance, args.residual_steps, args.residual_cap, 2)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(sf, scene, args.cpu_steps)
    sim.close()
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
