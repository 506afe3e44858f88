"""Benchmark: steps/s of the stable-fluids step at 256^3 on B200, with the
pressure iterated until the FP64 relative Poisson residual is <= 1e-3:
learned warm start vs plain Jacobi at equal residual.

Workload (one "step" = one stable_fluids_step_cuda call = one step-graph
launch): the seeded 256^3 buoyant plume -- dt 0.1, viscosity 1e-4, density
diffusion 1e-5, 20 diffusion iterations, Stam walls, two Gaussian sources
(radius 8) with upward forces U[1, 10] (seed 1). The pressure solve runs
inside the step graph until rel_res = ||b - A p|| / ||b|| <= 1e-3 (checked
every 16 sweeps). The working set (> 1 GB) is far larger than L2, so no
flush is needed between steps.

Solver variants, all timed the same way (W untimed steps, then K steps):
  learned  : Jacobi sweeps from the learned warm start (the network is
             trained inside this run, before any timing, on pairs the solver
             generates at 128^3; its trial-and-select against the previous
             pressure runs every step) -- the headline `value`;
  plain    : Jacobi sweeps from zero (the reference's start: it resets the
             pressure every step) -- the comparison the metric names;
  previous : Jacobi sweeps from the previous step's pressure;
  rbgs     : red-black Gauss-Seidel from zero, the reference's own arithmetic.

  value : whole-job steps/s of the learned variant, inputs resident on the
          device, CUDA events on the simulation stream, max over ranks.
  e2e   : the learned variant through the public C ABI with host buffers,
          on a fresh context that replays the device-timed steps (same W
          untimed steps, same K timed steps, so the same solves): every step
          uploads the force field from pinned host memory
          (stable_fluids_update_vector_field_cuda with host pointers), reads
          the step's statistics and reads the density back to pinned host
          memory; one pair of CUDA events around the K steps.
  roofline : the dominant kernel, the Jacobi pressure sweep (12 B/cell),
          timed with CUDA events on the context stream; the network's
          convolutions are reported beside it against the bf16 peak.
  fixed_iterations : the reference's own configuration (80 red-black
          pressure iterations per step) for a like-for-like kernel comparison.
  batched : 64 uneven simulations (sizes over {32..128}^3, config-0
          coefficients) stepped by one batch graph launch per step; aggregate
          cell-updates/s (the reference arm steps its contexts in turn).
  bf16_storage : the 384^3 plume (20/80 red-black iterations) with FP32 and
          with BF16 storage of velocity and density: steps/s and the fields'
          relative difference.
  cpu_baseline : the FP32 C++/OpenMP transcription of the step (oracle/) on a
          bounded sample, scaled to the metric's unit.

--impl reference runs the reference's own implementation of the path -- its
CUDA backend compiled unmodified from backend-cuda.cu (oracle/_ref; the
reference has no CPU implementation) -- on the same scene through the same
C ABI. That process loads the reference library only. The reference cannot
iterate to a residual, so it runs with a fixed pressure-iteration count per
step: the counts the reference arithmetic (red-black Gauss-Seidel from zero,
bit-identical in this library) needs to reach the tolerance in each step are
read from bench_calibration.json, which `python bench.py --calibrate` writes
with this library's red-black variant. The line's value is the reference at
the mean of the timed steps' needs (the same total iterations as running
each step at its own need); the reference at the largest need (the fixed
count that reaches the tolerance in every timed step) is reported beside it.

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
CHECK_INTERVAL = 16
CALIBRATION = ROOT / "bench_calibration.json"
ITERATIONS_PER_PASS = 0  # set from --iterations-per-pass
# DRAM bytes (read + write) of one single-sweep Jacobi pressure launch
# (k_jacobi_vec4, consecutive launches in alternating z directions, caches
# kept warm between launches) from an ncu capture, by grid size.
PASS_TRAFFIC: dict[int, tuple[float, str]] = {
    256: (84.9e6 + 66.4e6, "profiles/k_jacobi_vec4_pressure_256.md: dram__bytes_read.sum + dram__bytes_write.sum, mean of four consecutive launches with --cache-control none"),
}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("b200", "reference"), default="b200")
    p.add_argument("--size", type=int, default=256)
    p.add_argument("--tolerance", type=float, default=1e-3)
    p.add_argument("--cap", type=int, default=100000, help="pressure-iteration cap of the residual-driven solve")
    p.add_argument("--variants", default="learned,plain,previous,rbgs")
    p.add_argument("--trial", type=int, default=CHECK_INTERVAL, help="learned start: sweeps of the trial against the previous pressure")
    p.add_argument("--weights", default=str(ROOT / "stable-fluids_b200" / "weights" / "warmstart_128.npy"),
                   help="trained warm-start parameters (stable-fluids_b200/train_warmstart.py); used when the file exists, unless --train-in-bench")
    p.add_argument("--train-in-bench", action="store_true", help="train the network inside this run instead of loading --weights")
    p.add_argument("--train-size", type=int, default=128)
    p.add_argument("--train-scenes", type=int, default=6)
    p.add_argument("--train-steps", type=int, default=32, help="pairs per training scene")
    p.add_argument("--train-sweeps", type=int, default=1000, help="Jacobi sweeps of the target solve")
    p.add_argument("--train-epochs", type=int, default=12)
    p.add_argument("--train-seconds", type=float, default=90.0)
    p.add_argument("--learning-rate", type=float, default=3e-4)
    p.add_argument("--e2e-steps", type=int, default=None, help="end-to-end timing through the C ABI: the first N of the device-timed steps (default: all K; 0: skip)")
    p.add_argument("--fixed-steps", type=int, default=20)
    p.add_argument("--batch-steps", type=int, default=100, help="steps of the batched 64-simulation workload (0: skip)")
    p.add_argument("--bf16-size", type=int, default=384)
    p.add_argument("--bf16-steps", type=int, default=50, help="timed steps of the FP32-vs-BF16-storage comparison (config 3: 50; 0: skip)")
    p.add_argument("--scene-steps", type=int, default=10, help="steps of the viewer-scene force generator comparison (0: skip)")
    p.add_argument("--render-frames", type=int, default=5, help="frames of the headless volume rendering measurement (0: skip)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-clocks", action="store_true")
    p.add_argument("--fixed-pressure-iterations", type=int, default=0,
                   help="profiling: run the variants with this fixed sweep count instead of the residual-driven solve (ncu cannot see kernels inside conditional graph nodes)")
    p.add_argument("--iterations-per-pass", type=int, default=0, help="stencil iterations per HBM pass of the variants' solves (0, 1: one launch per sweep; >= 2: z-wavefront passes)")
    p.add_argument("--calibrate", action="store_true", help="write bench_calibration.json: the red-black iterations each step of the scene needs (this library's rbgs variant), for --impl reference")
    p.add_argument("--calibrate-steps", type=int, default=40)
    a = p.parse_args()
    a.warmup = max(a.warmup, 3)
    global ITERATIONS_PER_PASS
    ITERATIONS_PER_PASS = a.iterations_per_pass
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


def dist_setup():
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int, device=None) -> float:
    """Max of a host float over the ranks (identity for one rank)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device if device is not None else "cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def solver_options(sf, variant, tol, cap, trial):
    o = sf.default_options()
    o.scheme = sf.SCHEME_RBGS if variant == "rbgs" else sf.SCHEME_JACOBI
    o.warm_start = {"learned": sf.WARM_START_LEARNED, "learned_coarse": sf.WARM_START_LEARNED, "plain": sf.WARM_START_ZERO, "previous": sf.WARM_START_PREVIOUS, "rbgs": sf.WARM_START_ZERO}[variant]
    o.warm_start_coarsening = 1 if variant == "learned_coarse" else 0
    o.compute_residual = 1
    o.residual_tolerance = tol
    o.residual_check_interval = CHECK_INTERVAL
    o.max_pressure_iterations = cap
    o.warm_start_trial_iterations = trial
    o.iterations_per_pass = ITERATIONS_PER_PASS
    return o


def launches_per_step(info, iterations, trial_done):
    """Kernels one residual-driven step launches: the captured step counts
    the loop body once; each further pass of the body launches the
    interval's stencil passes + the residual sums + the check
    (info.kernels_per_check)."""
    passes = max((iterations - trial_done) // CHECK_INTERVAL, 1)
    return info.kernels_per_step + (passes - 1) * info.kernels_per_check


def run_variant(sf, scene, variant, args, world, device, net=None):
    """W untimed steps then K timed steps (CUDA events per step on the
    simulation stream, summed); per-step iterations and residuals."""
    import torch

    opts = solver_options(sf, variant, 0.0 if args.fixed_pressure_iterations else args.tolerance, args.cap, args.trial)
    config = scene.config
    if args.fixed_pressure_iterations:
        config = type(scene.config).from_buffer_copy(scene.config)
        config.pressure_iterations = args.fixed_pressure_iterations
    sim = sf.Simulation(config, scene.scalars, scene.vectors, options=opts, device=device)
    if variant.startswith("learned"):
        net.attach(sim)
    sf.scenes.apply_inputs(sim, scene, 0)
    sim.step(args.warmup)
    torch.cuda.synchronize()
    info = sim.info()
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    its, res, fallback = [], [], []
    barrier(world)
    for k in range(args.steps):
        events[k][0].record(sim.stream)
        sim.step(1)
        events[k][1].record(sim.stream)
        st = sim.stats()  # waits for the step
        its.append(st.pressure_iterations)
        res.append(st.rel_residual)
        fallback.append(st.used_fallback)
    torch.cuda.synchronize()
    barrier(world)
    per_step = [a.elapsed_time(b) for a, b in events]
    t = sum(per_step) / 1000.0
    t = max_over_ranks(t, world)
    trial_done = args.trial if variant.startswith("learned") else 0
    if args.fixed_pressure_iterations:
        launches = info.kernels_per_step * args.steps
    else:
        launches = sum(launches_per_step(info, i, trial_done) for i in its)
    out = {"steps_per_s": world * args.steps / t, "ms_per_step": 1000.0 * t / args.steps, "ms_per_step_median": statistics.median(per_step), "pressure_iterations": its, "rel_residual": res, "hit_cap": any(r > args.tolerance for r in res), "gpu_launches": launches}
    if variant.startswith("learned"):
        out["used_fallback"] = fallback
        out["trial_sweeps"] = args.trial
    return sim, out


def load_network(sf, args, device):
    """The warm-start network with the committed trained parameters
    (stable-fluids_b200/train_warmstart.py wrote them and their protocol)."""
    import hashlib

    import numpy as np

    params = np.load(args.weights)
    net = sf.WarmStartNetwork(seed=0, device=device)
    net.set_parameters(params)
    info = {"source": os.path.relpath(args.weights, ROOT), "sha256": hashlib.sha256(np.ascontiguousarray(params, np.float32).tobytes()).hexdigest()[:16]}
    try:
        meta = json.loads(pathlib.Path(args.weights).with_suffix(".json").read_text())
        info.update({"protocol": meta.get("protocol"), "target_rel_residual": meta.get("target_rel_residual"), "best_held_out_error": meta.get("best_held_out_error"),
                     "sha256_matches_record": meta.get("sha256", "")[:16] == info["sha256"]})
    except (OSError, ValueError):
        pass
    return net, info


def train_network(sf, args, device):
    """Pairs from seeded 128^3 training plumes (targets: the scene's own
    Jacobi solve of --train-sweeps sweeps from the previous pressure), then
    Adam; everything on the GPU through the library."""
    t0 = time.perf_counter()
    pairs = []
    for k in range(args.train_scenes):
        scene = sf.scenes.training_scene(k, n=args.train_size, pressure_iterations=args.train_sweeps)
        pairs += sf.warmstart.generate_pairs(sf, scene, steps=args.train_steps, skip=2)
    t_pairs = time.perf_counter() - t0
    net = sf.WarmStartNetwork(seed=0, device=device)
    h = float(sf.scenes.training_scene(0, n=args.train_size).config.cell_size)
    history = sf.warmstart.train(net, pairs, h, epochs=args.train_epochs, learning_rate=args.learning_rate, deadline=time.perf_counter() + args.train_seconds) if pairs else []
    info = {"pairs": len(pairs), "grid": [args.train_size] * 3, "target_sweeps": args.train_sweeps, "epochs_run": len(history), "loss_per_epoch": history,
            "pair_generation_s": t_pairs, "training_s": time.perf_counter() - t0 - t_pairs}
    del pairs
    return net, info


def time_pressure_sweep(sf, scene, device, sweeps=96):
    """The Jacobi pressure solve's kernel, timed with CUDA events on the
    context stream: the fixed-count pressure stage of a Jacobi context
    (`sweeps` sweeps, a multiple of every pass size) enqueued directly,
    three times. Returns (seconds per launch, sweeps per launch)."""
    import torch

    o = sf.default_options()
    o.scheme = sf.SCHEME_JACOBI
    o.warm_start = sf.WARM_START_PREVIOUS
    cfg = type(scene.config).from_buffer_copy(scene.config)
    cfg.pressure_iterations = sweeps
    sim = sf.Simulation(cfg, scene.scalars, scene.vectors, options=o, device=device)
    sf.scenes.apply_inputs(sim, scene, 0)
    sim.step(1)
    sim.enqueue_stage(sf.STAGE_PRESSURE)
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    start.record(sim.stream)
    for _ in range(3):
        launches += sim.enqueue_stage(sf.STAGE_PRESSURE)
    end.record(sim.stream)
    torch.cuda.synchronize()
    sim.close()
    launches = max(launches, 1)
    return start.elapsed_time(end) / 1000.0 / launches, 3 * sweeps / launches


def time_network(net, n, device, repeats=3):
    """Duration of one prediction at n^3 (CUDA events on the network stream)."""
    import torch

    b = torch.randn(n, n, n, device=device)
    p = 0.1 * torch.randn(n, n, n, device=device)
    out = torch.empty_like(b)
    lib = net.lib
    args = (net.handle, b.data_ptr(), p.data_ptr(), n, n, n, 1.0 / n, out.data_ptr(), net.stream.cuda_stream)
    lib.stable_fluids_b200_network_predict(*args)
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(net.stream)
    for _ in range(repeats):
        lib.stable_fluids_b200_network_predict(*args)
    end.record(net.stream)
    torch.cuda.synchronize()
    return start.elapsed_time(end) / 1000.0 / repeats


def network_flops(n):
    """Multiply-adds x 2 of one prediction at n^3, counting only real
    channels (2 input channels of the first layer, 1 output channel)."""
    v0, v1, v2 = n ** 3, (n // 2) ** 3, (n // 4) ** 3
    macs = 27 * (v0 * (2 * 16 + 16 * 16 + 48 * 16 + 16 * 16 + 16 * 1) + v1 * (16 * 32 + 32 * 32 + 96 * 32 + 32 * 32) + v2 * (32 * 64 + 64 * 64))
    return 2.0 * macs


def e2e_run(sf, scene, args, steps, device, net):
    """The learned variant through the public ABI with host buffers, on a
    fresh context replaying the device-timed run's steps: the same W untimed
    steps, then the first `steps` of its K timed steps (the same solves). Each
    step uploads the force field from pinned host memory
    (stable_fluids_b200_stage_vector_field on an upload stream, so the upload
    of step k runs while step k - 1 computes), steps, and reads the density
    back to pinned host memory (stable_fluids_b200_read_view_async on a
    read-back stream, overlapping step k + 1). The timed region runs from before the first upload to after
    the last read-back. Returns the time, the bytes moved per step and the
    pressure iterations of the last step (per-step statistics would need a
    synchronisation per step)."""
    import numpy as np
    import torch

    sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, options=solver_options(sf, "learned", args.tolerance, args.cap, args.trial), device=device)
    try:
        net.attach(sim)
        sf.scenes.apply_inputs(sim, scene, 0)
        sim.step(args.warmup)
        n = sim.cells
        host_force = [torch.from_numpy(np.ascontiguousarray(f, dtype=np.float32)).pin_memory() for f in scene.force]
        host_rho = torch.empty(n, dtype=torch.float32).pin_memory()
        h = sim.scalar_handles[0]
        # one copy stream per direction: an upload queued behind the previous
        # step's read-back would wait for that step to finish
        up, down = torch.cuda.Stream(device=device), torch.cuda.Stream(device=device)
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record(sim.stream)
        up.wait_event(start)
        down.wait_event(start)
        for _ in range(steps):
            sim.stage_vector(sim.vector_handles[0], host_force[0], host_force[1], host_force[2], up)
            sim.step(1)
            sim.read_view_async(sf.VIEW_SCALAR_FIELD_DATA, [host_rho], down, handle=h)
        sim.stream.wait_stream(up)
        sim.stream.wait_stream(down)
        end.record(sim.stream)
        torch.cuda.synchronize()
        t = start.elapsed_time(end) / 1000.0
        its = [sim.stats().pressure_iterations]
    finally:
        sim.close()
    return t, 3 * n * 4, n * 4, its


def fixed_iterations(sf, lib, scene, steps, warmup, device, world):
    """The reference's configuration as it is: 80 red-black pressure
    iterations from zero per step (results bit-identical to the reference)."""
    import torch

    sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, lib=lib, device=device)
    sf.scenes.apply_inputs(sim, scene, 0)
    sim.step(warmup)
    torch.cuda.synchronize()
    barrier(world)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(sim.stream)
    sim.step(steps)
    end.record(sim.stream)
    torch.cuda.synchronize()
    barrier(world)
    t = max_over_ranks(start.elapsed_time(end) / 1000.0, world)
    sim.close()
    return {"steps_per_s": world * steps / t, "ms_per_step": 1000.0 * t / steps, "steps": steps, "pressure_iterations": scene.config.pressure_iterations, "scheme": "rbgs"}


def l2_copy_bandwidth(device, mib=24, repeats=50):
    """Bandwidth of a device copy whose source and destination (2 x `mib`
    MiB) stay in L2: bytes read + written per second, CUDA events. The
    denominator of the batched workload's L2 roofline."""
    import torch

    n = mib * 1024 * 1024 // 4
    a = torch.rand(n, device=device)
    b = torch.empty_like(a)
    for _ in range(5):
        b.copy_(a)
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(repeats):
        b.copy_(a)
    end.record()
    torch.cuda.synchronize()
    return 2 * 4 * n * repeats / (start.elapsed_time(end) / 1000.0) / 1e9


def batch_step_bytes(config):
    """Algorithmic bytes of one step of a red-black simulation (the bench's
    batched workload) per cell: 6 B per cell and colour launch (x of the
    colour read and written, the other colour and b read once), force + pack
    40, advection 28, scalar source + advection 28, divergence 16, projection
    44, diagnostics 20, copies for the diffusion starts 4 x 8."""
    sweeps = 2 * (4 * config.diffuse_iterations + config.pressure_iterations)
    return 6 * sweeps + 40 + 28 + 28 + 16 + 44 + 20 + 32


def batched(sf, lib, steps, warmup, count=64, mode=None, options=None, net=None, device=0):
    """Batched workload: `count` uneven plumes (sizes over {32..128}^3,
    config-0 coefficients, 20 diffusion / 40 red-black pressure iterations).
    mode: "work_table" (one persistent launch per stage over all
    simulations, z chunks from the tile autotuner), "graphs" (the step graphs
    as children of one graph), or None (each context stepped in turn on its
    own stream: how a caller drives the reference library). Timed with CUDA
    events on the batch stream (work table, graphs) or by the host clock
    around device synchronizations (contexts in turn). Returns aggregate
    cell-updates/s."""
    import torch

    scenes = sf.scenes.batch_scenes(count=count)
    sims = [sf.Simulation(sc.config, sc.scalars, sc.vectors, lib=lib, options=options) for sc in scenes]
    for sim, sc in zip(sims, scenes):
        if net is not None:
            net.attach(sim)
        sf.scenes.apply_inputs(sim, sc, 0)
    cells = sum(sim.cells for sim in sims)
    batch, extra = None, {}
    if mode is not None:
        t0 = time.perf_counter()
        with tempfile.TemporaryDirectory() as tmp:
            batch = sf.Batch(sims, mode=sf.BATCH_WORK_TABLE if mode == "work_table" else sf.BATCH_GRAPHS, autotune=mode == "work_table", tile_cache=os.path.join(tmp, "tiles.json") if mode == "work_table" else None)
        extra = {"kernels_per_step": batch.kernels_per_step, "layout_create_s": time.perf_counter() - t0, "l2_groups": batch.groups}
        if mode == "work_table":
            extra["z_chunks_by_size"] = {f"{sc.config.nx}^3": z for sc, z in sorted(zip(scenes, batch.z_chunks), key=lambda p: p[0].config.nx)}
    step = batch.step if batch is not None else (lambda: [sim.step(1) for sim in sims])
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    if batch is not None:
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(batch.stream)
        for _ in range(steps):
            step()
        end.record(batch.stream)
        torch.cuda.synchronize()
        t = start.elapsed_time(end) / 1000.0
        timing = "CUDA events on the batch stream"
    else:
        t0 = time.perf_counter()
        for _ in range(steps):
            step()
        torch.cuda.synchronize()
        t = time.perf_counter() - t0
        timing = "host clock around the steps with a device synchronize on both sides (work spans many streams)"
    residual = None
    if options is not None and options.compute_residual:
        r = sorted(sim.stats().rel_residual for sim in sims)
        residual = {"min": r[0], "median": statistics.median(r), "max": r[-1]}
    if batch is not None:
        batch.close()
    for sim in sims:
        sim.close()
    if residual is not None:
        extra["rel_residual_per_sim"] = residual
    if options is None or options.scheme == sf.SCHEME_RBGS:
        extra["algorithmic_bytes_per_s"] = sum(sim.cells * batch_step_bytes(sc.config) for sim, sc in zip(sims, scenes)) * steps / t
    sizes = sorted({sc.config.nx for sc in scenes})
    label = {"work_table": "one persistent launch per stage over a work table of L2-sized groups of simulations, groups on 4 concurrent streams (autotuned z chunks)", "graphs": "one graph of the simulations' step graphs per batch step", None: "each context stepped on its own stream"}[mode]
    if net is not None:
        label += "; Jacobi from one shared learned warm start (trial of 16 sweeps against the previous pressure), config-0 iteration count"
    return {"cell_updates_per_s": cells * steps / t, "steps_per_s": steps / t, "sims": count, "cells": cells, "sizes": sizes, "steps": steps, "timing": timing, "mode": label, **extra}


def bf16_storage(sf, n, steps, warmup, device):
    """Mixed precision at n^3 (the config-1 plume generator, 20 diffusion /
    80 red-black pressure iterations): steps/s with FP32 and with BF16
    storage of velocity and density, and the BF16 run's relative L2
    difference from the FP32 run per field after warmup + steps steps --
    beside the difference a one-ulp change of one force value makes to the
    FP32 run over the same steps (the flow's own amplification of a
    rounding-sized difference)."""
    import numpy as np
    import torch

    scene = sf.scenes.config1(n=n)
    out = {"grid": [n, n, n], "steps": steps, "warmup": warmup}
    fields = {}
    for name, storage in (("fp32", sf.STORAGE_FP32), ("bf16", sf.STORAGE_BF16), ("fp32_perturbed", sf.STORAGE_FP32)):
        opts = sf.default_options()
        opts.storage = storage
        sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, options=opts, device=device)
        sf.scenes.apply_inputs(sim, scene, 0)
        if name == "fp32_perturbed":
            # the same FP32 run with the force's largest component one ulp larger:
            # how far the flow itself carries a rounding-sized difference
            fx, fy, fz = (np.array(f, np.float32, copy=True) for f in scene.force)
            k = np.unravel_index(np.argmax(np.abs(fy)), fy.shape)
            fy[k] = np.nextafter(fy[k], np.float32(np.inf))
            sim.set_vector(sim.vector_handles[0], fx, fy, fz)
        sim.step(warmup)
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(sim.stream)
        sim.step(steps)
        end.record(sim.stream)
        torch.cuda.synchronize()
        if name != "fp32_perturbed":
            out[f"{name}_steps_per_s"] = steps / (start.elapsed_time(end) / 1000.0)
            out[f"{name}_device_bytes"] = sim.info().device_bytes
        fields[name] = {"density": sim.fetch(sf.VIEW_SCALAR_FIELD_DATA, sim.scalar_handles[0]), "velocity": np.stack(sim.fetch(sf.VIEW_FLOW_VELOCITY)), "pressure": sim.fetch(sf.VIEW_FLOW_PRESSURE)}
        sim.close()
    out["speedup"] = out["bf16_steps_per_s"] / out["fp32_steps_per_s"]
    rel = lambda a, b: float(np.linalg.norm(a.astype(np.float64) - b) / max(np.linalg.norm(b.astype(np.float64)), 1e-30))
    out["rel_l2_bf16_vs_fp32"] = {k: rel(fields["bf16"][k], fields["fp32"][k]) for k in fields["fp32"]}
    out["rel_l2_fp32_one_ulp_force_vs_fp32"] = {k: rel(fields["fp32_perturbed"][k], fields["fp32"][k]) for k in fields["fp32"]}
    return out


def scene_generator(sf, n, steps, device):
    """The reference viewer's per-step force update (vulkan-app/scene_plume.cpp:
    323-335) at n^3: the library's device generator (one kernel writing force x
    and z into the context) against the viewer's host path -- force x and z
    from the host masks (vectorised NumPy here, faster than the viewer's scalar
    loop), then two host-to-device copies through update_vector_field. The
    device path is timed with CUDA events, the host path with the host clock
    around device synchronizations. The host path's cost does not depend on
    the mask values, so it runs on seeded random masks of the same size."""
    import numpy as np
    import torch

    scene = sf.scenes.plume("viewer", (n, n, n), diffuse_iterations=20, pressure_iterations=40)
    sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, device=device)
    sim.plume_scene_setup()
    sim.plume_scene_forces(0)
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(sim.stream)
    for k in range(steps):
        sim.plume_scene_forces(k + 1)
    end.record(sim.stream)
    torch.cuda.synchronize()
    dev_s = start.elapsed_time(end) / 1000.0 / steps
    rng = np.random.default_rng(0)
    drift, swirl_x, swirl_z, fy = (rng.random((n, n, n), dtype=np.float32) for _ in range(4))
    t0 = time.perf_counter()
    for k in range(steps):
        phase = np.float32(k + 1) * np.float32(0.045)
        dx, dz, sw = np.float32(1.15) * np.sin(phase), np.float32(0.85) * np.cos(phase * np.float32(0.71)), np.float32(1.65) * np.cos(phase * np.float32(0.53))
        fx = dx * drift + sw * swirl_x
        fz = dz * drift + sw * swirl_z
        sim.set_vector(sim.vector_handles[0], fx, fy, fz)
    torch.cuda.synchronize()
    host_s = (time.perf_counter() - t0) / steps
    sim.close()
    bytes_written = 2 * 4 * n ** 3
    return {"grid": [n, n, n], "steps": steps, "device_us_per_step": dev_s * 1e6, "device_gbs": bytes_written / dev_s / 1e9, "host_path_ms_per_step": host_s * 1e3,
            "speedup": host_s / dev_s, "h2d_bytes_saved_per_step": bytes_written}


def volume_render(sf, n, device, width=1920, height=1080, steps=256, frames=5):
    """Headless ray-march of the density of an n^3 plume (the viewer's volume
    shader restated in CUDA) into a width x height RGBA float image:
    ms per frame (CUDA events) and samples per second (width * height *
    steps is the bound; rays leave the box or stop early)."""
    import numpy as np
    import torch

    scene = sf.scenes.config1(n=n)
    sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, device=device)
    sf.scenes.run(sim, scene, 3)
    ext = np.array([n * scene.config.cell_size] * 3, np.float32)
    centre = ext / 2
    eye = centre + np.array([0.35, 0.25, -1.6], np.float32) * ext.max()
    fwd = (centre - eye) / np.linalg.norm(centre - eye)
    right = np.cross(np.array([0, 1, 0], np.float32), fwd)
    right /= np.linalg.norm(right)
    up = np.cross(fwd, right)
    p = sf.B200VolumeRender()
    for k, val in {"eye": eye, "right": right, "up": up, "forward": fwd, "volume_min": np.zeros(3), "volume_max": ext, "color_a": (0.1, 0.2, 0.9), "color_b": (1.0, 0.6, 0.1)}.items():
        getattr(p, k)[:] = [float(t) for t in val]
    p.aspect, p.tan_half_fov, p.value_scale, p.density = width / height, 0.55, 1.0, 40.0
    p.value_min, p.value_max, p.steps, p.projection, p.width, p.height = 0.0, 2.0, steps, 0, width, height
    img = sim.render_volume(sf.VIEW_SCALAR_FIELD_DATA, p, sim.scalar_handles[0])
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(sim.stream)
    for _ in range(frames):
        sim.render_volume(sf.VIEW_SCALAR_FIELD_DATA, p, sim.scalar_handles[0], out=img)
    end.record(sim.stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(end) / frames
    coverage = float((img[..., 3] > 0).float().mean())
    sim.close()
    return {"grid": [n, n, n], "image": [width, height], "steps": steps, "ms_per_frame": ms, "frames_per_s": 1000.0 / ms,
            "max_samples_per_s": width * height * steps / (ms / 1000.0), "pixels_with_density": coverage}


def cpu_baseline(sf, scene, plain_iterations):
    """The FP32 C++/OpenMP transcription of the step (oracle/) on all host
    cores: one step without pressure sweeps and one with 16 Jacobi sweeps,
    scaled to the plain variant's mean sweep count."""
    from oracle import oracle as orc

    threads = orc.set_threads(os.cpu_count() or 1)
    times = {}
    for p in (0, 0, 48):  # the first run warms the host (page faults, thread pool)
        cfg = type(scene.config).from_buffer_copy(scene.config)
        cfg.pressure_iterations = p
        o = orc.Oracle(cfg, scene.scalars, scene.vectors, precision=32, scheme=orc.JACOBI)
        sf.scenes.apply_inputs(o, scene, 0)
        t0 = time.perf_counter()
        o.step(1)
        times[p] = time.perf_counter() - t0
        o.close()
    sweep = max(times[48] - times[0], 0.0) / 48
    n = scene.config.nx
    value = 1.0 / (times[0] + plain_iterations * sweep)
    return {"value": value, "unit": "steps/s", "cores": threads, "kind": "port",
            "sample": f"1 step of the {n}^3 plume without pressure sweeps ({times[0]:.2f} s) and 1 with 48 Jacobi sweeps ({times[48]:.2f} s) on {threads} threads; steps/s = 1 / (t_step + N x t_sweep) with N = {plain_iterations:.0f}, the mean sweep count of the plain variant (same arithmetic)"}


def calibration_key(args):
    return {"grid": [args.size] * 3, "tolerance": args.tolerance, "check_interval": CHECK_INTERVAL, "cap": args.cap, "scene": "config1 plume, seed 1"}


def calibrate(sf, args, scene, local):
    """Writes bench_calibration.json: the red-black iterations each step of
    the benchmark scene needs to reach the tolerance, from zero (this
    library's rbgs variant, bit-identical to the reference's arithmetic),
    stepping from the scene's first step on."""
    opts = solver_options(sf, "rbgs", args.tolerance, args.cap, 0)
    sim = sf.Simulation(scene.config, scene.scalars, scene.vectors, options=opts, device=local)
    sf.scenes.apply_inputs(sim, scene, 0)
    needs = []
    for _ in range(args.calibrate_steps):
        sim.step(1)
        needs.append(sim.stats().pressure_iterations)
    sim.close()
    doc = {**calibration_key(args), "rbgs_iterations_per_step": needs,
           "written_by": "python bench.py --calibrate (the library's red-black variant, residual-driven, from zero)"}
    CALIBRATION.write_text(json.dumps(doc, indent=1) + "\n")
    return doc


def read_calibration(args, first, count):
    """Per-step red-black needs of steps first .. first + count - 1 (0-based)
    from bench_calibration.json, or None if the file does not cover them."""
    try:
        doc = json.loads(CALIBRATION.read_text())
    except (OSError, ValueError):
        return None
    if any(doc.get(k) != v for k, v in calibration_key(args).items()):
        return None
    needs = doc.get("rbgs_iterations_per_step", [])
    return needs[first:first + count] if len(needs) >= first + count else None


def time_reference(sf, lib, scene, iterations, steps, warmup, local):
    """Steps/s of the reference library with a fixed pressure-iteration count."""
    import torch

    cfg = type(scene.config).from_buffer_copy(scene.config)
    cfg.pressure_iterations = iterations
    sim = sf.Simulation(cfg, scene.scalars, scene.vectors, lib=lib, device=local)
    sf.scenes.apply_inputs(sim, scene, 0)
    sim.step(warmup)
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(sim.stream)
    sim.step(steps)
    end.record(sim.stream)
    torch.cuda.synchronize()
    t = start.elapsed_time(end) / 1000.0
    sim.close()
    return steps / t


def reference_arm(sf, args, scene, world, rank, local):
    """The reference backend (oracle/_ref) at equal residual, with the
    per-step iteration needs read from bench_calibration.json. Only the
    reference library is loaded in this process."""
    from oracle import oracle as orc

    if rank != 0:
        return None
    n = args.size
    needs = read_calibration(args, args.warmup, args.steps)
    if needs is None:
        return {"impl": "reference", "unavailable": f"bench_calibration.json does not cover steps {args.warmup}..{args.warmup + args.steps - 1} of the {n}^3 scene at tolerance {args.tolerance:g}; run `python bench.py --calibrate --calibrate-steps {args.warmup + args.steps}`"}
    lib = sf.load_library(orc.REF_LIB_PATH)
    mean_need = int(round(statistics.mean(needs)))
    with Clocks(local, not args.no_clocks) as clk:
        value = time_reference(sf, lib, scene, mean_need, args.steps, args.warmup, local)
    at_max = time_reference(sf, lib, scene, max(needs), args.steps, args.warmup, local)
    config = {"workload": f"plume {n}^3 FP32, 20 diffusion its, pressure to rel_res <= {args.tolerance:g}, Stam walls", "grid": [n, n, n],
              "solver": f"reference red-black Gauss-Seidel from zero, {mean_need} iterations per step: the mean of the timed steps' needs {needs} (bench_calibration.json)",
              "l2": "working set > L2 (no flush needed)", "parallelism": "single GPU"}
    line = {"metric": METRIC, "value": value, "unit": "steps/s", "impl": "reference", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 / value, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded plume)",
            "config": config, "cell_updates_per_s": value * n ** 3,
            "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "at_max_need": {"steps_per_s": at_max, "pressure_iterations": max(needs), "note": "the fixed count that reaches the tolerance in every timed step"},
            "reference_run": {"kind": "reference", "device": "the same B200 (the reference has no CPU implementation; backend-cuda.cu built unmodified for sm_100a, oracle/_ref)",
                              "sample": f"{args.warmup} untimed + {args.steps} timed steps per iteration count"}}
    line["fixed_iterations"] = fixed_iterations(sf, lib, scene, args.fixed_steps, args.warmup, local, 1)
    if args.batch_steps > 0:
        line["batched"] = batched(sf, lib, args.batch_steps, args.warmup, mode=None)
    c = clk.summary()
    if c:
        line["clocks"] = c
    return line


def main():
    args = parse()
    import torch

    world, rank, local = dist_setup()
    sf = importlib.import_module("stable-fluids_b200")
    scene = sf.scenes.config1(n=args.size)
    n = args.size

    if args.calibrate:
        if rank == 0:
            doc = calibrate(sf, args, scene, local)
            print(json.dumps({"calibration": str(CALIBRATION.name), "rbgs_iterations_per_step": doc["rbgs_iterations_per_step"]}))
        return
    if args.impl == "reference":
        line = reference_arm(sf, args, scene, world, rank, local)
        if line is not None:
            print(json.dumps(line))
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return

    variants = [v for v in args.variants.split(",") if v]
    headline = "learned" if "learned" in variants else variants[0]  # profiling runs may leave the network out
    net, train_info = None, None
    if any(v.startswith("learned") for v in variants):
        net, train_info = load_network(sf, args, local) if (os.path.exists(args.weights) and not args.train_in_bench) else train_network(sf, args, local)

    results = {}
    with Clocks(local, not args.no_clocks and rank == 0) as clk:
        for v in variants:
            sim, out = run_variant(sf, scene, v, args, world, local, net if v.startswith("learned") else None)
            results[v] = out
            sim.close()
    learned = results[headline]
    value = learned["steps_per_s"]

    # roofline: the Jacobi sweep dominates every variant's step
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    tc_peak = float(peaks.get("bf16_tflops", 1590.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    launch_s, sweeps_per_launch = time_pressure_sweep(sf, scene, local)
    cells = n ** 3
    bytes_per_launch = 12 * cells
    achieved = bytes_per_launch / launch_s / 1e9
    traffic = PASS_TRAFFIC.get(n) if sweeps_per_launch == 1 else None
    kernel_name = "k_jacobi_vec4 (Jacobi pressure sweep)" if sweeps_per_launch == 1 else f"k_wave (Jacobi pressure pass, {sweeps_per_launch:g} sweeps per launch)"
    roofline = {"bound": "hbm", "kernel": kernel_name, "achieved": achieved, "peak": hbm_peak, "peak_source": peak_src, "unit": "GB/s", "frac": achieved / hbm_peak,
                "traffic": traffic[0] if traffic else None, "traffic_source": traffic[1] if traffic else None, "bytes_per_launch": bytes_per_launch, "launch_us": launch_s * 1e6,
                "sweeps_per_launch": sweeps_per_launch, "sweep_us": launch_s * 1e6 / sweeps_per_launch,
                "unit_of_work": f"one pass of {sweeps_per_launch:g} Jacobi sweeps over {n}^3 cells: read p + rhs, write p = 12 B/cell"}
    roofline_network = None
    if net is not None:
        net_s = time_network(net, n, torch.device("cuda", local))
        flops = network_flops(n)
        roofline_network = {"bound": "tensor", "kernel": "warm-start network prediction (all layers)", "achieved": flops / net_s / 1e12, "peak": tc_peak, "peak_source": peak_src, "unit": "TFLOP/s",
                            "frac": flops / net_s / 1e12 / tc_peak, "flop_per_launch": flops, "launch_ms": net_s * 1e3, "unit_of_work": f"one prediction at {n}^3, real channels only"}

    e2e = None
    e2e_steps = args.steps if args.e2e_steps is None else min(args.e2e_steps, args.steps)
    if e2e_steps > 0 and "learned" in results and not args.fixed_pressure_iterations:
        te, h2d, d2h, e2e_its = e2e_run(sf, scene, args, e2e_steps, local, net)
        te = max_over_ranks(te, world)
        e2e = {"value": world * e2e_steps / te, "unit": "steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": e2e_steps, "pressure_iterations_last_step": e2e_its, "io": "inputs staged on a copy stream (stable_fluids_b200_stage_vector_field), density read back asynchronously (stable_fluids_b200_read_view_async)"}
    fixed = fixed_iterations(sf, None, scene, args.fixed_steps, args.warmup, local, world) if args.fixed_steps > 0 else None
    batch = None
    if args.batch_steps > 0:
        rbgs = sf.default_options()
        rbgs.compute_residual = 1
        batch = batched(sf, None, args.batch_steps, args.warmup, mode="work_table", options=rbgs)
        l2 = l2_copy_bandwidth(torch.device("cuda", local))
        batch["roofline_l2"] = {"achieved_gbs": batch["algorithmic_bytes_per_s"] / 1e9, "peak_gbs": l2, "frac": batch["algorithmic_bytes_per_s"] / 1e9 / l2,
                                "peak_source": "measured here: device copy of 2 x 24 MiB resident in L2"}
        batch["graphs_layout"] = {k: v for k, v in batched(sf, None, args.batch_steps, args.warmup, mode="graphs", options=rbgs).items() if k in ("steps_per_s", "cell_updates_per_s", "kernels_per_step", "mode", "layout_create_s", "rel_residual_per_sim")}
        if net is not None:
            learned_opts = solver_options(sf, "learned", 0.0, args.cap, args.trial)
            learned_opts.compute_residual = 1
            previous_opts = solver_options(sf, "previous", 0.0, args.cap, args.trial)
            previous_opts.compute_residual = 1
            keys = ("steps_per_s", "cell_updates_per_s", "kernels_per_step", "mode", "rel_residual_per_sim")
            batch["shared_network"] = {k: v for k, v in batched(sf, None, args.batch_steps, args.warmup, mode="graphs", options=learned_opts, net=net).items() if k in keys}
            batch["previous_start_same_iterations"] = {k: v for k, v in batched(sf, None, args.batch_steps, args.warmup, mode="graphs", options=previous_opts).items() if k in keys}
    mixed = bf16_storage(sf, args.bf16_size, args.bf16_steps, args.warmup, local) if args.bf16_steps > 0 else None
    viewer = scene_generator(sf, n, args.scene_steps, local) if args.scene_steps > 0 else None
    render = volume_render(sf, n, local, frames=args.render_frames) if args.render_frames > 0 else None

    config = {"workload": f"plume {n}^3 FP32, 20 diffusion its, pressure to rel_res <= {args.tolerance:g} (checked every {CHECK_INTERVAL} sweeps), Stam walls",
              "grid": [n, n, n], "solver": {"learned": "Jacobi sweeps from the learned warm start", "plain": "Jacobi sweeps from zero", "previous": "Jacobi sweeps from the previous pressure", "rbgs": "red-black Gauss-Seidel from zero"}[headline]
            + (f", {args.fixed_pressure_iterations} sweeps per step (profiling)" if args.fixed_pressure_iterations else ""), "l2": "working set > L2 (no flush needed)",
              "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}
    # the rbgs variant must still need what bench_calibration.json (the
    # reference arm's iteration counts) says
    calibration_check = None
    if "rbgs" in results and not args.fixed_pressure_iterations:
        expected = read_calibration(args, args.warmup, args.steps)
        got = results["rbgs"]["pressure_iterations"]
        calibration_check = "no calibration for these steps" if expected is None else ("match" if expected == got else f"MISMATCH: calibration {expected}, this run {got}")
        if expected is not None and expected != got:
            print(f"bench: rbgs iterations differ from {CALIBRATION.name}: {expected} vs {got}", file=sys.stderr)
    ratios = {"speedup_vs_plain_jacobi": value / results["plain"]["steps_per_s"] if "plain" in results else None,
              "learned_vs_previous": value / results["previous"]["steps_per_s"] if "previous" in results and headline == "learned" else None,
              "mean_sweeps": {v: statistics.mean(r["pressure_iterations"]) for v, r in results.items()}}
    # Bulky per-step detail first; the compact summary of every leg last, so
    # that it survives in a record that keeps only the end of the line.
    line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": learned["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded plume)", "config": config,
            "variants": results, "training": train_info, "batched": batch, "bf16_storage": mixed, "viewer_scene_forces": viewer, "volume_render": render, "roofline_network": roofline_network,
            "e2e": e2e, "roofline": roofline, "cell_updates_per_s": value * cells, "gpu_launches": learned["gpu_launches"]}
    c = clk.summary() if rank == 0 else None
    if c:
        line["clocks"] = c
    if rank == 0 and world == 1 and not args.no_cpu_baseline and "plain" in results and not args.fixed_pressure_iterations:
        line["cpu_baseline"] = cpu_baseline(sf, scene, statistics.mean(results["plain"]["pressure_iterations"]))
    line["summary"] = {**ratios, "steps_per_s": {v: round(r["steps_per_s"], 3) for v, r in results.items()}, "calibration_check": calibration_check,
                       "e2e_steps_per_s": e2e["value"] if e2e else None, "jacobi_sweep_us": roofline["sweep_us"], "roofline_frac": roofline["frac"],
                       "network_ms": roofline_network["launch_ms"] if roofline_network else None,
                       "fixed_iterations_steps_per_s": fixed["steps_per_s"] if fixed else None,
                       "batched_gcups": {"work_table": batch["cell_updates_per_s"] / 1e9, "graphs": batch["graphs_layout"]["cell_updates_per_s"] / 1e9,
                                         "shared_network": batch["shared_network"]["cell_updates_per_s"] / 1e9 if "shared_network" in batch else None} if batch else None,
                       "batched_l2_frac": batch["roofline_l2"]["frac"] if batch else None,
                       "batched_rel_residual_median": {k: b["rel_residual_per_sim"]["median"] for k, b in (("work_table", batch), ("shared_network", batch.get("shared_network")), ("previous", batch.get("previous_start_same_iterations"))) if b} if batch else None,
                       "bf16": {k: mixed[k] for k in ("fp32_steps_per_s", "bf16_steps_per_s", "rel_l2_bf16_vs_fp32", "rel_l2_fp32_one_ulp_force_vs_fp32")} if mixed else None}
    if net is not None:
        net.close()
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
